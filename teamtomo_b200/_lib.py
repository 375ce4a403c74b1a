"""ctypes binding of the C ABI declared in ``include/teamtomo_b200.h``.

The CUDA library is required: there is no CPU fallback.  Importing the
package succeeds without a GPU (so CPU-side checks can run), but every call
that launches work needs the built ``libteamtomo_b200.so`` and CUDA tensors.
"""

from __future__ import annotations

import ctypes
import os

import torch

from . import _build

TT_OK, TT_ERR_INVALID, TT_ERR_CUDA, TT_ERR_WORKSPACE = 0, 1, 2, 3

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_f32 = ctypes.c_float
_sz = ctypes.c_size_t


class SliceParams(ctypes.Structure):
    """Mirror of ``tt_slice_params``."""

    _fields_ = [
        ("n", _i64), ("img_d", _i64), ("img_h", _i64), ("img_w", _i64),
        ("vol_d", _i64), ("vol_h", _i64), ("vol_w", _i64),
        ("has_fftfreq_max", _i32), ("fftfreq_max", _f32),
        ("zyx_matrices", _i32),
        ("x_tolerance", _f32), ("x_tolerance10", _f32),
        ("has_rot_tolerance", _i32), ("rot_tolerance", _f32),
        ("rotation_f64", _i32), ("volume_unshifted", _i32), ("slices_unshifted", _i32),
        ("deterministic", _i32), ("volume_layout", _i32),
    ]


class CtfParams(ctypes.Structure):
    """Mirror of ``tt_ctf_params`` (8 float32, the row layout of CTF tensors)."""

    _fields_ = [(name, _f32) for name in (
        "defocus_um", "astigmatism_um", "astigmatism_angle_deg", "voltage_kv",
        "spherical_aberration_mm", "amplitude_contrast", "phase_shift_deg", "pixel_size_a")]


class BatchVolume(ctypes.Structure):
    """Mirror of ``tt_batch_volume``."""

    _fields_ = [
        ("params", SliceParams),
        ("volume_rfft", _vp), ("slices", _vp), ("accumulator", _vp),
        ("rotation_matrices", _vp), ("ctf", _vp),
    ]


MAX_BATCH_VOLUMES = 96

# name -> (argtypes, restype); every symbol the header declares
SIGNATURES = {
    "tt_version": ([], _i32),
    "tt_last_error": ([], ctypes.c_char_p),
    "tt_extract_central_slices_rfft_3d": ([_vp, _vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_slice_geometry": ([_vp, _i32, _vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_volume_xpairs_bytes": ([ctypes.POINTER(SliceParams)], _sz),
    "tt_pack_volume_xpairs": ([_vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_volume_bricks_bytes": ([ctypes.POINTER(SliceParams)], _sz),
    "tt_pack_volume_bricks": ([_vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_extract_backward_workspace_bytes": ([ctypes.POINTER(SliceParams)], _sz),
    "tt_extract_central_slices_rfft_3d_backward": (
        [_vp, _vp, _vp, _vp, _vp, _vp, _sz, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_extract_central_slices_rfft_3d_backward_noalloc": (
        [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_central_slice_mse_workspace_bytes": ([ctypes.POINTER(SliceParams)], _sz),
    "tt_central_slice_mse": ([_vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_insert_central_slices_rfft_3d": (
        [_vp, _i32, _vp, _vp, _vp, _vp, _sz, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_insert_accumulator_bytes": ([_i32, _i64, _i64, _i64, _i64], _sz),
    "tt_insert_central_slices_rfft_3d_backward": ([_vp, _i32, _vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_insert_accumulate": ([_vp, _i32, _vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_insert_finalize": ([_vp, _i32, _i64, _i64, _i64, _i64, _vp, _vp, _vp], _i32),
    "tt_insert_accumulator_layout": ([ctypes.POINTER(SliceParams)], _i32),
    "tt_insert_bricked_accumulator_bytes": ([_i64, _i64, _i64], _sz),
    "tt_insert_finalize_bricked": ([_vp, _i64, _i64, _i64, _vp, _vp, _vp], _i32),
    "tt_probe_l2_reductions": ([_vp, _sz, _i64, _i32, ctypes.c_uint64, _vp], _i32),
    "tt_friedel_mirror_x0": ([_vp, _vp, _i32, _i64, _i64, _i64, _i64, _vp], _i32),
    "tt_insert_workspace_bytes": ([_i32, ctypes.POINTER(SliceParams)], _sz),
    "tt_fixed_absmax": ([_vp, _i32, _i64, _vp, _vp], _i32),
    "tt_insert_fixed_accumulator_bytes": ([_i64, _i64, _i64, _i64], _sz),
    "tt_insert_fixed_accumulate": ([_vp, _i32, _vp, _vp, _vp, _i64, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_insert_fixed_finalize": ([_vp, _i32, _i64, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _vp], _i32),
    "tt_extract_central_slices_rfft_3d_multichannel": ([_vp, _i64, _vp, _vp, ctypes.POINTER(SliceParams), _vp],
                                                       _i32),
    "tt_extract_central_slices_rfft_3d_multichannel_backward": (
        [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _sz, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_insert_accumulate_multichannel": ([_vp, _i64, _vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_insert_central_slices_rfft_3d_multichannel_backward": (
        [_vp, _i64, _vp, _vp, ctypes.POINTER(SliceParams), _vp], _i32),
    "tt_extract_central_lines_rfft_2d": ([_vp, _i64, _i64, _vp, _i32, _i64, _i64, _i64, _i32, _f32, _i32, _vp, _vp],
                                         _i32),
    "tt_extract_central_lines_rfft_2d_backward": (
        [_vp, _i64, _i64, _vp, _i32, _i64, _i64, _i64, _i32, _f32, _i32, _vp, _vp, _vp, _vp], _i32),
    "tt_batch_workspace_bytes": ([], _sz),
    "tt_extract_central_slices_rfft_3d_batched": (
        [ctypes.POINTER(BatchVolume), _i32, _i32, _vp, _sz, _vp], _i32),
    "tt_insert_central_slices_rfft_3d_batched": (
        [ctypes.POINTER(BatchVolume), _i32, _i32, _vp, _sz, _vp], _i32),
    "tt_sample_image_3d": ([_vp, _i32, _i64, _i64, _i64, _i64, _vp, _i64, _vp, _i32, _vp], _i32),
    "tt_sample_image_3d_backward": ([_vp, _i32, _i64, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _vp, _i32, _vp], _i32),
    "tt_insert_into_image_3d": (
        [_vp, _i32, _vp, _i64, _vp, _i64, _i64, _i64, _i64, _vp, _i32, _i32, _vp], _i32),
    "tt_affine_transform_image_3d": ([_vp, _i32, _i64, _i64, _i64, _i64, _vp, _i64, _i64, _i64, _i64, _i32, _vp,
                                      _vp], _i32),
    "tt_insert_into_image_3d_backward": ([_vp, _i32, _vp, _i64, _i64, _i64, _i64, _i64, _i32, _vp, _vp], _i32),
    "tt_project_prepare": ([_vp, _i32, _i64, _i64, _vp, _vp], _i32),
    "tt_recentre_crop_2d": ([_vp, _i32, _i64, _i64, _i64, _i64, _vp, _vp], _i32),
    "tt_pad_fftshift_2d": ([_vp, _i32, _i64, _i64, _i64, _vp, _vp], _i32),
    "tt_backproject_normalize": ([_vp, _i32, _i64, _i64, _i64, _i64, _vp, _vp], _i32),
    "tt_backproject_finish": ([_vp, _i32, _i64, _i64, _i64, _i64, _i64, _vp, _vp], _i32),
}

_lib = None


def lib_path() -> str:
    return _build.LIB


def load() -> ctypes.CDLL:
    """Load the CUDA library (building it first if the sources are newer)."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path) or _build.needs_build():
            try:
                _build.build()
            except Exception as exc:  # no nvcc or a compile error: fail loudly
                if not os.path.exists(path):
                    raise RuntimeError(
                        f"teamtomo_b200 CUDA library missing at {path} and could not be built: {exc}"
                    ) from exc
        L = ctypes.CDLL(path)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(status: int, what: str) -> None:
    if status == TT_OK:
        return
    msg = load().tt_last_error().decode(errors="replace")
    if status == TT_ERR_INVALID:
        raise ValueError(f"{what}: {msg}")
    raise RuntimeError(f"{what}: {msg}")


def dense(t: torch.Tensor) -> torch.Tensor:
    """``t`` as a C-contiguous tensor whose memory holds its values: lazy
    conjugate / negative views (``x.conj()``, and the gradients autograd
    passes through them) are materialised first."""
    return t.resolve_conj().resolve_neg().contiguous()


def ptr(t: torch.Tensor | None):
    if t is None:
        return None
    if t.is_conj() or t.is_neg():
        # the memory of a lazy view does not hold its values
        raise ValueError("tensor is a lazy conjugate/negative view; materialise it with dense()")
    return ctypes.c_void_p(t.data_ptr())


def stream_of(device: torch.device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda(*tensors: torch.Tensor) -> torch.device:
    dev = None
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda:
            raise RuntimeError(
                "teamtomo_b200 runs on CUDA tensors only (got a tensor on "
                f"{t.device}); there is no CPU fallback"
            )
        dev = t.device if dev is None else dev
    return dev
