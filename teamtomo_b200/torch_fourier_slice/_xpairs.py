"""x-paired volume copies for the extraction gathers.

A trilinear sample reads the corners (x0, x0 + 1) of four volume rows.  In the
x-paired copy, entry (z, y, x) holds the complex64 pair (V[z, y, x],
V[z, y, x + 1]) as four floats, so each row is one 16-byte gather instead of
two 8-byte ones: fewer L1 wavefronts for the same scattered addresses, the
limit of the extraction and of the rotation gradient.  Values and operation
order are unchanged, so results are bit-identical to the plain layout.

The copy costs one streaming pass over the volume (8 bytes read and 16
written per voxel, 0.05 ms at 256^3) and twice the volume's footprint in L2
while it is read.  Measured on a B200 (4096 slices, 2048 at 320; plain ->
x-paired, each kernel alone, the pack not included):

    box    copy     extraction   backward (dV + dR)   fused MSE
    128    17 MB    -11 %        -6 %                 -12 %
    192    57 MB    -12 %        -6.5 %               -13 %
    256    135 MB   -8 %         -1.5 %               -5 %
    320    264 MB   -8 %         +9.5 %               +6 %

Once the copy no longer fits in L2 its misses double the DRAM traffic of the
gathers; in a full training step (extraction, backward, insertion at 256^3)
that traffic slows the other kernels and pushes the GPU onto its power cap,
and the step is as fast or faster without the copy (372.9K vs 371.7K
slices/s).  Policy (``TT_VOLUME_XPAIRS`` = ``auto``, the default): gather
from a copy when the call's slices hold at least two pixels per voxel and the
copy fits in half the L2 (boxes up to about 192^3 on a B200); ``1`` always,
``0`` never.
"""

from __future__ import annotations

import ctypes
import os

import torch

from .. import _lib

MIN_PIXELS_PER_VOXEL = 2
_l2_bytes: dict[int, int] = {}


def l2_bytes(device: torch.device) -> int:
    """L2 cache size of a CUDA device (0 when unknown)."""
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if idx not in _l2_bytes:
        _l2_bytes[idx] = int(getattr(torch.cuda.get_device_properties(idx), "L2_cache_size", 0))
    return _l2_bytes[idx]


def copy_budget(volume: torch.Tensor) -> int:
    """Largest x-paired copy (bytes) worth making for ``volume``: half the L2
    of its GPU (0 for a CPU tensor)."""
    return l2_bytes(volume.device) // 2 if volume.is_cuda else 0


def use_xpairs(n_pixels: int, volume: torch.Tensor) -> bool:
    """Whether a call sampling ``n_pixels`` slice pixels from ``volume``
    (complex64, (d, h, w//2+1)) should gather from an x-paired copy."""
    mode = os.environ.get("TT_VOLUME_XPAIRS", "auto").strip().lower()
    if mode in ("0", "off", "false", "no"):
        return False
    if volume.dtype != torch.complex64 or volume.ndim != 3:
        return False
    if mode in ("1", "on", "true", "yes"):
        return True
    return n_pixels >= MIN_PIXELS_PER_VOXEL * volume.numel() and 16 * volume.numel() <= copy_budget(volume)


def with_xpairs(params: _lib.SliceParams, flag: bool) -> _lib.SliceParams:
    """Copy of ``params`` with ``volume_xpairs`` set to ``flag``."""
    q = _lib.SliceParams()
    ctypes.pointer(q)[0] = params
    q.volume_xpairs = int(bool(flag))
    return q


def pack(volume: torch.Tensor, params: _lib.SliceParams) -> torch.Tensor:
    """The x-paired copy of a contiguous complex64 volume: float32
    (d, h, w//2+1, 4), on the volume's device and current stream."""
    xp = torch.empty(tuple(volume.shape) + (4,), dtype=torch.float32, device=volume.device)
    L = _lib.load()
    _lib.check(L.tt_pack_volume_xpairs(_lib.ptr(volume), _lib.ptr(xp), params, _lib.stream_of(volume.device)),
               "pack_volume_xpairs")
    return xp
