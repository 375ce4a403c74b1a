"""CPU checks of the C ABI and the host layer (no GPU, no kernel launches).

* the library loads and exports every function include/teamtomo_b200.h declares,
  and the ctypes layer binds exactly those;
* argument validation fails with TT_ERR_INVALID before anything is launched;
* the workspace query and the parameter struct layout;
* host-side errors of the Python API raise the reference's exception types;
* the product refuses CPU tensors (no CPU fallback).
"""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "teamtomo_b200.h")


def declared_functions() -> set[str]:
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"\b(tt_[a-z0-9_]+)\s*\(", src))


def test_library_exports_every_declared_symbol():
    from teamtomo_b200 import _lib

    L = _lib.load()
    declared = declared_functions()
    assert len(declared) >= 10
    for name in declared:
        assert hasattr(L, name), name
    assert set(_lib.SIGNATURES) == declared
    assert L.tt_version() >= 100


def _params(**kw):
    from teamtomo_b200 import _lib

    p = _lib.SliceParams()
    p.n, p.img_d, p.img_h, p.img_w = 4, 16, 16, 16
    p.vol_d, p.vol_h, p.vol_w = 16, 16, 9
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_param_struct_layout():
    from teamtomo_b200 import _lib

    # 7 int64 + 12 four-byte fields (the last one in what was the tail padding)
    assert ctypes.sizeof(_lib.SliceParams) == 104
    assert _lib.SliceParams.fftfreq_max.offset == 60 and _lib.SliceParams.deterministic.offset == 96
    assert _lib.SliceParams.volume_layout.offset == 100


@pytest.mark.fake_pointers
@pytest.mark.parametrize("layout", [1, 2])
def test_volume_layout_validation(layout):
    """volume_layout: the copies are accepted by the extraction entry points
    (the multichannel ones take the bricked copies only), refused by the
    others, and codes outside {0, 1, 2} are refused; the packs check their
    pointers and alignment."""
    from teamtomo_b200 import _lib

    L = _lib.load()
    fake = ctypes.c_void_p(16)
    p = _params(volume_layout=layout)
    assert L.tt_volume_xpairs_bytes(ctypes.byref(p)) == 16 * 16 * 9 * 16
    assert L.tt_volume_bricks_bytes(ctypes.byref(p)) == 8 * 8 * 5 * 64
    assert L.tt_insert_accumulate(fake, 0, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert b"volume_layout" in L.tt_last_error()
    assert L.tt_insert_central_slices_rfft_3d(fake, 0, fake, fake, fake, fake, 1 << 30, ctypes.byref(p),
                                              None) == _lib.TT_ERR_INVALID
    if layout == 1:
        assert L.tt_extract_central_slices_rfft_3d_multichannel(fake, 2, fake, fake, ctypes.byref(p),
                                                                None) == _lib.TT_ERR_INVALID
        assert b"plain or bricked" in L.tt_last_error()
    # accepted (fails later, on the missing workspace, not on the layout)
    assert L.tt_extract_central_slices_rfft_3d_backward(fake, fake, fake, None, fake, None, 0,
                                                        ctypes.byref(p), None) == _lib.TT_ERR_WORKSPACE
    for bad in (3, -1):
        p = _params(volume_layout=bad)
        assert L.tt_extract_central_slices_rfft_3d(fake, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    p = _params()
    for pack in (L.tt_pack_volume_xpairs, L.tt_pack_volume_bricks):
        assert pack(None, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
        assert pack(fake, ctypes.c_void_p(24), ctypes.byref(p), None) == _lib.TT_ERR_INVALID
        assert b"16-byte" in L.tt_last_error()
        assert pack(ctypes.c_void_p(20), fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
        assert b"8-byte" in L.tt_last_error()


def test_volume_layout_policy(monkeypatch):
    from teamtomo_b200.torch_fourier_slice import _layout

    vol = torch.zeros((16, 16, 9), dtype=torch.complex64)
    monkeypatch.delenv("TT_VOLUME_LAYOUT", raising=False)
    # auto: the bricked copy from half a slice pixel per voxel up
    assert _layout.choose(vol.numel() // 2, vol) == _layout.BRICKS
    assert _layout.choose(vol.numel() // 2 - 1, vol) == _layout.PLAIN
    assert _layout.choose(10**9, vol.to(torch.complex128)) == _layout.PLAIN
    assert _layout.choose(10**9, vol[None]) == _layout.PLAIN
    for mode, code in (("plain", _layout.PLAIN), ("xpairs", _layout.XPAIRS), ("bricks", _layout.BRICKS)):
        monkeypatch.setenv("TT_VOLUME_LAYOUT", mode)
        assert _layout.choose(1, vol) == code
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "bogus")
    with pytest.raises(ValueError):
        _layout.choose(1, vol)
    assert _layout.pack(vol, None, _layout.PLAIN) is None
    from teamtomo_b200 import _lib

    p = _lib.SliceParams()
    p.n, p.deterministic = 7, 1
    q = _layout.with_layout(p, _layout.BRICKS)
    assert (q.n, q.deterministic, q.volume_layout, p.volume_layout) == (7, 1, 2, 0)


@pytest.mark.fake_pointers
def test_validation_rejects_before_launch():
    from teamtomo_b200 import _lib

    L = _lib.load()
    fake = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    p = _params(n=-1)
    assert L.tt_extract_central_slices_rfft_3d(fake, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert b"n must be" in L.tt_last_error()
    p = _params(img_h=0)
    assert L.tt_extract_central_slices_rfft_3d(fake, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    p = _params()
    assert L.tt_extract_central_slices_rfft_3d(None, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert b"NULL" in L.tt_last_error()
    p = _params(vol_w=8)  # insertion needs the rfft of volume_shape
    assert L.tt_insert_central_slices_rfft_3d(fake, 0, fake, fake, fake, fake, 1 << 30, ctypes.byref(p),
                                              None) == _lib.TT_ERR_INVALID
    p = _params()
    assert L.tt_insert_central_slices_rfft_3d(fake, 0, fake, fake, fake, fake, 16, ctypes.byref(p),
                                              None) == _lib.TT_ERR_WORKSPACE
    assert L.tt_insert_accumulate(fake, 0, fake, None, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert L.tt_insert_finalize(fake, 0, 0, 4, 4, 3, fake, fake, None) == _lib.TT_ERR_INVALID
    p = _params()
    assert L.tt_extract_central_slices_rfft_3d_backward(fake, fake, fake, None, fake, None, 0,
                                                        ctypes.byref(p), None) == _lib.TT_ERR_WORKSPACE
    assert L.tt_friedel_mirror_x0(None, None, 0, 1, 4, 4, 3, None) == _lib.TT_ERR_INVALID
    assert L.tt_slice_geometry(fake, 7, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert L.tt_sample_image_3d(fake, 9, 1, 4, 4, 4, fake, 1, fake, 0, None) == _lib.TT_ERR_INVALID
    assert L.tt_backproject_finish(fake, 0, 1, 8, 8, 8, 4, fake, None) == _lib.TT_ERR_INVALID
    assert L.tt_recentre_crop_2d(fake, 0, 1, 8, 7, 4, fake, None) == _lib.TT_ERR_INVALID
    # n == 0 is a successful no-op that touches nothing
    p = _params(n=0)
    assert L.tt_extract_central_slices_rfft_3d(fake, fake, fake, ctypes.byref(p), None) == _lib.TT_OK


@pytest.mark.fake_pointers
def test_batched_validation_and_layout():
    from teamtomo_b200 import _lib

    L = _lib.load()
    assert ctypes.sizeof(_lib.CtfParams) == 32
    assert ctypes.sizeof(_lib.BatchVolume) == 104 + 5 * 8
    assert L.tt_batch_workspace_bytes() >= 8
    fake = ctypes.c_void_p(16)
    arr = (_lib.BatchVolume * 1)(_lib.BatchVolume(_params(), fake, fake, fake, fake, None))
    assert L.tt_extract_central_slices_rfft_3d_batched(arr, 97, 0, fake, 256, None) == _lib.TT_ERR_INVALID
    assert L.tt_extract_central_slices_rfft_3d_batched(arr, 1, 3, fake, 256, None) == _lib.TT_ERR_INVALID
    assert L.tt_extract_central_slices_rfft_3d_batched(arr, 1, 0, None, 0, None) == _lib.TT_ERR_WORKSPACE
    bad = (_lib.BatchVolume * 1)(_lib.BatchVolume(_params(vol_w=8), None, fake, fake, fake, None))
    assert L.tt_insert_central_slices_rfft_3d_batched(bad, 1, 0, fake, 256, None) == _lib.TT_ERR_INVALID
    assert L.tt_extract_central_slices_rfft_3d_batched(bad, 1, 0, fake, 256, None) == _lib.TT_ERR_INVALID
    # layouts: the extraction takes plain or bricked volumes, one layout per call; the insertion plain
    # or bricked accumulators (fftshifted volumes), mixed in one call
    xp = (_lib.BatchVolume * 1)(_lib.BatchVolume(_params(volume_layout=1), fake, fake, fake, fake, None))
    assert L.tt_extract_central_slices_rfft_3d_batched(xp, 1, 0, fake, 256, None) == _lib.TT_ERR_INVALID
    assert b"plain or bricked" in L.tt_last_error()
    assert L.tt_insert_central_slices_rfft_3d_batched(xp, 1, 0, fake, 256, None) == _lib.TT_ERR_INVALID
    assert b"bricked" in L.tt_last_error()
    unshifted = (_lib.BatchVolume * 1)(_lib.BatchVolume(_params(volume_layout=2, volume_unshifted=1), fake, fake,
                                                        fake, fake, None))
    assert L.tt_insert_central_slices_rfft_3d_batched(unshifted, 1, 0, fake, 256, None) == _lib.TT_ERR_INVALID
    mixed = (_lib.BatchVolume * 2)(_lib.BatchVolume(_params(volume_layout=2), fake, fake, fake, fake, None),
                                   _lib.BatchVolume(_params(), fake, fake, fake, fake, None))
    assert L.tt_extract_central_slices_rfft_3d_batched(mixed, 2, 0, fake, 256, None) == _lib.TT_ERR_INVALID
    assert b"one volume_layout" in L.tt_last_error()
    # accepted: with no CUDA device visible it fails on the first CUDA call, not in validation
    assert L.tt_insert_central_slices_rfft_3d_batched(mixed, 2, 0, fake, 256, None) not in (_lib.TT_OK,
                                                                                          _lib.TT_ERR_INVALID)
    assert b"memset" in L.tt_last_error()


@pytest.mark.fake_pointers
def test_insert_backward_gradient_layouts():
    from teamtomo_b200 import _lib

    L = _lib.load()
    fake = ctypes.c_void_p(16)
    # the gradient volume is plain or, complex64 and fftshifted, its bricked copy; never x-paired
    for kw, c128 in ((dict(volume_layout=1), 0), (dict(volume_layout=2), 1),
                     (dict(volume_layout=2, volume_unshifted=1), 0), (dict(volume_layout=3), 0)):
        p = _params(**kw)
        assert L.tt_insert_central_slices_rfft_3d_backward(fake, c128, fake, fake, ctypes.byref(p),
                                                           None) == _lib.TT_ERR_INVALID, kw
    p = _params(volume_layout=2, vol_w=8)
    assert L.tt_insert_central_slices_rfft_3d_backward(fake, 0, fake, fake, ctypes.byref(p),
                                                       None) == _lib.TT_ERR_INVALID
    p = _params(volume_layout=2, n=0)
    assert L.tt_insert_central_slices_rfft_3d_backward(fake, 0, fake, fake, ctypes.byref(p), None) == _lib.TT_OK


@pytest.mark.fake_pointers
def test_probe_validation():
    from teamtomo_b200 import _lib

    L = _lib.load()
    fake = ctypes.c_void_p(1 << 20)
    assert L.tt_probe_l2_reductions(None, 1 << 20, 8, 8, 0, None) == _lib.TT_ERR_INVALID
    assert L.tt_probe_l2_reductions(ctypes.c_void_p((1 << 20) + 16), 1 << 20, 8, 8, 0, None) == _lib.TT_ERR_INVALID
    assert L.tt_probe_l2_reductions(fake, 1000, 8, 8, 0, None) == _lib.TT_ERR_INVALID
    assert L.tt_probe_l2_reductions(fake, 1 << 20, 8, 3, 0, None) == _lib.TT_ERR_INVALID
    assert L.tt_probe_l2_reductions(fake, 1 << 20, -1, 8, 0, None) == _lib.TT_ERR_INVALID
    assert L.tt_probe_l2_reductions(fake, 1 << 20, 4, 8, 0, None) == _lib.TT_OK  # fewer than one group


def test_bricked_insert_accumulator_policy():
    from teamtomo_b200 import _lib

    L = _lib.load()
    # plain below 64 MB of bricked accumulator, bricked from there up (fftshifted, float) while the
    # accumulator fits one z-phase of the L2 (a B200's 126 MB: 256^3 does, 320^3 does not; with no
    # device to ask, one phase is assumed)
    import torch

    phased = 0 if torch.cuda.is_available() else 2
    for n, want in ((64, 0), (128, 0), (200, 0), (216, 2), (256, 2), (320, phased)):
        p = _params(img_d=n, img_h=n, img_w=n, vol_d=n, vol_h=n, vol_w=n // 2 + 1)
        assert L.tt_insert_accumulator_layout(ctypes.byref(p)) == want, n
        assert L.tt_insert_bricked_accumulator_bytes(n, n, n // 2 + 1) == (
            ((n + 1) // 2) * ((n + 1) // 2) * ((n // 2 + 2) // 2) * 8 * 16)
        p.volume_unshifted = 1
        assert L.tt_insert_accumulator_layout(ctypes.byref(p)) == 0
        p.volume_unshifted, p.deterministic = 0, 1
        assert L.tt_insert_accumulator_layout(ctypes.byref(p)) == 0
    assert L.tt_insert_bricked_accumulator_bytes(0, 4, 4) == 0
    assert L.tt_insert_finalize_bricked(None, 4, 4, 3, None, None, None) == _lib.TT_ERR_INVALID


@pytest.mark.fake_pointers
def test_deterministic_mode_workspace_and_validation():
    from teamtomo_b200 import _lib

    L = _lib.load()
    fake = ctypes.c_void_p(16)
    vox = 16 * 16 * 9
    p = _params()
    assert L.tt_insert_workspace_bytes(0, ctypes.byref(p)) == vox * 16
    assert L.tt_insert_workspace_bytes(1, ctypes.byref(p)) == vox * 32
    base = L.tt_extract_backward_workspace_bytes(ctypes.byref(p))
    p = _params(deterministic=1)
    assert L.tt_insert_workspace_bytes(0, ctypes.byref(p)) == 256 + vox * 32
    assert L.tt_extract_backward_workspace_bytes(ctypes.byref(p)) == base + 256 + vox * 16
    assert L.tt_insert_fixed_accumulator_bytes(2, 16, 16, 9) == 2 * vox * 32
    # a deterministic one-shot insertion checks its larger workspace
    assert L.tt_insert_central_slices_rfft_3d(fake, 0, fake, fake, fake, fake, vox * 16, ctypes.byref(p),
                                              None) == _lib.TT_ERR_WORKSPACE
    # the float two-stage API refuses the flag; the fixed one checks max_slices and pointers
    assert L.tt_insert_accumulate(fake, 0, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert L.tt_insert_fixed_accumulate(fake, 0, fake, fake, fake, 3, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert b"max_slices" in L.tt_last_error()
    assert L.tt_insert_fixed_accumulate(fake, 0, fake, fake, None, 4, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert L.tt_insert_fixed_finalize(fake, 0, 1, 16, 16, 9, fake, 0, fake, fake, None) == _lib.TT_ERR_INVALID
    assert L.tt_fixed_absmax(fake, 0, -1, fake, None) == _lib.TT_ERR_INVALID
    assert L.tt_fixed_absmax(None, 0, 0, None, None) == _lib.TT_OK  # empty: nothing to do
    # the no-allocation backward cannot hold a fixed-point volume gradient
    assert L.tt_extract_central_slices_rfft_3d_backward_noalloc(fake, fake, fake, fake, None, ctypes.byref(p),
                                                                None) == _lib.TT_ERR_INVALID
    arr = (_lib.BatchVolume * 1)(_lib.BatchVolume(p, fake, fake, fake, fake, None))
    assert L.tt_extract_central_slices_rfft_3d_batched(arr, 1, 0, fake, 256, None) == _lib.TT_ERR_INVALID
    p = _params(deterministic=2)
    assert L.tt_extract_central_slices_rfft_3d(fake, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID


def test_deterministic_flag_follows_torch():
    from teamtomo_b200.torch_fourier_slice._params import resolve_deterministic

    assert resolve_deterministic(True) and not resolve_deterministic(False)
    before = torch.are_deterministic_algorithms_enabled()
    try:
        torch.use_deterministic_algorithms(True)
        assert resolve_deterministic(None)
        torch.use_deterministic_algorithms(False)
        assert not resolve_deterministic(None)
    finally:
        torch.use_deterministic_algorithms(before)


def test_lazy_conjugate_views_are_materialised():
    """x.conj() is a lazy view whose memory holds x: the pointer layer refuses
    it and dense() resolves it (autograd passes such views as gradients)."""
    from teamtomo_b200 import _lib

    x = torch.tensor([1 + 2j, 3 - 4j], dtype=torch.complex64)
    with pytest.raises(ValueError, match="lazy conjugate"):
        _lib.ptr(x.conj())
    with pytest.raises(ValueError, match="lazy conjugate"):
        _lib.ptr(torch.view_as_real(x)._neg_view())
    y = _lib.dense(x.conj())
    assert not y.is_conj() and torch.equal(y, torch.conj_physical(x))
    assert _lib.dense(x) is x  # nothing to do: no copy


def test_ctf_params_rows():
    from teamtomo_b200.batched import ctf_params

    rows = ctf_params([1.0, 2.0, 3.0], astigmatism_um=0.1)
    assert rows.shape == (3, 8) and rows.dtype == torch.float32
    assert torch.equal(rows[:, 0], torch.tensor([1.0, 2.0, 3.0]))
    assert torch.allclose(rows[:, 1], torch.full((3,), 0.1))
    assert torch.equal(rows[:, 3], torch.full((3,), 300.0))
    with pytest.raises(ValueError):
        ctf_params([1.0, 2.0], astigmatism_um=[0.1, 0.2, 0.3])


def test_workspace_query():
    from teamtomo_b200 import _lib

    L = _lib.load()
    p = _params(n=4096, img_d=256, img_h=256, img_w=256, vol_d=256, vol_h=256, vol_w=129)
    tiles = ((129 + 7) // 8) * ((256 + 31) // 32)  # 8 x 32 pixel tiles: one slot of 6 partial sums each
    assert L.tt_extract_backward_workspace_bytes(ctypes.byref(p)) == 4096 * tiles * 6 * 4
    assert L.tt_insert_accumulator_bytes(0, 1, 256, 256, 129) == 256 * 256 * 129 * 16
    assert L.tt_insert_accumulator_bytes(1, 2, 4, 4, 3) == 2 * 4 * 4 * 3 * 32
    p = _params(n=0)
    assert L.tt_extract_backward_workspace_bytes(ctypes.byref(p)) == 0


def test_slice_params_rounding():
    from teamtomo_b200.torch_fourier_slice._params import slice_params

    p = slice_params(n=3, image_shape=(16, 16, 16), volume=None, rotation=torch.zeros(3, 3, 3),
                     fftfreq_max=0.3, x_tolerance=1e-8, rot_tolerance=1e-8, vol_dims=(16, 16, 9))
    assert p.x_tolerance == float(np.float32(1e-8))
    assert p.x_tolerance10 == float(np.float32(1e-8 * 10))
    assert p.fftfreq_max == float(np.float32(0.3))
    assert p.has_rot_tolerance == 1 and p.rotation_f64 == 0
    p = slice_params(n=1, image_shape=(8, 8, 8), volume=None, rotation=torch.zeros(1, 3, 3, dtype=torch.float64),
                     rot_tolerance=None, vol_dims=(8, 8, 5))
    assert p.has_rot_tolerance == 0 and p.rotation_f64 == 1 and p.has_fftfreq_max == 0


def test_rotation_arg():
    from teamtomo_b200.torch_fourier_slice._params import rotation_arg

    R, stack = rotation_arg(torch.zeros(4, 5, 3, 3, dtype=torch.float16), torch.device("cpu"))
    assert R.shape == (20, 3, 3) and R.dtype == torch.float32 and stack == (4, 5)
    R, stack = rotation_arg(torch.zeros(3, 3, dtype=torch.float64), torch.device("cpu"))
    assert R.shape == (1, 3, 3) and R.dtype == torch.float64 and stack == ()
    with pytest.raises(ValueError):
        rotation_arg(torch.zeros(4, 3, 2), torch.device("cpu"))


def test_no_cpu_fallback():
    import teamtomo_b200 as tt

    vol = torch.zeros((8, 8, 5), dtype=torch.complex64)
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        tt.extract_central_slices_rfft_3d(vol, (8, 8, 8), torch.eye(3))
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        tt.insert_central_slices_rfft_3d(torch.zeros((1, 8, 5), dtype=torch.complex64), (8, 8, 8),
                                         torch.eye(3)[None])
    with pytest.raises(RuntimeError, match="CUDA tensors only"):
        tt.sample_image_3d(torch.zeros((4, 4, 4)), torch.zeros((2, 3)))


def test_reference_exceptions_on_host():
    import teamtomo_b200 as tt

    with pytest.raises(ValueError, match="all dimensions of volume must be equal"):
        tt.project_3d_to_2d(torch.zeros((8, 8, 9)), torch.eye(3))
    with pytest.raises(ValueError, match="pad_factor"):
        tt.project_3d_to_2d(torch.zeros((8, 8, 8)), torch.eye(3), pad_factor=0.5)
    with pytest.raises(ValueError, match="images must be square"):
        tt.backproject_2d_to_3d(torch.zeros((2, 8, 9)), torch.eye(3)[None])
    with pytest.raises(AssertionError):
        tt.extract_central_slices_rfft_3d(torch.zeros((8, 8)), (8, 8, 8), torch.eye(3))
    with pytest.raises(ValueError, match="One coordinate triplet"):
        tt.insert_into_image_3d(torch.zeros(3), torch.zeros((4, 3)), torch.zeros((4, 4, 4)))
    with pytest.raises(ValueError, match="same dtype"):
        tt.insert_into_image_3d(torch.zeros(4, dtype=torch.float64), torch.zeros((4, 3)), torch.zeros((4, 4, 4)))
    with pytest.raises(ValueError, match="shape \\(d, h, w\\)"):
        tt.sample_image_3d(torch.zeros((4, 4)), torch.zeros((2, 3)))


def test_streaming_host_checks():
    from teamtomo_b200 import streaming

    assert streaming.chunk_bounds(10, 4) == [(0, 4), (4, 8), (8, 10)]
    assert streaming.chunk_bounds(0, 4) == []
    with pytest.raises(ValueError):
        streaming.chunk_bounds(10, 0)
    with pytest.raises(ValueError, match="leading size"):
        next(streaming.prefetch_to_device([torch.zeros(3), torch.zeros(4)], 2, "cpu"))
    with pytest.raises(ValueError, match="data_bound"):
        streaming.InsertionAccumulator((8, 8, 8), "cpu", deterministic=True)


@pytest.mark.fake_pointers
def test_fused_mse_validation():
    from teamtomo_b200 import _lib

    L = _lib.load()
    fake = ctypes.c_void_p(16)
    p = _params()
    need = L.tt_central_slice_mse_workspace_bytes(ctypes.byref(p))
    rows = (16 + 31) // 32  # loss (double) and rotation partials per row of tiles
    assert need == 4 * rows * 8 + 4 * rows * 6 * 4
    assert L.tt_central_slice_mse(fake, fake, fake, fake, None, None, fake, 8, ctypes.byref(p),
                                  None) == _lib.TT_ERR_WORKSPACE
    assert L.tt_central_slice_mse(fake, fake, fake, None, None, None, fake, need, ctypes.byref(p),
                                  None) == _lib.TT_ERR_INVALID
    p = _params(deterministic=1)
    assert L.tt_central_slice_mse(fake, fake, fake, fake, None, None, fake, need, ctypes.byref(p),
                                  None) == _lib.TT_ERR_INVALID
    p = _params(n=0)
    assert L.tt_central_slice_mse(fake, fake, fake, fake, None, None, fake, need, ctypes.byref(p),
                                  None) == _lib.TT_ERR_INVALID


def test_multichannel_layout_policy(monkeypatch):
    """The multichannel extraction follows the single-volume policy per
    channel, except that it takes no x-paired copy."""
    from teamtomo_b200.torch_fourier_slice import _layout
    from teamtomo_b200.torch_fourier_slice.slice_extraction import _multichannel_layout

    vols = torch.zeros((3, 16, 16, 9), dtype=torch.complex64)
    per_channel = vols[0].numel()
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "auto")
    assert _multichannel_layout(per_channel, vols) == _layout.BRICKS
    assert _multichannel_layout(per_channel // 2 - 1, vols) == _layout.PLAIN
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "xpairs")
    assert _multichannel_layout(per_channel, vols) == _layout.PLAIN
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "bricks")
    assert _multichannel_layout(1, vols) == _layout.BRICKS
    with pytest.raises(ValueError):
        _layout.pack_channels(vols, None, _layout.XPAIRS)
    assert _layout.pack_channels(vols, None, _layout.PLAIN) is None


def test_bricks_slot_limit_in_policy(monkeypatch):
    """The gathers address a bricked copy with 32-bit slot offsets, so the
    auto policy keeps volumes whose copy would reach 2^31 slots plain (shapes
    only: meta tensors hold no memory)."""
    from teamtomo_b200.torch_fourier_slice import _layout

    monkeypatch.setenv("TT_VOLUME_LAYOUT", "auto")
    fits = torch.empty((1024, 1024, 513), dtype=torch.complex64, device="meta")
    too_big = torch.empty((2048, 2048, 1025), dtype=torch.complex64, device="meta")
    assert _layout.bricks_fit(fits) and not _layout.bricks_fit(too_big)
    assert _layout.choose(10**13, fits) == _layout.BRICKS
    assert _layout.choose(10**13, too_big) == _layout.PLAIN
    # a forced bricked layout names the limit instead of failing in the C ABI
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "bricks")
    assert _layout.choose(10**13, fits) == _layout.BRICKS
    with pytest.raises(ValueError, match="2\\^31"):
        _layout.choose(10**13, too_big)


@pytest.mark.fake_pointers
def test_bricks_slot_limit_in_the_c_abi():
    """A volume whose bricked copy would hold 2^31 slots or more (1500 x 1500
    x 1001: 2.25 G slots, below the 2^32-voxel volume limit) is refused with
    the bricked layout and by the pack, before any launch."""
    from teamtomo_b200 import _lib

    L = _lib.load()
    fake = ctypes.c_void_p(16)
    big = dict(vol_d=1500, vol_h=1500, vol_w=1001)
    p = _params(volume_layout=2, **big)
    assert L.tt_extract_central_slices_rfft_3d(fake, fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert b"2^31" in L.tt_last_error()
    p = _params(**big)
    assert L.tt_pack_volume_bricks(fake, fake, ctypes.byref(p), None) == _lib.TT_ERR_INVALID
    assert b"2^31" in L.tt_last_error()
