"""The allocation-free extraction backward, called through the C ABI.

Some callers of this library cannot allocate device memory when they run the
backward pass (a host or plugin framework that owns every device allocation
and only lends the buffers of one call, or a fixed memory budget that must not
grow).  tt_extract_central_slices_rfft_3d_backward_noalloc serves them with a
4 MiB scratch array built into the library instead of a caller workspace.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.  It must pass alone in a
fresh process as well as after the other tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu


def _params(n_slices, box, R):
    from teamtomo_b200.torch_fourier_slice._params import slice_params

    return slice_params(n=n_slices, image_shape=(box, box, box), volume=None, rotation=R,
                        rot_tolerance=1e-8, vol_dims=(box, box, box // 2 + 1))


def _reference_backward(L, V, R, G, params, stream):
    """The existing entry point, with a caller-provided workspace."""
    dv = torch.zeros_like(V)
    dr = torch.empty_like(R)
    nbytes = int(L.tt_extract_backward_workspace_bytes(params))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=V.device)
    st = L.tt_extract_central_slices_rfft_3d_backward(
        ctypes.c_void_p(V.data_ptr()), ctypes.c_void_p(R.data_ptr()), ctypes.c_void_p(G.data_ptr()),
        ctypes.c_void_p(dv.data_ptr()), ctypes.c_void_p(dr.data_ptr()), ctypes.c_void_p(ws.data_ptr()),
        nbytes, params, stream)
    assert st == 0, L.tt_last_error()
    return dv, dr


def _noalloc_backward(L, V, R, G, params, stream, dv, dr):
    return L.tt_extract_central_slices_rfft_3d_backward_noalloc(
        ctypes.c_void_p(V.data_ptr()), ctypes.c_void_p(R.data_ptr()), ctypes.c_void_p(G.data_ptr()),
        ctypes.c_void_p(dv.data_ptr()) if dv is not None else None,
        ctypes.c_void_p(dr.data_ptr()) if dr is not None else None, params, stream)


def test_noalloc_backward_matches_workspace_backward():
    from teamtomo_b200 import _lib

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    box = 64
    V = torch.tensor(rfft_volume_np(blob_volume(box, seed=41)), device=dev)
    for call, (n_slices, seed) in enumerate(((96, 1), (40, 2))):  # two calls in a row
        R = torch.tensor(rotations(n_slices, seed=seed), device=dev)
        g = torch.Generator(device=dev).manual_seed(seed)
        G = torch.randn((n_slices, box, box // 2 + 1), dtype=torch.complex64, device=dev, generator=g)
        params = _params(n_slices, box, R)
        dv_ref, dr_ref = _reference_backward(L, V, R, G, params, stream)
        dv = torch.zeros_like(V)
        dr = torch.empty_like(R)
        st = _noalloc_backward(L, V, R, G, params, stream, dv, dr)
        assert st == 0, L.tt_last_error()
        torch.cuda.synchronize(dev)
        assert rel_l2(dv.cpu().numpy(), dv_ref.cpu().numpy()) < 1e-5, call
        assert rel_l2(dr.cpu().numpy(), dr_ref.cpu().numpy()) < 1e-5, call
        assert torch.isfinite(dr).all()


SCRATCH_BYTES = 4 << 20


def _limit(box):
    """Most slices one call takes with the rotation gradient: 24 bytes of
    partial sums per row of 8 x 32 pixel tiles of a slice."""
    rows = -(-box // 32)
    return SCRATCH_BYTES // (24 * rows)


def _inputs(box, n_slices, seed, dev):
    R = torch.tensor(rotations(n_slices, seed=seed), device=dev)
    g = torch.Generator(device=dev).manual_seed(seed)
    G = torch.randn((n_slices, box, box // 2 + 1), dtype=torch.complex64, device=dev, generator=g)
    return R, G


def test_noalloc_backward_without_rotation_gradient_and_at_the_limit():
    """The volume gradient alone (no scratch used), and a call of exactly the
    largest slice count the array holds, against the workspace entry point;
    device memory in use is the same before and after each call."""
    from teamtomo_b200 import _lib

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    for box, n_slices in ((64, 200), (8, _limit(8))):
        V = torch.tensor(rfft_volume_np(blob_volume(box, seed=43)), device=dev)
        R, G = _inputs(box, n_slices, 5, dev)
        params = _params(n_slices, box, R)
        dv_ref, dr_ref = _reference_backward(L, V, R, G, params, stream)
        for want_dr in (False, True):
            # two calls in a row; the second one's device memory is watched
            # (the first may load the kernel's code into device memory)
            for call in range(2):
                dv = torch.zeros_like(V)
                dr = torch.empty_like(R) if want_dr else None
                torch.cuda.synchronize(dev)
                free_before = torch.cuda.mem_get_info(dev)[0]
                st = _noalloc_backward(L, V, R, G, params, stream, dv, dr)
                assert st == 0, L.tt_last_error()
                torch.cuda.synchronize(dev)
                if call == 1:
                    assert torch.cuda.mem_get_info(dev)[0] == free_before, (box, want_dr)
                assert rel_l2(dv.cpu().numpy(), dv_ref.cpu().numpy()) < 1e-5, (box, want_dr, call)
                if want_dr:
                    assert rel_l2(dr.cpu().numpy(), dr_ref.cpu().numpy()) < 1e-5, (box, call)


def test_noalloc_backward_from_the_bricked_copy():
    """The bricked volume copy (volume_layout 2) through the allocation-free
    entry point, against the workspace entry point on the plain volume."""
    from teamtomo_b200 import _lib
    from teamtomo_b200.torch_fourier_slice import _layout

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    box, n_slices = 48, 150
    V = torch.tensor(rfft_volume_np(blob_volume(box, seed=44)), device=dev)
    R, G = _inputs(box, n_slices, 6, dev)
    params = _params(n_slices, box, R)
    dv_ref, dr_ref = _reference_backward(L, V, R, G, params, stream)
    bricks = _layout.pack(V, params, _layout.BRICKS)
    pb = _layout.with_layout(params, _layout.BRICKS)
    dv = torch.zeros_like(V)
    dr = torch.empty_like(R)
    st = L.tt_extract_central_slices_rfft_3d_backward_noalloc(
        ctypes.c_void_p(bricks.data_ptr()), ctypes.c_void_p(R.data_ptr()), ctypes.c_void_p(G.data_ptr()),
        ctypes.c_void_p(dv.data_ptr()), ctypes.c_void_p(dr.data_ptr()), pb, stream)
    assert st == 0, L.tt_last_error()
    torch.cuda.synchronize(dev)
    assert rel_l2(dv.cpu().numpy(), dv_ref.cpu().numpy()) < 1e-5
    assert rel_l2(dr.cpu().numpy(), dr_ref.cpu().numpy()) < 1e-5


def test_noalloc_backward_rejects_oversized_calls():
    """One slice past the limit is refused before anything is launched.  The
    buffers are sized for the slice count asked for, so a regression of the
    check would give a wrong answer, never an out-of-bounds access."""
    from teamtomo_b200 import _lib

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    box = 32  # one row of tiles per slice: 174763 slices, 0.76 GB of gradient slices
    n_slices = _limit(box) + 1
    V = torch.zeros((box, box, box // 2 + 1), dtype=torch.complex64, device=dev)
    R = torch.tensor(rotations(n_slices, seed=3), device=dev)
    G = torch.zeros((n_slices, box, box // 2 + 1), dtype=torch.complex64, device=dev)
    params = _params(n_slices, box, R)
    dr = torch.empty_like(R)
    st = _noalloc_backward(L, V, R, G, params, stream, None, dr)
    assert st == _lib.TT_ERR_INVALID
    assert b"built-in array" in L.tt_last_error()
