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


def test_noalloc_backward_rejects_oversized_calls():
    from teamtomo_b200 import _lib

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    box = 256
    V = torch.zeros((box, box, box // 2 + 1), dtype=torch.complex64, device=dev)
    R = torch.tensor(rotations(4, seed=3), device=dev)
    G = torch.zeros((4, box, box // 2 + 1), dtype=torch.complex64, device=dev)
    params = _params(4096, box, R)  # 4096 slices of 256^3 need ~12.7 MB of scratch
    dr = torch.empty_like(R)
    st = _noalloc_backward(L, V, R, G, params, stream, None, dr)
    assert st == _lib.TT_ERR_INVALID
    assert b"built-in array" in L.tt_last_error()
