"""Insertion cases beyond the golden vectors: the one-shot C entry point
(tt_insert_central_slices_rfft_3d, its own workspace and finalize; for
accumulators of 64 MB and more a 2 x 2 x 2-bricked accumulator) against the
accumulate + finalize form (plain accumulator) and the oracle, on odd boxes,
fftfreq_max, zyx matrices, axis-aligned and 180-degree-apart rotations, many
slices of a small box, and several calls into one accumulator.

Both forms add the same (data * w, w) corner terms with the reference's
float32 weights; only the summation order differs, so volumes and weights
agree within float32 rounding (rel-L2 <= 1e-5) and the weights' non-zero
pattern is identical.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import rel_l2, rotations

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def tt():
    import teamtomo_b200

    return teamtomo_b200


def _images(n, nrot, seed):
    rng = np.random.default_rng(seed)
    imgs = rng.standard_normal((nrot, n, n // 2 + 1)) + 1j * rng.standard_normal((nrot, n, n // 2 + 1))
    return imgs.astype(np.complex64)


def _one_shot(imgs, n, rots, fftfreq_max=None, zyx_matrices=False):
    """Through the C ABI's one-shot entry point."""
    import ctypes

    from teamtomo_b200 import _lib
    from teamtomo_b200.torch_fourier_slice._params import rfft_shape, slice_params

    L = _lib.load()
    img = torch.tensor(imgs, device="cuda")
    R = torch.tensor(rots, device="cuda")
    p = slice_params(n=R.shape[0], image_shape=(n, n, n), volume=None, rotation=R, fftfreq_max=fftfreq_max,
                     zyx_matrices=zyx_matrices, vol_dims=rfft_shape((n, n, n)))
    d, h, w = rfft_shape((n, n, n))
    vol = torch.empty((d, h, w), dtype=torch.complex64, device="cuda")
    wts = torch.empty((d, h, w), dtype=torch.float32, device="cuda")
    nbytes = int(L.tt_insert_workspace_bytes(0, p))
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.tt_insert_central_slices_rfft_3d(_lib.ptr(img), 0, _lib.ptr(R), _lib.ptr(vol), _lib.ptr(wts),
                                              _lib.ptr(ws), nbytes, p, st) == 0, L.tt_last_error()
    return vol.cpu().numpy(), wts.cpu().numpy()


def _two_stage(imgs, n, rots, fftfreq_max=None, zyx_matrices=False):
    from teamtomo_b200.torch_fourier_slice import slice_insertion as si

    acc = si.new_accumulator((n, n, n), False, torch.device("cuda"))
    si.insert_accumulate(torch.tensor(imgs, device="cuda"), torch.tensor(rots, device="cuda"), (n, n, n), acc[0],
                         fftfreq_max, zyx_matrices)
    v, w = si.insert_finalize(acc, False)
    return v[0].cpu().numpy(), w.cpu().numpy()


@pytest.mark.parametrize("n,nrot,kw", [
    (32, 1, {}), (32, 7, {}), (48, 200, {}), (64, 300, {}), (63, 120, {}),  # odd box
    (65, 90, dict(fftfreq_max=0.3)), (64, 150, dict(zyx_matrices=True)),
    (96, 64, dict(fftfreq_max=0.45)), (128, 256, {}),
    # accumulators of 64 MB and more: the one-shot splat uses the bricked layout
    (201, 60, {}), (256, 30, dict(zyx_matrices=True)),
])
def test_one_shot_matches_two_stage_and_oracle(oracle, n, nrot, kw):
    imgs = _images(n, nrot, seed=n + nrot)
    rots = rotations(nrot, seed=n * 7 + nrot)
    v1, w1 = _one_shot(imgs, n, rots, **kw)
    v2, w2 = _two_stage(imgs, n, rots, **kw)
    rv, rw = oracle.insert(imgs, (n, n, n), rots, nthreads=8, **kw)
    assert rel_l2(v1, v2) < RTOL and rel_l2(w1, w2) < RTOL
    assert rel_l2(v1, rv) < RTOL and rel_l2(w1, rw) < RTOL
    assert np.array_equal(w1 != 0, rw != 0) and np.array_equal(w2 != 0, rw != 0)


def test_axis_aligned_and_conjugate_pair_rotations(oracle):
    """Planes along the grid axes (whole rows of points on integer
    coordinates and on the x = 0 plane, where both redirect branches meet)
    and rotations 180 degrees apart."""
    from scipy.spatial.transform import Rotation

    from helpers import PAIRS

    n = 64
    eul = [e for pair in PAIRS for e in pair] + [[0, 90, 0], [90, 0, 0], [0, 0, 90], [90, 90, 90]]
    rots = Rotation.from_euler("ZYZ", np.array(eul, float), degrees=True).as_matrix().astype(np.float32)
    imgs = _images(n, rots.shape[0], seed=3)
    v1, w1 = _one_shot(imgs, n, rots)
    rv, rw = oracle.insert(imgs, (n, n, n), rots, nthreads=8)
    assert rel_l2(v1, rv) < RTOL and rel_l2(w1, rw) < RTOL
    assert np.array_equal(w1 != 0, rw != 0)


def test_many_slices_small_box(oracle):
    n, nrot = 24, 9000
    imgs = _images(n, nrot, seed=9)
    rots = rotations(nrot, seed=10)
    v1, w1 = _one_shot(imgs, n, rots)
    rv, rw = oracle.insert(imgs, (n, n, n), rots, nthreads=8)
    assert rel_l2(v1, rv) < RTOL and rel_l2(w1, rw) < RTOL
    assert np.array_equal(w1 != 0, rw != 0)


def test_accumulate_across_calls(oracle):
    """Two accumulate calls into one accumulator, then one finalize: the
    streaming form of the insertion."""
    from teamtomo_b200.torch_fourier_slice import slice_insertion as si

    n = 48
    imgs = _images(n, 300, seed=12)
    rots = rotations(300, seed=13)
    acc = si.new_accumulator((n, n, n), False, torch.device("cuda"))
    for a, b in ((0, 170), (170, 300)):
        si.insert_accumulate(torch.tensor(imgs[a:b], device="cuda"), torch.tensor(rots[a:b], device="cuda"),
                             (n, n, n), acc[0])
    v, w = si.insert_finalize(acc, False)
    rv, rw = oracle.insert(imgs, (n, n, n), rots, nthreads=8)
    assert rel_l2(v[0].cpu().numpy(), rv) < RTOL and rel_l2(w.cpu().numpy(), rw) < RTOL
