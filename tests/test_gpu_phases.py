"""Insertion into accumulators larger than the L2, which the kernels fill in
z-phases (the tiles of each pass land in one z-slab of the accumulator).

Phasing only reorders the work, so a 320^3 insertion (a 264 MB float
accumulator: two phases on a B200) must equal the oracle, and the batched
CTF-weighted insertion must equal the single-volume one, as at sizes that
run in one phase.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import rel_l2, rotations

pytestmark = pytest.mark.gpu


def tt():
    import teamtomo_b200

    return teamtomo_b200


def test_large_accumulator_runs_in_phases():
    l2 = torch.cuda.get_device_properties(0).L2_cache_size
    assert 320 * 320 * 161 * 16 > 1.1 * l2, "the 320^3 accumulator should need more than one phase"


def test_phased_insertion_matches_oracle(oracle):
    n, k = 320, 48
    g = torch.Generator(device="cuda").manual_seed(11)
    imgs = torch.randn((k, n, n // 2 + 1), dtype=torch.complex64, device="cuda", generator=g)
    R = torch.as_tensor(rotations(k, seed=12)).float().cuda()
    vol, w = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), R)
    rv, rw = oracle.insert(imgs.cpu().numpy(), (n, n, n), R.cpu().numpy(), nthreads=8)
    assert rel_l2(vol.cpu().numpy(), rv) < 1e-5
    assert rel_l2(w.cpu().numpy(), rw) < 1e-5


def test_phased_batched_ctf_insertion_equals_single_volume():
    from teamtomo_b200 import batched as B

    n, k = 320, 256
    g = torch.Generator(device="cuda").manual_seed(13)
    imgs = torch.randn((k, n, n // 2 + 1), dtype=torch.complex64, device="cuda", generator=g)
    R = torch.as_tensor(rotations(k, seed=14)).float().cuda()
    ctf = B.ctf_params(np.random.default_rng(15).uniform(0.8, 2.5, k), device="cuda")
    (vb, wb), = B.insert_central_slices_rfft_3d_batched([imgs], [R], ctf=[ctf])
    (v1, w1), = B.insert_central_slices_rfft_3d_batched([imgs[:100]], [R[:100]], ctf=[ctf[:100]])
    (v2, w2), = B.insert_central_slices_rfft_3d_batched([imgs[100:]], [R[100:]], ctf=[ctf[100:]])
    assert rel_l2(vb.cpu().numpy(), (v1 + v2).cpu().numpy()) < 1e-6
    assert rel_l2(wb.cpu().numpy(), (w1 + w2).cpu().numpy()) < 1e-6
    # without a CTF the batched insertion equals the single-volume one
    (vp, wp), = B.insert_central_slices_rfft_3d_batched([imgs], [R])
    vs, ws = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), R)
    assert rel_l2(vp.cpu().numpy(), vs.cpu().numpy()) < 1e-6
    assert rel_l2(wp.cpu().numpy(), ws.cpu().numpy()) < 1e-6


def test_phased_complex128_insertion_matches_oracle(oracle):
    """complex128 images fill a 32-byte-slot accumulator (527 MB at 320^3: four
    z-phases); values and float64 weights equal the oracle's."""
    n, k = 320, 24
    g = torch.Generator(device="cuda").manual_seed(17)
    imgs = torch.randn((k, n, n // 2 + 1), dtype=torch.complex128, device="cuda", generator=g)
    R = torch.as_tensor(rotations(k, seed=18)).float().cuda()
    vol, w = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), R)
    assert vol.dtype == torch.complex128 and w.dtype == torch.float64
    rv, rw = oracle.insert(imgs.cpu().numpy(), (n, n, n), R.cpu().numpy(), nthreads=8)
    assert rel_l2(vol.cpu().numpy(), rv) < 1e-10
    assert rel_l2(w.cpu().numpy(), rw) < 1e-10
