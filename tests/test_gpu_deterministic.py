"""Deterministic (64-bit fixed-point) insertion and volume gradient on the GPU.

* the fixed-point accumulator equals the oracle's integer sums bit for bit, and
  the finalized volume / weights equal the oracle's conversion bit for bit;
* the outputs are identical across runs, slice orders and splits into calls;
* they agree with the float path and the reference-pinned float oracle within
  float32 summation noise (rel-L2 1e-6).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.as_tensor(np.asarray(a)).cuda()


def tt():
    import teamtomo_b200

    return teamtomo_b200


def ins():
    from teamtomo_b200.torch_fourier_slice import slice_insertion

    return slice_insertion


def _images(n, k, seed, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((k, n, n // 2 + 1)) + 1j * rng.standard_normal((k, n, n // 2 + 1))).astype(dtype)


CASES = [
    dict(n=32, k=40, dtype=np.complex64, fmax=None, zyx=False),
    dict(n=33, k=25, dtype=np.complex64, fmax=None, zyx=False),
    dict(n=32, k=30, dtype=np.complex64, fmax=0.3, zyx=True),
    dict(n=24, k=20, dtype=np.complex128, fmax=None, zyx=False),
]


@pytest.mark.parametrize("case", CASES,
                         ids=lambda c: f"n{c['n']}_{np.dtype(c['dtype']).name}_{c['fmax']}_{c['zyx']}")
def test_fixed_accumulator_bit_exact_with_oracle(oracle, case):
    n, k = case["n"], case["k"]
    imgs = _images(n, k, seed=n + k, dtype=case["dtype"])
    rot = rotations(k, seed=n)
    I = ins()
    img_d, rot_d = cuda(imgs), cuda(rot).float()
    absmax = I.fixed_absmax(img_d)
    bits = oracle.fixed_absmax_bits(imgs)
    assert (int(absmax.item()) & 0xFFFFFFFF) == bits
    acc = I.new_fixed_accumulator((n, n, n), "cuda")
    I.insert_fixed_accumulate(img_d, rot_d, (n, n, n), acc[0], absmax, k, case["fmax"], case["zyx"])
    ref = oracle.insert_fixed(imgs, (n, n, n), rot, bits, k, fftfreq_max=case["fmax"], zyx_matrices=case["zyx"])
    got = acc[0, ..., :3].cpu().numpy()
    assert np.array_equal(got, ref), f"{np.count_nonzero(got != ref)} integer sums differ"
    c128 = case["dtype"] == np.complex128
    vol, w = I.insert_fixed_finalize(acc, c128, absmax, k)
    rv, rw = oracle.fixed_finalize(ref, bits, k, complex128=c128)
    assert np.array_equal(vol[0].cpu().numpy(), rv) and np.array_equal(w.cpu().numpy(), rw)
    # the public one-shot call gives the same bits
    v2, w2 = tt().insert_central_slices_rfft_3d(img_d, (n, n, n), rot_d, fftfreq_max=case["fmax"],
                                                zyx_matrices=case["zyx"], deterministic=True)
    assert torch.equal(v2, vol[0]) and torch.equal(w2, w)
    # within float32 noise of the float oracle (the reference's semantics)
    fv, fw = oracle.insert(imgs, (n, n, n), rot, fftfreq_max=case["fmax"], zyx_matrices=case["zyx"])
    tol = 1e-12 if c128 else 1e-6
    assert rel_l2(vol[0].cpu().numpy(), fv) < tol and rel_l2(w.cpu().numpy(), fw) < tol


def test_deterministic_insert_invariant_to_order_and_split():
    n, k = 64, 300
    imgs = cuda(_images(n, k, seed=3))
    rot = cuda(rotations(k, seed=4)).float()
    v1, w1 = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), rot, deterministic=True)
    v2, w2 = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), rot, deterministic=True)
    perm = torch.randperm(k, generator=torch.Generator().manual_seed(0)).cuda()
    v3, w3 = tt().insert_central_slices_rfft_3d(imgs[perm].contiguous(), (n, n, n), rot[perm].contiguous(),
                                                deterministic=True)
    assert torch.equal(v1, v2) and torch.equal(w1, w2)
    assert torch.equal(v1, v3) and torch.equal(w1, w3)
    # split into three calls on one accumulator, same scale
    I = ins()
    absmax = I.fixed_absmax(imgs)
    acc = I.new_fixed_accumulator((n, n, n), "cuda")
    for s in (slice(0, 90), slice(90, 211), slice(211, k)):
        I.insert_fixed_accumulate(imgs[s].contiguous(), rot[s].contiguous(), (n, n, n), acc[0], absmax, k)
    v4, w4 = I.insert_fixed_finalize(acc, False, absmax, k)
    assert torch.equal(v1, v4[0]) and torch.equal(w1, w4)
    # the float path agrees within float32 noise
    vf, wf = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), rot, deterministic=False)
    assert rel_l2(v1.cpu().numpy(), vf.cpu().numpy()) < 1e-6
    assert rel_l2(w1.cpu().numpy(), wf.cpu().numpy()) < 1e-6


def test_use_deterministic_algorithms_selects_fixed_point():
    n, k = 32, 50
    imgs = cuda(_images(n, k, seed=9))
    rot = cuda(rotations(k, seed=9)).float()
    ref = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), rot, deterministic=True)
    before = torch.are_deterministic_algorithms_enabled()
    try:
        torch.use_deterministic_algorithms(True)
        got = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), rot)
    finally:
        torch.use_deterministic_algorithms(before)
    assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[1])


def test_deterministic_multichannel_insert(oracle):
    n, k, c = 32, 20, 3
    imgs = np.stack([_images(n, k, seed=s) for s in range(c)], axis=1)  # (k, c, h, w)
    rot = rotations(k, seed=1)
    vol, w = tt().insert_central_slices_rfft_3d_multichannel(cuda(imgs), (n, n, n), cuda(rot).float(),
                                                             deterministic=True)
    bits = oracle.fixed_absmax_bits(imgs)
    for ch in range(c):
        acc = oracle.insert_fixed(imgs[:, ch], (n, n, n), rot, bits, k)
        rv, rw = oracle.fixed_finalize(acc, bits, k)
        assert np.array_equal(vol[ch].cpu().numpy(), rv)
        assert np.array_equal(w.cpu().numpy(), rw)


def _loss(slices, G):
    # L = Re <G, S>  ->  dL/dS (PyTorch convention) = G
    return (slices * torch.conj(G)).real.sum()


def test_deterministic_volume_gradient(oracle):
    n, k = 48, 200
    vol = cuda(rfft_volume_np(blob_volume(n, seed=2, n_blobs=10)))
    rot = cuda(rotations(k, seed=6)).float()
    g = torch.randn((k, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(1))

    def grads(order, deterministic):
        v = vol.clone().requires_grad_(True)
        R = rot[order].contiguous().requires_grad_(True)
        s = tt().extract_central_slices_rfft_3d(v, (n, n, n), R, deterministic=deterministic)
        _loss(s, g[order]).backward()
        return v.grad, R.grad

    ident = torch.arange(k, device="cuda")
    perm = torch.randperm(k, generator=torch.Generator().manual_seed(2)).cuda()
    d1, r1 = grads(ident, True)
    d2, _ = grads(ident, True)
    d3, r3 = grads(perm, True)
    assert torch.equal(d1, d2) and torch.equal(d1, d3)
    assert torch.equal(r1[perm], r3)  # the rotation gradient is per slice and reduced in a fixed order
    dref, _ = oracle.extract_grad(vol.cpu().numpy(), (n, n, n), rot.cpu().numpy(), g.cpu().numpy(),
                                  want_drot=False)
    assert rel_l2(d1.cpu().numpy(), dref) < 1e-6
    df, rf = grads(ident, False)
    assert rel_l2(d1.cpu().numpy(), df.cpu().numpy()) < 1e-6
    assert rel_l2(r1.cpu().numpy(), rf.cpu().numpy()) < 1e-6
