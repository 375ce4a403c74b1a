"""Parity at the sizes of the benchmark configurations.

Each configuration runs at its full size on the GPU; the oracle checks sampled
slices / images where running all of them on the CPU would take too long, and
size-independent properties cover the rest: adjoint identities, linearity,
and bitwise invariance of the deterministic mode to how the work is split.
"""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu


def tt():
    import teamtomo_b200

    return teamtomo_b200


def cuda(a):
    return torch.as_tensor(np.asarray(a)).cuda()


def test_project_64cube_100_rotations(oracle):
    """project_3d_to_2d of a 64^3 Gaussian-blob volume at 100 rotations, pad 2."""
    vol = blob_volume(64, seed=1001)
    rot = rotations(100, seed=1001)
    out = tt().project_3d_to_2d(cuda(vol), cuda(rot))
    assert out.shape == (100, 64, 64)
    ref = oracle.project_3d_to_2d(vol, rot)
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("pad", [1.0, 2.0])
def test_backproject_10000_images_128(oracle, pad):
    """backproject_2d_to_3d of 10,000 128^2 images: linear in the images (same
    rotations, same weights) and equal to the oracle on a 300-image subset."""
    n, k = 128, 10_000
    g = torch.Generator(device="cuda").manual_seed(1002)
    X = torch.randn((k, n, n), device="cuda", generator=g)
    Y = torch.randn((k, n, n), device="cuda", generator=g)
    R = cuda(rotations(k, seed=1002)).float()
    bx = tt().backproject_2d_to_3d(X, R, pad_factor=pad)
    by = tt().backproject_2d_to_3d(Y, R, pad_factor=pad)
    bxy = tt().backproject_2d_to_3d(2.0 * X - 0.5 * Y, R, pad_factor=pad)
    assert rel_l2(bxy.cpu().numpy(), (2.0 * bx - 0.5 * by).cpu().numpy()) < 1e-5
    m = 300
    sub = tt().backproject_2d_to_3d(X[:m], R[:m], pad_factor=pad)
    ref = oracle.backproject_2d_to_3d(X[:m].cpu().numpy(), R[:m].cpu().numpy(), pad_factor=pad)
    assert rel_l2(sub.cpu().numpy(), ref) < 1e-5


def test_differentiation_256cube_4096_slices(oracle):
    """The headline configuration: 256^3, 4096 rotations.  Sampled slices and
    their gradients vs the oracle; the adjoint identity of the full extraction
    and of the full insertion."""
    n, k = 256, 4096
    vol = rfft_volume_np(blob_volume(n, seed=1003))
    R = cuda(rotations(k, seed=1003)).float()
    V = cuda(vol)
    S = tt().extract_central_slices_rfft_3d(V, (n, n, n), R)
    pick = np.random.default_rng(3).choice(k, 24, replace=False)
    ref = oracle.extract(vol, (n, n, n), R[pick].cpu().numpy())
    assert rel_l2(S[pick].cpu().numpy(), ref) < 1e-6
    G = torch.randn(S.shape, dtype=S.dtype, device="cuda", generator=torch.Generator(device="cuda").manual_seed(5))
    Vg = V.clone().requires_grad_(True)
    Rg = R.clone().requires_grad_(True)
    S2 = tt().extract_central_slices_rfft_3d(Vg, (n, n, n), Rg)
    (S2 * G.conj()).real.sum().backward()
    lhs = torch.sum(S.to(torch.complex128) * G.to(torch.complex128).conj()).real.item()
    rhs = torch.sum(Vg.grad.to(torch.complex128) * V.to(torch.complex128).conj()).real.item()
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    _, dr = oracle.extract_grad(vol, (n, n, n), R[pick].cpu().numpy(), G[pick].cpu().numpy(), want_dvol=False)
    assert rel_l2(Rg.grad[pick].cpu().numpy(), dr) < 1e-5
    # insertion of all 4096 slices: Re<H, insert(X)> = Re<insert_bwd(H), X>
    H = torch.randn(V.shape, dtype=V.dtype, device="cuda", generator=torch.Generator(device="cuda").manual_seed(6))
    Xg = G.clone().requires_grad_(True)
    vol_i, _ = tt().insert_central_slices_rfft_3d(Xg, (n, n, n), R)
    lhs = torch.sum(vol_i.detach().to(torch.complex128) * H.to(torch.complex128).conj()).real.item()
    (vol_i * H.conj()).real.sum().backward()
    rhs = torch.sum(G.to(torch.complex128) * Xg.grad.to(torch.complex128).conj()).real.item()
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    # the full d/dvolume and the full insertion (volume and weights) of all
    # 4096 slices against the oracle (OpenMP, a few seconds each)
    threads = os.cpu_count() or 1
    G_np, R_np = G.cpu().numpy(), R.cpu().numpy()
    ref_dv, _ = oracle.extract_grad(vol, (n, n, n), R_np, G_np, want_drot=False, nthreads=threads)
    assert rel_l2(Vg.grad.cpu().numpy(), ref_dv) < 1e-5
    w_i = tt().insert_central_slices_rfft_3d(G, (n, n, n), R)[1]
    rv, rw = oracle.insert(G_np, (n, n, n), R_np, nthreads=threads)
    assert rel_l2(vol_i.detach().cpu().numpy(), rv) < 1e-5
    assert rel_l2(w_i.cpu().numpy(), rw) < 1e-5
    assert np.array_equal(w_i.cpu().numpy() != 0, rw != 0)


def test_batched_uneven_ctf_configuration(oracle):
    """32 volumes with boxes from {64, 96, 128, 160, 200, 256}, 500-20,000
    rotations each, per-image CTF: every volume's slices equal the
    single-volume call bitwise; CTF-weighted slices of sampled images equal
    the oracle."""
    from teamtomo_b200 import batched as B

    rng = np.random.default_rng(1004)
    boxes = [int(b) for b in rng.choice([64, 96, 128, 160, 200, 256], size=32)]
    counts = [int(c) for c in rng.integers(500, 20_001, size=32)]
    vols = [cuda(rfft_volume_np(blob_volume(b, seed=2000 + i, n_blobs=6))) for i, b in enumerate(boxes)]
    rots = [cuda(rotations(c, seed=3000 + i)).float() for i, c in enumerate(counts)]
    ctfs = [B.ctf_params(rng.uniform(0.5, 3.0, c), device="cuda") for c in counts]
    plain = B.extract_central_slices_rfft_3d_batched(vols, rots)
    weighted = B.extract_central_slices_rfft_3d_batched(vols, rots, ctf=ctfs)
    for i in range(0, 32, 5):
        n = boxes[i]
        assert torch.equal(plain[i], tt().extract_central_slices_rfft_3d(vols[i], (n, n, n), rots[i]))
        j = int(rng.integers(counts[i]))
        ref = oracle.extract(vols[i].cpu().numpy(), (n, n, n), rots[i][j:j + 1].cpu().numpy())[0]
        ref = ref * oracle.ctf_2d(*ctfs[i][j].cpu().numpy(), image_shape=(n, n))
        assert rel_l2(weighted[i][j].cpu().numpy(), ref) < 1e-4


def test_full_scale_320cube_streamed_insertion():
    """320^3 volume, 40,000 streamed CTF-less images (a fifth of the
    configuration's 200,000): the deterministic insertion is bitwise the same
    for two different chunkings, and the float insertion agrees with it."""
    n, k = 320, 40_000
    g = torch.Generator().manual_seed(1005)
    imgs = torch.randn((k, n, n // 2 + 1), dtype=torch.complex64, generator=g).pin_memory()
    R = torch.as_tensor(rotations(k, seed=1005)).float().pin_memory()
    bound = float(torch.view_as_real(imgs).abs().max())
    S = tt().streaming
    out = []
    for chunk in (5_000, 7_919):
        acc = S.InsertionAccumulator((n, n, n), "cuda", deterministic=True, data_bound=bound, max_slices=k)
        for _, _, (x, r) in S.prefetch_to_device([imgs, R], chunk, "cuda"):
            acc.add(x, r)
        out.append(acc.finalize())
    assert torch.equal(out[0][0], out[1][0]) and torch.equal(out[0][1], out[1][1])
    accf = S.InsertionAccumulator((n, n, n), "cuda")
    for _, _, (x, r) in S.prefetch_to_device([imgs, R], 10_000, "cuda"):
        accf.add(x, r)
    vf, wf = accf.finalize()
    # float32 sums of 40,000 terms per low-frequency voxel: summation noise, within 1e-5
    assert rel_l2(vf.cpu().numpy(), out[0][0].cpu().numpy()) < 1e-5
    assert rel_l2(wf.cpu().numpy(), out[0][1].cpu().numpy()) < 1e-5


def test_full_scale_320cube_ctf_insertion_vs_oracle(oracle):
    """The full-scale configuration's CTF-weighted insertion (per-image
    defocus U(0.8, 2.5) um, 300 kV, Cs 2.7 mm, Ac 0.07, 1 A/px) at 320^3, on
    3,000 images, against the oracle: volume = insertion of ctf * image,
    weights = insertion of ctf^2."""
    from teamtomo_b200 import batched as B

    n, k = 320, 3_000
    rng = np.random.default_rng(1005)
    imgs = (rng.standard_normal((k, n, n // 2 + 1)) + 1j * rng.standard_normal((k, n, n // 2 + 1)))
    imgs = imgs.astype(np.complex64)
    rots = rotations(k, seed=1005).astype(np.float32)
    defocus = rng.uniform(0.8, 2.5, k)
    ctf = B.ctf_params(defocus, voltage_kv=300.0, spherical_aberration_mm=2.7, amplitude_contrast=0.07,
                       pixel_size_a=1.0, device="cuda")
    (vol, w), = B.insert_central_slices_rfft_3d_batched([cuda(imgs)], [cuda(rots)], ctf=[ctf])
    threads = os.cpu_count() or 1
    cc = ctf.cpu().numpy()
    rv = np.zeros((n, n, n // 2 + 1), np.complex128)
    rw = np.zeros((n, n, n // 2 + 1), np.float64)
    for a in range(0, k, 500):  # the insertion is linear: sum the chunks' volumes
        c = np.stack([oracle.ctf_2d(*cc[j], image_shape=(n, n)) for j in range(a, min(a + 500, k))])
        v1, _ = oracle.insert((imgs[a:a + 500] * c).astype(np.complex64), (n, n, n), rots[a:a + 500],
                              nthreads=threads)
        v2, _ = oracle.insert((c * c).astype(np.complex64), (n, n, n), rots[a:a + 500], nthreads=threads)
        rv += v1
        rw += v2.real
    assert rel_l2(vol.cpu().numpy(), rv) < 1e-5
    assert rel_l2(w.cpu().numpy(), rw) < 1e-5


def test_full_scale_320cube_100k_orientation_extraction(oracle):
    """The full-scale configuration's 100,000-orientation extraction with
    forward and backward at 320^3, in chunks of 10,000: sampled slices and
    their rotation gradients against the oracle, the volume gradient of the
    first 1,000 slices against the oracle, and the adjoint identity of the
    whole pass."""
    n, k, chunk = 320, 100_000, 10_000
    vol = rfft_volume_np(blob_volume(n, seed=1005))
    V = cuda(vol)
    R_all = cuda(rotations(k, seed=1006)).float()
    Vg = V.clone().requires_grad_(True)
    pick = np.sort(np.random.default_rng(7).choice(k, 16, replace=False))
    lhs = 0.0
    S_pick, G_pick, dR_pick = [], [], []
    for a in range(0, k, chunk):
        Rc = R_all[a:a + chunk].clone().requires_grad_(True)
        S = tt().extract_central_slices_rfft_3d(Vg, (n, n, n), Rc)
        G = torch.randn(S.shape, dtype=S.dtype, device="cuda",
                        generator=torch.Generator(device="cuda").manual_seed(a))
        (S * G.conj()).real.sum().backward()
        lhs += torch.sum(S.detach().to(torch.complex128) * G.to(torch.complex128).conj()).real.item()
        sel = [int(i) - a for i in pick if a <= i < a + chunk]
        S_pick.append(S.detach()[sel].cpu().numpy())
        G_pick.append(G[sel].cpu().numpy())
        dR_pick.append(Rc.grad[sel].cpu().numpy())
        del S, G
    rhs = torch.sum(Vg.grad.to(torch.complex128) * V.to(torch.complex128).conj()).real.item()
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    Rp = R_all[pick].cpu().numpy()
    threads = os.cpu_count() or 1
    assert rel_l2(np.concatenate(S_pick), oracle.extract(vol, (n, n, n), Rp, nthreads=threads)) < 1e-6
    _, dr = oracle.extract_grad(vol, (n, n, n), Rp, np.concatenate(G_pick), want_dvol=False, nthreads=threads)
    assert rel_l2(np.concatenate(dR_pick), dr) < 1e-5
    # volume gradient of the first 1,000 slices
    m = 1_000
    Vm = V.clone().requires_grad_(True)
    Sm = tt().extract_central_slices_rfft_3d(Vm, (n, n, n), R_all[:m])
    Gm = torch.randn(Sm.shape, dtype=Sm.dtype, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
    (Sm * Gm.conj()).real.sum().backward()
    ref_dv, _ = oracle.extract_grad(vol, (n, n, n), R_all[:m].cpu().numpy(), Gm.cpu().numpy(), want_drot=False,
                                    nthreads=threads)
    assert rel_l2(Vm.grad.cpu().numpy(), ref_dv) < 1e-5
