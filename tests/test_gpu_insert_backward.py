"""Backward of the insertion w.r.t. the slices (the gather adjoint of the
splat and of the Friedel completion) against the reference's autograd, the
oracle, and the adjoint identity."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import rel_l2, rotations

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.as_tensor(np.asarray(a)).cuda()


def tt():
    import teamtomo_b200

    return teamtomo_b200


def _grad(imgs, rot, gvol, n, **kw):
    x = cuda(imgs).requires_grad_(True)
    vol, w = tt().insert_central_slices_rfft_3d(x, (n, n, n), cuda(rot), **kw)
    assert not w.requires_grad
    (vol * cuda(gvol).conj()).real.sum().backward()
    return x.grad.cpu().numpy()


def test_matches_reference_autograd_golden(golden):
    for name in golden["insgrad_cases"]:
        name = str(name)
        imgs = golden[f"insgrad_{name}_images"]
        n = imgs.shape[-2]
        fmax = float(golden[f"insgrad_{name}_fmax"])
        got = _grad(imgs, golden[f"insgrad_{name}_rot"], golden[f"insgrad_{name}_gvol"], n,
                    fftfreq_max=None if fmax < 0 else fmax, zyx_matrices=bool(int(golden[f"insgrad_{name}_zyx"])))
        ref = golden[f"insgrad_{name}_out"]
        tol = 1e-12 if imgs.dtype == np.complex128 else 1e-6
        assert rel_l2(got, ref) < tol, name
        assert np.array_equal(got == 0, ref == 0), name


@pytest.mark.parametrize("n,k,kw", [(64, 40, {}), (33, 30, {}), (48, 25, dict(fftfreq_max=0.3)),
                                    (40, 20, dict(zyx_matrices=True))])
def test_matches_oracle(oracle, n, k, kw):
    rng = np.random.default_rng(n + k)
    shape = (k, n, n // 2 + 1)
    imgs = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    gvol = (rng.standard_normal((n, n, n // 2 + 1)) + 1j * rng.standard_normal((n, n, n // 2 + 1))).astype(
        np.complex64)
    rot = rotations(k, seed=n)
    got = _grad(imgs, rot, gvol, n, **kw)
    ref = oracle.insert_grad_images(gvol, (n, n, n), rot, **kw)
    assert rel_l2(got, ref) < 1e-6
    assert np.array_equal(got == 0, ref == 0)


@pytest.mark.parametrize("n,k,kw", [(64, 200, {}), (33, 90, {}), (48, 150, dict(fftfreq_max=0.3)),
                                    (40, 120, dict(zyx_matrices=True))])
def test_bricked_gradient_copy_is_bitwise_plain(oracle, monkeypatch, n, k, kw):
    """From half a slice pixel per voxel the backward gathers from a bricked
    copy of the gradient volume: the same values and sums as from the plain
    volume, bit for bit (odd box included: the copy is padded to even dims)."""
    rng = np.random.default_rng(n * k)
    shape = (k, n, n // 2 + 1)
    imgs = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    gvol = (rng.standard_normal((n, n, n // 2 + 1)) + 1j * rng.standard_normal((n, n, n // 2 + 1))).astype(
        np.complex64)
    rot = rotations(k, seed=n + 1)
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "plain")
    plain = _grad(imgs, rot, gvol, n, **kw)
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "bricks")
    bricked = _grad(imgs, rot, gvol, n, **kw)
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "auto")
    auto = _grad(imgs, rot, gvol, n, **kw)
    assert np.array_equal(plain, bricked) and np.array_equal(plain, auto)
    ref = oracle.insert_grad_images(gvol, (n, n, n), rot, **kw)
    assert rel_l2(bricked, ref) < 1e-6
    assert np.array_equal(bricked == 0, ref == 0)


@pytest.mark.parametrize("n", [128, 65])
def test_adjoint_identity(n):
    """Re<G, insert(X)> = Re<insert_bwd(G), X>, in complex128."""
    k = 64
    g = torch.Generator(device="cuda").manual_seed(n)
    X = torch.randn((k, n, n // 2 + 1), dtype=torch.complex128, device="cuda", generator=g)
    G = torch.randn((n, n, n // 2 + 1), dtype=torch.complex128, device="cuda", generator=g)
    R = cuda(rotations(k, seed=7)).float()
    vol, _ = tt().insert_central_slices_rfft_3d(X, (n, n, n), R)
    from teamtomo_b200.torch_fourier_slice.slice_insertion import insert_backward

    gx = insert_backward(G, R, (n, n, n))
    lhs = torch.sum(vol * G.conj()).real.item()
    rhs = torch.sum(X * gx.conj()).real.item()
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_multichannel_and_deterministic_gradients():
    n, k, c = 32, 24, 3
    g = torch.Generator(device="cuda").manual_seed(3)
    X = torch.randn((k, c, n, n // 2 + 1), dtype=torch.complex64, device="cuda", generator=g)
    G = torch.randn((c, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda", generator=g)
    R = cuda(rotations(k, seed=9)).float()
    Xm = X.clone().requires_grad_(True)
    vols, _ = tt().insert_central_slices_rfft_3d_multichannel(Xm, (n, n, n), R)
    (vols * G.conj()).real.sum().backward()
    for ch in range(c):
        Xc = X[:, ch].clone().requires_grad_(True)
        v, _ = tt().insert_central_slices_rfft_3d(Xc, (n, n, n), R, deterministic=True)
        (v * G[ch].conj()).real.sum().backward()
        # the backward is a gather: identical in both modes
        assert torch.equal(Xc.grad, Xm.grad[:, ch])
