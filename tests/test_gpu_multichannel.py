"""Fused multichannel kernels (one geometry pass per pixel for all channels)
against per-channel single-volume calls."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu


def tt():
    import teamtomo_b200

    return teamtomo_b200


def _vols(n, c):
    return torch.stack([torch.as_tensor(rfft_volume_np(blob_volume(n, seed=10 + i, n_blobs=6))) for i in range(c)]).cuda()


@pytest.mark.parametrize("n,k,c,kw", [(48, 30, 3, {}), (33, 20, 2, dict(fftfreq_max=0.3)),
                                      (32, 16, 4, dict(zyx_matrices=True))])
def test_multichannel_extraction_and_gradients(n, k, c, kw):
    vols = _vols(n, c)
    R = torch.as_tensor(rotations(k, seed=n)).float().cuda()
    G = torch.randn((k, c, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(1))
    Vm, Rm = vols.clone().requires_grad_(True), R.clone().requires_grad_(True)
    out = tt().extract_central_slices_rfft_3d_multichannel(Vm, (n, n, n), Rm, **kw)
    assert out.shape == (k, c, n, n // 2 + 1)
    (out * G.conj()).real.sum().backward()
    dR = torch.zeros_like(R)
    for ch in range(c):
        V1, R1 = vols[ch].clone().requires_grad_(True), R.clone().requires_grad_(True)
        s1 = tt().extract_central_slices_rfft_3d(V1, (n, n, n), R1, **kw)
        assert torch.equal(out[:, ch].detach(), s1.detach())
        (s1 * G[:, ch].conj()).real.sum().backward()
        assert rel_l2(Vm.grad[ch].cpu().numpy(), V1.grad.cpu().numpy()) < 1e-6
        dR += R1.grad
    assert rel_l2(Rm.grad.cpu().numpy(), dR.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("n,k,c", [(48, 40, 3), (33, 25, 2)])
def test_multichannel_insertion_and_gradient(n, k, c):
    g = torch.Generator(device="cuda").manual_seed(2)
    X = torch.randn((k, c, n, n // 2 + 1), dtype=torch.complex64, device="cuda", generator=g)
    Gv = torch.randn((c, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda", generator=g)
    R = torch.as_tensor(rotations(k, seed=n + 1)).float().cuda()
    Xm = X.clone().requires_grad_(True)
    vols, w = tt().insert_central_slices_rfft_3d_multichannel(Xm, (n, n, n), R)
    (vols * Gv.conj()).real.sum().backward()
    for ch in range(c):
        X1 = X[:, ch].clone().requires_grad_(True)
        v1, w1 = tt().insert_central_slices_rfft_3d(X1, (n, n, n), R)
        assert rel_l2(vols[ch].detach().cpu().numpy(), v1.detach().cpu().numpy()) < 1e-6
        assert rel_l2(w.cpu().numpy(), w1.cpu().numpy()) < 1e-6
        (v1 * Gv[ch].conj()).real.sum().backward()
        assert torch.equal(Xm.grad[:, ch], X1.grad)


def test_multichannel_project_and_backproject():
    n, k, c = 32, 12, 3
    vol = torch.stack([torch.as_tensor(blob_volume(n, seed=20 + i, n_blobs=5)) for i in range(c)]).cuda()
    R = torch.as_tensor(rotations(k, seed=4)).float().cuda()
    proj = tt().project_3d_to_2d_multichannel(vol, R)
    assert proj.shape == (k, c, n, n)
    for ch in range(c):
        assert rel_l2(proj[:, ch].cpu().numpy(), tt().project_3d_to_2d(vol[ch], R).cpu().numpy()) < 1e-6
    rec = tt().backproject_2d_to_3d_multichannel(proj, R)
    assert rec.shape == (c, n, n, n)
    for ch in range(c):
        assert rel_l2(rec[ch].cpu().numpy(), tt().backproject_2d_to_3d(proj[:, ch], R).cpu().numpy()) < 1e-6
