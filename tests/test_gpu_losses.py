"""Fused extraction + MSE + backward against the unfused composition
(extract_central_slices_rfft_3d -> torch MSE -> autograd)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu


def tt():
    import teamtomo_b200

    return teamtomo_b200


def _case(n, k, seed):
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=seed, n_blobs=8))).cuda()
    R = torch.as_tensor(rotations(k, seed=seed)).float().cuda()
    g = torch.Generator(device="cuda").manual_seed(seed)
    with torch.no_grad():
        T = tt().extract_central_slices_rfft_3d(vol * 1.1, (n, n, n), R)
        T = T + 0.3 * T.abs().mean() * torch.randn(T.shape, dtype=T.dtype, device="cuda", generator=g)
    return vol, R, T


@pytest.mark.parametrize("n,k,kw", [(64, 50, {}), (33, 40, dict(fftfreq_max=0.3)),
                                    (48, 30, dict(zyx_matrices=True)), (256, 16, {})])
def test_fused_mse_equals_composition(n, k, kw):
    vol, R, T = _case(n, k, seed=n)
    V1, R1 = vol.clone().requires_grad_(True), R.clone().requires_grad_(True)
    ref = (tt().extract_central_slices_rfft_3d(V1, (n, n, n), R1, **kw) - T).abs().square().mean()
    ref.backward()
    V2, R2 = vol.clone().requires_grad_(True), R.clone().requires_grad_(True)
    loss = tt().losses.central_slice_mse(V2, (n, n, n), R2, T, **kw)
    (3.0 * loss).backward()  # the upstream gradient scales both gradients
    assert abs(loss.item() - ref.item()) <= 1e-6 * ref.item()
    assert rel_l2(V2.grad.cpu().numpy() / 3.0, V1.grad.cpu().numpy()) < 1e-6
    assert rel_l2(R2.grad.cpu().numpy() / 3.0, R1.grad.cpu().numpy()) < 1e-5


def test_fused_mse_partial_gradients_and_float64_rotations():
    n, k = 40, 24
    vol, R, T = _case(n, k, seed=5)
    Rd = R.double().requires_grad_(True)
    loss = tt().losses.central_slice_mse(vol, (n, n, n), Rd, T)  # volume without grad
    loss.backward()
    assert Rd.grad.dtype == torch.float64
    R1 = R.double().requires_grad_(True)
    (tt().extract_central_slices_rfft_3d(vol, (n, n, n), R1) - T).abs().square().mean().backward()
    assert rel_l2(Rd.grad.cpu().numpy(), R1.grad.cpu().numpy()) < 1e-5
    V = vol.clone().requires_grad_(True)
    tt().losses.central_slice_mse(V, (n, n, n), R, T).backward()  # rotations without grad
    assert V.grad is not None
    with torch.no_grad():
        l0 = tt().losses.central_slice_mse(vol, (n, n, n), R, T)
    assert abs(l0.item() - loss.item()) <= 1e-6 * loss.item()


def test_fused_mse_loss_is_deterministic():
    n, k = 64, 64
    vol, R, T = _case(n, k, seed=7)
    a = [tt().losses.central_slice_mse(vol, (n, n, n), R, T).item() for _ in range(3)]
    assert a[0] == a[1] == a[2]
