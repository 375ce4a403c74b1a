"""GPU gradients of the extraction (autograd Function -> fused backward kernel).

Checked against (a) the reference's own autograd (golden vectors),
(b) the CPU oracle, (c) float64 finite differences of a float64 forward
(relative error <= 1e-3 at N <= 16), and (d) at full size through the
size-independent adjoint identity Re<G, extract(V)> = Re<dV(G), V>.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def tt():
    import teamtomo_b200

    return teamtomo_b200


def cuda(a):
    return torch.as_tensor(np.asarray(a)).cuda()


def _loss(slices, G):
    # L = Re <G, S>  ->  dL/dS (PyTorch convention) = G
    return (slices * torch.conj(G)).real.sum()


def test_grad_rotation_matches_reference_autograd(golden):
    vol = cuda(golden["grad_drot_volume"])
    n = vol.shape[0]
    R = cuda(golden["grad_drot_rot"]).requires_grad_(True)  # float64 leaf, as the reference test
    s = tt().extract_central_slices_rfft_3d(vol, (n, n, n), R)
    _loss(s, cuda(golden["grad_drot_G"])).backward()
    assert R.grad.dtype == torch.float64
    assert rel_l2(R.grad.cpu().numpy(), golden["grad_drot_out"]) < RTOL


def test_grad_volume_matches_reference_autograd(golden):
    vol = cuda(golden["grad_dvol_volume"]).requires_grad_(True)
    n = vol.shape[0]
    s = tt().extract_central_slices_rfft_3d(vol, (n, n, n), cuda(golden["grad_dvol_rot"]))
    _loss(s, cuda(golden["grad_dvol_G"])).backward()
    assert rel_l2(vol.grad.cpu().numpy(), golden["grad_dvol_out"]) < RTOL


@pytest.mark.parametrize("n,nrot,kw", [(64, 48, {}), (33, 20, dict(fftfreq_max=0.3)),
                                       (48, 16, dict(zyx_matrices=True)),
                                       (256, 12, {})])
def test_gradients_match_oracle(oracle, n, nrot, kw):
    vol = rfft_volume_np(blob_volume(n, seed=n))
    rots = rotations(nrot, seed=n + 3).astype(np.float32)
    rng = np.random.default_rng(n)
    G = (rng.standard_normal((nrot, n, n // 2 + 1)) + 1j * rng.standard_normal((nrot, n, n // 2 + 1)))
    G = G.astype(np.complex64)
    V = cuda(vol).requires_grad_(True)
    R = cuda(rots).requires_grad_(True)
    _loss(tt().extract_central_slices_rfft_3d(V, (n, n, n), R, **kw), cuda(G)).backward()
    dv, dr = oracle.extract_grad(vol, (n, n, n), rots, G, **kw)
    assert R.grad.dtype == torch.float32
    assert rel_l2(V.grad.cpu().numpy(), dv) < RTOL
    assert rel_l2(R.grad.cpu().numpy(), dr) < RTOL


def _clean_rotations(count, seed, n):
    """Random rotations with no slice pixel near the x' = 0 redirect boundary."""
    out = []
    s = seed
    h = n
    k = np.arange(h)
    fy = np.fft.fftshift(np.where(k < (h + 1) // 2, k, k - h) / h)
    fx = np.arange(n // 2 + 1) / n
    while len(out) < count:
        r = rotations(1, seed=s)[0]
        s += 1
        m = r[::-1, ::-1]
        px = m[2, 1] * fy[:, None] + m[2, 2] * fx[None, :]
        px[(fy[:, None] == 0) & (fx[None, :] == 0)] = 1.0
        if np.abs(px).min() > 1e-3:
            out.append(r)
    return np.stack(out)


def test_grad_rotation_finite_differences(oracle):
    n = 16
    vol = rfft_volume_np(blob_volume(n, seed=16)).astype(np.complex128)
    rots = _clean_rotations(4, seed=100, n=n)
    rng = np.random.default_rng(1)
    G = rng.standard_normal((4, n, n // 2 + 1)) + 1j * rng.standard_normal((4, n, n // 2 + 1))
    R = cuda(rots).requires_grad_(True)
    _loss(tt().extract_central_slices_rfft_3d(cuda(vol.astype(np.complex64)), (n, n, n), R),
          cuda(G.astype(np.complex64))).backward()
    grad = R.grad.cpu().numpy()

    def L(r):
        return float(np.real(np.sum(np.conj(G) * oracle.extract_f64(vol, (n, n, n), r))))

    eps = 1e-6
    fd = np.zeros_like(rots)
    for b in range(4):
        for i in range(3):
            for j in range(3):
                rp, rm = rots.copy(), rots.copy()
                rp[b, i, j] += eps
                rm[b, i, j] -= eps
                fd[b, i, j] = (L(rp) - L(rm)) / (2 * eps)
    assert rel_l2(grad, fd) < 1e-3


def test_grad_volume_finite_differences(oracle):
    n = 12
    vol = rfft_volume_np(blob_volume(n, seed=12)).astype(np.complex128)
    rots = _clean_rotations(5, seed=200, n=n)
    rng = np.random.default_rng(2)
    G = rng.standard_normal((5, n, n // 2 + 1)) + 1j * rng.standard_normal((5, n, n // 2 + 1))
    V = cuda(vol.astype(np.complex64)).requires_grad_(True)
    _loss(tt().extract_central_slices_rfft_3d(V, (n, n, n), cuda(rots)), cuda(G.astype(np.complex64))).backward()
    dv = V.grad.cpu().numpy().astype(np.complex128)
    for t in range(3):
        delta = rng.standard_normal(vol.shape) + 1j * rng.standard_normal(vol.shape)
        eps = 1e-3

        def L(v):
            return float(np.real(np.sum(np.conj(G) * oracle.extract_f64(v, (n, n, n), rots))))

        fd = (L(vol + eps * delta) - L(vol - eps * delta)) / (2 * eps)
        an = float(np.real(np.sum(np.conj(dv) * delta)))  # Re <dV, delta>
        assert abs(an - fd) <= 1e-3 * abs(fd), (t, an, fd)


@pytest.mark.parametrize("n,nrot", [(256, 256), (512, 8)])
def test_adjoint_identity_full_size(n, nrot):
    """Re<G, extract(V)> == Re<dV(G), V> (dV = the insert-adjoint backward)."""
    g = torch.Generator(device="cuda").manual_seed(n)
    shape = (n, n, n // 2 + 1)
    V = torch.randn(shape, dtype=torch.complex64, device="cuda", generator=g)
    G = torch.randn((nrot, n, n // 2 + 1), dtype=torch.complex64, device="cuda", generator=g)
    R = cuda(rotations(nrot, seed=n)).float()
    Vg = V.clone().requires_grad_(True)
    S = tt().extract_central_slices_rfft_3d(Vg, (n, n, n), R)
    lhs = torch.sum(S.detach().to(torch.complex128) * torch.conj(G.to(torch.complex128))).real.item()
    _loss(S, G).backward()
    rhs = torch.sum(Vg.grad.to(torch.complex128) * torch.conj(V.to(torch.complex128))).real.item()
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_rotation_gradient_is_deterministic():
    n, nrot = 128, 64
    V = cuda(rfft_volume_np(blob_volume(n, seed=5)))
    G = torch.randn((nrot, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    grads = []
    for _ in range(2):
        R = cuda(rotations(nrot, seed=9)).float().requires_grad_(True)
        _loss(tt().extract_central_slices_rfft_3d(V, (n, n, n), R), G).backward()
        grads.append(R.grad.clone())
    assert torch.equal(grads[0], grads[1])


def test_gradient_through_lazy_conjugate():
    """A loss written with s.conj() hands the backward a lazy conjugate view;
    the gradients must equal those of the same loss written without it."""
    n, k = 32, 20
    vol = cuda(rfft_volume_np(blob_volume(n, seed=4)))
    rots = cuda(rotations(k, seed=5)).float()
    G = torch.randn((k, n, n // 2 + 1), dtype=torch.complex64, device="cuda")

    def grads(conj_form):
        V = vol.clone().requires_grad_(True)
        R = rots.clone().requires_grad_(True)
        s = tt().extract_central_slices_rfft_3d(V, (n, n, n), R)
        loss = (s.conj() * G).real.sum() if conj_form else _loss(s, G)
        loss.backward()
        return V.grad, R.grad

    (a, ra), (b, rb) = grads(True), grads(False)
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-6
    assert rel_l2(ra.cpu().numpy(), rb.cpu().numpy()) < 1e-6
    # a conjugated volume view is read as its values
    out = tt().extract_central_slices_rfft_3d(vol.conj(), (n, n, n), rots)
    ref = tt().extract_central_slices_rfft_3d(vol.conj().resolve_conj(), (n, n, n), rots)
    assert torch.equal(out, ref)


def test_grad_rotation_on_the_border_matches_reference_autograd(golden):
    vol = cuda(golden["grad_axes_volume"])
    n = vol.shape[0]
    R = cuda(golden["grad_axes_rot"]).requires_grad_(True)
    _loss(tt().extract_central_slices_rfft_3d(vol, (n, n, n), R), cuda(golden["grad_axes_G"])).backward()
    assert rel_l2(R.grad.cpu().numpy(), golden["grad_axes_out"]) < RTOL
    # the fused MSE kernel shares the rule
    T = torch.zeros((R.shape[0], n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    R2 = cuda(golden["grad_axes_rot"]).requires_grad_(True)
    R3 = cuda(golden["grad_axes_rot"]).requires_grad_(True)
    tt().losses.central_slice_mse(vol, (n, n, n), R2, T).backward()
    (tt().extract_central_slices_rfft_3d(vol, (n, n, n), R3) - T).abs().square().mean().backward()
    assert rel_l2(R2.grad.cpu().numpy(), R3.grad.cpu().numpy()) < RTOL
