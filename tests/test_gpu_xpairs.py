"""The x-paired volume layout (tt_pack_volume_xpairs, p->volume_xpairs).

The gathers read the same values in the same order from either layout, so
the extraction, the rotation gradient and the fused MSE are BIT-identical
between the plain and the x-paired volume; the float d/dvolume scatter does
not read the volume and is compared within float-atomic reordering noise.
The oracle pins the x-paired path at sizes the CPU finishes in seconds.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu


def _lib():
    from teamtomo_b200 import _lib

    return _lib


def _params(n, shape, vol, R, **kw):
    from teamtomo_b200.torch_fourier_slice._params import slice_params

    return slice_params(n=n, image_shape=shape, volume=vol, rotation=R, **kw)


def _pack(vol, p):
    from teamtomo_b200.torch_fourier_slice import _xpairs

    return _xpairs.pack(vol, p)


def _xp(p, flag=True):
    from teamtomo_b200.torch_fourier_slice import _xpairs

    return _xpairs.with_xpairs(p, flag)


def _extract(vol_arg, R, p, out_shape):
    L = _lib().load()
    out = torch.empty(out_shape, dtype=torch.complex64, device="cuda")
    _lib().check(L.tt_extract_central_slices_rfft_3d(_lib().ptr(vol_arg), _lib().ptr(R), _lib().ptr(out),
                                                     ctypes.byref(p), None), "extract")
    return out


@pytest.mark.parametrize("n", [32, 33, 64])
@pytest.mark.parametrize("unshifted", [False, True])
def test_pack_layout(n, unshifted):
    vol = torch.randn((n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    R = torch.eye(3, device="cuda")[None]
    p = _params(1, (n, n, n), vol, R, volume_unshifted=unshifted)
    L = _lib().load()
    assert L.tt_volume_xpairs_bytes(ctypes.byref(p)) == vol.numel() * 16
    xp = _pack(vol, p)
    re = torch.view_as_real(vol)
    assert torch.equal(xp[..., 0:2], re)
    assert torch.equal(xp[..., :-1, 2:4], re[..., 1:, :])
    assert torch.all(xp[..., -1, 2:4] == 0)


@pytest.mark.parametrize("n,img", [(64, 64), (63, 63), (48, 40)])
@pytest.mark.parametrize("kw", [dict(), dict(fftfreq_max=0.3), dict(zyx_matrices=True), dict(x_tolerance=1e-3)])
def test_extract_bitwise_equal_to_plain_layout(oracle, n, img, kw):
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=400 + n))).cuda()
    R = torch.as_tensor(rotations(40, seed=401 + n)).float().cuda()
    shape = (img, img, img)
    p = _params(40, shape, vol, R, **kw)
    plain = _extract(vol, R, p, (40, img, img // 2 + 1))
    paired = _extract(_pack(vol, p), R, _xp(p), (40, img, img // 2 + 1))
    assert torch.equal(plain, paired)
    ref = oracle.extract(vol.cpu().numpy(), shape, R.cpu().numpy(), **kw)
    assert rel_l2(paired.cpu().numpy(), ref) < 1e-5


def test_extract_unshifted_volume_bitwise(oracle):
    """The projection path reads the plain rfftn output (volume_unshifted):
    the x-paired copy keeps that (z, y) order."""
    n = 48
    shifted = rfft_volume_np(blob_volume(n, seed=410))
    plain_rfftn = np.fft.ifftshift(shifted, axes=(0, 1))
    R = torch.as_tensor(rotations(30, seed=411)).float().cuda()
    v_s = torch.as_tensor(shifted).cuda()
    v_u = torch.as_tensor(np.ascontiguousarray(plain_rfftn)).cuda()
    p_s = _params(30, (n, n, n), v_s, R)
    p_u = _params(30, (n, n, n), v_u, R, volume_unshifted=True)
    a = _extract(v_s, R, p_s, (30, n, n // 2 + 1))
    b = _extract(_pack(v_u, p_u), R, _xp(p_u), (30, n, n // 2 + 1))
    assert torch.equal(a, b)


@pytest.mark.parametrize("n", [64, 63])
def test_backward_rotation_gradient_bitwise(n):
    """d/drotation is reduced in a fixed order: bitwise equal between layouts;
    d/dvolume (no volume read) equal within float-atomic reordering."""
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=420 + n))).cuda()
    R = torch.as_tensor(rotations(64, seed=421 + n)).float().cuda()
    G = torch.randn((64, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(7))
    from teamtomo_b200.torch_fourier_slice.slice_extraction import extract_backward

    p = _params(64, (n, n, n), vol, R)
    dv0, dr0 = extract_backward(vol, R, G, p)
    dv1, dr1 = extract_backward(vol, R, G, p, xpairs=_pack(vol, p))
    assert torch.equal(dr0, dr1)
    assert rel_l2(dv1.cpu().numpy(), dv0.cpu().numpy()) < 1e-6
    # deterministic volume gradient: bitwise
    pd = _params(64, (n, n, n), vol, R, deterministic=True)
    dv0, _ = extract_backward(vol, R, G, pd)
    dv1, _ = extract_backward(vol, R, G, pd, xpairs=_pack(vol, pd))
    assert torch.equal(dv0, dv1)


def test_autograd_path_selects_xpairs(monkeypatch, oracle):
    """Through the drop-in API: forced on and off give the same slices
    bitwise and the same rotation gradient bitwise; the oracle agrees."""
    import teamtomo_b200 as tt

    n = 48
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=430))).cuda()
    Rn = rotations(24, seed=431)
    G = torch.randn((24, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(9))
    res = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("TT_VOLUME_XPAIRS", mode)
        R = torch.as_tensor(Rn).float().cuda().requires_grad_(True)
        S = tt.extract_central_slices_rfft_3d(vol, (n, n, n), R)
        (S * G.conj()).real.sum().backward()
        res[mode] = (S.detach(), R.grad.detach())
    assert torch.equal(res["0"][0], res["1"][0])
    assert torch.equal(res["0"][1], res["1"][1])
    _, dr = oracle.extract_grad(vol.cpu().numpy(), (n, n, n), Rn.astype(np.float32), G.cpu().numpy(),
                                want_dvol=False)
    assert rel_l2(res["1"][1].cpu().numpy(), dr) < 1e-5


def test_fused_mse_bitwise(monkeypatch):
    import teamtomo_b200 as tt

    n = 64
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=440))).cuda()
    Rn = rotations(32, seed=441)
    T = torch.randn((32, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(11))
    res = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("TT_VOLUME_XPAIRS", mode)
        R = torch.as_tensor(Rn).float().cuda().requires_grad_(True)
        V = vol.clone().requires_grad_(True)
        loss = tt.losses.central_slice_mse(V, (n, n, n), R, T)
        loss.backward()
        res[mode] = (loss.detach(), R.grad.detach(), V.grad.detach())
    assert torch.equal(res["0"][0], res["1"][0])
    assert torch.equal(res["0"][1], res["1"][1])
    assert rel_l2(res["1"][2].cpu().numpy(), res["0"][2].cpu().numpy()) < 1e-6


def test_noalloc_backward_accepts_xpairs():
    n = 40
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=450))).cuda()
    R = torch.as_tensor(rotations(16, seed=451)).float().cuda()
    G = torch.randn((16, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(13))
    p = _params(16, (n, n, n), vol, R)
    L = _lib().load()
    out = []
    for v, q in ((vol, p), (_pack(vol, p), _xp(p))):
        dr = torch.empty_like(R)
        _lib().check(L.tt_extract_central_slices_rfft_3d_backward_noalloc(
            _lib().ptr(v), _lib().ptr(R), _lib().ptr(G), None, _lib().ptr(dr), ctypes.byref(q), None), "noalloc")
        out.append(dr)
    assert torch.equal(out[0], out[1])


def test_full_size_headline_bitwise():
    """256^3 volume, 1024 rotations: forward slices bitwise equal between the
    layouts (the headline workload's path), rotation gradient too."""
    n = 256
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=460))).cuda()
    R = torch.as_tensor(rotations(1024, seed=461)).float().cuda()
    p = _params(1024, (n, n, n), vol, R)
    xp = _pack(vol, p)
    a = _extract(vol, R, p, (1024, n, n // 2 + 1))
    b = _extract(xp, R, _xp(p), (1024, n, n // 2 + 1))
    assert torch.equal(a, b)
    from teamtomo_b200.torch_fourier_slice.slice_extraction import extract_backward

    G = torch.randn(a.shape, dtype=a.dtype, device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    _, dr0 = extract_backward(vol, R, G, p, want_volume=False)
    _, dr1 = extract_backward(vol, R, G, p, want_volume=False, xpairs=xp)
    assert torch.equal(dr0, dr1)


def _auto_run(monkeypatch, n, k, seed):
    """Forward + backward (d/drotation) through the drop-in API under the auto
    policy and with the plain volume; returns (results, number of packs)."""
    import teamtomo_b200 as tt
    from teamtomo_b200.torch_fourier_slice import _xpairs

    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=seed))).cuda()
    Rn = rotations(k, seed=seed + 1)
    G = torch.randn((k, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(seed + 2))
    packs = []
    real_pack = _xpairs.pack
    monkeypatch.setattr(_xpairs, "pack", lambda v, p: packs.append(1) or real_pack(v, p))
    res = {}
    for mode in ("auto", "0"):
        monkeypatch.setenv("TT_VOLUME_XPAIRS", mode)
        R = torch.as_tensor(Rn).float().cuda().requires_grad_(True)
        S = tt.extract_central_slices_rfft_3d(vol, (n, n, n), R)
        (S * G.conj()).real.sum().backward()
        res[mode] = (S.detach(), R.grad.detach())
    return vol, res, len(packs)


def test_auto_policy_shares_the_copy_with_the_backward(monkeypatch):
    """192^3 x 400 slices: the forward gathers from an x-paired copy (57 MB)
    and the backward reuses it (one pack); results equal the plain path
    bitwise."""
    from teamtomo_b200.torch_fourier_slice import _xpairs

    n, k = 192, 400
    vol, res, packs = _auto_run(monkeypatch, n, k, 470)
    npix = k * n * (n // 2 + 1)
    monkeypatch.setenv("TT_VOLUME_XPAIRS", "auto")
    assert _xpairs.use_xpairs(npix, vol)
    assert packs == 1
    assert torch.equal(res["auto"][0], res["0"][0]) and torch.equal(res["auto"][1], res["0"][1])


@pytest.mark.parametrize("n,k", [(256, 520), (320, 700)])
def test_auto_policy_plain_volume_for_large_boxes(monkeypatch, n, k):
    """At least two pixels per voxel, but a copy larger than half the L2 (135 MB
    at 256^3, 264 MB at 320^3): forward and backward read the plain volume; the
    results equal the forced plain path bitwise."""
    from teamtomo_b200.torch_fourier_slice import _xpairs

    vol, res, packs = _auto_run(monkeypatch, n, k, 480 + n)
    npix = k * n * (n // 2 + 1)
    monkeypatch.setenv("TT_VOLUME_XPAIRS", "auto")
    assert not _xpairs.use_xpairs(npix, vol)
    assert packs == 0
    assert torch.equal(res["auto"][0], res["0"][0]) and torch.equal(res["auto"][1], res["0"][1])
