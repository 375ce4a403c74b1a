"""Volume copies for the extraction gathers (p->volume_layout): the x-paired
copy (tt_pack_volume_xpairs) and the bricked copy (tt_pack_volume_bricks).

The gathers read the same values in the same order from every layout, so
the extraction, the rotation gradient and the fused MSE are BIT-identical
between the plain volume and either copy; the float d/dvolume scatter does
not read the volume and is compared within float-atomic reordering noise.
The oracle pins the copies' paths at sizes the CPU finishes in seconds.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu

XPAIRS, BRICKS = 1, 2
COPIES = pytest.mark.parametrize("layout", [XPAIRS, BRICKS], ids=["xpairs", "bricks"])


def _lib():
    from teamtomo_b200 import _lib

    return _lib


def _params(n, shape, vol, R, **kw):
    from teamtomo_b200.torch_fourier_slice._params import slice_params

    return slice_params(n=n, image_shape=shape, volume=vol, rotation=R, **kw)


def _pack(vol, p, layout):
    from teamtomo_b200.torch_fourier_slice import _layout

    return _layout.pack(vol, p, layout)


def _with(p, layout):
    from teamtomo_b200.torch_fourier_slice import _layout

    return _layout.with_layout(p, layout)


def _extract(vol_arg, R, p, out_shape):
    L = _lib().load()
    out = torch.empty(out_shape, dtype=torch.complex64, device="cuda")
    _lib().check(L.tt_extract_central_slices_rfft_3d(_lib().ptr(vol_arg), _lib().ptr(R), _lib().ptr(out),
                                                     ctypes.byref(p), None), "extract")
    return out


@pytest.mark.parametrize("n", [32, 33, 64])
@pytest.mark.parametrize("unshifted", [False, True])
def test_pack_xpairs(n, unshifted):
    vol = torch.randn((n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    R = torch.eye(3, device="cuda")[None]
    p = _params(1, (n, n, n), vol, R, volume_unshifted=unshifted)
    L = _lib().load()
    assert L.tt_volume_xpairs_bytes(ctypes.byref(p)) == vol.numel() * 16
    xp = _pack(vol, p, XPAIRS)
    re = torch.view_as_real(vol)
    assert torch.equal(xp[..., 0:2], re)
    assert torch.equal(xp[..., :-1, 2:4], re[..., 1:, :])
    assert torch.all(xp[..., -1, 2:4] == 0)


@pytest.mark.parametrize("d,h,w", [(32, 32, 17), (33, 33, 17), (64, 64, 33), (20, 18, 11)])
@pytest.mark.parametrize("unshifted", [False, True])
def test_pack_bricks(d, h, w, unshifted):
    """Voxel (z, y, x) (fftshifted order) at complex64 index
    ((z/2 * ceil(h/2) + y/2) * ceil(w/2) + x/2) * 8 + (z%2)*4 + (y%2)*2 + x%2,
    zeros in the slots past an odd dimension."""
    vol = torch.randn((d, h, w), dtype=torch.complex64, device="cuda")
    R = torch.eye(3, device="cuda")[None]
    p = _params(1, (d, h, 2 * (w - 1)), vol, R, volume_unshifted=unshifted)
    L = _lib().load()
    bd, bh, bw = (d + 1) // 2, (h + 1) // 2, (w + 1) // 2
    assert L.tt_volume_bricks_bytes(ctypes.byref(p)) == bd * bh * bw * 64
    b = _pack(vol, p, BRICKS).cpu().numpy().reshape(bd, bh, bw, 2, 2, 2)
    src = vol.cpu().numpy()
    if unshifted:  # the copy is always in fftshifted (z, y) order
        src = np.fft.fftshift(src, axes=(0, 1))
    ref = np.zeros((2 * bd, 2 * bh, 2 * bw), dtype=np.complex64)
    ref[:d, :h, :w] = src
    ref = ref.reshape(bd, 2, bh, 2, bw, 2).transpose(0, 2, 4, 1, 3, 5)
    assert np.array_equal(b, ref)


@COPIES
@pytest.mark.parametrize("n,img", [(64, 64), (63, 63), (48, 40)])
@pytest.mark.parametrize("kw", [dict(), dict(fftfreq_max=0.3), dict(zyx_matrices=True), dict(x_tolerance=1e-3)])
def test_extract_bitwise_equal_to_plain_layout(oracle, layout, n, img, kw):
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=400 + n))).cuda()
    R = torch.as_tensor(rotations(40, seed=401 + n)).float().cuda()
    shape = (img, img, img)
    p = _params(40, shape, vol, R, **kw)
    plain = _extract(vol, R, p, (40, img, img // 2 + 1))
    copied = _extract(_pack(vol, p, layout), R, _with(p, layout), (40, img, img // 2 + 1))
    assert torch.equal(plain, copied)
    ref = oracle.extract(vol.cpu().numpy(), shape, R.cpu().numpy(), **kw)
    assert rel_l2(copied.cpu().numpy(), ref) < 1e-5


@COPIES
def test_extract_unshifted_volume_bitwise(layout):
    """The projection path reads the plain rfftn output (volume_unshifted):
    the copies read it in the same (z, y) order."""
    n = 48
    shifted = rfft_volume_np(blob_volume(n, seed=410))
    plain_rfftn = np.fft.ifftshift(shifted, axes=(0, 1))
    R = torch.as_tensor(rotations(30, seed=411)).float().cuda()
    v_s = torch.as_tensor(shifted).cuda()
    v_u = torch.as_tensor(np.ascontiguousarray(plain_rfftn)).cuda()
    p_s = _params(30, (n, n, n), v_s, R)
    p_u = _params(30, (n, n, n), v_u, R, volume_unshifted=True)
    a = _extract(v_s, R, p_s, (30, n, n // 2 + 1))
    b = _extract(_pack(v_u, p_u, layout), R, _with(p_u, layout), (30, n, n // 2 + 1))
    assert torch.equal(a, b)


@COPIES
@pytest.mark.parametrize("n", [64, 63])
def test_backward_rotation_gradient_bitwise(layout, n):
    """d/drotation is reduced in a fixed order: bitwise equal between layouts;
    d/dvolume (no volume read) equal within float-atomic reordering."""
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=420 + n))).cuda()
    R = torch.as_tensor(rotations(64, seed=421 + n)).float().cuda()
    G = torch.randn((64, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(7))
    from teamtomo_b200.torch_fourier_slice.slice_extraction import extract_backward

    p = _params(64, (n, n, n), vol, R)
    dv0, dr0 = extract_backward(vol, R, G, p)
    dv1, dr1 = extract_backward(vol, R, G, p, copy=_pack(vol, p, layout), layout=layout)
    assert torch.equal(dr0, dr1)
    assert rel_l2(dv1.cpu().numpy(), dv0.cpu().numpy()) < 1e-6
    # deterministic volume gradient: bitwise
    pd = _params(64, (n, n, n), vol, R, deterministic=True)
    dv0, _ = extract_backward(vol, R, G, pd)
    dv1, _ = extract_backward(vol, R, G, pd, copy=_pack(vol, pd, layout), layout=layout)
    assert torch.equal(dv0, dv1)


def test_autograd_path_layouts(monkeypatch, oracle):
    """Through the drop-in API: every forced layout gives the same slices
    bitwise and the same rotation gradient bitwise; the oracle agrees."""
    import teamtomo_b200 as tt

    n = 48
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=430))).cuda()
    Rn = rotations(24, seed=431)
    G = torch.randn((24, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(9))
    res = {}
    for mode in ("plain", "xpairs", "bricks"):
        monkeypatch.setenv("TT_VOLUME_LAYOUT", mode)
        R = torch.as_tensor(Rn).float().cuda().requires_grad_(True)
        S = tt.extract_central_slices_rfft_3d(vol, (n, n, n), R)
        (S * G.conj()).real.sum().backward()
        res[mode] = (S.detach(), R.grad.detach())
    for mode in ("xpairs", "bricks"):
        assert torch.equal(res["plain"][0], res[mode][0])
        assert torch.equal(res["plain"][1], res[mode][1])
    _, dr = oracle.extract_grad(vol.cpu().numpy(), (n, n, n), Rn.astype(np.float32), G.cpu().numpy(),
                                want_dvol=False)
    assert rel_l2(res["bricks"][1].cpu().numpy(), dr) < 1e-5


def test_fused_mse_bitwise(monkeypatch):
    import teamtomo_b200 as tt

    n = 64
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=440))).cuda()
    Rn = rotations(32, seed=441)
    T = torch.randn((32, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(11))
    res = {}
    for mode in ("plain", "xpairs", "bricks"):
        monkeypatch.setenv("TT_VOLUME_LAYOUT", mode)
        R = torch.as_tensor(Rn).float().cuda().requires_grad_(True)
        V = vol.clone().requires_grad_(True)
        loss = tt.losses.central_slice_mse(V, (n, n, n), R, T)
        loss.backward()
        res[mode] = (loss.detach(), R.grad.detach(), V.grad.detach())
    for mode in ("xpairs", "bricks"):
        assert torch.equal(res["plain"][0], res[mode][0])
        assert torch.equal(res["plain"][1], res[mode][1])
        assert rel_l2(res[mode][2].cpu().numpy(), res["plain"][2].cpu().numpy()) < 1e-6


def test_noalloc_backward_accepts_copies():
    n = 40
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=450))).cuda()
    R = torch.as_tensor(rotations(16, seed=451)).float().cuda()
    G = torch.randn((16, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(13))
    p = _params(16, (n, n, n), vol, R)
    L = _lib().load()
    out = []
    for v, q in ((vol, p), (_pack(vol, p, XPAIRS), _with(p, XPAIRS)), (_pack(vol, p, BRICKS), _with(p, BRICKS))):
        dr = torch.empty_like(R)
        _lib().check(L.tt_extract_central_slices_rfft_3d_backward_noalloc(
            _lib().ptr(v), _lib().ptr(R), _lib().ptr(G), None, _lib().ptr(dr), ctypes.byref(q), None), "noalloc")
        out.append(dr)
    assert torch.equal(out[0], out[1]) and torch.equal(out[0], out[2])


@COPIES
def test_full_size_headline_bitwise(layout):
    """256^3 volume, 1024 rotations: forward slices bitwise equal between the
    layouts (the headline workload's path), rotation gradient too."""
    n = 256
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=460))).cuda()
    R = torch.as_tensor(rotations(1024, seed=461)).float().cuda()
    p = _params(1024, (n, n, n), vol, R)
    copy = _pack(vol, p, layout)
    a = _extract(vol, R, p, (1024, n, n // 2 + 1))
    b = _extract(copy, R, _with(p, layout), (1024, n, n // 2 + 1))
    assert torch.equal(a, b)
    from teamtomo_b200.torch_fourier_slice.slice_extraction import extract_backward

    G = torch.randn(a.shape, dtype=a.dtype, device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    _, dr0 = extract_backward(vol, R, G, p, want_volume=False)
    _, dr1 = extract_backward(vol, R, G, p, want_volume=False, copy=copy, layout=layout)
    assert torch.equal(dr0, dr1)


def _auto_run(monkeypatch, n, k, seed):
    """Forward + backward (d/drotation) through the drop-in API under the auto
    policy and with the plain volume; returns (volume, results, packs made)."""
    import teamtomo_b200 as tt
    from teamtomo_b200.torch_fourier_slice import _layout

    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=seed))).cuda()
    Rn = rotations(k, seed=seed + 1)
    G = torch.randn((k, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(seed + 2))
    packs = []
    real_pack = _layout.pack
    monkeypatch.setattr(_layout, "pack", lambda v, p, lay: (packs.append(lay) if lay else None) or real_pack(v, p, lay))
    res = {}
    for mode in ("auto", "plain"):
        monkeypatch.setenv("TT_VOLUME_LAYOUT", mode)
        R = torch.as_tensor(Rn).float().cuda().requires_grad_(True)
        S = tt.extract_central_slices_rfft_3d(vol, (n, n, n), R)
        (S * G.conj()).real.sum().backward()
        res[mode] = (S.detach(), R.grad.detach())
    return vol, res, packs


@pytest.mark.parametrize("n,k", [(128, 160), (256, 300)])
def test_auto_policy_shares_the_copy_with_the_backward(monkeypatch, n, k):
    """At least half a pixel per voxel: the forward gathers from the bricked copy
    and the backward reuses it (one pack); results equal the plain path
    bitwise."""
    from teamtomo_b200.torch_fourier_slice import _layout

    vol, res, packs = _auto_run(monkeypatch, n, k, 470 + n)
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "auto")
    assert _layout.choose(k * n * (n // 2 + 1), vol) == _layout.BRICKS
    assert packs == [_layout.BRICKS]
    assert torch.equal(res["auto"][0], res["plain"][0]) and torch.equal(res["auto"][1], res["plain"][1])


def test_auto_policy_plain_volume_for_few_slices(monkeypatch):
    """Fewer than half a pixel per voxel (256^3, 100 slices): no copy is made."""
    from teamtomo_b200.torch_fourier_slice import _layout

    n, k = 256, 100
    vol, res, packs = _auto_run(monkeypatch, n, k, 490)
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "auto")
    assert _layout.choose(k * n * (n // 2 + 1), vol) == _layout.PLAIN
    assert packs == []
    assert torch.equal(res["auto"][0], res["plain"][0]) and torch.equal(res["auto"][1], res["plain"][1])


@pytest.mark.parametrize("n,c", [(64, 3), (63, 2)])
def test_multichannel_bricks_bitwise(monkeypatch, oracle, n, c):
    """The multichannel extraction from the channels' bricked copies equals
    the plain volumes bitwise (slices, d/drotation; d/dvolume within
    float-atomic reordering), and the oracle per channel; the multichannel
    projection (an unshifted rfft source) too."""
    import teamtomo_b200 as tt

    vols = torch.stack([torch.as_tensor(rfft_volume_np(blob_volume(n, seed=500 + n + i))) for i in range(c)]).cuda()
    Rn = rotations(40, seed=501 + n)
    G = torch.randn((40, c, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(17))
    real = torch.as_tensor(np.stack([blob_volume(n, seed=520 + i) for i in range(c)])).float().cuda()
    res = {}
    for mode in ("plain", "bricks"):
        monkeypatch.setenv("TT_VOLUME_LAYOUT", mode)
        R = torch.as_tensor(Rn).float().cuda().requires_grad_(True)
        V = vols.clone().requires_grad_(True)
        S = tt.extract_central_slices_rfft_3d_multichannel(V, (n, n, n), R)
        (S * G.conj()).real.sum().backward()
        P = tt.project_3d_to_2d_multichannel(real, torch.as_tensor(Rn).float().cuda())
        res[mode] = (S.detach(), R.grad.detach(), V.grad.detach(), P)
    a, b = res["plain"], res["bricks"]
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]) and torch.equal(a[3], b[3])
    assert rel_l2(b[2].cpu().numpy(), a[2].cpu().numpy()) < 1e-6
    for ch in range(c):
        ref = oracle.extract(vols[ch].cpu().numpy(), (n, n, n), Rn.astype(np.float32))
        assert rel_l2(b[0][:, ch].cpu().numpy(), ref) < 1e-5


def test_multichannel_auto_policy_packs_once(monkeypatch):
    """At least half a pixel per voxel: one bricked pack of all channels in
    the forward, reused by the backward."""
    import teamtomo_b200 as tt
    from teamtomo_b200.torch_fourier_slice import _layout

    n, k, c = 64, 64, 2
    vols = torch.randn((c, n, n, n // 2 + 1), dtype=torch.complex64, device="cuda",
                       generator=torch.Generator(device="cuda").manual_seed(19))
    packs = []
    real_pack = _layout.pack_channels
    monkeypatch.setattr(_layout, "pack_channels",
                        lambda v, p, lay: (packs.append(lay) if lay else None) or real_pack(v, p, lay))
    monkeypatch.setenv("TT_VOLUME_LAYOUT", "auto")
    R = torch.as_tensor(rotations(k, seed=530)).float().cuda().requires_grad_(True)
    S = tt.extract_central_slices_rfft_3d_multichannel(vols, (n, n, n), R)
    S.real.sum().backward()
    assert packs == [_layout.BRICKS] and torch.isfinite(R.grad).all()
