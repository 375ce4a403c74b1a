"""Batched, CTF-weighted extraction / insertion over uneven volumes (one
persistent launch), its CUDA-graph plan and the tile-shape autotuner."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.as_tensor(np.asarray(a)).cuda()


def B():
    from teamtomo_b200 import batched

    return batched


def tt():
    import teamtomo_b200

    return teamtomo_b200


def _ctf_row(params):
    return B().ctf_params(*[float(x) for x in params], n=1, device="cuda")


def test_in_kernel_ctf_matches_reference_golden(golden, oracle):
    """Extracting a constant volume with the identity rotation returns the CTF
    itself on the image's rfft / fftshift grid (where the slice lies inside the
    volume: for odd boxes the last row maps past the edge and reads zero)."""
    for i in range(int(golden["ctf_cases"])):
        rf, fs = (bool(x) for x in golden[f"ctf_{i}_flags"])
        if not (rf and fs):
            continue  # the slice grid is always rfft + fftshifted
        h, w = (int(x) for x in golden[f"ctf_{i}_shape"])
        vol = torch.ones((h, h, w // 2 + 1), dtype=torch.complex64, device="cuda")
        out = B().extract_central_slices_rfft_3d_batched(
            [vol], [torch.eye(3, device="cuda")[None]], image_shapes=[(h, h, w)],
            ctf=[_ctf_row(golden[f"ctf_{i}_params"])])[0][0].cpu().numpy()
        flags, _ = oracle.slice_geometry(np.eye(3)[None], (h, h, w), (h, h, w // 2 + 1), 0)
        inside = (flags[0] & 4) != 0
        assert inside.mean() > 0.9
        ref = golden[f"ctf_{i}_out"]
        assert np.all(out.imag == 0) and np.all(out[~inside] == 0)
        np.testing.assert_allclose(out.real[inside], ref[inside], atol=1e-4)


def _uneven_batch(seed=0):
    rng = np.random.default_rng(seed)
    boxes = [64, 96, 40, 128, 65, 100]
    vols, rots, ctfs = [], [], []
    for i, n in enumerate(boxes):
        vols.append(cuda(rfft_volume_np(blob_volume(n, seed=n, n_blobs=8))))
        k = int(rng.integers(5, 40))
        rots.append(cuda(rotations(k, seed=100 + i)).float())
        ctfs.append(B().ctf_params(rng.uniform(0.5, 3.0, k), astigmatism_um=rng.uniform(0, 0.3, k),
                                   astigmatism_angle_deg=rng.uniform(0, 180, k), amplitude_contrast=0.07,
                                   pixel_size_a=1.0, device="cuda"))
    return boxes, vols, rots, ctfs


@pytest.mark.parametrize("tile_shape", [0, 1, 2])
def test_batched_extract_equals_single_volume_calls(tile_shape):
    boxes, vols, rots, _ = _uneven_batch()
    outs = B().extract_central_slices_rfft_3d_batched(vols, rots, tile_shape=tile_shape)
    for n, v, R, o in zip(boxes, vols, rots, outs):
        single = tt().extract_central_slices_rfft_3d(v, (n, n, n), R)
        assert torch.equal(o, single), n


def test_batched_extract_with_ctf(oracle):
    boxes, vols, rots, ctfs = _uneven_batch(1)
    outs = B().extract_central_slices_rfft_3d_batched(vols, rots, ctf=ctfs)
    for n, v, R, c, o in zip(boxes, vols, rots, ctfs, outs):
        plain = oracle.extract(v.cpu().numpy(), (n, n, n), R.cpu().numpy())
        cc = c.cpu().numpy()
        ref = np.stack([plain[j] * oracle.ctf_2d(*cc[j], image_shape=(n, n)) for j in range(len(cc))])
        assert rel_l2(o.cpu().numpy(), ref) < 1e-4, n


def test_batched_insert_equals_single_volume_calls():
    boxes, vols, rots, _ = _uneven_batch(2)
    imgs = [tt().extract_central_slices_rfft_3d(v, (n, n, n), R) for n, v, R in zip(boxes, vols, rots)]
    outs = B().insert_central_slices_rfft_3d_batched(imgs, rots)
    for n, im, R, (vol, w) in zip(boxes, imgs, rots, outs):
        v1, w1 = tt().insert_central_slices_rfft_3d(im, (n, n, n), R)
        assert rel_l2(vol.cpu().numpy(), v1.cpu().numpy()) < 1e-6
        assert rel_l2(w.cpu().numpy(), w1.cpu().numpy()) < 1e-6


def test_batched_insert_with_ctf(oracle):
    """CTF-weighted insertion = insertion of ctf*image; weights = insertion of ctf^2."""
    boxes, vols, rots, ctfs = _uneven_batch(3)
    imgs = [tt().extract_central_slices_rfft_3d(v, (n, n, n), R) for n, v, R in zip(boxes, vols, rots)]
    outs = B().insert_central_slices_rfft_3d_batched(imgs, rots, ctf=ctfs)
    for n, im, R, c, (vol, w) in zip(boxes, imgs, rots, ctfs, outs):
        cc = c.cpu().numpy()
        ctf = np.stack([oracle.ctf_2d(*cc[j], image_shape=(n, n)) for j in range(len(cc))])
        rv, _ = oracle.insert((im.cpu().numpy() * ctf).astype(np.complex64), (n, n, n), R.cpu().numpy())
        rw, _ = oracle.insert((ctf * ctf).astype(np.complex64), (n, n, n), R.cpu().numpy())
        assert rel_l2(vol.cpu().numpy(), rv) < 1e-4, n
        assert rel_l2(w.cpu().numpy(), rw.real) < 1e-4, n


def test_batched_insert_bricked_accumulators(oracle):
    """Volumes with 64 MB of accumulator and more go to bricked accumulators
    (lane-octet splat, bricked finalize), the small ones stay plain, in one
    launch: each against the one-shot single-volume insertion (also bricked
    from that size) and, with a CTF, against the oracle's insertions of
    ctf * image and ctf^2."""
    from teamtomo_b200 import _lib
    from teamtomo_b200.torch_fourier_slice._params import rfft_shape, slice_params

    L = _lib.load()
    boxes, counts = [216, 48, 230], [40, 30, 25]
    vols = [cuda(rfft_volume_np(blob_volume(b, seed=b, n_blobs=8))) for b in boxes]
    rots = [cuda(rotations(k, seed=b + k)).float() for b, k in zip(boxes, counts)]
    layouts = [L.tt_insert_accumulator_layout(ctypes.byref(slice_params(
        n=k, image_shape=(b, b, b), volume=None, rotation=R, vol_dims=rfft_shape((b, b, b)))))
        for b, k, R in zip(boxes, counts, rots)]
    assert layouts == [2, 0, 2]
    imgs = [tt().extract_central_slices_rfft_3d(v, (n, n, n), R) for n, v, R in zip(boxes, vols, rots)]
    for n, im, R, (vol, w) in zip(boxes, imgs, rots, B().insert_central_slices_rfft_3d_batched(imgs, rots)):
        v1, w1 = tt().insert_central_slices_rfft_3d(im, (n, n, n), R)
        assert rel_l2(vol.cpu().numpy(), v1.cpu().numpy()) < 1e-6, n
        assert rel_l2(w.cpu().numpy(), w1.cpu().numpy()) < 1e-6, n
        assert torch.equal(w != 0, w1 != 0), n
    ctfs = [B().ctf_params(np.linspace(0.8, 2.5, k), n=k, device="cuda") for k in counts]
    outs = B().insert_central_slices_rfft_3d_batched(imgs, rots, ctf=ctfs)
    for n, im, R, c, (vol, w) in zip(boxes, imgs, rots, ctfs, outs):
        cc = c.cpu().numpy()
        ctf = np.stack([oracle.ctf_2d(*cc[j], image_shape=(n, n)) for j in range(len(cc))])
        rv, _ = oracle.insert((im.cpu().numpy() * ctf).astype(np.complex64), (n, n, n), R.cpu().numpy(),
                              nthreads=8)
        rw, _ = oracle.insert((ctf * ctf).astype(np.complex64), (n, n, n), R.cpu().numpy(), nthreads=8)
        assert rel_l2(vol.cpu().numpy(), rv) < 1e-4, n
        assert rel_l2(w.cpu().numpy(), rw.real) < 1e-4, n


def test_bricked_finalize_without_weights():
    """tt_insert_finalize_bricked with weights NULL writes the same volume."""
    from teamtomo_b200 import _lib
    from teamtomo_b200.torch_fourier_slice._params import rfft_shape, slice_params

    L = _lib.load()
    n, k = 216, 12
    shape = (n, n, n)
    d, h, w = rfft_shape(shape)
    R = cuda(rotations(k, seed=5)).float()
    img = tt().extract_central_slices_rfft_3d(cuda(rfft_volume_np(blob_volume(n, seed=3, n_blobs=6))), shape, R)
    p = slice_params(n=k, image_shape=shape, volume=None, rotation=R, vol_dims=(d, h, w))
    p.volume_layout = 2
    acc = torch.zeros(int(L.tt_insert_bricked_accumulator_bytes(d, h, w)) // 4, dtype=torch.float32, device="cuda")
    ws = torch.empty(int(L.tt_batch_workspace_bytes()), dtype=torch.uint8, device="cuda")
    arr = (_lib.BatchVolume * 1)(_lib.BatchVolume(p, None, img.data_ptr(), acc.data_ptr(), R.data_ptr(), None))
    st = _lib.stream_of(torch.device("cuda"))
    assert L.tt_insert_central_slices_rfft_3d_batched(arr, 1, 0, _lib.ptr(ws), ws.numel(), st) == 0
    v1 = torch.empty((d, h, w), dtype=torch.complex64, device="cuda")
    v2 = torch.empty_like(v1)
    wt = torch.empty((d, h, w), dtype=torch.float32, device="cuda")
    assert L.tt_insert_finalize_bricked(_lib.ptr(acc), d, h, w, _lib.ptr(v1), _lib.ptr(wt), st) == 0
    assert L.tt_insert_finalize_bricked(_lib.ptr(acc), d, h, w, _lib.ptr(v2), None, st) == 0
    assert torch.equal(v1, v2)
    v0, w0 = tt().insert_central_slices_rfft_3d(img, shape, R)
    assert rel_l2(v1.cpu().numpy(), v0.cpu().numpy()) < 1e-6 and rel_l2(wt.cpu().numpy(), w0.cpu().numpy()) < 1e-6


def test_batched_chunks_beyond_one_launch():
    """More volumes than one launch carries (96) are split into launches."""
    vols = [cuda(rfft_volume_np(blob_volume(8, seed=s, n_blobs=2))) for s in range(100)]
    rots = [cuda(rotations(2, seed=s)).float() for s in range(100)]
    outs = B().extract_central_slices_rfft_3d_batched(vols, rots)
    for v, R, o in zip(vols, rots, outs):
        assert torch.equal(o, tt().extract_central_slices_rfft_3d(v, (8, 8, 8), R))


def test_graph_plan_replays_like_eager():
    boxes, n_slices = [64, 96, 40], [12, 7, 20]
    plan = B().BatchedSlicePlan(boxes, n_slices, mode="extract", with_ctf=True)
    for i, (b, k) in enumerate(zip(boxes, n_slices)):
        plan.volumes[i].copy_(cuda(rfft_volume_np(blob_volume(b, seed=b, n_blobs=6))))
        plan.rotations[i].copy_(cuda(rotations(k, seed=i)).float())
        plan.ctf[i].copy_(B().ctf_params(np.linspace(1.0, 2.0, k), n=k, device="cuda"))
    outs = [o.clone() for o in plan.run()]
    eager = B().extract_central_slices_rfft_3d_batched(plan.volumes, plan.rotations, ctf=plan.ctf)
    for a, b in zip(outs, eager):
        assert torch.equal(a, b)
    plan.rotations[0].copy_(cuda(rotations(12, seed=99)).float())  # new inputs, same graph
    again = plan.run()[0]
    assert not torch.equal(again, outs[0])
    assert torch.equal(again, B().extract_central_slices_rfft_3d_batched(
        plan.volumes[:1], plan.rotations[:1], ctf=plan.ctf[:1])[0])


def test_graph_plan_insert():
    boxes, n_slices = [32, 48], [10, 6]
    plan = B().BatchedSlicePlan(boxes, n_slices, mode="insert", with_ctf=False)
    for i, (b, k) in enumerate(zip(boxes, n_slices)):
        plan.images[i].copy_(torch.randn((k, b, b // 2 + 1), dtype=torch.complex64, device="cuda"))
        plan.rotations[i].copy_(cuda(rotations(k, seed=i)).float())
    outs = [(v.clone(), w.clone()) for v, w in plan.run()]
    for (v, w), im, R, b in zip(outs, plan.images, plan.rotations, boxes):
        v1, w1 = tt().insert_central_slices_rfft_3d(im, (b, b, b), R)
        assert rel_l2(v.cpu().numpy(), v1.cpu().numpy()) < 1e-6
        assert rel_l2(w.cpu().numpy(), w1.cpu().numpy()) < 1e-6


def test_autotuner_caches_the_fastest_shape(tmp_path, monkeypatch):
    from teamtomo_b200 import autotune

    monkeypatch.setenv("TT_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(autotune, "_mem", None)
    times = autotune.tune("extract", 48, n_slices=32, repeats=2)
    # every tile shape with both volume layouts
    assert set(times) == {(t, lay) for t in (0, 1, 2) for lay in ("plain", "bricks")}
    assert all(t > 0 for t in times.values())
    best_ts, best_lay = min(times, key=times.get)
    dev = torch.device("cuda")
    assert autotune.cached_tile_shape("extract", 48, dev) == best_ts
    assert autotune.cached_layout("extract", 48, dev) == (2 if best_lay == "bricks" else 0)
    assert (tmp_path / "tune.json").exists()
    monkeypatch.setattr(autotune, "_mem", None)  # reload from disk
    assert autotune.cached_tile_shape("extract", 48, dev) == best_ts
    assert autotune.cached_tile_shape("insert", 48, dev) == autotune.DEFAULT_TILE_SHAPE
    assert autotune.cached_layout("insert", 48, dev) is None


def test_batched_extraction_from_bricked_copies_is_bitwise_plain():
    """The bricked copies give the same slices bit for bit, CTF included."""
    boxes, vols, rots, ctfs = _uneven_batch(4)
    plain = B().extract_central_slices_rfft_3d_batched(vols, rots, ctf=ctfs, volume_layout="plain")
    bricks = B().extract_central_slices_rfft_3d_batched(vols, rots, ctf=ctfs, volume_layout="bricks")
    for a, b in zip(plain, bricks):
        assert torch.equal(a, b)
    with pytest.raises(ValueError):
        B().extract_central_slices_rfft_3d_batched(vols, rots, volume_layout="xpairs")


@pytest.mark.parametrize("lanes", [1, 2, 4, 8])
def test_l2_reduction_probe_adds_every_reduction(lanes):
    """The probe's reductions all land in the buffer: the x components sum to
    the count (whole groups), the fourth components stay zero."""
    from teamtomo_b200 import _lib

    L = _lib.load()
    nbytes, count = 1 << 20, (1 << 18) + 5
    buf = torch.zeros(nbytes // 4, dtype=torch.float32, device="cuda")
    assert L.tt_probe_l2_reductions(_lib.ptr(buf), nbytes, count, lanes, 7, _lib.stream_of(buf.device)) == 0
    q = buf.view(-1, 4).double()
    assert q[:, 0].sum().item() == (count // lanes) * lanes
    assert torch.equal(q[:, 0], q[:, 1]) and torch.equal(q[:, 0], q[:, 2]) and q[:, 3].abs().sum().item() == 0
