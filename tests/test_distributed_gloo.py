"""Multi-process (gloo, CPU) tests of the data-parallel host logic.

The ranks run ``teamtomo_b200.distributed`` with its splat stages replaced by
the oracle on CPU tensors (the CUDA kernels themselves are covered by the GPU
tests); what is checked here is the sharding, the agreement on one
fixed-point scale, the collectives and their order:

* sharded deterministic insertion equals the single-process fixed-point
  insertion of all images bit for bit, on every rank, for 2 and 3 ranks
  (including a rank with no images);
* sharded float insertion equals the single-process insertion within float32
  noise;
* ``replicate_volume`` sums the volume gradient over the ranks.
"""

from __future__ import annotations

import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from helpers import rel_l2, rotations

N, K = 16, 13


def _data(k=K, n=N):
    rng = np.random.default_rng(11)
    imgs = (rng.standard_normal((k, n, n // 2 + 1)) + 1j * rng.standard_normal((k, n, n // 2 + 1))).astype(
        np.complex64)
    return imgs, rotations(k, seed=12).astype(np.float32)


def _install_oracle_stages():
    """Replace the CUDA splat stages of slice_insertion by the oracle (CPU)."""
    from oracle import oracle as O
    from teamtomo_b200.torch_fourier_slice import slice_insertion as I

    def fixed_absmax(*images, out=None):
        return torch.tensor([O.fixed_absmax_bits(*[t.numpy() for t in images])], dtype=torch.int32)

    def insert_fixed_accumulate(img, R, shape, acc, absmax, max_slices, fftfreq_max=None, zyx_matrices=False):
        if R.shape[0] == 0:
            return
        part = O.insert_fixed(img.numpy(), shape, R.numpy(), int(absmax.item()), max_slices,
                              fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices)
        acc[..., :3] += torch.from_numpy(part)

    def insert_fixed_finalize(acc, complex128, absmax, max_slices):
        vol, w = O.fixed_finalize(acc[0, ..., :3].numpy(), int(absmax.item()), max_slices, complex128)
        return torch.from_numpy(vol)[None], torch.from_numpy(w)

    def insert_float(img, shape, R, fftfreq_max=None, zyx_matrices=False, deterministic=False):
        d, h, w = shape
        if R.shape[0] == 0:
            return torch.zeros((d, h, w // 2 + 1), dtype=torch.complex64), torch.zeros((d, h, w // 2 + 1))
        vol, wts = O.insert(img.numpy(), shape, R.numpy(), fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices)
        return torch.from_numpy(vol), torch.from_numpy(wts)

    I.fixed_absmax = fixed_absmax
    I.insert_fixed_accumulate = insert_fixed_accumulate
    I.insert_fixed_finalize = insert_fixed_finalize
    I.insert_central_slices_rfft_3d = insert_float


def _worker(rank, world, port, outdir, k):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        _install_oracle_stages()
        from teamtomo_b200 import distributed as D

        imgs, rot = _data(k)
        s0, s1 = D.shard_bounds(k, rank, world)
        img_t, rot_t = torch.from_numpy(imgs[s0:s1]), torch.from_numpy(rot[s0:s1])
        vd, wd = D.insert_central_slices_rfft_3d(img_t, (N, N, N), rot_t, deterministic=True)
        vf, wf = D.insert_central_slices_rfft_3d(img_t, (N, N, N), rot_t, deterministic=False)
        v = torch.ones(5, requires_grad=True)
        (D.replicate_volume(v) * float(rank + 1)).sum().backward()
        torch.save(dict(vd=vd, wd=wd, vf=vf, wf=wf, vgrad=v.grad, n_local=s1 - s0),
                   os.path.join(outdir, f"r{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(world, tmp_path, k=K):
    out = tmp_path / f"w{world}"
    out.mkdir()
    mp.spawn(_worker, args=(world, _free_port(), str(out), k), nprocs=world, join=True)
    return [torch.load(out / f"r{r}.pt") for r in range(world)]


def test_shard_bounds_cover_everything():
    from teamtomo_b200.distributed import shard_bounds

    for n in (0, 1, 7, 4096):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(4, 2, 2)


def test_sharded_insertion_over_gloo(tmp_path, oracle):
    imgs, rot = _data()
    bits = oracle.fixed_absmax_bits(imgs)
    ref_vd, ref_wd = oracle.fixed_finalize(oracle.insert_fixed(imgs, (N, N, N), rot, bits, K), bits, K)
    ref_vf, ref_wf = oracle.insert(imgs, (N, N, N), rot)
    for world in (2, 3):
        res = _run(world, tmp_path)
        assert sum(r["n_local"] for r in res) == K
        for r in res:
            assert np.array_equal(r["vd"].numpy(), ref_vd) and np.array_equal(r["wd"].numpy(), ref_wd)
            assert rel_l2(r["vf"].numpy(), ref_vf) < 1e-6 and rel_l2(r["wf"].numpy(), ref_wf) < 1e-6
            assert torch.equal(r["vgrad"], torch.full((5,), float(sum(range(1, world + 1)))))


def test_rank_without_images(tmp_path, oracle):
    imgs, rot = _data(2)
    res = _run(3, tmp_path, k=2)
    assert [r["n_local"] for r in res] == [0, 1, 1]
    bits = oracle.fixed_absmax_bits(imgs)
    ref_vd, _ = oracle.fixed_finalize(oracle.insert_fixed(imgs, (N, N, N), rot, bits, 2), bits, 2)
    for r in res:
        assert np.array_equal(r["vd"].numpy(), ref_vd)
