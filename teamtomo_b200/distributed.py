"""Data-parallel Fourier-slice operations over ``torch.distributed``.

One process per GPU; every rank holds the whole rfft volume (68 MB at a 256^3
box, 132 MB at 320^3) and a shard of the slices / images.

* Extraction and its rotation gradient are independent per slice: each rank
  extracts its own shard and no collective runs.
* The volume gradient of a replicated volume is the sum of the per-rank
  partial gradients: ``replicate_volume`` marks the volume so that its
  gradient is all-reduced (SUM) in the backward pass.
* Insertion: each rank splats its shard; one all-reduce sums the partial
  volume and weights, packed side by side.  The Friedel completion is
  linear, so it is applied before the sum.
* Deterministic insertion: the ranks first agree on one fixed-point scale
  (MAX all-reduce of the absmax word, SUM of the slice counts), accumulate
  64-bit integers, and all-reduce the three live integer words per voxel.  Integer sums are exact, so
  the result is bit-identical for any number of ranks and any sharding.

The collectives are the only data exchanged; nothing crosses NVLink in the
slice kernels themselves.  The helpers also run on CPU tensors over ``gloo``
(the host logic; the splat kernels need CUDA tensors).
"""

from __future__ import annotations

import torch
import torch.distributed as dist

from . import _lib
from .torch_fourier_slice import slice_insertion as _ins
from .torch_fourier_slice._params import resolve_deterministic, rotation_arg


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of rank's contiguous share of n items (sizes differ by at most 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return (n * rank) // world, (n * (rank + 1)) // world


def shard(tensor: torch.Tensor, group=None, dim: int = 0) -> torch.Tensor:
    """This rank's contiguous share of ``tensor`` along ``dim``."""
    start, stop = shard_bounds(tensor.shape[dim], dist.get_rank(group), dist.get_world_size(group))
    return tensor.narrow(dim, start, stop - start)


def _sum_count(n: int, device, group) -> int:
    t = torch.tensor([n], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return int(t.item())


def _all_reduce_sum(t: torch.Tensor, group) -> torch.Tensor:
    dist.all_reduce(torch.view_as_real(t) if t.is_complex() else t, op=dist.ReduceOp.SUM, group=group)
    return t


class _ReplicatedVolume(torch.autograd.Function):
    """Identity forward; the backward sums the gradient over the ranks."""

    @staticmethod
    def forward(ctx, volume, group):
        ctx.group = group
        return volume.view_as(volume)

    @staticmethod
    def backward(ctx, grad):
        return _all_reduce_sum(_lib.dense(grad).clone(), ctx.group), None


def replicate_volume(volume: torch.Tensor, group=None) -> torch.Tensor:
    """Use ``volume`` (identical on every rank) in a sharded computation whose
    volume gradient must be the sum over all ranks' shards."""
    return _ReplicatedVolume.apply(volume, group)


def all_reduce_volume_gradient(grad: torch.Tensor, group=None) -> torch.Tensor:
    """In-place SUM of per-rank partial volume gradients."""
    return _all_reduce_sum(grad, group)


def all_reduce_sum(t: torch.Tensor, group=None) -> torch.Tensor:
    """In-place SUM over the ranks of a (complex or real) partial volume."""
    return _all_reduce_sum(t, group)


def insert_central_slices_rfft_3d(
    image_rfft: torch.Tensor,
    volume_shape: tuple[int, int, int],
    rotation_matrices: torch.Tensor,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    deterministic: bool | None = None,
    group=None,
) -> tuple[torch.Tensor, torch.Tensor]:
    """Insertion of the images of ALL ranks: each rank passes its own shard
    (any size, possibly empty) and every rank receives the summed
    ``(volume, weights)``, as ``insert_central_slices_rfft_3d`` of the
    concatenated stacks would return them."""
    dev = image_rfft.device
    R, _ = rotation_arg(rotation_matrices, dev)
    n = R.shape[0]
    img = _lib.dense(image_rfft.reshape(n, *image_rfft.shape[-2:]))
    c128 = image_rfft.dtype == torch.complex128
    if not resolve_deterministic(deterministic):
        volume, weights = _ins.insert_central_slices_rfft_3d(img, volume_shape, R, fftfreq_max=fftfreq_max,
                                                             zyx_matrices=zyx_matrices, deterministic=False)
        # one collective for both: (re, im) of the volume and the weights side by side
        re_im = torch.view_as_real(volume).reshape(-1)
        flat = torch.cat([re_im, weights.reshape(-1).to(re_im.dtype)])
        dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
        re_im.copy_(flat[:re_im.numel()])
        weights.reshape(-1).copy_(flat[re_im.numel():])
        return volume, weights
    # one scale for all ranks: the largest |re|, |im| anywhere and the total slice count
    absmax = _ins.fixed_absmax(img)
    dist.all_reduce(absmax, op=dist.ReduceOp.MAX, group=group)
    total = max(_sum_count(n, dev, group), 1)
    acc = _ins.new_fixed_accumulator(volume_shape, dev)
    _ins.insert_fixed_accumulate(img, R, volume_shape, acc[0], absmax, total, fftfreq_max, zyx_matrices)
    # exact integer sum of the three live words per voxel (re, im, w), without
    # the slot's pad word: a quarter fewer bytes on the wire
    live = acc[..., :3].contiguous()
    dist.all_reduce(live, op=dist.ReduceOp.SUM, group=group)
    acc[..., :3] = live
    volume, weights = _ins.insert_fixed_finalize(acc, c128, absmax, total)
    return volume[0], weights
