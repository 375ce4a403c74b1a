"""Streaming host-resident slice stacks through the GPU.

Particle stacks are often larger than the GPU's memory, or simply live on the
host; the copies over PCIe then cost more than the slice kernels.  Two pieces
keep the GPU busy while the next chunk is in flight:

* ``prefetch_to_device`` copies fixed-size chunks of pinned host tensors on a
  side stream, ``depth`` chunks ahead of the consumer, into a ring of device
  buffers.  The consumer's stream waits for each chunk's copy; a buffer is
  refilled only after the work the consumer queued on it has run.
* ``InsertionAccumulator`` adds the insertions of any number of chunks into
  one accumulator and finalizes once (Friedel completion, split into volume
  and weights) — float accumulation, or the deterministic fixed-point mode
  with a data bound given up front.

All ordering is by CUDA events; the host waits only in the deterministic
``finalize``, to check the data bound.
"""

from __future__ import annotations

from typing import Iterator, Sequence

import torch

from . import _lib
from .torch_fourier_slice import slice_insertion as _ins
from .torch_fourier_slice._params import rfft_shape


def chunk_bounds(n: int, chunk: int) -> list[tuple[int, int]]:
    """[start, stop) of consecutive chunks of at most ``chunk`` items covering n."""
    if chunk < 1:
        raise ValueError(f"chunk must be >= 1, got {chunk}")
    return [(s, min(s + chunk, n)) for s in range(0, n, chunk)]


def prefetch_to_device(
    host_tensors: Sequence[torch.Tensor],
    chunk: int,
    device: torch.device | str | int,
    depth: int = 2,
) -> Iterator[tuple[int, int, list[torch.Tensor]]]:
    """Yield ``(start, stop, device_chunks)`` for consecutive chunks along dim 0.

    ``host_tensors`` share their leading size; pin them (``.pin_memory()``)
    for the copies to overlap with compute.  Each yielded device tensor is a
    view of a ring buffer that is overwritten ``depth`` chunks later: work on
    it must be queued before the next item is requested, and anything kept
    beyond that must be cloned."""
    if not host_tensors:
        return
    device = torch.device(device)
    n = host_tensors[0].shape[0]
    if any(t.shape[0] != n for t in host_tensors):
        raise ValueError("host tensors must share their leading size")
    if depth < 1:
        raise ValueError(f"depth must be >= 1, got {depth}")
    spans = chunk_bounds(n, chunk)
    if not spans:
        return
    compute = torch.cuda.current_stream(device)
    copy = torch.cuda.Stream(device)
    rows = min(chunk, n)
    bufs = [[torch.empty((rows, *t.shape[1:]), dtype=t.dtype, device=device) for t in host_tensors]
            for _ in range(min(depth, len(spans)))]
    for group in bufs:
        for b in group:
            b.record_stream(copy)
    ready = [torch.cuda.Event() for _ in bufs]
    free = [torch.cuda.Event() for _ in bufs]

    def issue(i: int) -> None:
        k = i % len(bufs)
        s, e = spans[i]
        with torch.cuda.stream(copy):
            if i >= len(bufs):
                copy.wait_event(free[k])  # the consumer's work on this buffer has run
            for dst, src in zip(bufs[k], host_tensors):
                dst[: e - s].copy_(src[s:e], non_blocking=True)
            ready[k].record(copy)

    for i in range(len(bufs)):
        issue(i)
    for i, (s, e) in enumerate(spans):
        k = i % len(bufs)
        compute.wait_event(ready[k])
        yield s, e, [b[: e - s] for b in bufs[k]]
        free[k].record(compute)
        if i + len(bufs) < len(spans):
            issue(i + len(bufs))


class InsertionAccumulator:
    """Insertion of many chunks of slices into one volume.

    ``add(images, rotation_matrices)`` splats a chunk ((..., h, w//2+1)
    complex slices, (..., 3, 3) rotations); ``finalize()`` returns
    ``(volume, weights)`` as ``insert_central_slices_rfft_3d`` of all chunks
    together would.  ``deterministic=True`` accumulates in 64-bit fixed point;
    its scale must be known before the first chunk: ``data_bound`` >= every
    |re|, |im| that will be added and ``max_slices`` >= the total slice count.
    The largest value actually added is tracked on the device, and
    ``finalize`` raises if it exceeded ``data_bound``.
    """

    def __init__(self, volume_shape, device, complex128: bool = False, fftfreq_max: float | None = None,
                 zyx_matrices: bool = False, deterministic: bool = False, data_bound: float | None = None,
                 max_slices: int | None = None):
        self.volume_shape = tuple(int(s) for s in volume_shape)
        self.device = torch.device(device)
        self.complex128 = bool(complex128)
        self.fftfreq_max = fftfreq_max
        self.zyx_matrices = zyx_matrices
        self.deterministic = bool(deterministic)
        self.count = 0
        if self.deterministic:
            if data_bound is None or max_slices is None:
                raise ValueError("deterministic accumulation needs data_bound and max_slices up front")
            bound = torch.tensor([abs(float(data_bound))], dtype=torch.float32)
            if float(bound) < abs(float(data_bound)):  # round the bound up to float32
                bound = torch.nextafter(bound, torch.tensor([float("inf")]))
            self.absmax = bound.view(torch.int32).to(self.device)
            self.max_slices = int(max_slices)
            self.acc = _ins.new_fixed_accumulator(self.volume_shape, self.device)
            self.seen = torch.zeros(1, dtype=torch.int32, device=self.device)
        else:
            self.acc = _ins.new_accumulator(self.volume_shape, self.complex128, self.device)

    def add(self, image_rfft: torch.Tensor, rotation_matrices: torch.Tensor) -> None:
        from .torch_fourier_slice._params import rotation_arg

        _lib.require_cuda(image_rfft)
        R, _ = rotation_arg(rotation_matrices, self.device)
        n = R.shape[0]
        if n == 0:
            return
        want = torch.complex128 if self.complex128 else torch.complex64
        if image_rfft.dtype != want:
            raise ValueError(f"accumulator takes {want} slices, got {image_rfft.dtype}")
        h, w = rfft_shape(self.volume_shape)[-2:]
        img = _lib.dense(image_rfft.reshape(n, h, w))
        if self.deterministic:
            if self.count + n > self.max_slices:
                raise ValueError(f"more than max_slices={self.max_slices} slices added")
            _ins.fixed_absmax(img, out=self.seen)
            _ins.insert_fixed_accumulate(img, R, self.volume_shape, self.acc[0], self.absmax, self.max_slices,
                                         self.fftfreq_max, self.zyx_matrices)
        else:
            _ins.insert_accumulate(img, R, self.volume_shape, self.acc[0], self.fftfreq_max, self.zyx_matrices)
        self.count += n

    def finalize(self) -> tuple[torch.Tensor, torch.Tensor]:
        if self.deterministic:
            # non-negative float32 values order like their bit patterns
            if int(self.seen.item()) > int(self.absmax.item()):
                raise ValueError("a slice value exceeded data_bound: the fixed-point sums may have overflowed")
            volume, weights = _ins.insert_fixed_finalize(self.acc, self.complex128, self.absmax, self.max_slices)
        else:
            volume, weights = _ins.insert_finalize(self.acc, self.complex128)
        return volume[0], weights
