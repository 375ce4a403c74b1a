"""Batched, CTF-weighted central-slice extraction and insertion.

Many volumes of uneven box size, each with its own rotations and an optional
per-image CTF, run in ONE persistent kernel launch that takes slices from a
work queue (``csrc/batched.cu``).  The reference has no batched API: for each
volume these compute exactly what ``extract_central_slices_rfft_3d`` /
``insert_central_slices_rfft_3d`` compute, with the CTF of torch-ctf's
``calculate_ctf_2d`` (rfft, fftshifted grid of the image shape) applied in the
kernel:

* extraction returns ``ctf * slice``;
* insertion accumulates ``ctf * image`` and the interpolation weights times
  ``ctf**2`` (the usual CTF-weighted backprojection numerator/denominator).

``BatchedSlicePlan`` captures a fixed-shape batch into a CUDA graph for
repeated replay.  The tile shape of the launch is chosen per box size by the
autotuner in ``teamtomo_b200.autotune`` (cached; 8x32 when never tuned).
"""

from __future__ import annotations

import ctypes
import math
from typing import Sequence

import torch

from . import _lib
from .torch_fourier_slice._params import rfft_shape, rotation_arg, slice_params
from .torch_fourier_slice._layout import BRICKS as _BRICKS
from .torch_fourier_slice.slice_insertion import insert_finalize, new_accumulator

CTF_FIELDS = ("defocus_um", "astigmatism_um", "astigmatism_angle_deg", "voltage_kv",
              "spherical_aberration_mm", "amplitude_contrast", "phase_shift_deg", "pixel_size_a")


def ctf_params(defocus_um, astigmatism_um=0.0, astigmatism_angle_deg=0.0, voltage_kv=300.0,
               spherical_aberration_mm=2.7, amplitude_contrast=0.07, phase_shift_deg=0.0,
               pixel_size_a=1.0, n: int | None = None, device=None) -> torch.Tensor:
    """Per-image CTF parameter rows, shape (n, 8) float32, in the field order of
    ``tt_ctf_params`` (the scalar arguments of torch-ctf's calculate_ctf_2d).
    Each argument is a scalar or a length-n sequence/tensor."""
    vals = [defocus_um, astigmatism_um, astigmatism_angle_deg, voltage_kv, spherical_aberration_mm,
            amplitude_contrast, phase_shift_deg, pixel_size_a]
    cols = [torch.as_tensor(v, dtype=torch.float32).reshape(-1) for v in vals]
    m = max(c.numel() for c in cols) if n is None else n
    cols = [c.expand(m) if c.numel() == 1 else c for c in cols]
    for c in cols:
        if c.numel() != m:
            raise ValueError(f"CTF parameter of length {c.numel()}, expected {m}")
    out = torch.stack(cols, dim=-1).contiguous()
    return out.to(device) if device is not None else out


def _ws(device) -> torch.Tensor:
    return torch.empty(int(_lib.load().tt_batch_workspace_bytes()), dtype=torch.uint8, device=device)


def _tile_shape(kind: str, boxes: Sequence[int], device, tile_shape):
    if tile_shape is not None:
        return int(tile_shape)
    from . import autotune

    return autotune.cached_tile_shape(kind, max(boxes), device)


def _layout(boxes: Sequence[int], n_pixels: int, n_voxels: int, device, volume_layout):
    """Volume layout the batched extraction gathers from: ``volume_layout``
    ('plain' or 'bricks') when given, else the autotuner's choice for the
    largest box when it has one, else the single-volume policy (the bricked
    copies from half a slice pixel per voxel)."""
    from .torch_fourier_slice import _layout as lay

    if volume_layout is not None:
        if volume_layout not in ("plain", "bricks"):
            raise ValueError(f"volume_layout must be 'plain' or 'bricks', got {volume_layout!r}")
        return lay.BRICKS if volume_layout == "bricks" else lay.PLAIN
    from . import autotune

    tuned = autotune.cached_layout("extract", max(boxes), device)
    if tuned is not None:
        return tuned
    return lay.BRICKS if n_pixels >= lay.MIN_PIXELS_PER_VOXEL * n_voxels else lay.PLAIN


def _check_ctf(ctf, n, device):
    if ctf is None:
        return None
    ctf = torch.as_tensor(ctf, dtype=torch.float32).to(device).reshape(-1, 8).contiguous()
    if ctf.shape[0] != n:
        raise ValueError(f"{ctf.shape[0]} CTF rows for {n} slices")
    return ctf


def _batches(items, size=_lib.MAX_BATCH_VOLUMES):
    for i in range(0, len(items), size):
        yield items[i:i + size]


def _run(fn_name, entries, tile_shape, device, what):
    L = _lib.load()
    arr = (_lib.BatchVolume * len(entries))(*entries)
    ws = _ws(device)
    _lib.check(getattr(L, fn_name)(arr, len(entries), int(tile_shape), _lib.ptr(ws), ws.numel(),
                                   _lib.stream_of(device)), what)


def extract_central_slices_rfft_3d_batched(
    volumes: Sequence[torch.Tensor],
    rotation_matrices: Sequence[torch.Tensor],
    image_shapes: Sequence[tuple[int, int, int]] | None = None,
    ctf: Sequence[torch.Tensor | None] | None = None,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    x_tolerance: float = 1e-8,
    rot_tolerance: float | None = 1e-8,
    tile_shape: int | None = None,
    volume_layout: str | None = None,
) -> list[torch.Tensor]:
    """Extract slices from every volume in one launch.

    ``volumes[i]`` is an fftshifted rfft volume (d, d, d//2+1) complex64,
    ``rotation_matrices[i]`` (n_i, 3, 3), ``image_shapes[i]`` defaults to
    (d, d, d), ``ctf[i]`` is None or (n_i, 8) CTF rows (see ``ctf_params``).
    ``volume_layout`` ('plain' or 'bricks', default: autotuned or by the
    pixels-per-voxel policy) selects whether the gathers read the volumes or
    their bricked copies (packed here; the results are the same bit for bit).
    Returns the list of (n_i, h_i, w_i//2+1) complex64 slice stacks."""
    from .torch_fourier_slice import _layout as lay

    if not volumes:
        return []
    dev = _lib.require_cuda(*volumes)
    ctf = list(ctf) if ctf is not None else [None] * len(volumes)
    shapes = list(image_shapes) if image_shapes is not None else [
        (v.shape[0], v.shape[0], v.shape[0]) for v in volumes]
    Rs = [rotation_arg(R, dev)[0] for R in rotation_matrices]
    n_pixels = sum(R.shape[0] * int(sh[-2]) * (int(sh[-1]) // 2 + 1) for R, sh in zip(Rs, shapes))
    layout = _layout([v.shape[0] for v in volumes], n_pixels, sum(v.numel() for v in volumes), dev,
                     volume_layout)
    if layout == lay.BRICKS and not all(lay.bricks_fit(v) for v in volumes):
        layout = lay.PLAIN
    outs, entries, keep = [], [], []
    for vol, Rm, shape, c in zip(volumes, Rs, shapes, ctf):
        if vol.ndim != 3 or vol.dtype != torch.complex64:
            raise ValueError("batched extraction takes complex64 (d, h, w//2+1) volumes")
        vol = _lib.dense(vol)
        n = Rm.shape[0]
        h, w = int(shape[-2]), int(shape[-1])
        out = torch.empty((n, h, w // 2 + 1), dtype=torch.complex64, device=dev)
        cc = _check_ctf(c, n, dev)
        p = slice_params(n=n, image_shape=shape, volume=vol, rotation=Rm, fftfreq_max=fftfreq_max,
                         zyx_matrices=zyx_matrices, x_tolerance=x_tolerance,
                         rot_tolerance=rot_tolerance)
        src = vol
        if layout == lay.BRICKS and n > 0:
            src = lay.pack(vol, p, lay.BRICKS)
            p = lay.with_layout(p, lay.BRICKS)
        entries.append(_lib.BatchVolume(p, src.data_ptr(), out.data_ptr(), None, Rm.data_ptr(),
                                        cc.data_ptr() if cc is not None else None))
        keep += [vol, src, Rm, cc]
        outs.append(out)
    ts = _tile_shape("extract", [v.shape[0] for v in volumes], dev, tile_shape)
    for chunk in _batches(entries):
        _run("tt_extract_central_slices_rfft_3d_batched", chunk, ts, dev,
             "extract_central_slices_rfft_3d_batched")
    return outs


def insert_central_slices_rfft_3d_batched(
    images: Sequence[torch.Tensor],
    rotation_matrices: Sequence[torch.Tensor],
    volume_shapes: Sequence[tuple[int, int, int]] | None = None,
    ctf: Sequence[torch.Tensor | None] | None = None,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    tile_shape: int | None = None,
) -> list[tuple[torch.Tensor, torch.Tensor]]:
    """Insert every image stack into its own volume in one launch.

    ``images[i]`` (n_i, h, w//2+1) complex64 fftshifted rffts,
    ``volume_shapes[i]`` defaults to (h, h, h).  Returns a list of
    (volume (d, h, w//2+1) complex64, weights float32), Friedel-completed;
    with a CTF the weights are sums of CTF^2-weighted interpolation weights."""
    if not images:
        return []
    dev = _lib.require_cuda(*images)
    ctf = list(ctf) if ctf is not None else [None] * len(images)
    shapes = list(volume_shapes) if volume_shapes is not None else [
        (im.shape[-2], im.shape[-2], im.shape[-2]) for im in images]
    accs, entries, keep = [], [], []
    L = _lib.load()
    for img, R, shape, c in zip(images, rotation_matrices, shapes, ctf):
        if img.dtype != torch.complex64:
            raise ValueError("batched insertion takes complex64 slices")
        h, w = int(shape[-2]), int(shape[-1])
        if tuple(img.shape[-2:]) != (h, w // 2 + 1):
            raise ValueError(f"slices of shape {tuple(img.shape[-2:])} for volume_shape {tuple(shape)}")
        Rm, _ = rotation_arg(R, dev)
        n = Rm.shape[0]
        if math.prod(img.shape[:-2]) != n:
            raise ValueError(f"{n} rotation matrices for {math.prod(img.shape[:-2])} slices")
        img = _lib.dense(img.reshape(n, *img.shape[-2:]))
        cc = _check_ctf(c, n, dev)
        p = slice_params(n=n, image_shape=shape, volume=None, rotation=Rm, fftfreq_max=fftfreq_max,
                         zyx_matrices=zyx_matrices, vol_dims=rfft_shape(shape))
        # large accumulators are 2 x 2 x 2-bricked (the library's policy, as the one-shot insertion)
        p.volume_layout = int(L.tt_insert_accumulator_layout(ctypes.byref(p)))
        if p.volume_layout == _BRICKS:
            d, h, w = rfft_shape(shape)
            acc = torch.zeros(int(L.tt_insert_bricked_accumulator_bytes(d, h, w)) // 4, dtype=torch.float32,
                              device=dev)
        else:
            acc = new_accumulator(shape, False, dev)
        entries.append(_lib.BatchVolume(p, None, img.data_ptr(), acc.data_ptr(), Rm.data_ptr(),
                                        cc.data_ptr() if cc is not None else None))
        keep += [img, Rm, cc]
        accs.append((acc, p.volume_layout, rfft_shape(shape)))
    ts = _tile_shape("insert", [s[-2] for s in shapes], dev, tile_shape)
    for chunk in _batches(entries):
        _run("tt_insert_central_slices_rfft_3d_batched", chunk, ts, dev,
             "insert_central_slices_rfft_3d_batched")
    out = []
    for acc, layout, (d, h, w) in accs:
        if layout == _BRICKS:
            vol = torch.empty((d, h, w), dtype=torch.complex64, device=dev)
            wts = torch.empty((d, h, w), dtype=torch.float32, device=dev)
            _lib.check(L.tt_insert_finalize_bricked(_lib.ptr(acc), d, h, w, _lib.ptr(vol), _lib.ptr(wts),
                                                    _lib.stream_of(dev)),
                       "insert_central_slices_rfft_3d_batched finalize")
            out.append((vol, wts))
        else:
            v, wt = insert_finalize(acc, False)
            out.append((v[0], wt))
    return out


class BatchedSlicePlan:
    """A fixed-shape batch of volumes captured into one CUDA graph.

    Allocates static buffers for the volumes, rotations and CTF rows (fill
    them in place: ``plan.volumes[i].copy_(...)``), captures the batched
    launch (extraction, or insertion + per-volume finalize) once, and replays
    it with ``run()``.  Outputs live in ``plan.outputs``."""

    def __init__(self, box_sizes: Sequence[int], n_slices: Sequence[int], mode: str = "extract",
                 with_ctf: bool = True, device=None, tile_shape: int | None = None):
        if mode not in ("extract", "insert"):
            raise ValueError("mode must be 'extract' or 'insert'")
        self.device = torch.device(device or "cuda")
        self.mode = mode
        dev = self.device
        self.rotations = [torch.zeros((n, 3, 3), device=dev) for n in n_slices]
        for r in self.rotations:
            r[:] = torch.eye(3, device=dev)
        self.ctf = [ctf_params(1.5, n=n, device=dev) for n in n_slices] if with_ctf else None
        if mode == "extract":
            self.volumes = [torch.zeros(rfft_shape((b, b, b)), dtype=torch.complex64, device=dev)
                            for b in box_sizes]
            call = lambda: extract_central_slices_rfft_3d_batched(  # noqa: E731
                self.volumes, self.rotations, ctf=self.ctf, tile_shape=tile_shape)
        else:
            self.images = [torch.zeros((n, b, b // 2 + 1), dtype=torch.complex64, device=dev)
                           for b, n in zip(box_sizes, n_slices)]
            call = lambda: insert_central_slices_rfft_3d_batched(  # noqa: E731
                self.images, self.rotations, ctf=self.ctf, tile_shape=tile_shape)
        # warm up (tuner cache lookup, library load) outside the capture
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            call()
        torch.cuda.current_stream(dev).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.outputs = call()

    def run(self):
        self.graph.replay()
        return self.outputs
