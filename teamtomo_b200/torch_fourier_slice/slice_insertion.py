"""Central-slice insertion (drop-in for torch_fourier_slice.slice_insertion).

``insert_central_slices_rfft_3d`` keeps the reference signature and returns
``(volume, weights)`` like
torch_fourier_slice/slice_insertion/_insert_central_slices_rfft_3d.py:9-106:
complex64 slices give a complex64 volume with float32 weights, complex128
slices a complex128 volume with float64 weights.  The splat runs on the
sm_100a scatter kernel into an (re, im, w) accumulator; one finalize pass
applies the Friedel completion of the x=0 plane and writes the two outputs.
The insertion is differentiable w.r.t. the slices: the backward is the gather
adjoint of the splat and of the Friedel completion (one kernel, no atomics).

Deterministic mode (``deterministic=True``, or ``None`` with
``torch.use_deterministic_algorithms(True)``; not in the reference): the splat
accumulates in 64-bit fixed point, so the outputs are bit-identical for any
launch order, any split of the slices into calls and any slice order.  The
scale comes from max |re|, |im| of all images that go into one accumulator
(``fixed_absmax``) and the total slice count (``max_slices``).
"""

from __future__ import annotations

import math

import torch

from .. import _lib
from . import _layout
from ._params import resolve_deterministic, rfft_shape, rotation_arg, slice_params


def _check_image(image_rfft: torch.Tensor, volume_shape):
    if image_rfft.dtype not in (torch.complex64, torch.complex128):
        raise ValueError(f"image_rfft must be complex64 or complex128, got {image_rfft.dtype}")
    h, w = int(volume_shape[-2]), int(volume_shape[-1])
    if tuple(image_rfft.shape[-2:]) != (h, w // 2 + 1):
        raise ValueError(
            f"image_rfft has rfft shape {tuple(image_rfft.shape[-2:])}, expected {(h, w // 2 + 1)} "
            f"for volume_shape {tuple(volume_shape)}"
        )


def new_accumulator(volume_shape, complex128: bool, device, channels: int = 1) -> torch.Tensor:
    """Zeroed insertion accumulator: (channels, d, h, w//2+1) slots of
    (re, im, w, pad) in float32 (complex64 data) or float64 (complex128)."""
    d, h, w = rfft_shape(volume_shape)
    dt = torch.float64 if complex128 else torch.float32
    return torch.zeros((channels, d, h, w, 4), dtype=dt, device=device)


def insert_accumulate(image_rfft, R, volume_shape, acc, fftfreq_max=None, zyx_matrices=False,
                      images_unshifted=False):
    """Add the trilinear splat of (n, h, w//2+1) slices into one accumulator
    (no Friedel completion)."""
    dev = acc.device
    # the kernels index raw memory in C order
    if not (image_rfft.is_contiguous() and R.is_contiguous() and acc.is_contiguous()):
        raise ValueError("insertion needs C-contiguous slices, rotations and accumulator")
    params = slice_params(n=R.shape[0], image_shape=volume_shape, volume=None, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          slices_unshifted=images_unshifted, vol_dims=rfft_shape(volume_shape))
    L = _lib.load()
    _lib.check(
        L.tt_insert_accumulate(_lib.ptr(image_rfft), int(image_rfft.dtype == torch.complex128),
                               _lib.ptr(R), _lib.ptr(acc), params, _lib.stream_of(dev)),
        "insert_central_slices_rfft_3d",
    )


def insert_finalize(acc: torch.Tensor, complex128: bool):
    """Accumulator (c, d, h, w, 4) -> volume (c, d, h, w) complex, weights (d, h, w)."""
    c, d, h, w = acc.shape[:4]
    cdt = torch.complex128 if complex128 else torch.complex64
    wdt = torch.float64 if complex128 else torch.float32
    volume = torch.empty((c, d, h, w), dtype=cdt, device=acc.device)
    weights = torch.empty((d, h, w), dtype=wdt, device=acc.device)
    L = _lib.load()
    _lib.check(L.tt_insert_finalize(_lib.ptr(acc), int(complex128), c, d, h, w, _lib.ptr(volume),
                                    _lib.ptr(weights), _lib.stream_of(acc.device)),
               "insert_central_slices_rfft_3d finalize")
    return volume, weights


def fixed_absmax(*images: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """Float32 bit pattern of max |re|, |im| over ``images`` as a (1,) int32
    device tensor (maxed into ``out`` when given): the scale input of the
    fixed-point accumulation.  All-reduce it with MAX to share one scale
    across processes."""
    dev = images[0].device
    if out is None:
        out = torch.zeros(1, dtype=torch.int32, device=dev)
    L = _lib.load()
    for t in images:
        t = _lib.dense(t)
        real = torch.view_as_real(t) if t.is_complex() else t
        _lib.check(L.tt_fixed_absmax(_lib.ptr(real), int(real.dtype == torch.float64), real.numel(),
                                     _lib.ptr(out), _lib.stream_of(dev)), "fixed_absmax")
    return out


def new_fixed_accumulator(volume_shape, device, channels: int = 1) -> torch.Tensor:
    """Zeroed fixed-point accumulator: (channels, d, h, w//2+1, 4) int64
    (re, im, w, pad)."""
    d, h, w = rfft_shape(volume_shape)
    return torch.zeros((channels, d, h, w, 4), dtype=torch.int64, device=device)


def insert_fixed_accumulate(image_rfft, R, volume_shape, acc, absmax, max_slices, fftfreq_max=None,
                            zyx_matrices=False, images_unshifted=False):
    """Deterministic splat of (n, h, w//2+1) slices into a fixed-point
    accumulator at the scale of ``absmax`` and ``max_slices``."""
    dev = acc.device
    if not (image_rfft.is_contiguous() and R.is_contiguous() and acc.is_contiguous()):
        raise ValueError("insertion needs C-contiguous slices, rotations and accumulator")
    params = slice_params(n=R.shape[0], image_shape=volume_shape, volume=None, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          slices_unshifted=images_unshifted, vol_dims=rfft_shape(volume_shape))
    L = _lib.load()
    _lib.check(
        L.tt_insert_fixed_accumulate(_lib.ptr(image_rfft), int(image_rfft.dtype == torch.complex128),
                                     _lib.ptr(R), _lib.ptr(acc), _lib.ptr(absmax), int(max_slices), params,
                                     _lib.stream_of(dev)),
        "insert_central_slices_rfft_3d (deterministic)",
    )


def insert_fixed_finalize(acc: torch.Tensor, complex128: bool, absmax, max_slices):
    """Fixed-point accumulator (c, d, h, w, 4) -> volume (c, d, h, w), weights (d, h, w)."""
    c, d, h, w = acc.shape[:4]
    cdt = torch.complex128 if complex128 else torch.complex64
    wdt = torch.float64 if complex128 else torch.float32
    volume = torch.empty((c, d, h, w), dtype=cdt, device=acc.device)
    weights = torch.empty((d, h, w), dtype=wdt, device=acc.device)
    L = _lib.load()
    _lib.check(L.tt_insert_fixed_finalize(_lib.ptr(acc), int(complex128), c, d, h, w, _lib.ptr(absmax),
                                          int(max(max_slices, 1)), _lib.ptr(volume), _lib.ptr(weights),
                                          _lib.stream_of(acc.device)),
               "insert_central_slices_rfft_3d finalize (deterministic)")
    return volume, weights


def friedel_mirror_x0(volume, weights):
    """In-place Friedel completion of the x=0 plane of (c?, d, h, w) volumes."""
    dev = volume.device
    d, h, w = volume.shape[-3:]
    channels = volume.numel() // (d * h * w)
    L = _lib.load()
    _lib.check(
        L.tt_friedel_mirror_x0(_lib.ptr(volume), _lib.ptr(weights),
                               int(volume.dtype == torch.complex128), channels, d, h, w,
                               _lib.stream_of(dev)),
        "friedel_mirror_x0",
    )


def _splat(chans, R, volume_shape, fftfreq_max, zyx_matrices, deterministic, c128, dev, unshifted=False):
    """Insertion of per-channel (n, h, w//2+1) stacks -> ((c, d, h, w) volumes, weights)."""
    n = R.shape[0]
    if deterministic:
        absmax = fixed_absmax(*chans)
        acc = new_fixed_accumulator(volume_shape, dev, channels=len(chans))
        for ch, img in enumerate(chans):
            insert_fixed_accumulate(img, R, volume_shape, acc[ch], absmax, max(n, 1), fftfreq_max, zyx_matrices,
                                    images_unshifted=unshifted)
        return insert_fixed_finalize(acc, c128, absmax, n)
    if len(chans) == 1 and not c128:
        return _insert_one_shot(chans[0], R, volume_shape, fftfreq_max, zyx_matrices, unshifted)
    acc = new_accumulator(volume_shape, c128, dev, channels=len(chans))
    for ch, img in enumerate(chans):
        insert_accumulate(img, R, volume_shape, acc[ch], fftfreq_max, zyx_matrices, images_unshifted=unshifted)
    return insert_finalize(acc, c128)


def _insert_one_shot(image_rfft, R, volume_shape, fftfreq_max, zyx_matrices, unshifted):
    """Float insertion of one (n, h, w//2+1) stack through the one-shot entry
    point, whose workspace holds the bricked accumulator."""
    dev = image_rfft.device
    if not (image_rfft.is_contiguous() and R.is_contiguous()):
        raise ValueError("insertion needs C-contiguous slices and rotations")
    params = slice_params(n=R.shape[0], image_shape=volume_shape, volume=None, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices, slices_unshifted=unshifted,
                          vol_dims=rfft_shape(volume_shape))
    d, h, w = rfft_shape(volume_shape)
    volume = torch.empty((1, d, h, w), dtype=torch.complex64, device=dev)
    weights = torch.empty((d, h, w), dtype=torch.float32, device=dev)
    L = _lib.load()
    nbytes = int(L.tt_insert_workspace_bytes(0, params))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    _lib.check(L.tt_insert_central_slices_rfft_3d(_lib.ptr(image_rfft), 0, _lib.ptr(R), _lib.ptr(volume),
                                                  _lib.ptr(weights), _lib.ptr(ws), nbytes, params,
                                                  _lib.stream_of(dev)),
               "insert_central_slices_rfft_3d")
    return volume, weights


def insert_backward(grad_volume, R, volume_shape, fftfreq_max=None, zyx_matrices=False,
                    images_unshifted=False) -> torch.Tensor:
    """dL/dslices (n, h, w//2+1) of one insertion for upstream dL/dvolume
    (d, h, w//2+1): the gather adjoint of the splat and of the Friedel
    completion (the weights output does not depend on the slices)."""
    dev = grad_volume.device
    grad_volume = _lib.dense(grad_volume)
    c128 = grad_volume.dtype == torch.complex128
    d, h, w = rfft_shape(volume_shape)
    out = torch.empty((R.shape[0], h, w), dtype=grad_volume.dtype, device=dev)
    params = slice_params(n=R.shape[0], image_shape=volume_shape, volume=None, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          slices_unshifted=images_unshifted, vol_dims=(d, h, w))
    # from half a slice pixel per voxel the gathers read a bricked copy of the
    # gradient volume (the extraction's layout policy; bit-identical results)
    src = grad_volume
    if not c128 and grad_volume.ndim == 3:
        layout = _layout.choose(R.shape[0] * h * w, grad_volume)
        if layout == _layout.BRICKS:
            params = _layout.with_layout(params, layout)
            src = _layout.pack(grad_volume, params, layout)
    L = _lib.load()
    _lib.check(L.tt_insert_central_slices_rfft_3d_backward(_lib.ptr(src), int(c128), _lib.ptr(R),
                                                           _lib.ptr(out), params, _lib.stream_of(dev)),
               "insert_central_slices_rfft_3d backward")
    return out


def insert_accumulate_multichannel(images, R, volume_shape, acc, fftfreq_max=None, zyx_matrices=False,
                                   images_unshifted=False):
    """Add the splat of (n, c, h, w//2+1) complex64 slices into c float
    accumulators (c, d, h, w//2+1, 4), one channel after the other (readers
    take the weights from channel 0)."""
    if not (images.is_contiguous() and R.is_contiguous() and acc.is_contiguous()):
        raise ValueError("insertion needs C-contiguous slices, rotations and accumulator")
    params = slice_params(n=R.shape[0], image_shape=volume_shape, volume=None, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          slices_unshifted=images_unshifted, vol_dims=rfft_shape(volume_shape))
    L = _lib.load()
    _lib.check(L.tt_insert_accumulate_multichannel(_lib.ptr(images), images.shape[1], _lib.ptr(R), _lib.ptr(acc),
                                                   params, _lib.stream_of(acc.device)),
               "insert_central_slices_rfft_3d_multichannel")


def insert_backward_multichannel(grad_volumes, R, volume_shape, fftfreq_max=None, zyx_matrices=False,
                                 images_unshifted=False) -> torch.Tensor:
    """dL/dslices (n, c, h, w//2+1) of a multichannel insertion for upstream
    dL/dvolumes (c, d, h, w//2+1), complex64."""
    dev = grad_volumes.device
    grad_volumes = _lib.dense(grad_volumes)
    c = grad_volumes.shape[0]
    d, h, w = rfft_shape(volume_shape)
    out = torch.empty((R.shape[0], c, h, w), dtype=torch.complex64, device=dev)
    params = slice_params(n=R.shape[0], image_shape=volume_shape, volume=None, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          slices_unshifted=images_unshifted, vol_dims=(d, h, w))
    L = _lib.load()
    _lib.check(L.tt_insert_central_slices_rfft_3d_multichannel_backward(
        _lib.ptr(grad_volumes), c, _lib.ptr(R), _lib.ptr(out), params, _lib.stream_of(dev)),
        "insert_central_slices_rfft_3d_multichannel backward")
    return out


class _InsertCentralSlices(torch.autograd.Function):
    """(n, c, h, w//2+1) slices -> ((c, d, h, w//2+1) volumes, weights),
    differentiable w.r.t. the slices (not the rotations, which are constants
    here; the weights carry no gradient).  ``unshifted``: slice rows stored
    ifftshifted (the plain rfft of a real image)."""

    @staticmethod
    def forward(ctx, images, R, volume_shape, fftfreq_max, zyx_matrices, deterministic, unshifted=False):
        c = images.shape[1]
        c128 = images.dtype == torch.complex128
        if c > 1 and not c128 and not deterministic:
            # one geometry pass per pixel for all channels
            acc = new_accumulator(volume_shape, False, images.device, channels=c)
            insert_accumulate_multichannel(_lib.dense(images), R, volume_shape, acc, fftfreq_max, zyx_matrices,
                                           unshifted)
            volumes, weights = insert_finalize(acc, False)
        else:
            chans = [_lib.dense(images[:, ch]) for ch in range(c)]
            volumes, weights = _splat(chans, R, volume_shape, fftfreq_max, zyx_matrices, deterministic, c128,
                                      images.device, unshifted)
        ctx.mark_non_differentiable(weights)
        ctx.save_for_backward(R)
        ctx.args = (volume_shape, fftfreq_max, zyx_matrices, unshifted)
        return volumes, weights

    @staticmethod
    def backward(ctx, grad_volumes, grad_weights):
        if grad_volumes is None or not ctx.needs_input_grad[0]:
            return None, None, None, None, None, None, None
        (R,) = ctx.saved_tensors
        c = grad_volumes.shape[0]
        if c > 1 and grad_volumes.dtype == torch.complex64:
            grads = insert_backward_multichannel(grad_volumes, R, *ctx.args)
        else:
            grads = torch.stack([insert_backward(grad_volumes[ch], R, *ctx.args) for ch in range(c)], dim=1)
        return grads, None, None, None, None, None, None


def insert_central_slices_rfft_3d(
    image_rfft: torch.Tensor,  # fftshifted rfft of (..., h, w) 2d image
    volume_shape: tuple[int, int, int],
    rotation_matrices: torch.Tensor,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    deterministic: bool | None = None,
) -> tuple[torch.Tensor, torch.Tensor]:
    """Insert central slices into an fftshifted rfft volume; returns
    ``(volume, weights)``.  Differentiable w.r.t. ``image_rfft`` (the gather
    adjoint, not in the reference's API but what its autograd computes);
    ``deterministic`` (not in the reference) selects the fixed-point splat."""
    _lib.require_cuda(image_rfft)
    _check_image(image_rfft, volume_shape)
    dev = image_rfft.device
    R, stack = rotation_arg(rotation_matrices, dev)
    n = R.shape[0]
    lead = image_rfft.shape[:-2]
    if math.prod(lead) != n:
        raise ValueError(f"{n} rotation matrices for image stack of shape {tuple(lead)}")
    img = image_rfft.reshape(n, 1, *image_rfft.shape[-2:])
    volumes, weights = _InsertCentralSlices.apply(img, R, tuple(int(x) for x in volume_shape), fftfreq_max,
                                                  zyx_matrices, resolve_deterministic(deterministic))
    return volumes[0], weights


def insert_central_slices_rfft_3d_multichannel(
    image_rfft: torch.Tensor,  # fftshifted rfft of (..., c, h, w) 2d images
    volume_shape: tuple[int, int, int],
    rotation_matrices: torch.Tensor,  # (..., 3, 3)
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    deterministic: bool | None = None,
) -> tuple[torch.Tensor, torch.Tensor]:
    """Multichannel insertion (_insert_central_slices_rfft_3d.py:109-210):
    returns ``(c, d, h, w//2+1)`` volumes and ONE ``(d, h, w//2+1)`` weight
    volume shared by the channels."""
    _lib.require_cuda(image_rfft)
    _check_image(image_rfft, volume_shape)
    dev = image_rfft.device
    c = image_rfft.shape[-3]
    R, stack = rotation_arg(rotation_matrices, dev)
    n = R.shape[0]
    img = image_rfft.reshape(n, c, *image_rfft.shape[-2:])
    return _InsertCentralSlices.apply(img, R, tuple(int(x) for x in volume_shape), fftfreq_max, zyx_matrices,
                                      resolve_deterministic(deterministic))
