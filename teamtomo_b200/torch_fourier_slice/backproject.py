"""Real-space reconstruction (drop-in for torch_fourier_slice.backproject_2d_to_3d).

Same steps as torch_fourier_slice/backproject.py:11-92 — pad, 2D rfft,
central-slice insertion, division by max(weights, 1), 3D irfft, division by
sinc^2, crop — with the fftshifts folded into kernel addressing: one kernel
pads and shifts the images, the insertion reads the unshifted 2D rfft, one
kernel applies the Friedel completion, the normalisation and the inverse
shift, and one kernel recentres, divides by sinc^2 and crops.

When the images require grad, the same steps run as differentiable pieces
(each fused pass has its exact adjoint; the insertion's backward is the
gather adjoint of the splat; the normalisation divides by the weights, which
do not depend on the images), so a reconstruction can be differentiated
w.r.t. its projections, as with the reference's torch code.
"""

from __future__ import annotations

import torch

from .. import _lib
from . import _wrappers
from ._params import rotation_arg
from .slice_insertion import (
    _InsertCentralSlices,
    insert_accumulate,
    insert_accumulate_multichannel,
    new_accumulator,
)


def _pad_amount(n: int, pad_factor: float) -> int:
    return int((n * (pad_factor - 1.0)) // 2)


def _backproject(images, rotation_matrices, pad_factor, fftfreq_max, zyx_matrices, channels):
    h, w = images.shape[-2:]
    if h != w:
        raise ValueError("images must be square.")
    if pad_factor < 1.0:
        raise ValueError("pad_factor must be >= 1.0")
    _lib.require_cuda(images)
    if images.dtype not in (torch.float32, torch.float64):
        images = images.to(torch.float32)
    dev = images.device
    p = _pad_amount(images.shape[-1], pad_factor) if pad_factor > 1.0 else 0
    d = images.shape[-1]
    n = d + 2 * p
    shape = (n, n, n)
    R, _ = rotation_arg(rotation_matrices, dev)
    nrot = R.shape[0]
    lead = images.shape[:-3] if channels else images.shape[:-2]
    c = images.shape[-3] if channels else 1
    flat = _lib.dense(images.reshape(-1, d, d))
    fft_in = _wrappers.pad_fftshift_2d(flat, p)
    spec = torch.fft.rfftn(fft_in, dim=(-2, -1)).reshape(*lead, c, n, n // 2 + 1)
    spec = spec.reshape(nrot, c, n, n // 2 + 1)
    if torch.is_grad_enabled() and images.requires_grad:
        vols, weights = _InsertCentralSlices.apply(spec, R, shape, fftfreq_max, zyx_matrices, False, True)
        dft = torch.fft.ifftshift(vols / torch.clamp(weights, min=1.0), dim=(-3, -2))
        real = _wrappers.irfftn_last(dft, 3)
        out = _wrappers.backproject_finish(real, p)
        return out if channels else out[0]
    c128 = spec.dtype == torch.complex128
    acc = new_accumulator(shape, c128, dev, channels=c)
    if c > 1 and not c128:
        insert_accumulate_multichannel(spec.contiguous(), R, shape, acc, fftfreq_max, zyx_matrices,
                                       images_unshifted=True)
    else:
        for ch in range(c):
            insert_accumulate(spec[:, ch].contiguous(), R, shape, acc[ch], fftfreq_max, zyx_matrices,
                              images_unshifted=True)
    dft = _wrappers.backproject_normalize(acc)
    # irfftn without an output size, as the reference (odd boxes lose one x column)
    real = _wrappers.irfftn_last(dft, 3)
    out = _wrappers.backproject_finish(real, p)
    return out if channels else out[0]


def backproject_2d_to_3d(
    images: torch.Tensor,  # (b, d, d)
    rotation_matrices: torch.Tensor,  # (b, 3, 3)
    pad_factor: float = 2.0,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
) -> torch.Tensor:
    """Reconstruct a (d, d, d) volume from (..., d, d) projection images."""
    return _backproject(images, rotation_matrices, pad_factor, fftfreq_max, zyx_matrices, False)


def backproject_2d_to_3d_multichannel(
    images: torch.Tensor,  # (..., c, d, d)
    rotation_matrices: torch.Tensor,  # (..., 3, 3)
    pad_factor: float = 2.0,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
) -> torch.Tensor:
    """Reconstruct (c, d, d, d) volumes from (..., c, d, d) images."""
    return _backproject(images, rotation_matrices, pad_factor, fftfreq_max, zyx_matrices, True)
