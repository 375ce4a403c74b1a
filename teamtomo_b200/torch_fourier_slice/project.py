"""Real-space projection (drop-in for torch_fourier_slice.project_3d_to_2d).

Same steps as torch_fourier_slice/project.py:12-93 — pad, premultiply by
sinc^2, 3D rfft, central-slice extraction, 2D irfft, crop — with the fftshift
bookkeeping folded into the kernels' addressing: the padded, sinc^2-weighted
volume is written directly in FFT order by one kernel, the extraction reads
the unshifted rfftn output and writes rows already ifftshifted for the 2D
irfft, and one kernel recentres and crops the projections.
"""

from __future__ import annotations

import torch

from . import _wrappers
from ._params import rotation_arg, slice_params
from .slice_extraction import _ExtractCentralSlices, _ExtractMultichannel


def _pad_amount(n: int, pad_factor: float) -> int:
    return int((n * (pad_factor - 1.0)) // 2)


def project_3d_to_2d(
    volume: torch.Tensor,
    rotation_matrices: torch.Tensor,
    pad_factor: float = 2.0,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
) -> torch.Tensor:
    """Project a cubic volume by sampling central slices through its DFT.

    ``volume`` (d, d, d) float32; ``rotation_matrices`` (..., 3, 3); returns
    (..., d, d) projections.  Differentiable w.r.t. volume and rotations."""
    d, h, w = volume.shape[-3:]
    if len({d, h, w}) != 1:
        raise ValueError("all dimensions of volume must be equal.")
    if pad_factor < 1.0:
        raise ValueError("pad_factor must be >= 1.0")
    p = _pad_amount(volume.shape[-1], pad_factor) if pad_factor > 1.0 else 0
    n_pad = d + 2 * p
    shape = (n_pad, n_pad, n_pad)
    fft_in = _wrappers.project_prepare(volume, p)  # padded * sinc^2, fftshifted
    # unshifted rfft; cuFFT may hand back a non-contiguous layout
    dft = torch.fft.rfftn(fft_in, dim=(-3, -2, -1)).contiguous()
    R, stack = rotation_arg(rotation_matrices, volume.device)
    params = slice_params(n=R.shape[0], image_shape=shape, volume=dft, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          rot_tolerance=1e-8, volume_unshifted=True, slices_unshifted=True)
    slices = _ExtractCentralSlices.apply(dft, R, params, (R.shape[0], n_pad, n_pad // 2 + 1))
    # irfftn without an output size, as the reference: an odd padded box
    # gives images one column narrower (2 * (n_pad // 2) wide)
    images = _wrappers.irfftn_last(slices, 2)
    out = _wrappers.recentre_crop_2d(images, p)
    return out.reshape(*stack, *out.shape[-2:])


def project_3d_to_2d_multichannel(
    volume: torch.Tensor,
    rotation_matrices: torch.Tensor,
    pad_factor: float = 2.0,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
) -> torch.Tensor:
    """(c, d, d, d) -> (..., c, d, d): every channel projected with the same
    rotations, one multichannel extraction for all channels."""
    c, d, h, w = volume.shape[-4:]
    if len({d, h, w}) != 1:
        raise ValueError("all dimensions of volume must be equal.")
    if pad_factor < 1.0:
        raise ValueError("pad_factor must be >= 1.0")
    p = _pad_amount(d, pad_factor) if pad_factor > 1.0 else 0
    n_pad = d + 2 * p
    shape = (n_pad, n_pad, n_pad)
    fft_in = torch.stack([_wrappers.project_prepare(volume[ch], p) for ch in range(c)])
    dft = torch.fft.rfftn(fft_in, dim=(-3, -2, -1)).contiguous()
    R, stack = rotation_arg(rotation_matrices, volume.device)
    params = slice_params(n=R.shape[0], image_shape=shape, volume=dft[0], rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          rot_tolerance=1e-8, volume_unshifted=True, slices_unshifted=True)
    slices = _ExtractMultichannel.apply(dft, R, params, (R.shape[0], c, n_pad, n_pad // 2 + 1))
    images = _wrappers.irfftn_last(slices, 2)
    out = _wrappers.recentre_crop_2d(images.reshape(-1, *images.shape[-2:]), p)
    return out.reshape(*stack, c, *out.shape[-2:])
