"""Central lines of 2D images: ``extract_central_slices_rfft_2d`` and
``project_2d_to_1d`` (drop-ins for torch_fourier_slice's 2D functions,
slice_extraction/_extract_central_slices_rfft_2d.py:9-84 and project.py).

The line sampling runs on a CUDA kernel (one thread per line sample) with a
fused backward (d/dimage scatter, per-line d/drotation reduced in a fixed
order); the padding, sinc^2 premultiplication and 1D/2D FFTs of the
projection are torch ops (they are not on the hot path).  Deliberate
difference: the reference raises for any ``fftfreq_max`` (it masks the
(w, 2) coordinate grid element-wise); here samples with frequency above
``fftfreq_max`` are zero.
"""

from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

from .. import _lib
from ._wrappers import irfftn_last


def _rotation_2d(rotation_matrices: torch.Tensor, device):
    R = torch.as_tensor(rotation_matrices)
    if R.shape[-2:] != (2, 2):
        raise ValueError(f"rotation matrices must have shape (..., 2, 2), got {tuple(R.shape)}")
    stack = tuple(R.shape[:-2])
    if R.dtype not in (torch.float32, torch.float64):
        R = R.to(torch.float32)
    return R.to(device).reshape(-1, 2, 2).contiguous(), stack


class _ExtractLines(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image_rfft, R, image_shape, fftfreq_max, yx_matrices):
        dev = image_rfft.device
        h, w = image_shape
        n = R.shape[0]
        out = torch.empty((n, w // 2 + 1), dtype=torch.complex64, device=dev)
        args = (image_rfft.shape[0], image_rfft.shape[1])
        flags = (int(fftfreq_max is not None), float(np.float32(fftfreq_max or 0.0)), int(bool(yx_matrices)))
        L = _lib.load()
        _lib.check(L.tt_extract_central_lines_rfft_2d(_lib.ptr(image_rfft), *args, _lib.ptr(R),
                                                      int(R.dtype == torch.float64), n, h, w, *flags,
                                                      _lib.ptr(out), _lib.stream_of(dev)),
                   "extract_central_slices_rfft_2d")
        ctx.save_for_backward(image_rfft, R)
        ctx.meta = (args, (h, w), flags)
        return out

    @staticmethod
    def backward(ctx, grad):
        image_rfft, R = ctx.saved_tensors
        want_i, want_r = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (want_i or want_r):
            return None, None, None, None, None
        args, (h, w), flags = ctx.meta
        dev = image_rfft.device
        grad = _lib.dense(grad.to(torch.complex64))
        dimg = torch.zeros_like(image_rfft) if want_i else None
        drot = torch.empty_like(R) if want_r else None
        L = _lib.load()
        _lib.check(L.tt_extract_central_lines_rfft_2d_backward(
            _lib.ptr(image_rfft), *args, _lib.ptr(R), int(R.dtype == torch.float64), R.shape[0], h, w, *flags,
            _lib.ptr(grad), _lib.ptr(dimg), _lib.ptr(drot), _lib.stream_of(dev)),
            "extract_central_slices_rfft_2d backward")
        return dimg, drot, None, None, None


def extract_central_slices_rfft_2d(
    image_rfft: torch.Tensor,
    image_shape: tuple[int, int],
    rotation_matrices: torch.Tensor,  # (..., 2, 2)
    fftfreq_max: float | None = None,
    yx_matrices: bool = False,
) -> torch.Tensor:
    """Extract central lines from an fftshifted 2D rfft: ``(h, w//2+1)``
    complex64 -> ``(..., w//2+1)``.  Differentiable w.r.t. the image and the
    rotation matrices."""
    _lib.require_cuda(image_rfft)
    if image_rfft.ndim != 2:
        raise ValueError(f"image_rfft must be (h, w//2+1), got {tuple(image_rfft.shape)}")
    if image_rfft.dtype != torch.complex64:
        raise RuntimeError(f"extract_central_slices_rfft_2d supports complex64 images (got {image_rfft.dtype})")
    R, stack = _rotation_2d(rotation_matrices, image_rfft.device)
    h, w = int(image_shape[-2]), int(image_shape[-1])
    out = _ExtractLines.apply(_lib.dense(image_rfft), R, (h, w), fftfreq_max, yx_matrices)
    return out.reshape(*stack, w // 2 + 1)


def _sinc2_2d(n: int, device, dtype) -> torch.Tensor:
    k = torch.arange(n, device=device)
    f = torch.where(k < (n + 1) // 2, k, k - n).to(torch.float32) * torch.tensor(1.0 / n, dtype=torch.float32)
    f = torch.fft.fftshift(f)
    r = torch.sqrt(f[:, None] ** 2 + f[None, :] ** 2)
    return (torch.sinc(r) ** 2).to(dtype)


def project_2d_to_1d(
    image: torch.Tensor,
    rotation_matrices: torch.Tensor,
    pad_factor: float = 2.0,
    fftfreq_max: float | None = None,
    yx_matrices: bool = False,
) -> torch.Tensor:
    """Project a square ``(d, d)`` image along rotated directions: ``(..., d)``
    lines (one sample narrower for odd padded sizes, as the reference's irfft
    without an output size).  Differentiable w.r.t. image and rotations."""
    h, w = image.shape[-2:]
    if h != w:
        raise ValueError("all dimensions of image must be equal.")
    if pad_factor < 1.0:
        raise ValueError("pad_factor must be >= 1.0")
    _lib.require_cuda(image)
    p = int((image.shape[-1] * (pad_factor - 1.0)) // 2) if pad_factor > 1.0 else 0
    if p:
        image = F.pad(image, pad=[p] * 4)
    n = image.shape[-1]
    image = image * _sinc2_2d(n, image.device, image.dtype)
    dft = torch.fft.rfftn(torch.fft.fftshift(image, dim=(-2, -1)), dim=(-2, -1))
    dft = torch.fft.fftshift(dft, dim=(-2,))
    lines = extract_central_slices_rfft_2d(dft.to(torch.complex64), (n, n), rotation_matrices,
                                           fftfreq_max=fftfreq_max, yx_matrices=yx_matrices)
    proj = torch.fft.ifftshift(irfftn_last(lines, 1), dim=(-1,))
    if p:
        proj = F.pad(proj, pad=[-p] * 2)
    return proj
