"""Host side of the elementwise passes around the FFTs of project / backproject.

Each forward runs one fused CUDA kernel (see ``csrc/wrappers.cu``).  The
passes of both projection and backprojection are differentiable; their
backward passes are the exact adjoints (a permutation, a crop or zero-pad and
a fixed sinc^2 weight), written with torch ops because they are off the hot
path.
"""

from __future__ import annotations

import torch
import torch.nn.functional as F

from .. import _lib


def _is_f64(t: torch.Tensor) -> int:
    return int(t.dtype == torch.float64)


def sinc2_grid(n: int, device, dtype=torch.float32) -> torch.Tensor:
    """sinc(|f|)^2 on the fftshifted n^3 frequency grid."""
    k = torch.arange(n, device=device)
    f = torch.where(k < (n + 1) // 2, k, k - n).to(torch.float32) * torch.tensor(
        1.0 / n, dtype=torch.float32)
    f = torch.fft.fftshift(f)
    r = torch.sqrt(f[:, None, None] ** 2 + f[None, :, None] ** 2 + f[None, None, :] ** 2)
    return (torch.sinc(r) ** 2).to(dtype)


def sinc2_grid_3(n0: int, n1: int, n2: int, device, dtype=torch.float32) -> torch.Tensor:
    """sinc(|f|)^2 on the fftshifted frequency grid of an (n0, n1, n2) array."""
    def axis(n):
        k = torch.arange(n, device=device)
        f = torch.where(k < (n + 1) // 2, k, k - n).to(torch.float32) * torch.tensor(1.0 / n, dtype=torch.float32)
        return torch.fft.fftshift(f)

    f0, f1, f2 = axis(n0), axis(n1), axis(n2)
    r = torch.sqrt(f0[:, None, None] ** 2 + f1[None, :, None] ** 2 + f2[None, None, :] ** 2)
    return (torch.sinc(r) ** 2).to(dtype)


def irfftn_last(x: torch.Tensor, ndim: int) -> torch.Tensor:
    """``irfftn`` over the last ``ndim`` axes (no output size), evaluated the way
    torch's CPU FFT evaluates it: inverse complex FFTs along the leading axes,
    then a 1D inverse real FFT along the last axis that ignores the imaginary
    parts of its DC and Nyquist bins.  Sampled central slices (and inserted
    volumes) are not exactly Hermitian, and for such inputs cuFFT's
    multi-dimensional complex-to-real transform differs from the CPU result
    by ~1e-4; this form matches it."""
    # a fresh tensor either way: the caller's input is never modified
    x = torch.fft.ifftn(x, dim=tuple(range(-ndim, -1))) if ndim > 1 else x.clone()
    xr = torch.view_as_real(x)
    xr[..., 0, 1].zero_()
    xr[..., -1, 1].zero_()  # the Nyquist bin of the default (even) output length
    return torch.fft.irfft(x, dim=-1)


class _ProjectPrepare(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volume, pad):
        d = volume.shape[-1]
        n = d + 2 * pad
        out = torch.empty((n, n, n), dtype=volume.dtype, device=volume.device)
        L = _lib.load()
        _lib.check(L.tt_project_prepare(_lib.ptr(volume), _is_f64(volume), d, pad, _lib.ptr(out),
                                        _lib.stream_of(volume.device)), "project_prepare")
        ctx.pad = pad
        return out

    @staticmethod
    def backward(ctx, g):
        p = ctx.pad
        n = g.shape[-1]
        g = torch.fft.ifftshift(g, dim=(-3, -2, -1)) * sinc2_grid(n, g.device, g.dtype)
        if p:
            g = g[p:-p, p:-p, p:-p]
        return g, None


class _RecentreCrop2d(torch.autograd.Function):
    @staticmethod
    def forward(ctx, images, pad):
        m, h, w = images.shape
        out = torch.empty((m, h - 2 * pad, w - 2 * pad), dtype=images.dtype, device=images.device)
        L = _lib.load()
        _lib.check(L.tt_recentre_crop_2d(_lib.ptr(images), _is_f64(images), m, h, w, pad,
                                         _lib.ptr(out), _lib.stream_of(images.device)),
                   "recentre_crop_2d")
        ctx.pad = pad
        return out

    @staticmethod
    def backward(ctx, g):
        p = ctx.pad
        if p:
            g = F.pad(g, [p] * 4)
        return torch.fft.fftshift(g, dim=(-2, -1)), None


def project_prepare(volume: torch.Tensor, pad: int) -> torch.Tensor:
    _lib.require_cuda(volume)
    if volume.dtype not in (torch.float32, torch.float64):
        volume = volume.to(torch.float32)
    return _ProjectPrepare.apply(_lib.dense(volume), int(pad))


def recentre_crop_2d(images: torch.Tensor, pad: int) -> torch.Tensor:
    h, w = images.shape[-2:]
    flat = _lib.dense(images.reshape(-1, h, w))
    return _RecentreCrop2d.apply(flat, int(pad))


class _PadFftshift2d(torch.autograd.Function):
    @staticmethod
    def forward(ctx, images, pad):
        m, d = images.shape[0], images.shape[-1]
        n = d + 2 * pad
        out = torch.empty((m, n, n), dtype=images.dtype, device=images.device)
        L = _lib.load()
        _lib.check(L.tt_pad_fftshift_2d(_lib.ptr(images), _is_f64(images), m, d, pad, _lib.ptr(out),
                                        _lib.stream_of(images.device)), "pad_fftshift_2d")
        ctx.pad = pad
        return out

    @staticmethod
    def backward(ctx, g):
        # adjoint of fftshift(pad(x)): crop(ifftshift(g))
        p = ctx.pad
        n = g.shape[-1]
        g = torch.fft.ifftshift(g, dim=(-2, -1))
        return g[..., p:n - p, p:n - p], None


def pad_fftshift_2d(images: torch.Tensor, pad: int) -> torch.Tensor:
    """(m, d, d) real -> fftshift(pad(images)) (m, n, n)."""
    return _PadFftshift2d.apply(_lib.dense(images), int(pad))


def backproject_normalize(acc: torch.Tensor) -> torch.Tensor:
    """Insertion accumulator (c, d, h, w, 4) -> Friedel completion, division by
    max(w, 1) and ifftshift(d, h): complex volumes (c, d, h, w)."""
    c, d, h, w = acc.shape[:4]
    c128 = acc.dtype == torch.float64
    out = torch.empty((c, d, h, w), dtype=torch.complex128 if c128 else torch.complex64,
                      device=acc.device)
    L = _lib.load()
    _lib.check(L.tt_backproject_normalize(_lib.ptr(acc), int(c128), c, d, h, w, _lib.ptr(out),
                                          _lib.stream_of(acc.device)),
               "backproject_normalize")
    return out


class _BackprojectFinish(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volume, pad):
        n0, n1, n2 = volume.shape[-3:]
        lead = volume.shape[:-3]
        channels = volume.numel() // (n0 * n1 * n2)
        out = torch.empty((*lead, n0 - 2 * pad, n1 - 2 * pad, n2 - 2 * pad), dtype=volume.dtype,
                          device=volume.device)
        L = _lib.load()
        _lib.check(L.tt_backproject_finish(_lib.ptr(volume), _is_f64(volume), channels, n0, n1, n2,
                                           pad, _lib.ptr(out), _lib.stream_of(volume.device)),
                   "backproject_finish")
        ctx.pad = pad
        ctx.dims = (n0, n1, n2)
        return out

    @staticmethod
    def backward(ctx, g):
        # adjoint of crop(ifftshift(v) / sinc^2): fftshift(pad(g) / sinc^2)
        p = ctx.pad
        n0, n1, n2 = ctx.dims
        if p:
            g = F.pad(g, [p] * 6)
        g = g / sinc2_grid_3(n0, n1, n2, g.device, g.dtype)
        return torch.fft.fftshift(g, dim=(-3, -2, -1)), None


def backproject_finish(volume: torch.Tensor, pad: int) -> torch.Tensor:
    """(c?, n0, n1, n2) irfft output -> crop(ifftshift(v) / sinc^2)."""
    return _BackprojectFinish.apply(_lib.dense(volume), int(pad))
