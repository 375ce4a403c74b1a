"""3D interpolation primitives (drop-in for torch_image_interpolation's 3D API).

``sample_image_3d`` and ``insert_into_image_3d`` keep the reference
signatures and semantics (torch_image_interpolation/image_interpolation_3d.py:11-101
and :104-275) and run on sm_100a gather / scatter kernels.  ``sample_image_3d``
is differentiable w.r.t. the image and the coordinates, as the reference's
grid_sample is (one backward kernel: a d/dimage scatter and the trilinear
coordinate gradient; no per-sample copy of the image).
"""

from __future__ import annotations

from typing import Literal

import torch

from .. import _lib

_DTYPE_CODES = {torch.float32: 0, torch.float64: 1, torch.complex64: 2, torch.complex128: 3}
_REAL = {torch.float32: torch.float32, torch.float64: torch.float64,
         torch.complex64: torch.float32, torch.complex128: torch.float64}


def _code(dtype: torch.dtype) -> int:
    if dtype not in _DTYPE_CODES:
        raise ValueError(f"unsupported dtype {dtype}; expected float32/64 or complex64/128")
    return _DTYPE_CODES[dtype]


class _SampleImage3d(torch.autograd.Function):
    @staticmethod
    def forward(ctx, img, coords, nearest):
        C, D, H, W = img.shape
        n = coords.shape[0]
        out = torch.empty((n, C), dtype=img.dtype, device=img.device)
        L = _lib.load()
        _lib.check(L.tt_sample_image_3d(_lib.ptr(img), _code(img.dtype), C, D, H, W, _lib.ptr(coords), n,
                                        _lib.ptr(out), int(nearest), _lib.stream_of(img.device)), "sample_image_3d")
        ctx.save_for_backward(img, coords)
        ctx.nearest = nearest
        return out

    @staticmethod
    def backward(ctx, grad):
        img, coords = ctx.saved_tensors
        want_i, want_c = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (want_i or want_c):
            return None, None, None
        C, D, H, W = img.shape
        grad = _lib.dense(grad.to(img.dtype))
        gimg = torch.zeros_like(img) if want_i else None
        gc = torch.empty_like(coords) if want_c else None
        L = _lib.load()
        _lib.check(L.tt_sample_image_3d_backward(_lib.ptr(img), _code(img.dtype), C, D, H, W, _lib.ptr(coords),
                                                 coords.shape[0], _lib.ptr(grad), _lib.ptr(gimg), _lib.ptr(gc),
                                                 int(ctx.nearest), _lib.stream_of(img.device)),
                   "sample_image_3d backward")
        return gimg, gc, None


def sample_image_3d(
    image: torch.Tensor,
    coordinates: torch.Tensor,
    interpolation: Literal["nearest", "trilinear"] = "trilinear",
) -> torch.Tensor:
    """Sample a (d, h, w) or (c, d, h, w) image at (..., 3) zyx array coordinates.

    Returns (...) or (..., c) samples; zero where a coordinate is outside
    [0, N-1]."""
    if image.ndim not in (3, 4):
        raise ValueError(f"image should have shape (d, h, w) or (c, d, h, w), got {image.shape}")
    if interpolation not in ("nearest", "trilinear"):
        raise ValueError(f"interpolation must be 'nearest' or 'trilinear', got {interpolation!r}")
    _lib.require_cuda(image)
    _code(image.dtype)  # validates the dtype
    multi = image.ndim == 4
    img = _lib.dense(image if multi else image[None])
    C, D, H, W = img.shape
    coords = torch.as_tensor(coordinates).to(image.device)
    batch = coords.shape[:-1]
    c = _lib.dense(coords.reshape(-1, 3).to(_REAL[image.dtype]))
    out = _SampleImage3d.apply(img, c, interpolation == "nearest")
    out = out.reshape(*batch, C)
    return out if multi else out[..., 0]


def insert_into_image_3d(
    values: torch.Tensor,
    coordinates: torch.Tensor,
    image: torch.Tensor,
    weights: torch.Tensor | None = None,
    interpolation: Literal["nearest", "trilinear"] = "trilinear",
) -> tuple[torch.Tensor, torch.Tensor]:
    """Insert values into a (d, h, w) or (c, d, h, w) image (in place).

    Returns ``(image, weights)``; ``weights`` (d, h, w) keeps its dtype and
    defaults to a new float32 zero volume.  As in the reference, an
    ``interpolation`` other than 'nearest' / 'trilinear' inserts nothing."""
    multi = image.ndim == 4
    d, h, w = image.shape[-3:]
    values_shape = values.shape[:-1] if multi else values.shape
    coordinates_shape, coordinates_ndim = coordinates.shape[:-1], coordinates.shape[-1]
    if values_shape != coordinates_shape:
        raise ValueError("One coordinate triplet is required for each value in data.")
    if coordinates_ndim != 3:
        raise ValueError("Coordinates must be 3D with shape (..., 3).")
    if image.dtype != values.dtype:
        raise ValueError("Image and values must have the same dtype.")
    _lib.require_cuda(image)
    if weights is None:
        weights = torch.zeros(size=(d, h, w), dtype=torch.float32, device=image.device)
    if interpolation not in ("nearest", "trilinear"):
        return image, weights
    if weights.dtype not in (torch.float32, torch.float64):
        raise ValueError(f"weights must be float32 or float64, got {weights.dtype}")
    C = image.shape[0] if multi else 1
    vals = values.to(image.device).reshape(-1, C)
    c = coordinates.to(image.device).reshape(-1, 3).float().contiguous()
    if image.is_contiguous() and weights.is_contiguous():
        return _InsertIntoImage3d.apply(vals, c, image, weights, C, interpolation == "nearest")
    img, wts = image.contiguous(), weights.contiguous()
    _InsertIntoImage3d.apply(vals, c, img, wts, C, interpolation == "nearest")
    image.copy_(img)
    weights.copy_(wts)
    return image, weights


class _InsertIntoImage3d(torch.autograd.Function):
    """In-place splat into (image, weights); differentiable w.r.t. the values
    (the reference's index_put_ backward: a gather with the same weights).
    The coordinates get no gradient."""

    @staticmethod
    def forward(ctx, vals, coords, image, weights, C, nearest):
        d, h, w = image.shape[-3:]
        v = _lib.dense(vals)
        L = _lib.load()
        _lib.check(L.tt_insert_into_image_3d(_lib.ptr(v), _code(image.dtype), _lib.ptr(coords), coords.shape[0],
                                             _lib.ptr(image), C, d, h, w, _lib.ptr(weights),
                                             int(weights.dtype == torch.float64), int(nearest),
                                             _lib.stream_of(image.device)), "insert_into_image_3d")
        ctx.mark_dirty(image, weights)
        ctx.mark_non_differentiable(weights)
        ctx.save_for_backward(coords)
        ctx.meta = (C, d, h, w, nearest, image.dtype, vals.shape)
        return image, weights

    @staticmethod
    def backward(ctx, grad_image, grad_weights):
        (coords,) = ctx.saved_tensors
        C, d, h, w, nearest, dtype, vshape = ctx.meta
        gv = None
        if ctx.needs_input_grad[0] and grad_image is not None:
            g = _lib.dense(grad_image.to(dtype))
            gv = torch.empty(vshape, dtype=dtype, device=g.device)
            L = _lib.load()
            _lib.check(L.tt_insert_into_image_3d_backward(_lib.ptr(g), _code(dtype), _lib.ptr(coords),
                                                          coords.shape[0], C, d, h, w, int(nearest), _lib.ptr(gv),
                                                          _lib.stream_of(g.device)), "insert_into_image_3d backward")
        return gv, None, grad_image, None, None, None


__all__ = ["sample_image_3d", "insert_into_image_3d"]
