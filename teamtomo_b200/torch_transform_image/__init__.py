"""Affine resampling of 3D images (drop-in for torch_transform_image's 3D transform).

``affine_transform_image_3d`` keeps the signature of
torch_transform_image/transforms_3d.py:10-40.  One CUDA kernel computes each
output voxel's homogeneous coordinate M (z, y, x, 1) in registers (float32,
the reference's operation order) and samples the image there (trilinear or
nearest, as ``sample_image_3d``); the (d, h, w, 3) coordinate grid the
reference builds is never written.  Matrices of other float dtypes are cast
to float32 (the reference's matmul with its float32 grid would raise).
"""

from __future__ import annotations

from typing import Literal, Optional

import torch

from .. import _lib

_CODE = {torch.float32: 0, torch.float64: 1, torch.complex64: 2, torch.complex128: 3}

__all__ = ["affine_transform_image_3d"]


def affine_transform_image_3d(
    image: torch.Tensor,
    matrices: torch.Tensor,
    interpolation: Literal["nearest", "trilinear"],
    output_shape: Optional[tuple] = None,
    zyx_matrices: bool = False,
) -> torch.Tensor:
    """Resample a (d, h, w) or (c, d, h, w) image at the positions that
    ``matrices`` (..., 4, 4) map each output voxel to; returns
    (..., d', h', w') or (..., d', h', w', c)."""
    if image.ndim not in (3, 4):
        raise ValueError(f"image should have shape (d, h, w) or (c, d, h, w), got {image.shape}")
    if interpolation not in ("nearest", "trilinear"):
        raise ValueError(f"interpolation must be 'nearest' or 'trilinear', got {interpolation!r}")
    _lib.require_cuda(image)
    if image.dtype not in _CODE:
        image = image.to(torch.float32)
    d, h, w = (int(s) for s in (output_shape if output_shape else image.shape[-3:]))
    M = torch.as_tensor(matrices, device=image.device).to(torch.float32)
    if M.shape[-2:] != (4, 4):
        raise ValueError(f"matrices must have shape (..., 4, 4), got {tuple(M.shape)}")
    if not zyx_matrices:
        M = M.clone()
        M[..., :3, :3] = torch.flip(M[..., :3, :3], dims=(-2, -1))
        M[..., :3, 3] = torch.flip(M[..., :3, 3], dims=(-1,))
    stack = tuple(M.shape[:-2])
    M = M.reshape(-1, 4, 4).contiguous()
    multi = image.ndim == 4
    img = _lib.dense(image if multi else image[None])
    C, D, H, W = img.shape
    out = torch.empty((M.shape[0], d, h, w, C), dtype=image.dtype, device=image.device)
    L = _lib.load()
    _lib.check(L.tt_affine_transform_image_3d(_lib.ptr(img), _CODE[image.dtype], C, D, H, W, _lib.ptr(M), M.shape[0],
                                              d, h, w, int(interpolation == "nearest"), _lib.ptr(out),
                                              _lib.stream_of(image.device)), "affine_transform_image_3d")
    out = out.reshape(*stack, d, h, w, C)
    return out if multi else out[..., 0]
