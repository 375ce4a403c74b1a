"""Host-side argument normalisation shared by the slice operators."""

from __future__ import annotations

import numpy as np
import torch

from .. import _lib


def rotation_arg(rotation_matrices: torch.Tensor, device: torch.device):
    """(..., 3, 3) -> contiguous (n, 3, 3) float32/float64 on ``device``.

    float64 matrices are passed as they are: the kernels round them to float32
    exactly as ``Tensor.to(torch.float32)`` does.  Other dtypes are cast to
    float32 first."""
    R = torch.as_tensor(rotation_matrices)
    if R.shape[-2:] != (3, 3):
        raise ValueError(f"rotation matrices must have shape (..., 3, 3), got {tuple(R.shape)}")
    stack = tuple(R.shape[:-2])
    if R.dtype not in (torch.float32, torch.float64):
        R = R.to(torch.float32)
    R = R.to(device).reshape(-1, 3, 3).contiguous()
    return R, stack


def _f32(x: float) -> float:
    return float(np.float32(x))


def slice_params(n, image_shape, volume, rotation, fftfreq_max=None, zyx_matrices=False,
                 x_tolerance=1e-8, rot_tolerance=None, volume_unshifted=False,
                 slices_unshifted=False, vol_dims=None, deterministic=False) -> _lib.SliceParams:
    d, h, w = (int(s) for s in image_shape)
    vd, vh, vw = vol_dims if vol_dims is not None else tuple(int(s) for s in volume.shape[-3:])
    p = _lib.SliceParams()
    p.n = int(n)
    p.img_d, p.img_h, p.img_w = d, h, w
    p.vol_d, p.vol_h, p.vol_w = vd, vh, vw
    p.has_fftfreq_max = int(fftfreq_max is not None)
    p.fftfreq_max = _f32(fftfreq_max) if fftfreq_max is not None else 0.0
    p.zyx_matrices = int(bool(zyx_matrices))
    p.x_tolerance = _f32(x_tolerance)
    p.x_tolerance10 = _f32(x_tolerance * 10)
    p.has_rot_tolerance = int(rot_tolerance is not None)
    p.rot_tolerance = _f32(rot_tolerance) if rot_tolerance is not None else 0.0
    p.rotation_f64 = int(rotation.dtype == torch.float64)
    p.volume_unshifted = int(bool(volume_unshifted))
    p.slices_unshifted = int(bool(slices_unshifted))
    p.deterministic = int(bool(deterministic))
    return p


def resolve_deterministic(flag: bool | None) -> bool:
    """``None`` follows ``torch.use_deterministic_algorithms``."""
    return torch.are_deterministic_algorithms_enabled() if flag is None else bool(flag)


def rfft_shape(shape):
    """Output shape of an rfft over ``shape`` (torch_grid_utils.rfft_shape)."""
    s = list(int(x) for x in shape)
    s[-1] = s[-1] // 2 + 1
    return tuple(s)
