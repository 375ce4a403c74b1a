"""Fused losses over central slices.

``central_slice_mse`` is ``mean(|extract_central_slices_rfft_3d(V, R) - T|^2)``
and its gradients w.r.t. the volume and the rotation matrices in ONE kernel:
the sample is rebuilt from the corner values the rotation gradient loads
anyway, so the slices are never written and the upstream gradient never read
back.  This is the objective of fitting a map and/or orientations to
observed slices; for any other loss, use ``extract_central_slices_rfft_3d``
(a differentiable op) and torch.

The gradients are computed with the loss (in the forward pass) when the
inputs require grad, and scaled by the upstream gradient in the backward.
"""

from __future__ import annotations

import math

import torch

from . import _lib
from .torch_fourier_slice import _layout
from .torch_fourier_slice._params import rotation_arg, slice_params


class _CentralSliceMSE(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volume_rfft, R, targets, params):
        dev = volume_rfft.device
        want_v, want_r = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        loss = torch.empty((), dtype=torch.float32, device=dev)
        dvol = torch.zeros_like(volume_rfft) if want_v else None
        drot = torch.empty_like(R) if want_r else None
        L = _lib.load()
        nbytes = int(L.tt_central_slice_mse_workspace_bytes(params))
        ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
        # large calls gather from a bricked copy of the volume (bit-identical results)
        layout = _layout.choose(targets.numel(), volume_rfft)
        copy = _layout.pack(volume_rfft, params, layout)
        _lib.check(L.tt_central_slice_mse(_lib.ptr(copy if copy is not None else volume_rfft), _lib.ptr(R),
                                          _lib.ptr(targets), _lib.ptr(loss), _lib.ptr(dvol), _lib.ptr(drot),
                                          _lib.ptr(ws), nbytes, _layout.with_layout(params, layout),
                                          _lib.stream_of(dev)), "central_slice_mse")
        ctx.save_for_backward(dvol, drot)
        return loss

    @staticmethod
    def backward(ctx, g):
        dvol, drot = ctx.saved_tensors
        return (dvol * g if dvol is not None else None), (drot * g if drot is not None else None), None, None


def central_slice_mse(
    volume_rfft: torch.Tensor,
    image_shape: tuple[int, int, int],
    rotation_matrices: torch.Tensor,  # (..., 3, 3)
    targets: torch.Tensor,  # (..., h, w // 2 + 1) complex64
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    x_tolerance: float = 1e-8,
    rot_tolerance: float | None = 1e-8,
) -> torch.Tensor:
    """Mean over all slice elements of |extract(volume_rfft, R) - targets|^2
    (a 0-dim float32 tensor), differentiable w.r.t. ``volume_rfft`` and
    ``rotation_matrices``.  Arguments as ``extract_central_slices_rfft_3d``."""
    assert volume_rfft.ndim == 3, "Input volume_rfft must be 3D tensor."
    _lib.require_cuda(volume_rfft, targets)
    if volume_rfft.dtype != torch.complex64 or targets.dtype != torch.complex64:
        raise RuntimeError("central_slice_mse takes complex64 volumes and targets")
    volume_rfft = _lib.dense(volume_rfft)
    R, stack = rotation_arg(rotation_matrices, volume_rfft.device)
    h, w = int(image_shape[-2]), int(image_shape[-1])
    n = R.shape[0]
    if n == 0:
        raise ValueError("central_slice_mse needs at least one slice")
    if tuple(targets.shape[-2:]) != (h, w // 2 + 1) or math.prod(targets.shape[:-2]) != n:
        raise ValueError(f"targets of shape {tuple(targets.shape)} for {n} slices of {(h, w // 2 + 1)}")
    T = _lib.dense(targets.reshape(n, h, w // 2 + 1))
    params = slice_params(n=n, image_shape=image_shape, volume=volume_rfft, rotation=R, fftfreq_max=fftfreq_max,
                          zyx_matrices=zyx_matrices, x_tolerance=x_tolerance, rot_tolerance=rot_tolerance)
    return _CentralSliceMSE.apply(volume_rfft, R, T, params)
