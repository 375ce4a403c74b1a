"""Central-slice extraction (drop-in for torch_fourier_slice.slice_extraction).

``extract_central_slices_rfft_3d`` keeps the reference signature, defaults and
semantics (torch_fourier_slice/slice_extraction/_extract_central_slices_rfft_3d.py:84-222)
and runs on the sm_100a gather kernel.  It is differentiable w.r.t. the volume
and the rotation matrices through one fused backward kernel; interpolation
weights are recomputed in the backward pass, not stored.

Deterministic mode (``deterministic=True``, or ``None`` with
``torch.use_deterministic_algorithms(True)``): the volume gradient is
accumulated in 64-bit fixed point and is bit-identical from run to run; the
rotation gradient is reduced in a fixed order in both modes.

Deliberate difference: the reference zeroes near-zero rotation elements IN
PLACE on the caller's float32 tensor (:147-151), which also raises for a leaf
that requires grad.  Here the caller's tensor is never modified; the zeroing
is applied to a private copy inside the kernel and the zeroed elements get a
zero gradient, as in the reference.
"""

from __future__ import annotations

import torch

from .. import _lib
from . import _layout
from ._params import resolve_deterministic, rotation_arg, slice_params


class _ExtractCentralSlices(torch.autograd.Function):
    @staticmethod
    def forward(ctx, volume_rfft, rotation_matrices, params, out_shape):
        # the kernels index raw memory in C order and sample complex64
        if not (volume_rfft.is_contiguous() and rotation_matrices.is_contiguous()):
            raise ValueError("extraction needs C-contiguous volume and rotation tensors")
        if volume_rfft.dtype != torch.complex64:
            raise RuntimeError(f"the extraction kernels sample complex64 volumes (got {volume_rfft.dtype})")
        dev = volume_rfft.device
        out = torch.empty(out_shape, dtype=torch.complex64, device=dev)
        L = _lib.load()
        # large calls gather from a bricked copy (bit-identical results)
        layout = _layout.choose(out.numel(), volume_rfft)
        copy = _layout.pack(volume_rfft, params, layout)
        _lib.check(
            L.tt_extract_central_slices_rfft_3d(_lib.ptr(copy if copy is not None else volume_rfft),
                                                _lib.ptr(rotation_matrices), _lib.ptr(out),
                                                _layout.with_layout(params, layout), _lib.stream_of(dev)),
            "extract_central_slices_rfft_3d",
        )
        ctx.params = params
        # the backward reads the volume only for d/drotation: keep the copy for it
        keep = copy is not None and ctx.needs_input_grad[1]
        ctx.layout = layout if keep else _layout.PLAIN
        ctx.save_for_backward(volume_rfft, rotation_matrices, *((copy,) if keep else ()))
        return out

    @staticmethod
    def backward(ctx, grad):
        saved = ctx.saved_tensors
        volume_rfft, rotation_matrices = saved[0], saved[1]
        want_v, want_r = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        dvol = drot = None
        if want_v or want_r:
            layout = ctx.layout
            copy = saved[2] if layout != _layout.PLAIN else None
            # direct calls of the backward alone (no forward copy) make their own
            if copy is None and want_r:
                layout = _layout.choose(grad.numel(), volume_rfft)
                copy = _layout.pack(volume_rfft, ctx.params, layout)
            dvol, drot = extract_backward(volume_rfft, rotation_matrices, grad, ctx.params,
                                          want_v, want_r, copy=copy, layout=layout)
        return dvol, drot, None, None


class _ExtractMultichannel(torch.autograd.Function):
    """(c, d, h, w//2+1) volumes -> (n, c, h, w//2+1) slices with one
    geometry pass per pixel; backward: d/dvolume per channel, d/drotation
    summed over the channels."""

    @staticmethod
    def forward(ctx, volumes, rotation_matrices, params, out_shape):
        if not (volumes.is_contiguous() and rotation_matrices.is_contiguous()):
            raise ValueError("extraction needs C-contiguous volume and rotation tensors")
        if volumes.dtype != torch.complex64:
            raise RuntimeError(f"the extraction kernels sample complex64 volumes (got {volumes.dtype})")
        dev = volumes.device
        out = torch.empty(out_shape, dtype=torch.complex64, device=dev)
        L = _lib.load()
        # large calls gather from the channels' bricked copies (bit-identical results)
        layout = _multichannel_layout(out_shape[0] * out_shape[2] * out_shape[3], volumes)
        copy = _layout.pack_channels(volumes, params, layout)
        _lib.check(L.tt_extract_central_slices_rfft_3d_multichannel(
            _lib.ptr(copy if copy is not None else volumes), volumes.shape[0], _lib.ptr(rotation_matrices),
            _lib.ptr(out), _layout.with_layout(params, layout), _lib.stream_of(dev)),
            "extract_central_slices_rfft_3d_multichannel")
        ctx.params = params
        # the backward reads the volumes only for d/drotation: keep the copies for it
        keep = copy is not None and ctx.needs_input_grad[1]
        ctx.layout = layout if keep else _layout.PLAIN
        ctx.save_for_backward(volumes, rotation_matrices, *((copy,) if keep else ()))
        return out

    @staticmethod
    def backward(ctx, grad):
        saved = ctx.saved_tensors
        volumes, R = saved[0], saved[1]
        want_v, want_r = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (want_v or want_r):
            return None, None, None, None
        layout = ctx.layout
        copy = saved[2] if layout != _layout.PLAIN else None
        if copy is None and want_r:
            layout = _multichannel_layout(grad.shape[0] * grad.shape[2] * grad.shape[3], volumes)
            copy = _layout.pack_channels(volumes, ctx.params, layout)
        dev = volumes.device
        grad = _lib.dense(grad.to(torch.complex64))
        L = _lib.load()
        dvol = torch.zeros_like(volumes) if want_v else None
        drot = torch.empty_like(R) if want_r else None
        nbytes = int(L.tt_extract_backward_workspace_bytes(ctx.params)) if want_r else 0
        ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev) if want_r else None
        _lib.check(L.tt_extract_central_slices_rfft_3d_multichannel_backward(
            _lib.ptr(copy if copy is not None else volumes), volumes.shape[0], _lib.ptr(R), _lib.ptr(grad),
            _lib.ptr(dvol), _lib.ptr(drot), _lib.ptr(ws), nbytes,
            _layout.with_layout(ctx.params, layout if copy is not None else _layout.PLAIN), _lib.stream_of(dev)),
            "extract_central_slices_rfft_3d_multichannel backward")
        return dvol, drot, None, None


def _multichannel_layout(n_pixels, volumes):
    """Layout of a multichannel call sampling ``n_pixels`` pixels per channel:
    the single-volume policy for one channel, the x-paired copy excepted."""
    layout = _layout.choose(n_pixels, volumes[0])
    return _layout.PLAIN if layout == _layout.XPAIRS else layout


def extract_backward(volume_rfft, rotation_matrices, grad, params, want_volume=True,
                     want_rotation=True, copy=None, layout=_layout.PLAIN):
    """Fused backward: (d/dvolume, d/drotation) for upstream slice gradient
    ``grad``.  ``copy``: the volume's ``layout`` copy (``_layout.pack``), read
    by the rotation gradient's gathers in place of ``volume_rfft``."""
    dev = volume_rfft.device
    grad = _lib.dense(grad.to(torch.complex64))
    L = _lib.load()
    if copy is None:
        layout = _layout.PLAIN
    params = _layout.with_layout(params, layout)
    dvol = torch.zeros_like(volume_rfft) if want_volume else None
    drot = torch.empty_like(rotation_matrices) if want_rotation else None
    ws = None
    nbytes = 0
    if want_rotation or (want_volume and params.deterministic):
        nbytes = int(L.tt_extract_backward_workspace_bytes(params))
        ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=dev)
    _lib.check(
        L.tt_extract_central_slices_rfft_3d_backward(
            _lib.ptr(copy if copy is not None else volume_rfft), _lib.ptr(rotation_matrices),
            _lib.ptr(grad), _lib.ptr(dvol),
            _lib.ptr(drot), _lib.ptr(ws), nbytes, params, _lib.stream_of(dev)),
        "extract_central_slices_rfft_3d backward",
    )
    return dvol, drot


def extract_central_slices_rfft_3d(
    volume_rfft: torch.Tensor,
    image_shape: tuple[int, int, int],
    rotation_matrices: torch.Tensor,  # (..., 3, 3)
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    x_tolerance: float = 1e-8,
    rot_tolerance: float | None = 1e-8,
    deterministic: bool | None = None,
) -> torch.Tensor:
    """Extract central slices from an fftshifted rfft volume.

    Parameters and return value as in the reference: ``volume_rfft`` is
    ``(d, d, d//2+1)`` complex64 (fftshifted in the first two dims),
    ``image_shape`` the real-space shape defining the slice grid,
    ``rotation_matrices`` ``(..., 3, 3)``; returns ``(..., h, w//2+1)``
    complex64 slices (zero outside ``fftfreq_max``).  ``deterministic``
    (not in the reference) selects the fixed-point volume gradient.
    """
    assert volume_rfft.ndim == 3, "Input volume_rfft must be 3D tensor."
    _lib.require_cuda(volume_rfft)
    if volume_rfft.dtype != torch.complex64:
        raise RuntimeError(
            f"extract_central_slices_rfft_3d supports complex64 volumes (got {volume_rfft.dtype})"
        )
    volume_rfft = _lib.dense(volume_rfft)
    R, stack = rotation_arg(rotation_matrices, volume_rfft.device)
    h, w = int(image_shape[-2]), int(image_shape[-1])
    params = slice_params(n=R.shape[0], image_shape=image_shape, volume=volume_rfft,
                          rotation=R, fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          x_tolerance=x_tolerance, rot_tolerance=rot_tolerance,
                          deterministic=resolve_deterministic(deterministic))
    out = _ExtractCentralSlices.apply(volume_rfft, R, params, (R.shape[0], h, w // 2 + 1))
    return out.reshape(*stack, h, w // 2 + 1)


def central_slice_geometry(
    rotation_matrices: torch.Tensor,
    image_shape: tuple[int, int, int],
    volume_dims: tuple[int, int, int],
    mode: str = "extract",
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    x_tolerance: float = 1e-8,
    rot_tolerance: float | None = 1e-8,
) -> tuple[torch.Tensor, torch.Tensor]:
    """Per-pixel geometry of the slice grid, computed by the CUDA kernels.

    Returns ``(flags, coords)``: flags (n, h, w//2+1) uint8 with bit0 = pixel
    kept, bit1 = conjugate redirect, bit2 = inside the volume; coords
    (n, h, w//2+1, 3) float32 redirected zyx array coordinates.  ``mode`` is
    'extract' (tolerance rules of the extraction) or 'insert' (strict x<0 rule,
    Friedel-redundant source pixels dropped, no rot_tolerance)."""
    R, _ = rotation_arg(rotation_matrices, rotation_matrices.device)
    _lib.require_cuda(R)
    h, w = int(image_shape[-2]), int(image_shape[-1])
    n = R.shape[0]
    params = slice_params(n=n, image_shape=image_shape, volume=None, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          x_tolerance=x_tolerance, rot_tolerance=rot_tolerance,
                          vol_dims=tuple(int(v) for v in volume_dims))
    flags = torch.empty((n, h, w // 2 + 1), dtype=torch.uint8, device=R.device)
    coords = torch.empty((n, h, w // 2 + 1, 3), dtype=torch.float32, device=R.device)
    L = _lib.load()
    _lib.check(L.tt_slice_geometry(_lib.ptr(R), 0 if mode == "extract" else 1, _lib.ptr(flags),
                                   _lib.ptr(coords), params, _lib.stream_of(R.device)),
               "central_slice_geometry")
    return flags, coords


def extract_central_slices_rfft_3d_multichannel(
    volume_rfft: torch.Tensor,  # (c, d, d, d)
    image_shape: tuple[int, int, int],
    rotation_matrices: torch.Tensor,  # (..., 3, 3)
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
    x_tolerance: float = 1e-8,
    rot_tolerance: float | None = 1e-8,
    deterministic: bool | None = None,
) -> torch.Tensor:  # (..., c, h, w)
    """Multichannel extraction (_extract_central_slices_rfft_3d.py:225-367):
    ``(c, d, d, d//2+1)`` -> ``(..., c, h, w//2+1)``, the same rotations for
    every channel, each pixel's geometry computed once for all channels (the
    deterministic mode runs the channels one by one)."""
    assert volume_rfft.ndim == 4, "Input volume_rfft must be 4D tensor."
    if not resolve_deterministic(deterministic):
        _lib.require_cuda(volume_rfft)
        if volume_rfft.dtype != torch.complex64:
            raise RuntimeError(
                f"extract_central_slices_rfft_3d supports complex64 volumes (got {volume_rfft.dtype})")
        vols = _lib.dense(volume_rfft)
        R, stack = rotation_arg(rotation_matrices, vols.device)
        h, w = int(image_shape[-2]), int(image_shape[-1])
        c = vols.shape[0]
        params = slice_params(n=R.shape[0], image_shape=image_shape, volume=vols[0], rotation=R,
                              fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices, x_tolerance=x_tolerance,
                              rot_tolerance=rot_tolerance)
        out = _ExtractMultichannel.apply(vols, R, params, (R.shape[0], c, h, w // 2 + 1))
        return out.reshape(*stack, c, h, w // 2 + 1)
    slices = [
        extract_central_slices_rfft_3d(volume_rfft[c], image_shape, rotation_matrices,
                                       fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                                       x_tolerance=x_tolerance, rot_tolerance=rot_tolerance,
                                       deterministic=deterministic)
        for c in range(volume_rfft.shape[0])
    ]
    return torch.stack(slices, dim=-3)
