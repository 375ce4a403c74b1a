"""x-paired volume copies for the extraction gathers.

A trilinear sample reads the corners (x0, x0 + 1) of four volume rows.  In the
x-paired copy, entry (z, y, x) holds the complex64 pair (V[z, y, x],
V[z, y, x + 1]) as four floats, so each row is one 16-byte gather instead of
two 8-byte ones: fewer L1 wavefronts for the same scattered addresses, the
limit of the extraction and of the rotation gradient.  Values and operation
order are unchanged, so results are bit-identical to the plain layout.

The copy costs one streaming pass over the volume (8 bytes read and 16
written per voxel, 0.05 ms at 256^3) and twice the volume's footprint in L2
while it is read.  Measured on a B200 (4096 slices, 2048 at 320; plain ->
x-paired, the pack not included):

    box    copy     extraction   backward (dV + dR)   fused MSE
    128    17 MB    -11 %        -6 %                 -12 %
    192    57 MB    -12 %        -6.5 %               -13 %
    256    135 MB   -8 %         -1.5 %               -5 %
    320    264 MB   -8 %         +9.5 %               +6 %

The forward gathers (8 resident blocks per SM, L1-bound) gain at every size.
The gradient kernels also scatter into d/dvolume: once copy and gradient no
longer fit in L2 they gain little in isolation (256^3) or lose (320^3), and
the extra DRAM traffic costs clock speed under the power cap in a full step
(256^3 training step: 368K slices/s with the gradients on the plain volume at
1965 MHz, 363K on the copy at 1890-1950 MHz).  Policy (``TT_VOLUME_XPAIRS``
= ``auto``, the default): pack when the call's slices hold at least two
pixels per voxel, and for the gradient kernels only when the copy fits in
half the L2; ``1`` always packs, ``0`` never.
"""

from __future__ import annotations

import ctypes
import os

import torch

from .. import _lib

MIN_PIXELS_PER_VOXEL = 2
_l2_bytes: dict[int, int] = {}


def l2_bytes(device: torch.device) -> int:
    """L2 cache size of a CUDA device (0 when unknown)."""
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if idx not in _l2_bytes:
        _l2_bytes[idx] = int(getattr(torch.cuda.get_device_properties(idx), "L2_cache_size", 0))
    return _l2_bytes[idx]


def use_xpairs(n_pixels: int, volume: torch.Tensor, purpose: str = "grad") -> bool:
    """Whether a call sampling ``n_pixels`` slice pixels from ``volume``
    (complex64, (d, h, w//2+1)) should gather from an x-paired copy.
    ``purpose``: ``"forward"`` (the extraction's gathers alone) or ``"grad"``
    (the rotation gradient and the fused MSE)."""
    if purpose not in ("forward", "grad"):
        raise ValueError(f"purpose must be 'forward' or 'grad', got {purpose!r}")
    mode = os.environ.get("TT_VOLUME_XPAIRS", "auto").strip().lower()
    if mode in ("0", "off", "false", "no"):
        return False
    if volume.dtype != torch.complex64 or volume.ndim != 3:
        return False
    if mode in ("1", "on", "true", "yes"):
        return True
    if n_pixels < MIN_PIXELS_PER_VOXEL * volume.numel():
        return False
    if purpose == "forward":
        return True
    return volume.is_cuda and 16 * volume.numel() <= l2_bytes(volume.device) // 2


def with_xpairs(params: _lib.SliceParams, flag: bool) -> _lib.SliceParams:
    """Copy of ``params`` with ``volume_xpairs`` set to ``flag``."""
    q = _lib.SliceParams()
    ctypes.pointer(q)[0] = params
    q.volume_xpairs = int(bool(flag))
    return q


def pack(volume: torch.Tensor, params: _lib.SliceParams) -> torch.Tensor:
    """The x-paired copy of a contiguous complex64 volume: float32
    (d, h, w//2+1, 4), on the volume's device and current stream."""
    xp = torch.empty(tuple(volume.shape) + (4,), dtype=torch.float32, device=volume.device)
    L = _lib.load()
    _lib.check(L.tt_pack_volume_xpairs(_lib.ptr(volume), _lib.ptr(xp), params, _lib.stream_of(volume.device)),
               "pack_volume_xpairs")
    return xp
