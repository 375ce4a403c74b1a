"""Volume copies for the extraction gathers (tt_slice_params.volume_layout).

A trilinear sample reads the corners (x0, x0 + 1) of four volume rows, and
the gathers of the extraction, its rotation gradient and the fused MSE are
bound by the L1 wavefronts of those scattered reads.  Two copies of the
volume lower them; values and operation order are unchanged, so results are
bit-identical to the plain layout:

* x-paired (``XPAIRS``, tt_pack_volume_xpairs): entry (z, y, x) holds the
  complex64 pair (V[z, y, x], V[z, y, x + 1]), so each row is one 16-byte
  gather instead of two 8-byte ones.  Twice the volume's size.
* bricked (``BRICKS``, tt_pack_volume_bricks): 2 x 2 x 2 voxel bricks of 64
  bytes, two x-adjacent bricks per 128-byte line, so a line holds a 4 x 2 x 2
  block of voxels instead of 16 voxels of one row and the corners of a warp's
  8 x 4 pixels touch fewer lines.  The volume's size (padded to even dims).

Each copy costs one streaming pass over the volume.  Measured on a B200
(ms, each kernel alone, 4096 slices, 2048 at 320; plain / x-paired / bricked):

    box   extraction           backward (dV + dR)   fused MSE            pack (x-pairs, bricks)
    128   0.46 / 0.41 / 0.38   1.07 / 0.98 / 0.92   1.03 / 0.92 / 0.88   0.010, 0.010
    192   1.00 / 0.89 / 0.80   2.35 / 2.15 / 2.01   2.29 / 2.02 / 1.90   0.023, 0.021
    256   1.78 / 1.67 / 1.58   4.08 / 4.06 / 3.85   3.99 / 4.17 / 3.46   0.054, 0.043
    320   1.51 / 1.42 / 1.25   3.55 / 3.89 / 3.25   3.59 / 3.96 / 3.19   0.101, 0.074

The bricked copy is the volume's size, so it stays as cacheable as the volume
(the x-paired copy, twice the size, misses L2 from 256^3 up).  Policy
(``TT_VOLUME_LAYOUT``): ``auto`` (the default) gathers from the bricked copy
when the call's slices hold at least half a pixel per voxel (the pack pays
for itself from about a fifth) and from the volume itself otherwise;
``plain``, ``xpairs`` or ``bricks`` force a layout.
"""

from __future__ import annotations

import ctypes
import os

import torch

from .. import _lib

PLAIN, XPAIRS, BRICKS = 0, 1, 2
_MODES = {"plain": PLAIN, "xpairs": XPAIRS, "bricks": BRICKS}
MIN_PIXELS_PER_VOXEL = 0.5


def choose(n_pixels: int, volume: torch.Tensor) -> int:
    """Layout a call sampling ``n_pixels`` slice pixels from ``volume``
    (complex64, (d, h, w//2+1)) should gather from."""
    mode = os.environ.get("TT_VOLUME_LAYOUT", "auto").strip().lower()
    if mode != "auto" and mode not in _MODES:
        raise ValueError(f"TT_VOLUME_LAYOUT must be auto, plain, xpairs or bricks (got {mode!r})")
    if volume.dtype != torch.complex64 or volume.ndim != 3:
        return PLAIN
    if mode != "auto":
        if _MODES[mode] == BRICKS and not bricks_fit(volume):
            raise ValueError(f"TT_VOLUME_LAYOUT=bricks: the bricked copy of a {tuple(volume.shape)} volume "
                             "would hold 2^31 slots or more (the gathers' 32-bit slot offsets); "
                             "use auto or plain for this volume")
        return _MODES[mode]
    return BRICKS if n_pixels >= MIN_PIXELS_PER_VOXEL * volume.numel() and bricks_fit(volume) else PLAIN


def bricks_fit(volume: torch.Tensor) -> bool:
    """Whether the bricked copy of ``volume`` has fewer than 2^31 slots (the
    range of the gathers' 32-bit slot offsets)."""
    d, h, w = volume.shape[-3:]
    return ((d + 1) // 2) * ((h + 1) // 2) * ((w + 1) // 2) * 8 < 2**31


def with_layout(params: _lib.SliceParams, layout: int) -> _lib.SliceParams:
    """Copy of ``params`` with ``volume_layout`` set to ``layout``."""
    q = _lib.SliceParams()
    ctypes.pointer(q)[0] = params
    q.volume_layout = int(layout)
    return q


def pack(volume: torch.Tensor, params: _lib.SliceParams, layout: int) -> torch.Tensor | None:
    """The ``layout`` copy of a contiguous complex64 volume (None for
    ``PLAIN``), on the volume's device and current stream: float32
    (d, h, w//2+1, 4) x-pairs, or the bricks as a flat complex64 tensor."""
    if layout == PLAIN:
        return None
    L = _lib.load()
    st = _lib.stream_of(volume.device)
    if layout == XPAIRS:
        out = torch.empty(tuple(volume.shape) + (4,), dtype=torch.float32, device=volume.device)
        _lib.check(L.tt_pack_volume_xpairs(_lib.ptr(volume), _lib.ptr(out), params, st), "pack_volume_xpairs")
        return out
    if layout == BRICKS:
        nbytes = int(L.tt_volume_bricks_bytes(params))
        out = torch.empty(nbytes // 8, dtype=torch.complex64, device=volume.device)
        _lib.check(L.tt_pack_volume_bricks(_lib.ptr(volume), _lib.ptr(out), params, st), "pack_volume_bricks")
        return out
    raise ValueError(f"unknown volume layout {layout}")


def pack_channels(volumes: torch.Tensor, params: _lib.SliceParams, layout: int) -> torch.Tensor | None:
    """The channels' bricked copies back to back, as the multichannel
    extraction takes them (one flat complex64 tensor), for ``layout`` =
    ``BRICKS``; None for ``PLAIN`` (the multichannel kernels take no
    x-paired copy)."""
    if layout == PLAIN:
        return None
    if layout != BRICKS:
        raise ValueError("the multichannel extraction takes plain or bricked volumes")
    L = _lib.load()
    st = _lib.stream_of(volumes.device)
    slots = int(L.tt_volume_bricks_bytes(params)) // 8
    out = torch.empty((volumes.shape[0], slots), dtype=torch.complex64, device=volumes.device)
    for ch in range(volumes.shape[0]):
        _lib.check(L.tt_pack_volume_bricks(_lib.ptr(volumes[ch]), _lib.ptr(out[ch]), params, st),
                   "pack_volume_bricks")
    return out
