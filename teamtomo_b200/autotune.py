"""Tile-shape and volume-layout autotuner for the batched slice kernels.

The batched kernels are compiled for three tile shapes (8x32, 16x16 and 32x8
pixels per 256-thread block), and the batched extraction gathers either from
the volumes themselves or from their 2 x 2 x 2 bricked copies.  Which
combination is fastest depends on the box size (how a warp's pixels spread
over the volume's cache lines).  ``tune`` times every combination on
synthetic data of a given box size with CUDA events and records the winner in
a JSON cache keyed by (GPU name, kind, box); the batched API looks the cache
up (``cached_tile_shape``, ``cached_layout``) and falls back to 8x32 (shape 0)
and the pixels-per-voxel layout policy for box sizes never tuned.

Cache file: ``$TT_AUTOTUNE_CACHE`` or ``~/.cache/teamtomo_b200/autotune.json``.
"""

from __future__ import annotations

import json
import os
import threading

import torch

TILE_SHAPES = {0: (8, 32), 1: (16, 16), 2: (32, 8)}
DEFAULT_TILE_SHAPE = 0
_lock = threading.Lock()
_mem: dict[str, int] | None = None


def cache_path() -> str:
    return os.environ.get("TT_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "teamtomo_b200", "autotune.json"))


def _key(kind: str, box: int, device) -> str:
    return f"{torch.cuda.get_device_name(device)}:{kind}:{int(box)}"


def _load() -> dict[str, int]:
    global _mem
    if _mem is None:
        try:
            with open(cache_path()) as f:
                _mem = {k: int(v) for k, v in json.load(f).items()}
        except (OSError, ValueError):
            _mem = {}
    return _mem


def _save() -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(_load(), f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only loses the cache, not the result


def cached_tile_shape(kind: str, box: int, device) -> int:
    with _lock:
        return _load().get(_key(kind, box, device), DEFAULT_TILE_SHAPE)


def cached_layout(kind: str, box: int, device) -> int | None:
    """Tuned volume layout (0 plain, 2 bricked) of the batched extraction at
    this box size, or None when never tuned."""
    with _lock:
        return _load().get(_key(kind, box, device) + ":layout")


def tune(kind: str, box: int, n_slices: int = 512, device=None, repeats: int = 5) -> dict[int, float]:
    """Time every tile shape for `kind` ('extract' or 'insert') at box size
    `box`, store the fastest in the cache and return {shape: ms}."""
    from . import batched

    dev = torch.device(device or "cuda")
    # time the kernels where the per-call work (the bricked layout's pack, the
    # insertion's accumulator zeroing and finalize) is amortised as in use:
    # four slice pixels per voxel or more (with 256 slices of a 256^3 box the
    # insertion's fixed costs hid a 3 % difference between tile shapes)
    n_slices = max(n_slices, 4 * box)
    g = torch.Generator(device=dev).manual_seed(box)
    shape3 = (box, box, box // 2 + 1)
    R = torch.linalg.qr(torch.randn((n_slices, 3, 3), device=dev, generator=g))[0].contiguous()
    ctf = batched.ctf_params(1.5, n=n_slices, device=dev)
    layouts = (None,)
    if kind == "extract":
        vol = torch.randn(shape3, dtype=torch.complex64, device=dev, generator=g)
        layouts = ("plain", "bricks")
        run = lambda ts, lay: batched.extract_central_slices_rfft_3d_batched(  # noqa: E731
            [vol], [R], ctf=[ctf], tile_shape=ts, volume_layout=lay)
    elif kind == "insert":
        img = torch.randn((n_slices, box, box // 2 + 1), dtype=torch.complex64, device=dev, generator=g)
        run = lambda ts, lay: batched.insert_central_slices_rfft_3d_batched(  # noqa: E731
            [img], [R], ctf=[ctf], tile_shape=ts)
    else:
        raise ValueError("kind must be 'extract' or 'insert'")
    times = {}
    for lay in layouts:
        for ts in TILE_SHAPES:
            run(ts, lay)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(dev)
            start.record()
            for _ in range(repeats):
                run(ts, lay)
            end.record()
            torch.cuda.synchronize(dev)
            times[(ts, lay)] = start.elapsed_time(end) / repeats
    best_ts, best_lay = min(times, key=times.get)
    with _lock:
        _load()[_key(kind, box, dev)] = best_ts
        if best_lay is not None:
            _load()[_key(kind, box, dev) + ":layout"] = 2 if best_lay == "bricks" else 0
        _save()
    return times
