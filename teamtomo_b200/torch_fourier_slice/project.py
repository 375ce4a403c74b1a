"""Real-space projection (drop-in for torch_fourier_slice.project_3d_to_2d).

Same steps as torch_fourier_slice/project.py:12-93 — pad, premultiply by
sinc^2, 3D rfft, central-slice extraction, 2D irfft, crop — with the fftshift
bookkeeping folded into the kernels' addressing: the padded, sinc^2-weighted
volume is written directly in FFT order by one kernel, the extraction reads
the unshifted rfftn output and writes rows already ifftshifted for the 2D
irfft, and one kernel recentres and crops the projections.
"""

from __future__ import annotations

import os
import threading
from collections import OrderedDict

import torch

from . import _wrappers
from ._params import rotation_arg, slice_params
from .slice_extraction import _ExtractCentralSlices, _ExtractMultichannel


def _pad_amount(n: int, pad_factor: float) -> int:
    return int((n * (pad_factor - 1.0)) // 2)


# float64 volumes: the padding, sinc^2 weighting and 3D rfft run in float64,
# the central slices are sampled from the complex64 rounding of that rfft (the
# extraction kernels sample complex64) and the projections are returned as
# float64.  The reference raises RuntimeError for float64 volumes (its
# grid_sample gets a float64 volume and float32 coordinates); projecting them
# is a deliberate extension.
def _slice_source(dft: torch.Tensor) -> torch.Tensor:
    if dft.dtype == torch.complex128:
        dft = dft.to(torch.complex64)
    return dft.contiguous()


def _out_dtype(volume: torch.Tensor) -> torch.dtype:
    return torch.float64 if volume.dtype == torch.float64 else torch.float32


# CUDA-graph replay of small projections.  A projection of a small volume is
# a chain of about ten short kernels (the padding / sinc^2 pass, the 3D rfft,
# the extraction, the 2D inverse FFTs, the crop) whose host-side launch cost
# exceeds their GPU time: 64^3 at pad 2, 100 rotations took 220 us per call
# eagerly and 122 us as one graph replay on a B200.  Calls without autograd on
# small volumes therefore replay a graph captured once per (device, shapes,
# dtypes, arguments), copying the inputs into its static buffers and cloning
# the output; ``TT_PROJECT_GRAPHS=0`` turns this off.
_GRAPH_MAX_DFT_BYTES = 64 << 20  # padded rfft size up to which calls are graph-replayed
_GRAPH_CACHE_SIZE = 8
_graphs: "OrderedDict[tuple, _ProjectionGraph]" = OrderedDict()
_graphs_lock = threading.Lock()


class _ProjectionGraph:
    """One captured projection with its static input / output buffers."""

    def __init__(self, volume, R, kwargs):
        self.volume = torch.empty_like(volume, memory_format=torch.contiguous_format)
        self.R = torch.empty_like(R, memory_format=torch.contiguous_format)
        self.volume.copy_(volume)
        self.R.copy_(R)
        side = torch.cuda.Stream(device=volume.device)
        side.wait_stream(torch.cuda.current_stream(volume.device))
        with torch.cuda.stream(side):  # warm-up outside capture: FFT plans, library loading
            for _ in range(2):
                _project_eager(self.volume, self.R, **kwargs)
        torch.cuda.current_stream(volume.device).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        # thread-local: CUDA calls other threads make meanwhile are not part of the capture
        with torch.cuda.graph(self.graph, capture_error_mode="thread_local"):
            self.out = _project_eager(self.volume, self.R, **kwargs)
        self.done = None  # event after the last replay's output copy

    def __call__(self, volume, R):
        stream = torch.cuda.current_stream(volume.device)
        if self.done is not None:  # an earlier call on another stream may still read the buffers
            stream.wait_event(self.done)
        self.volume.copy_(volume)
        self.R.copy_(R)
        self.graph.replay()
        out = self.out.clone()
        self.done = torch.cuda.Event()
        self.done.record(stream)
        return out


def _graph_eligible(volume, R, n_pad) -> bool:
    if os.environ.get("TT_PROJECT_GRAPHS", "1").strip().lower() in ("0", "off", "false", "no"):
        return False
    if not (volume.is_cuda and R.is_cuda) or volume.device != R.device:
        return False
    if torch.is_grad_enabled() and (volume.requires_grad or R.requires_grad):
        return False
    if torch.cuda.is_current_stream_capturing():
        return False
    return n_pad * n_pad * (n_pad // 2 + 1) * 8 <= _GRAPH_MAX_DFT_BYTES


def project_3d_to_2d(
    volume: torch.Tensor,
    rotation_matrices: torch.Tensor,
    pad_factor: float = 2.0,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
) -> torch.Tensor:
    """Project a cubic volume by sampling central slices through its DFT.

    ``volume`` (d, d, d) float32 or float64; ``rotation_matrices`` (..., 3, 3);
    returns (..., d, d) projections in the volume's dtype (float64 volumes are
    sampled in single precision).  Differentiable w.r.t. volume and rotations."""
    d, h, w = volume.shape[-3:]
    if len({d, h, w}) != 1:
        raise ValueError("all dimensions of volume must be equal.")
    if pad_factor < 1.0:
        raise ValueError("pad_factor must be >= 1.0")
    kwargs = dict(pad_factor=pad_factor, fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices)
    p = _pad_amount(volume.shape[-1], pad_factor) if pad_factor > 1.0 else 0
    R_in = torch.as_tensor(rotation_matrices)
    if _graph_eligible(volume, R_in, d + 2 * p):
        key = (volume.device, tuple(volume.shape), volume.dtype, tuple(R_in.shape), R_in.dtype,
               float(pad_factor), fftfreq_max, bool(zyx_matrices), os.environ.get("TT_VOLUME_LAYOUT", "auto"))
        with _graphs_lock:
            entry = _graphs.get(key)
            if entry is None:
                entry = _ProjectionGraph(volume, R_in, kwargs)
                _graphs[key] = entry
                while len(_graphs) > _GRAPH_CACHE_SIZE:
                    _graphs.popitem(last=False)
            else:
                _graphs.move_to_end(key)
            return entry(volume, R_in)
    return _project_eager(volume, rotation_matrices, **kwargs)


def _project_eager(volume, rotation_matrices, pad_factor, fftfreq_max, zyx_matrices):
    d = volume.shape[-1]
    p = _pad_amount(volume.shape[-1], pad_factor) if pad_factor > 1.0 else 0
    n_pad = d + 2 * p
    shape = (n_pad, n_pad, n_pad)
    fft_in = _wrappers.project_prepare(volume, p)  # padded * sinc^2, fftshifted
    # unshifted rfft; cuFFT may hand back a non-contiguous layout
    dft = _slice_source(torch.fft.rfftn(fft_in, dim=(-3, -2, -1)))
    R, stack = rotation_arg(rotation_matrices, volume.device)
    params = slice_params(n=R.shape[0], image_shape=shape, volume=dft, rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          rot_tolerance=1e-8, volume_unshifted=True, slices_unshifted=True)
    slices = _ExtractCentralSlices.apply(dft, R, params, (R.shape[0], n_pad, n_pad // 2 + 1))
    # irfftn without an output size, as the reference: an odd padded box
    # gives images one column narrower (2 * (n_pad // 2) wide)
    images = _wrappers.irfftn_last(slices, 2)
    out = _wrappers.recentre_crop_2d(images, p).to(_out_dtype(volume))
    return out.reshape(*stack, *out.shape[-2:])


def project_3d_to_2d_multichannel(
    volume: torch.Tensor,
    rotation_matrices: torch.Tensor,
    pad_factor: float = 2.0,
    fftfreq_max: float | None = None,
    zyx_matrices: bool = False,
) -> torch.Tensor:
    """(c, d, d, d) -> (..., c, d, d): every channel projected with the same
    rotations, one multichannel extraction for all channels."""
    c, d, h, w = volume.shape[-4:]
    if len({d, h, w}) != 1:
        raise ValueError("all dimensions of volume must be equal.")
    if pad_factor < 1.0:
        raise ValueError("pad_factor must be >= 1.0")
    p = _pad_amount(d, pad_factor) if pad_factor > 1.0 else 0
    n_pad = d + 2 * p
    shape = (n_pad, n_pad, n_pad)
    fft_in = torch.stack([_wrappers.project_prepare(volume[ch], p) for ch in range(c)])
    dft = _slice_source(torch.fft.rfftn(fft_in, dim=(-3, -2, -1)))
    R, stack = rotation_arg(rotation_matrices, volume.device)
    params = slice_params(n=R.shape[0], image_shape=shape, volume=dft[0], rotation=R,
                          fftfreq_max=fftfreq_max, zyx_matrices=zyx_matrices,
                          rot_tolerance=1e-8, volume_unshifted=True, slices_unshifted=True)
    slices = _ExtractMultichannel.apply(dft, R, params, (R.shape[0], c, n_pad, n_pad // 2 + 1))
    images = _wrappers.irfftn_last(slices, 2)
    out = _wrappers.recentre_crop_2d(images.reshape(-1, *images.shape[-2:]), p).to(_out_dtype(volume))
    return out.reshape(*stack, c, *out.shape[-2:])
