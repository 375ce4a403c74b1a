#!/usr/bin/env python
"""Throughput of the Fourier-slice hot path on B200: extract + insert + backward.

Workload (one "step", the 256^3 differentiation configuration):
  * volume: 256^3 real Gaussian-blob volume (20 blobs, sigma U(2,6)*4 px,
    centres uniform in a ball of radius 96, + N(0, 0.01^2)), seeded, as its
    fftshifted rfft, complex64 (256, 256, 129);
  * 4096 rotation matrices drawn uniformly on SO(3)
    (scipy special_ortho_group, random_state=1003);
  * targets: central slices of a second blob volume plus complex white noise;
  * step = extract_central_slices_rfft_3d (forward) -> MSE loss against the
    targets -> backward (d/dvolume via the insert-adjoint scatter and
    d/drotation, one fused kernel) -> insert_central_slices_rfft_3d of the
    targets into a fresh (volume, weights) pair.
  slices/s = 4096 / step time.  Synthetic data stand in for the reference's
  simulated maps (no network, no dataset).

--impl reference times the reference's own torch code (baseline/_ref,
unmodified) on the host CPU cores on a bounded sample of the same workload,
with the same metric and unit (the oracle's C restatement stands in when
baseline/_ref is absent).

Prints ONE JSON line (rank 0).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "slices/s extract+insert+bwd @256³ fp32 vs plain torch-GPU; % HBM roofline"
UNIT = "slices/s"
N_BOX = 256
N_SLICES = 4096
ROT_SEED = 1003
WORKLOAD = ("extract_central_slices_rfft_3d fwd + MSE vs noisy targets + bwd (d/dvolume, "
            "d/drotation) + insert_central_slices_rfft_3d of the targets; 256^3 complex64 rfft "
            "volume (256x256x129), 4096 seeded SO(3) rotations")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--box", type=int, default=N_BOX)
    ap.add_argument("--slices", type=int, default=N_SLICES)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fused", action="store_true", help="skip the fused-MSE leg")
    ap.add_argument("--no-torch-gpu", action="store_true", help="skip timing the reference's torch code on the GPU")
    ap.add_argument("--torch-gpu-sample", type=int, default=512, help="slices timed on the reference's torch path")
    ap.add_argument("--e2e-chunk", type=int, default=256, help="slices per streamed chunk in the e2e leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-probe", action="store_true", help="skip the L2 reduction-rate probe")
    ap.add_argument("--cpu-sample", type=int, default=1024, help="slices of the oracle-port CPU sample")
    ap.add_argument("--ref-cpu-sample", type=int, default=32,
                    help="slices of the reference-torch-on-CPU sample (cpu_baseline)")
    ap.add_argument("--deterministic", action="store_true",
                    help="64-bit fixed-point insertion and volume gradient (bit-reproducible)")
    ap.add_argument("--case", choices=KERNEL_CASES, default=None,
                    help="with --workload kernels: run only this case")
    ap.add_argument("--workload", choices=["differentiation", "batched", "project", "backproject", "fullscale",
                                           "kernels"],
                    default="differentiation",
                    help="differentiation: the 256^3 extract+insert+bwd step (headline); batched: 32 "
                         "uneven CTF-weighted volumes in one graph-captured launch per stage")
    return ap.parse_args()


# ----------------------------------------------------------------------------
# synthetic data
# ----------------------------------------------------------------------------

def rotations(n: int, seed: int) -> np.ndarray:
    from scipy.stats import special_ortho_group

    return special_ortho_group.rvs(3, size=n, random_state=seed).reshape(n, 3, 3).astype(np.float32)


def blob_volume_torch(n: int, seed: int, device):
    import torch

    rng = np.random.default_rng(seed)
    ax = torch.arange(n, device=device, dtype=torch.float32)
    vol = torch.zeros((n, n, n), device=device, dtype=torch.float32)
    for _ in range(20):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        c = n / 2 + u * 0.375 * n * rng.uniform() ** (1.0 / 3.0)
        s = rng.uniform(2, 6) * n / 64
        g = [torch.exp(-((ax - float(c[i])) ** 2) / (2 * s * s)) for i in range(3)]
        vol += g[0][:, None, None] * g[1][None, :, None] * g[2][None, None, :]
    gen = torch.Generator(device=device).manual_seed(seed)
    vol += 0.01 * torch.randn(vol.shape, device=device, generator=gen)
    return vol


def rfft_volume_torch(vol):
    import torch

    f = torch.fft.rfftn(torch.fft.fftshift(vol, dim=(-3, -2, -1)), dim=(-3, -2, -1))
    return torch.fft.fftshift(f, dim=(-3, -2)).contiguous()


# ----------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# CPU legs: the reference's own torch code on the host cores (the reported
# baseline) and the oracle's C restatement of it (a second figure)
# ----------------------------------------------------------------------------

REF_DIR = os.path.join(ROOT, "baseline", "_ref")


def reference_modules():
    """The unmodified reference slice functions from baseline/_ref (placed
    there by baseline/install_reference.py), or None when absent."""
    if not os.path.isdir(os.path.join(REF_DIR, "torch_fourier_slice")):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    from torch_fourier_slice import extract_central_slices_rfft_3d as ref_extract
    from torch_fourier_slice import insert_central_slices_rfft_3d as ref_insert

    return ref_extract, ref_insert


def reference_ctf():
    """calculate_ctf_2d of the reference's torch-ctf from baseline/_ref, or None."""
    if not os.path.isdir(os.path.join(REF_DIR, "torch_ctf")):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    from torch_ctf import calculate_ctf_2d

    return calculate_ctf_2d


def reference_ctf_images(calc, rows, box):
    """(n, box, box//2+1) CTF images of the reference's calculate_ctf_2d
    (rfft, fftshifted) for (n, 8) rows of batched.ctf_params.  Each argument
    goes in as its own copy: calculate_ctf_2d subtracts the astigmatism from
    its defocus argument in place, which on views of one rows tensor also
    corrupts the other columns it reads."""
    c = rows.detach().float()
    col = lambda i: c[:, i].clone()  # noqa: E731
    return calc(defocus=col(0), astigmatism=col(1), astigmatism_angle=col(2), voltage=col(3),
                spherical_aberration=col(4), amplitude_contrast=col(5), phase_shift=col(6),
                pixel_size=col(7), image_shape=(box, box), rfft=True, fftshift=True)


def reference_ctf_insert(mods, calc, images, R, rows, box):
    """CTF-weighted insertion in the reference's own code: the CTF images,
    then one insertion of images x CTF (the volume) and one of CTF^2 (whose
    real part is the weights); the rotations go in as a copy (the reference
    zeroes near-zero elements of its argument in place)."""
    import torch

    _, ref_insert = mods
    shape = (box, box, box)
    with torch.no_grad():
        ctf = reference_ctf_images(calc, rows, box)
        v, _ = ref_insert(images * ctf, shape, R.clone())
        w, _ = ref_insert((ctf * ctf).to(images.dtype), shape, R.clone())
    return v, w.real


def reference_ctf_extract_insert(mods, calc, vol, R, rows, box):
    """One volume of the batched step in the reference's own code: CTF
    images, the CTF-weighted extraction, then the CTF-weighted insertion of
    those slices."""
    import torch

    ref_extract, _ = mods
    with torch.no_grad():
        ctf = reference_ctf_images(calc, rows, box)
        S = ref_extract(vol, (box, box, box), R.clone()) * ctf
    return reference_ctf_insert(mods, calc, S, R, rows, box)


def reference_extract_fwd_bwd(mods, V, R, T, box):
    """Extraction, MSE against T and the autograd backward for d/drotation in
    the reference's own code (d/dvolume left out: its autograd expands the
    volume per sample point)."""
    ref_extract, _ = mods
    Rg = R.double().clone().requires_grad_(True)
    S = ref_extract(V, (box, box, box), Rg)
    (S - T).abs().square().mean().backward()


def _host_seconds(fn, warm=None):
    """Wall time of fn() on the host (one untimed call of warm() first)."""
    if warm is not None:
        warm()
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


def cpu_workload(box, sample, mods, seed=ROT_SEED):
    """The GPU arm's workload on the host: the same seeded blob volumes, the
    first ``sample`` of its 4096 rotations, targets = central slices of the
    second volume (taken with the reference's extraction when ``mods`` holds
    it, else with the oracle port) plus complex noise at the same relative
    level.  Input preparation, outside every timed region."""
    import torch

    cpu = torch.device("cpu")
    V0 = rfft_volume_torch(blob_volume_torch(box, seed, cpu))
    Vt = rfft_volume_torch(blob_volume_torch(box, seed + 1000, cpu))
    R = torch.tensor(rotations(N_SLICES, seed)[:sample])
    if mods is not None:
        with torch.no_grad():
            T = mods[0](Vt, (box, box, box), R.double())
    else:
        from oracle import oracle as O

        T = torch.from_numpy(O.extract(Vt.numpy(), (box, box, box), R.numpy(), nthreads=os.cpu_count() or 1))
    gen = torch.Generator().manual_seed(7)
    T = T + 0.5 * T.abs().mean() * torch.randn(T.shape, dtype=T.dtype, generator=gen)
    return V0, R, T


def reference_cpu_step(mods, V0, R, T, box):
    """One sample step of the reference's own code on the CPU: extraction,
    the MSE against the targets, its autograd backward for d/drotation, and
    the insertion of the targets.  Its autograd w.r.t. the volume expands the
    volume per sample point (4.5 TB at 128^3 x 64 slices), so d/dvolume is
    left out; the rotations go in as float64 (the reference zeroes near-zero
    elements of its argument in place, which a float32 leaf refuses)."""
    ref_extract, ref_insert = mods
    shape = (box, box, box)
    Rg = R.double().clone().requires_grad_(True)
    S = ref_extract(V0, shape, Rg)
    loss = (S - T).abs().square().mean()
    loss.backward()
    ref_insert(T, shape, Rg.detach())


def port_cpu_step(O, vol_np, rots_np, targets_np, nthreads):
    """One bounded sample of the oracle's C restatement: extract + grad
    (dV, dR) + insert."""
    n = vol_np.shape[0]
    s = O.extract(vol_np, (n, n, n), rots_np, nthreads=nthreads)
    g = (2.0 / s.size) * (s - targets_np)
    O.extract_grad(vol_np, (n, n, n), rots_np, g.astype(np.complex64), nthreads=nthreads)
    O.insert(targets_np, (n, n, n), rots_np, nthreads=nthreads)


def run_port_baseline(V0, R, T, repeats=1):
    from oracle import oracle as O

    O.lib()
    threads = os.cpu_count() or 1
    vol, rots, tg = V0.numpy(), R.numpy(), T.numpy()
    port_cpu_step(O, vol, rots[:4], tg[:4], threads)  # warm
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        port_cpu_step(O, vol, rots, tg, threads)
        times.append(time.perf_counter() - t0)
    t = min(times)
    return {"value": len(rots) / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(rots)} slices of the {vol.shape[0]}^3 step (extract + dV/dR + insert), oracle C "
                      f"restatement, OpenMP {threads} threads, best of {repeats}"}


def run_cpu_baseline(box, ref_sample, port_sample):
    """cpu_baseline of the GPU arm's line: the reference's torch code on the
    host cores (kind "reference"), with the oracle port beside it."""
    import torch

    mods = reference_modules()
    V0, R, T = cpu_workload(box, max(ref_sample, port_sample), mods)
    port = run_port_baseline(V0, R[:port_sample], T[:port_sample])
    if mods is None:
        port["reference"] = {"unavailable": "baseline/_ref missing (run baseline/install_reference.py)"}
        return port
    reference_cpu_step(mods, V0, R[:2], T[:2], box)  # warm
    t0 = time.perf_counter()
    reference_cpu_step(mods, V0, R[:ref_sample], T[:ref_sample], box)
    t = time.perf_counter() - t0
    return {"value": ref_sample / t, "unit": UNIT, "cores": torch.get_num_threads(), "kind": "reference",
            "host_cpus": os.cpu_count(),
            "sample": f"{ref_sample} of the 4096 slices of the {box}^3 step: the reference's torch code "
                      f"(baseline/_ref, unmodified) on the CPU, extraction + MSE + autograd d/drotation + "
                      f"insertion; d/dvolume excluded (the reference's autograd expands the volume per point)",
            "port": port}


def reference_arm(args):
    """--impl reference: the reference's own torch code on the host cores,
    every step a bounded sample of the 4096-slice step sized so that the
    whole run stays within about two minutes (the oracle port stands in when
    baseline/_ref is absent)."""
    import torch

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    mods = reference_modules()
    probe = 2
    V0, R, T = cpu_workload(args.box, 64, mods)
    if mods is not None:
        kind, threads = "reference", torch.get_num_threads()

        def step(k):
            reference_cpu_step(mods, V0, R[:k], T[:k], args.box)
    else:
        from oracle import oracle as O

        O.lib()
        kind, threads = "port", os.cpu_count() or 1
        vol, rots, tg = V0.numpy(), R.numpy(), T.numpy()

        def step(k):
            port_cpu_step(O, vol, rots[:k], tg[:k], threads)
    t0 = time.perf_counter()
    step(probe)
    per_slice = (time.perf_counter() - t0) / probe
    total_steps = max(args.steps, 1) + max(args.warmup, 0)
    sample = int(max(2, min(64, 120.0 / total_steps / max(per_slice, 1e-6))))
    for _ in range(args.warmup):
        step(sample)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(sample)
    dt = time.perf_counter() - t0
    value = sample * args.steps / dt
    what = ("the reference's torch code (baseline/_ref, unmodified) on the CPU: extraction + MSE + autograd "
            "d/drotation + insertion; d/dvolume excluded (the reference's autograd expands the volume per "
            "point)") if kind == "reference" else "oracle C restatement (baseline/_ref absent), OpenMP"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "box": args.box, "slices_per_step": sample,
                   "note": "each step is a bounded sample of the 4096-slice step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "host_cpus": os.cpu_count(),
                         "sample": f"{sample} slices per step of the {args.box}^3 step: {what}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------

def torch_gpu_reference(dev, n, V0, R0, T, sample, chunk=128):
    """The reference's own torch code (baseline/_ref, unmodified, placed there
    by baseline/install_reference.py) run on the GPU for the same step:
    extraction, the same MSE, its autograd backward for d/drotation, and the
    insertion of the targets (partial volumes summed), chunked over slices.
    Its autograd w.r.t. the volume expands the volume per sample (4.5 TB at
    128^3 x 64 slices), so d/dvolume is left out of this leg."""
    import torch

    mods = reference_modules()
    if mods is None:
        return {"unavailable": "baseline/_ref missing (run baseline/install_reference.py where the reference is)"}
    ref_extract, ref_insert = mods

    shape = (n, n, n)
    sample = min(sample, R0.shape[0])
    Rs = R0[:sample].detach().double()  # a float32 leaf would be zeroed in place by the reference and raise

    def step():
        vol_sum = None
        for s0 in range(0, sample, chunk):
            R = Rs[s0:s0 + chunk].clone().requires_grad_(True)
            S = ref_extract(V0, shape, R)
            loss = (S - T[s0:s0 + chunk]).abs().square().mean()
            loss.backward()
            vol, w = ref_insert(T[s0:s0 + chunk], shape, R.detach())
            vol_sum = vol if vol_sum is None else vol_sum + vol
        return vol_sum

    step()
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 2
    a.record()
    for _ in range(reps):
        step()
    b.record()
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b) / reps
    return {"value": sample / (ms / 1e3), "unit": UNIT, "ms_per_sample": ms,
            "sample": f"{sample} of the 4096 slices, chunks of {chunk}, volume without grad",
            "excluded": "d/dvolume (the reference's autograd expands the volume per sample)",
            "code": "reference torch_fourier_slice, unmodified, CUDA tensors"}


def l2_reduction_ceiling(dev, n, R, insert_ms, reps=3):
    """The insertion's trilinear-corner reductions per second beside the L2's
    float4 reduction rate (tt_probe_l2_reductions) for the same number of
    reductions: eight lanes per 128-byte line on random lines of a buffer of
    the insertion accumulator's size and of one that fits the L2 (32 MB), and
    two lanes per line (the x-paired rows' pattern) on the accumulator-sized
    buffer.  The corner count is exact: every kept source pixel whose point
    lies inside the volume adds its corners of non-zero weight (an axis whose
    coordinate is an integer has one).  Outside the timed region."""
    import ctypes

    import torch

    from teamtomo_b200 import _lib
    from teamtomo_b200.torch_fourier_slice import slice_extraction as se
    from teamtomo_b200.torch_fourier_slice._params import rfft_shape, slice_params

    L = _lib.load()
    shape = (n, n, n)
    dims = rfft_shape(shape)
    count = 0
    for i in range(0, R.shape[0], 256):
        flags, c = se.central_slice_geometry(R[i:i + 256], shape, dims, mode="insert")
        ok = ((flags & 1) != 0) & ((flags & 4) != 0)
        corners = (1 + (c != torch.floor(c)).to(torch.int64)).prod(dim=-1)
        count += int((corners * ok).sum().item())
        del flags, c
    p = slice_params(n=R.shape[0], image_shape=shape, volume=None, rotation=R, vol_dims=dims)
    acc_bytes = int(L.tt_insert_workspace_bytes(0, ctypes.byref(p)))
    st = _lib.stream_of(dev)
    out = {"insert_corner_reductions": count,
           "insert_g_per_s": round(count / (insert_ms / 1e3) / 1e9, 1), "probe_g_per_s": {}}
    for label, nbytes, lanes in ((f"8 lanes/line, {acc_bytes >> 20} MiB", acc_bytes, 8),
                                 ("8 lanes/line, 32 MiB", 32 << 20, 8),
                                 (f"2 lanes/line, {acc_bytes >> 20} MiB", acc_bytes, 2)):
        buf = torch.zeros(nbytes // 4, dtype=torch.float32, device=dev)
        run = lambda: _lib.check(L.tt_probe_l2_reductions(_lib.ptr(buf), nbytes, count, lanes, 1234, st),  # noqa
                                 "probe_l2_reductions")
        ms = _time_device(run, reps, 1, dev)
        out["probe_g_per_s"][label] = round(count / (ms / 1e3) / 1e9, 1)
        del buf
    first = next(iter(out["probe_g_per_s"].values()))
    out["insert_over_probe_8_lanes_same_size"] = round(out["insert_g_per_s"] / first, 3)
    return out


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def copy_launches(n_pixels, volume):
    """1 when an extraction of n_pixels slice pixels (its forward and backward,
    or the fused MSE) gathers from a copy of the volume (one pack launch),
    else 0."""
    from teamtomo_b200.torch_fourier_slice import _layout

    return int(_layout.choose(n_pixels, volume) != _layout.PLAIN)


def load_traffic():
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


BATCH_BOXES = (64, 96, 128, 160, 200, 256)


def batched_workload(args):
    """32 volumes, box sizes drawn from BATCH_BOXES, 500-20,000 rotations each,
    per-image CTF (defocus U(0.5, 3.0) um, 300 kV, Cs 2.7 mm, Ac 0.07, 1 A/px).
    One step = CTF-weighted extraction of every slice of every volume (one
    persistent launch) + CTF-weighted insertion of those slices into fresh
    volumes (one launch + per-volume finalize), replayed from one CUDA graph."""
    import torch

    from teamtomo_b200 import autotune, batched

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(1004)
    nvol = 32
    boxes = [int(b) for b in rng.choice(BATCH_BOXES, size=nvol)]
    counts = [int(c) for c in rng.integers(500, 20001, size=nvol)]
    vols = [rfft_volume_torch(blob_volume_torch(b, 2000 + i, dev)) for i, b in enumerate(boxes)]
    rots = [torch.tensor(rotations(c, 3000 + i), device=dev) for i, c in enumerate(counts)]
    ctfs = [batched.ctf_params(rng.uniform(0.5, 3.0, c), voltage_kv=300.0, spherical_aberration_mm=2.7,
                               amplitude_contrast=0.07, pixel_size_a=1.0, device=dev) for c in counts]
    tuned = {}
    for kind in ("extract", "insert"):
        for b in sorted(set(boxes)):
            tuned[f"{kind}:{b}"] = autotune.tune(kind, b, n_slices=256, device=dev, repeats=3)
    ts_e = autotune.cached_tile_shape("extract", max(boxes), dev)
    ts_i = autotune.cached_tile_shape("insert", max(boxes), dev)

    def step():
        slices = batched.extract_central_slices_rfft_3d_batched(vols, rots, ctf=ctfs, tile_shape=ts_e)
        return batched.insert_central_slices_rfft_3d_batched(slices, rots, ctf=ctfs, tile_shape=ts_i)

    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        step()
    torch.cuda.current_stream(dev).wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        outs = step()
    for _ in range(max(args.warmup, 0)):
        graph.replay()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev.index)
    clocks.start()
    time.sleep(0.3)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        graph.replay()
    end.record()
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    ms = start.elapsed_time(end) / args.steps
    total = sum(counts)
    P = [b * (b // 2 + 1) for b in boxes]
    vox = [b * b * (b // 2 + 1) for b in boxes]
    # extraction writes 8P per slice + reads the volume once; insertion reads 8P
    # per slice + writes volume and weights once
    algo_e = sum(c * 8 * p for c, p in zip(counts, P)) + sum(8 * v for v in vox)
    algo_i = sum(c * 8 * p for c, p in zip(counts, P)) + sum(12 * v for v in vox)
    algo = algo_e + algo_i
    peak, peak_kind = load_peaks()
    gbs = algo / (ms / 1e3) / 1e9
    # DRAM traffic: the ncu captures' traffic per algorithmic byte of each stage
    # (8 volumes x 2000 slices, profiles/ncu_batched_*), scaled to this step
    tr = load_traffic()
    re_, ri_ = tr.get("batched_extract_per_algorithmic_byte"), tr.get("batched_insert_per_algorithmic_byte")
    traffic = int(re_ * algo_e + ri_ * algo_i) if re_ and ri_ else None
    ref_gpu, ref_cpu = batched_reference_legs(args, dev, vols, rots, ctfs, boxes, counts)
    line = {
        "metric": "slices/s CTF-weighted extract+insert, 32 uneven volumes, one launch per stage",
        "value": total / (ms / 1e3), "unit": "slices/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched", "volumes": nvol, "boxes": boxes, "slices": counts,
                   "total_slices": total, "tile_shapes": {"extract": ts_e, "insert": ts_i},
                   "l2": "inputs larger than L2"},
        "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(gbs / peak, 4), "traffic": traffic, "kernel": "extract+insert step",
                     "peak_source": peak_kind,
                     "traffic_source": "ncu per-algorithmic-byte traffic of the batched stages at 8 volumes x "
                                       "2000 slices, scaled to this step's algorithmic bytes"},
        "autotune_ms": {k: {(f"{s[0]}/{s[1]}" if s[1] else str(s[0])): round(t, 4) for s, t in v.items()}
                        for k, v in tuned.items()},
        "clocks": clk, "gpu_launches": args.steps * (3 + nvol),
        "torch_gpu_reference": ref_gpu, "cpu_baseline": ref_cpu,
    }
    del outs
    print(json.dumps(line))
    return 0


def batched_reference_legs(args, dev, vols, rots, ctfs, boxes, counts, gpu_sample=256, cpu_sample=4):
    """The batched step in the reference's own code (per volume: CTF images,
    CTF-weighted extraction, CTF-weighted insertion as two insertions), timed
    on the first ``gpu_sample`` slices of every volume on this GPU and the
    first ``cpu_sample`` on the host cores; each volume's time is scaled
    linearly to its slice count and the rate is the step's slices over the
    sum.  Returns (torch_gpu_reference, cpu_baseline), None where skipped."""
    import torch

    mods, calc = reference_modules(), reference_ctf()
    if mods is None or calc is None:
        why = {"unavailable": "baseline/_ref missing (run baseline/install_reference.py)"}
        return why, why
    total = sum(counts)
    gpu = cpu = None
    if not args.no_torch_gpu:
        est = 0.0
        for v, r, c, b, n in zip(vols, rots, ctfs, boxes, counts):
            k = min(n, gpu_sample)
            fn = lambda: reference_ctf_extract_insert(mods, calc, v, r[:k], c[:k], b)  # noqa: E731
            est += _time_device(fn, 1, 1, dev) / 1e3 * n / k
        gpu = {"value": total / est, "unit": "slices/s",
               "sample": f"first {gpu_sample} slices of each volume (all of smaller ones), each volume's time "
                         "scaled linearly to its slice count (extrapolated)",
               "code": "reference torch_fourier_slice + torch_ctf, unmodified, CUDA tensors: calculate_ctf_2d, "
                       "extract x CTF, insert(slices x CTF) + insert(CTF^2) for the weights"}
    if not args.no_cpu_baseline:
        est = 0.0
        for v, r, c, b, n in zip(vols, rots, ctfs, boxes, counts):
            k = min(n, cpu_sample)
            vc, rc, cc = v.cpu(), r[:k].cpu(), c[:k].cpu()
            est += _host_seconds(lambda: reference_ctf_extract_insert(mods, calc, vc, rc, cc, b),
                                 warm=lambda: reference_ctf_extract_insert(mods, calc, vc, rc[:1], cc[:1], b)) * n / k
        cpu = {"value": total / est, "unit": "slices/s", "cores": torch.get_num_threads(), "kind": "reference",
               "host_cpus": os.cpu_count(),
               "sample": f"first {cpu_sample} slices of each volume on the host cores, each volume's time scaled "
                         "linearly to its slice count (extrapolated); the reference's torch code as in "
                         "torch_gpu_reference"}
    return gpu, cpu


def fullscale_reference_legs(args, dev, images, V, n, gpu=(256, 256), cpu=(16, 8)):
    """The full-scale workload in the reference's own code on a prefix:
    the CTF-weighted insertion (CTF images, insert(images x CTF),
    insert(CTF^2) for the weights) of the first images, and the extraction
    with MSE and autograd d/drotation (d/dvolume left out) of the first
    orientations, on this GPU (``gpu`` = images, orientations) and on the
    host cores (``cpu``); rates per image / orientation, extrapolated
    linearly to the workload.  Returns (torch_gpu_reference, cpu_baseline)."""
    import torch

    mods, calc = reference_modules(), reference_ctf()
    if mods is None or calc is None:
        why = {"unavailable": "baseline/_ref missing (run baseline/install_reference.py)"}
        return why, why
    R, ctf, S = images(0, max(gpu))
    out_gpu = out_cpu = None
    if not args.no_torch_gpu:
        ni, ne = gpu
        ti = _time_device(lambda: reference_ctf_insert(mods, calc, S[:ni], R[:ni], ctf[:ni], n), 1, 1, dev)
        te = _time_device(lambda: reference_extract_fwd_bwd(mods, V, R[:ne], S[:ne], n), 1, 1, dev)
        out_gpu = {"value": ni / (ti / 1e3), "unit": "images/s",
                   "extract_fwd_bwd": {"value": ne / (te / 1e3), "unit": "slices/s",
                                       "excluded": "d/dvolume (the reference's autograd expands the volume per "
                                                   "sample point)"},
                   "sample": f"first {ni} images / {ne} orientations, extrapolated linearly",
                   "code": "reference torch_fourier_slice + torch_ctf, unmodified, CUDA tensors"}
    if not args.no_cpu_baseline:
        ni, ne = cpu
        Vc, Rc, Sc, Cc = V.cpu(), R[:max(cpu)].cpu(), S[:max(cpu)].cpu(), ctf[:max(cpu)].cpu()
        ti = _host_seconds(lambda: reference_ctf_insert(mods, calc, Sc[:ni], Rc[:ni], Cc[:ni], n),
                           warm=lambda: reference_ctf_insert(mods, calc, Sc[:1], Rc[:1], Cc[:1], n))
        te = _host_seconds(lambda: reference_extract_fwd_bwd(mods, Vc, Rc[:ne], Sc[:ne], n),
                           warm=lambda: reference_extract_fwd_bwd(mods, Vc, Rc[:1], Sc[:1], n))
        out_cpu = {"value": ni / ti, "unit": "images/s", "cores": torch.get_num_threads(), "kind": "reference",
                   "host_cpus": os.cpu_count(),
                   "extract_fwd_bwd": {"value": ne / te, "unit": "slices/s"},
                   "sample": f"first {ni} images / {ne} orientations on the host cores, extrapolated linearly; "
                             "the reference's torch code as in torch_gpu_reference (d/dvolume left out)"}
    return out_gpu, out_cpu


def _ref_module():
    """The reference's torch_fourier_slice from baseline/_ref, or None."""
    ref_dir = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref_dir, "torch_fourier_slice")):
        return None
    if ref_dir not in sys.path:
        sys.path.insert(0, ref_dir)
    import torch_fourier_slice

    return torch_fourier_slice


def _time_device(fn, steps, warmup, dev):
    import torch

    for _ in range(max(warmup, 0)):
        fn()
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        fn()
    b.record()
    torch.cuda.synchronize(dev)
    return a.elapsed_time(b) / steps


def config_workload(args):
    """The other configurations of the path, one JSON line each:
    project     project_3d_to_2d of a 64^3 Gaussian-blob volume at 100 rotations (pad 2.0)
    backproject backproject_2d_to_3d of 10,000 128^2 noisy projections (SNR 0.1), pad 1.0 and 2.0
    fullscale   CTF-weighted insertion of 200,000 320^2 noisy images (SNR 0.05, defocus U(0.8, 2.5) um)
                into a 320^3 volume, then 100,000-orientation extraction with forward + backward
                (fused MSE against the images), generated on the GPU chunk by chunk (82 GB of images)
    Each times our path with CUDA events and, where the reference can run on this GPU, the
    reference's own torch code (baseline/_ref) on a bounded sample."""
    import torch

    import teamtomo_b200 as tt

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    ref = _ref_module()
    peak, peak_kind = load_peaks()
    clocks = ClockSampler(dev.index)
    out = {"n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    if args.workload == "project":
        n, k = 64, 100
        vol = blob_volume_torch(n, 1001, dev)
        R = torch.tensor(rotations(k, 1001), device=dev)
        clocks.start()
        ms = _time_device(lambda: tt.project_3d_to_2d(vol, R), args.steps, args.warmup, dev)
        clk = clocks.stop()
        ref_ms = (_time_device(lambda: ref.project_3d_to_2d(vol, R), 5, 2, dev) if ref else None)
        cpu = None
        if ref is not None and not args.no_cpu_baseline:
            vc, Rc = vol.cpu(), R.cpu()
            t = _host_seconds(lambda: ref.project_3d_to_2d(vc, Rc), warm=lambda: ref.project_3d_to_2d(vc, Rc[:2]))
            cpu = {"value": k / t, "unit": "slices/s", "cores": torch.get_num_threads(), "kind": "reference",
                   "host_cpus": os.cpu_count(), "sample": f"the whole workload ({k} rotations), reference "
                   "project_3d_to_2d (baseline/_ref, unmodified) on the host cores"}
        out.update({"metric": "slices/s project_3d_to_2d 64^3 pad 2.0", "value": k / (ms / 1e3), "unit": "slices/s",
                    "ms_per_step": ms, "config": {"workload": "project 64^3 x 100 rotations, pad 2.0"},
                    "torch_gpu_reference": None if ref is None else {"value": k / (ref_ms / 1e3), "ms": ref_ms},
                    "cpu_baseline": cpu, "clocks": clk, "gpu_launches": 4 * args.steps})
    elif args.workload == "backproject":
        n, k = 128, 10_000
        vol = blob_volume_torch(n, 1002, dev)
        R = torch.tensor(rotations(k, 1002), device=dev)
        with torch.no_grad():
            proj = torch.cat([tt.project_3d_to_2d(vol, R[i:i + 1000]) for i in range(0, k, 1000)])
            gen = torch.Generator(device=dev).manual_seed(1002)
            noise = torch.randn(proj.shape, device=dev, generator=gen) * (proj.var() / 0.1).sqrt()
            imgs = (proj + noise).contiguous()
        del proj, noise
        res = {}
        clocks.start()
        for pf in (1.0, 2.0):
            ms = _time_device(lambda: tt.backproject_2d_to_3d(imgs, R, pad_factor=pf), args.steps, args.warmup,
                              dev)
            res[f"pad{pf:g}"] = {"value": k / (ms / 1e3), "ms_per_step": ms}
        clk = clocks.stop()
        refres = None
        if ref is not None:
            m = 1000  # bounded sample of the reference
            refres = {}
            for pf in (1.0, 2.0):
                rms = _time_device(lambda: ref.backproject_2d_to_3d(imgs[:m], R[:m], pad_factor=pf), 2, 1, dev)
                refres[f"pad{pf:g}"] = {"value": m / (rms / 1e3), "sample": m}
        cpu = None
        if ref is not None and not args.no_cpu_baseline:
            m = 100  # prefix of the images on the host cores, extrapolated linearly
            ic, Rc = imgs[:m].cpu(), R[:m].cpu()
            cpu = {"unit": "images/s", "cores": torch.get_num_threads(), "kind": "reference",
                   "host_cpus": os.cpu_count(),
                   "sample": f"first {m} of the {k} images on the host cores, extrapolated linearly; reference "
                             "backproject_2d_to_3d (baseline/_ref, unmodified); value at pad 1.0"}
            for pf in (1.0, 2.0):
                t = _host_seconds(lambda: ref.backproject_2d_to_3d(ic, Rc, pad_factor=pf),
                                  warm=lambda: ref.backproject_2d_to_3d(ic[:2], Rc[:2], pad_factor=pf))
                cpu[f"pad{pf:g}"] = m / t
            cpu["value"] = cpu["pad1"]
        out.update({"metric": "images/s backproject_2d_to_3d 10,000 x 128^2", "value": res["pad1"]["value"],
                    "unit": "images/s", "ms_per_step": res["pad1"]["ms_per_step"],
                    "config": {"workload": "backproject 10,000 x 128^2 (SNR 0.1); value at pad 1.0 "
                               "(128x128x65 volume), pad 2.0 beside it"},
                    "pads": res, "torch_gpu_reference": refres, "cpu_baseline": cpu, "clocks": clk,
                    "gpu_launches": 5 * args.steps})
    else:
        n, n_img, n_ext, chunk = 320, 200_000, 100_000, 10_000
        vol_real = blob_volume_torch(n, 1005, dev)
        V = rfft_volume_torch(vol_real)
        shape = (n, n, n)
        from teamtomo_b200 import batched

        def images(i0, m):
            """Chunk [i0, i0+m): rotations, CTF rows, noisy CTF-modulated slices of the map."""
            R = torch.tensor(rotations(m, 50_000 + i0), device=dev)
            rng = np.random.default_rng(60_000 + i0)
            ctf = batched.ctf_params(rng.uniform(0.8, 2.5, m), voltage_kv=300.0, spherical_aberration_mm=2.7,
                                     amplitude_contrast=0.07, pixel_size_a=1.0, device=dev)
            with torch.no_grad():
                S = batched.extract_central_slices_rfft_3d_batched([V], [R], ctf=[ctf])[0]
                gen = torch.Generator(device=dev).manual_seed(70_000 + i0)
                S = S + torch.randn(S.shape, dtype=S.dtype, device=dev, generator=gen) * (
                    S.abs().square().mean() / 0.05).sqrt()
            return R, ctf, S

        torch.cuda.synchronize(dev)
        ins_ms = ext_ms = 0.0
        vol_sum = w_sum = None
        clocks.start()
        for i0 in range(0, n_img, chunk):
            R, ctf, S = images(i0, chunk)
            torch.cuda.synchronize(dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            (v, w), = batched.insert_central_slices_rfft_3d_batched([S], [R], ctf=[ctf])
            vol_sum = v if vol_sum is None else vol_sum.add_(v)
            w_sum = w if w_sum is None else w_sum.add_(w)
            b.record()
            torch.cuda.synchronize(dev)
            ins_ms += a.elapsed_time(b)
        Vfit = (vol_sum / torch.clamp(w_sum, min=1.0)).detach().requires_grad_(True)
        for i0 in range(0, n_ext, chunk):
            R, ctf, S = images(i0, chunk)
            Rg = R.float().requires_grad_(True)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            tt.losses.central_slice_mse(Vfit, shape, Rg, S).backward()
            b.record()
            torch.cuda.synchronize(dev)
            ext_ms += a.elapsed_time(b)
        clk = clocks.stop()
        ref_gpu, ref_cpu = fullscale_reference_legs(args, dev, images, Vfit.detach(), n)
        out.update({"metric": "images/s CTF-weighted insertion, 320^3, 200,000 images; then slices/s extract "
                              "fwd+bwd, 100,000 orientations",
                    "value": n_img / (ins_ms / 1e3), "unit": "images/s", "ms_per_step": ins_ms + ext_ms,
                    "steps": 1, "warmup": 0,
                    "extract_fwd_bwd": {"value": n_ext / (ext_ms / 1e3), "unit": "slices/s", "ms": ext_ms},
                    "insert_ms": ins_ms,
                    "config": {"workload": "full scale: 320^3 complex64 rfft volume (320x320x161), "
                               f"images generated on the GPU in chunks of {chunk} (not timed)",
                               "images": n_img, "orientations": n_ext},
                    "torch_gpu_reference": ref_gpu, "cpu_baseline": ref_cpu, "clocks": clk,
                    # insertion: splat, finalize, sum; fused MSE: loss kernel, loss and rotation finish
                    # (+ the pack of the volume copy the gathers read)
                    "gpu_launches": n_img // chunk * 3
                    + n_ext // chunk * (3 + copy_launches(chunk * n * (n // 2 + 1), Vfit))})
    print(json.dumps(out))
    return 0


# ----------------------------------------------------------------------------
# per-kernel cases: one small invocation of each kernel, for ncu captures
# (``--workload kernels --case NAME``) and live per-kernel timings (all cases)
# ----------------------------------------------------------------------------

KERNEL_CASES = ("extract", "backward", "mse", "insert", "insert_bwd", "det_insert", "det_backward",
                "batched_extract", "batched_insert", "sample3d", "insert3d", "affine3d", "mc_extract",
                "mc_backward", "mc_insert", "lines", "project", "backproject", "pack_bricks")


def kernel_case(name, dev):
    """Inputs and one call of case ``name``: returns (fn, algorithmic bytes
    per call, the kernels the call launches).  Inputs exceed the L2 (126 MB)
    where the kernel's own data allow, but stay at a few GB on the device."""
    import torch

    import teamtomo_b200 as tt
    from teamtomo_b200 import batched as B
    from teamtomo_b200.torch_fourier_slice import _layout
    from teamtomo_b200.torch_fourier_slice._params import slice_params

    n, ns = 256, 512
    P, vox = n * (n // 2 + 1), n * n * (n // 2 + 1)
    shape = (n, n, n)
    gen = torch.Generator(device=dev).manual_seed(11)

    def crandn(*sh):
        return torch.randn(sh, dtype=torch.complex64, device=dev, generator=gen)

    V = rfft_volume_torch(blob_volume_torch(n, ROT_SEED, dev))
    R = torch.tensor(rotations(ns, ROT_SEED), device=dev)
    if name == "extract":
        return (lambda: tt.extract_central_slices_rfft_3d(V, shape, R)), ns * 8 * P + 8 * vox, \
            "pack_bricks_kernel, extract_fwd_kernel<VoxBrick2>"
    if name in ("backward", "det_backward"):
        Vg = V.clone().requires_grad_(True)
        Rg = R.clone().requires_grad_(True)
        G = crandn(ns, n, n // 2 + 1)
        det = name == "det_backward"

        def fn():
            Vg.grad = None
            Rg.grad = None
            S = tt.extract_central_slices_rfft_3d(Vg, shape, Rg, deterministic=det)
            S.backward(G)
        return fn, ns * 8 * P + 16 * vox, "extract_bwd_kernel (+ forward, pack, drot_finish)"
    if name == "mse":
        Vg = V.clone().requires_grad_(True)
        Rg = R.clone().requires_grad_(True)
        T = crandn(ns, n, n // 2 + 1)

        def fn():
            Vg.grad = None
            Rg.grad = None
            tt.losses.central_slice_mse(Vg, shape, Rg, T).backward()
        return fn, ns * 8 * P + 16 * vox, "slice_mse_kernel (+ pack, loss and drot finish)"
    if name in ("insert", "det_insert"):
        T = crandn(ns, n, n // 2 + 1)
        det = name == "det_insert"
        return (lambda: tt.insert_central_slices_rfft_3d(T, shape, R, deterministic=det)), \
            ns * 8 * P + 12 * vox, "insert_accumulate_kernel / insert_fixed_kernel + finalize"
    if name == "insert_bwd":
        T = crandn(ns, n, n // 2 + 1).requires_grad_(True)
        H = crandn(n, n, n // 2 + 1)

        def fn():
            T.grad = None
            v, _ = tt.insert_central_slices_rfft_3d(T, shape, R)
            v.backward(H)
        return fn, 8 * vox + ns * 8 * P, "insert_bwd_kernel (+ the insertion)"
    return kernel_case_more(name, dev, V, R, crandn, gen)


def kernel_case_more(name, dev, V, R, crandn, gen):
    """The cases of kernel_case beyond the single-volume slice kernels."""
    import torch

    import teamtomo_b200 as tt
    from teamtomo_b200 import batched as B
    from teamtomo_b200.torch_fourier_slice import _layout
    from teamtomo_b200.torch_fourier_slice._params import slice_params

    n = 256
    P, vox = n * (n // 2 + 1), n * n * (n // 2 + 1)
    if name in ("batched_extract", "batched_insert"):
        boxes = (64, 96, 128, 160, 200, 256, 96, 128)
        counts = (2000,) * len(boxes)
        vols = [rfft_volume_torch(blob_volume_torch(b, 2000 + i, dev)) for i, b in enumerate(boxes)]
        rots = [torch.tensor(rotations(c, 3000 + i), device=dev) for i, c in enumerate(counts)]
        rng = np.random.default_rng(1004)
        ctfs = [B.ctf_params(rng.uniform(0.5, 3.0, c), device=dev) for c in counts]
        slice_bytes = sum(c * 8 * b * (b // 2 + 1) for c, b in zip(counts, boxes))
        vb = sum(b * b * (b // 2 + 1) for b in boxes)
        if name == "batched_extract":
            return (lambda: B.extract_central_slices_rfft_3d_batched(vols, rots, ctf=ctfs)), slice_bytes + 8 * vb, \
                "batched_slices_kernel<extract>"
        sl = B.extract_central_slices_rfft_3d_batched(vols, rots, ctf=ctfs)
        return (lambda: B.insert_central_slices_rfft_3d_batched(sl, rots, ctf=ctfs)), slice_bytes + 12 * vb, \
            "batched_slices_kernel<insert> + insert_finalize_kernel"
    if name in ("sample3d", "insert3d"):
        m = 1 << 24
        img = torch.randn((n, n, n), device=dev, generator=gen)
        coords = torch.rand((m, 3), device=dev, generator=gen) * (n - 1)
        if name == "sample3d":
            return (lambda: tt.sample_image_3d(img, coords)), 4 * n ** 3 + 16 * m, "sample3d_kernel"
        vals = torch.randn(m, device=dev, generator=gen)
        return (lambda: tt.insert_into_image_3d(vals, coords, torch.zeros_like(img))), 16 * m + 8 * n ** 3, \
            "insert3d_kernel"
    if name == "affine3d":
        img = torch.randn((n, n, n), device=dev, generator=gen)
        M = torch.eye(4, device=dev)
        M[:3, :3] = torch.tensor(rotations(1, 5)[0], device=dev, dtype=torch.float32)
        return (lambda: tt.torch_transform_image.affine_transform_image_3d(img, M, "trilinear")), 8 * n ** 3, \
            "affine3d_kernel"
    if name.startswith("mc_"):
        c, ns = 4, 256
        vols = torch.stack([rfft_volume_torch(blob_volume_torch(n, 4000 + i, dev)) for i in range(c)])
        Rm = R[:ns]
        if name == "mc_extract":
            return (lambda: tt.extract_central_slices_rfft_3d_multichannel(vols, (n, n, n), Rm)), \
                c * (ns * 8 * P + 8 * vox), "multichannel extraction kernel"
        if name == "mc_backward":
            Vg = vols.clone().requires_grad_(True)
            Rg = Rm.clone().requires_grad_(True)
            G = crandn(ns, c, n, n // 2 + 1)

            def fn():
                Vg.grad = None
                Rg.grad = None
                tt.extract_central_slices_rfft_3d_multichannel(Vg, (n, n, n), Rg).backward(G)
            return fn, c * (ns * 8 * P + 16 * vox), "multichannel backward kernel"
        T = crandn(ns, c, n, n // 2 + 1)
        return (lambda: tt.insert_central_slices_rfft_3d_multichannel(T, (n, n, n), Rm)), \
            c * (ns * 8 * P + 8 * vox) + 4 * vox, "insert_accumulate_kernel per channel + finalize"
    if name == "lines":
        h = 4096
        img = crandn(h, h // 2 + 1)
        th = torch.rand(65536, device=dev, generator=gen) * 6.283185307
        R2 = torch.stack([torch.stack([th.cos(), -th.sin()], -1), torch.stack([th.sin(), th.cos()], -1)], -2)
        return (lambda: tt.extract_central_slices_rfft_2d(img, (h, h), R2)), 65536 * 8 * (h // 2 + 1) + 8 * h * (
            h // 2 + 1), "line_extract_kernel"
    if name == "project":
        b, k = 128, 2048
        vol = blob_volume_torch(b, 1001, dev)
        Rp = torch.tensor(rotations(k, 1001), device=dev)
        # non-FFT bytes: pad x sinc^2 (read b^3, write (2b)^3), extraction (write k (2b)(b+1)),
        # recentre / crop (read k (2b)^2, write k b^2), all float32 / complex64
        return (lambda: tt.project_3d_to_2d(vol, Rp)), 4 * b ** 3 + 4 * (2 * b) ** 3 + k * 8 * 2 * b * (b + 1) + \
            k * 4 * ((2 * b) ** 2 + b * b), "project_prepare_kernel, extraction, recentre_crop_2d_kernel"
    if name == "backproject":
        b, k = 128, 2048
        imgs = torch.randn((k, b, b), device=dev, generator=gen)
        Rp = torch.tensor(rotations(k, 1002), device=dev)
        return (lambda: tt.backproject_2d_to_3d(imgs, Rp)), k * 4 * (b * b + (2 * b) ** 2) + k * 8 * 2 * b * (
            b + 1) + 20 * (2 * b) ** 2 * (b + 1) + 8 * (2 * b) ** 3, \
            "pad_fftshift_2d_kernel, insertion, normalize_unshift_kernel, backproject_finish_kernel"
    if name == "pack_bricks":
        p = slice_params(n=1, image_shape=(n, n, n), volume=V, rotation=R)
        return (lambda: _layout.pack(V, p, _layout.BRICKS)), 16 * vox, "pack_bricks_kernel"
    raise ValueError(f"unknown kernel case {name!r}")


def kernels_workload(args):
    """--workload kernels: each case (or --case NAME) once for warm-up, then
    the measured calls inside an NVTX range named "measured" (ncu:
    --nvtx --nvtx-include measured/), with CUDA-event times on the current
    stream; one JSON line per case."""
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    names = [args.case] if args.case else list(KERNEL_CASES)
    for name in names:
        fn, algo, kernels = kernel_case(name, dev)
        fn()
        torch.cuda.synchronize(dev)
        reps = max(args.steps, 1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("measured")
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize(dev)
        ms = a.elapsed_time(b) / reps
        peak, kind = load_peaks()
        print(json.dumps({"case": name, "kernels": kernels, "ms_per_call": round(ms, 4), "algorithmic_bytes": algo,
                          "achieved_gbs": round(algo / ms / 1e6, 1), "frac_of_peak": round(algo / ms / 1e6 / peak, 4),
                          "peak_gbs": peak, "peak_source": kind}), flush=True)
        del fn
        torch.cuda.empty_cache()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batched":
        return batched_workload(args)
    if args.workload in ("project", "backproject", "fullscale"):
        return config_workload(args)
    if args.workload == "kernels":
        return kernels_workload(args)

    import torch
    import torch.distributed as dist

    import teamtomo_b200 as tt

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n, ns = args.box, args.slices
    shape = (n, n, n)

    # ---- inputs resident in HBM (targets > L2 per step) ----
    V0 = rfft_volume_torch(blob_volume_torch(n, ROT_SEED, dev))
    Vt = rfft_volume_torch(blob_volume_torch(n, ROT_SEED + 1000, dev))
    R0 = torch.tensor(rotations(ns, ROT_SEED + rank), device=dev)
    with torch.no_grad():
        T = tt.extract_central_slices_rfft_3d(Vt, shape, R0)
        gen = torch.Generator(device=dev).manual_seed(7 + rank)
        T = T + 0.5 * T.abs().mean() * torch.randn(T.shape, dtype=T.dtype, device=dev, generator=gen)
    del Vt
    V = V0.clone().requires_grad_(True)
    R = R0.clone().requires_grad_(True)
    stream = torch.cuda.current_stream(dev)
    marks = {}

    def on_grad(g):
        e = torch.cuda.Event(enable_timing=True)
        e.record(stream)
        marks["bwd_start"] = e
        return g

    class _ResidualMSE(torch.autograd.Function):
        @staticmethod
        def forward(ctx, s, t, m):
            # m: element count of the whole step (a chunk's share of the mean)
            r = s - t
            ctx.save_for_backward(r)
            ctx.m = m
            return torch.linalg.vector_norm(torch.view_as_real(r)).square() / m

        @staticmethod
        def backward(ctx, g):
            # loss = mean |S - T|^2  ->  PyTorch complex gradient 2 (S - T) / M
            (r,) = ctx.saved_tensors
            return r.mul_(g * (2.0 / ctx.m)), None, None

    det = bool(args.deterministic)

    def insert(images, rot):
        # N > 1: every rank splats its own targets, one all-reduce sums the volumes
        if world > 1:
            return tt.distributed.insert_central_slices_rfft_3d(images, shape, rot, deterministic=det)
        return tt.insert_central_slices_rfft_3d(images, shape, rot, deterministic=det)

    def step(with_events=False):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if with_events else None
        V.grad = None
        R.grad = None
        if ev:
            ev[0].record(stream)
        S = tt.extract_central_slices_rfft_3d(V, shape, R, deterministic=det)
        if ev:
            ev[1].record(stream)
            S.register_hook(on_grad)
        loss = _ResidualMSE.apply(S, T, T.numel())
        loss.backward()
        if ev:
            ev[2].record(stream)
        vol, w = insert(T, R.detach())
        if ev:
            ev[3].record(stream)
        if world > 1:
            tt.distributed.all_reduce_volume_gradient(V.grad)
        return loss, ev, (vol, w)

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    time.sleep(0.3)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sections = {"extract": [], "backward": [], "insert": []}
    evs = []
    start.record(stream)
    for _ in range(args.steps):
        loss, ev, _ = step(with_events=True)
        evs.append((ev, marks["bwd_start"]))
    end.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    elapsed = start.elapsed_time(end)  # ms
    for ev, b in evs:
        sections["extract"].append(ev[0].elapsed_time(ev[1]))
        sections["backward"].append(b.elapsed_time(ev[2]))
        sections["insert"].append(ev[2].elapsed_time(ev[3]))
    if world > 1:
        t = torch.tensor([elapsed], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    ms_step = elapsed / args.steps
    value = world * ns * args.steps / (elapsed / 1e3)

    # ---- per-kernel roofline (algorithmic bytes per launch) ----
    P = n * (n // 2 + 1)
    vox = n * n * (n // 2 + 1)
    algo = {
        "extract": ns * 8 * P + 8 * vox,          # slices written + volume read once
        "backward": ns * 8 * P + 16 * vox,        # grad read + dV written + volume read once
        "insert": ns * 8 * P + 12 * vox,          # slices read + volume and weights written
    }
    peak, peak_kind = load_peaks()
    traffic = load_traffic()
    kernels = {}
    for k, v in sections.items():
        ms = statistics.mean(v)
        gbs = algo[k] / (ms / 1e3) / 1e9
        kernels[k] = {"ms": round(ms, 4), "algorithmic_bytes": algo[k], "achieved_gbs": round(gbs, 1),
                      "frac": round(gbs / peak, 4)}
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    roof = {"bound": "hbm", "achieved": kernels[dom]["achieved_gbs"], "peak": peak, "unit": "GB/s",
            "frac": kernels[dom]["frac"], "traffic": traffic.get(dom), "kernel": dom,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6.65 TB/s"}

    # ---- the same step with the fused loss op (losses.central_slice_mse) ----
    # extraction, squared error and both gradients in one kernel (the slices
    # are never written, the upstream gradient never read); then the insertion.
    fused = None
    if not args.no_fused and not det:
        def fused_step(ev=None):
            V.grad = None
            R.grad = None
            if ev:
                ev[0].record(stream)
            lf = tt.losses.central_slice_mse(V, shape, R, T)
            lf.backward()
            if ev:
                ev[1].record(stream)
            insert(T, R.detach())
            if ev:
                ev[2].record(stream)
            if world > 1:
                tt.distributed.all_reduce_volume_gradient(V.grad)
            return lf

        for _ in range(max(args.warmup, 0)):
            fused_step()
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        f_ev = []
        fs, fe = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        fs.record(stream)
        for _ in range(args.steps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            fused_step(ev)
            f_ev.append(ev)
        fe.record(stream)
        torch.cuda.synchronize(dev)
        el_f = fs.elapsed_time(fe)
        if world > 1:
            t = torch.tensor([el_f], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el_f = float(t.item())
        fused = {"value": world * ns * args.steps / (el_f / 1e3), "unit": UNIT, "ms_per_step": el_f / args.steps,
                 "op": "losses.central_slice_mse (extract + MSE + d/dvolume + d/drotation, one kernel) + insert",
                 "kernels_ms": {"fused_mse": round(statistics.mean(e[0].elapsed_time(e[1]) for e in f_ev), 4),
                                "insert": round(statistics.mean(e[1].elapsed_time(e[2]) for e in f_ev), 4)}}

    # ---- end to end through the public API with host buffers ----
    # The targets and rotations stream from pinned host memory in chunks; the
    # copy of chunk k+1 overlaps the extract / backward / insert of chunk k.
    e2e = None
    if not args.no_e2e:
        hV = V0.detach().cpu().pin_memory()
        hR = R0.detach().cpu().pin_memory()
        hT = T.cpu().pin_memory()
        h_loss = torch.empty((), dtype=torch.float32).pin_memory()
        h_dR = torch.empty_like(hR).pin_memory()
        # every result of the step comes back: loss, d/drotation, d/dvolume and
        # the inserted (volume, weights)
        h_dV = torch.empty_like(hV).pin_memory()
        h_vol = torch.empty_like(hV).pin_memory()
        h_w = torch.empty(hV.shape, dtype=torch.float32).pin_memory()
        h2d = hV.numel() * 8 + hR.numel() * 4 + hT.numel() * 8
        d2h = 4 + h_dR.numel() * 4 + h_dV.numel() * 8 + h_vol.numel() * 8 + h_w.numel() * 4
        bound = float(torch.view_as_real(hT).abs().max()) if det else None  # input property, outside the timing
        m_total = hT.numel()

        def e2e_step():
            Vd = hV.to(dev, non_blocking=True).requires_grad_(True)
            acc = tt.streaming.InsertionAccumulator(shape, dev, deterministic=det, data_bound=bound,
                                                    max_slices=ns)
            loss = torch.zeros((), dtype=torch.float32, device=dev)
            for s0, s1, (Tc, Rc_buf) in tt.streaming.prefetch_to_device([hT, hR], args.e2e_chunk, dev):
                Rc = Rc_buf.clone().requires_grad_(True)
                S = tt.extract_central_slices_rfft_3d(Vd, shape, Rc, deterministic=det)
                lc = _ResidualMSE.apply(S, Tc, m_total)
                lc.backward()
                loss += lc.detach()
                acc.add(Tc, Rc.detach())
                h_dR[s0:s1].copy_(Rc.grad, non_blocking=True)
            if world > 1:
                tt.distributed.all_reduce_volume_gradient(Vd.grad)
            vol, w = acc.finalize()
            if world > 1:
                tt.distributed.all_reduce_sum(vol)
                tt.distributed.all_reduce_sum(w)
            # the results go out on their own stream: the device-to-host copies
            # of this step overlap the host-to-device copies of the next one
            out_stream.wait_stream(stream)
            with torch.cuda.stream(out_stream):
                for src, dst in ((Vd.grad, h_dV), (vol, h_vol), (w, h_w), (loss, h_loss)):
                    src.record_stream(out_stream)
                    dst.copy_(src, non_blocking=True)

        out_stream = torch.cuda.Stream(device=dev)
        e2e_steps = max(3, min(args.steps, 10))
        e2e_step()
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s2.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        stream.wait_stream(out_stream)  # the last step's results are on the host before the clock stops
        e2.record(stream)
        torch.cuda.synchronize(dev)
        el2 = s2.elapsed_time(e2)
        if world > 1:
            t = torch.tensor([el2], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el2 = float(t.item())
        e2e = {"value": world * ns * e2e_steps / (el2 / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": e2e_steps, "chunk_slices": args.e2e_chunk,
               "overlap": "H2D of chunk k+1 on a copy stream during compute of chunk k; D2H of a step's "
                          "results on a third stream during the next step's H2D",
               "d2h": "loss, d/drotation, d/dvolume, inserted volume and weights"}

    torch_gpu = None
    if rank == 0 and world == 1 and not args.no_torch_gpu:
        with torch.no_grad():
            V_ref = V.detach().clone()
        torch_gpu = torch_gpu_reference(dev, n, V_ref, R0, T, args.torch_gpu_sample)
        if "value" in torch_gpu:
            torch_gpu["ours_over_torch_gpu"] = round(value / torch_gpu["value"], 1)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_baseline(n, args.ref_cpu_sample, args.cpu_sample)

    reductions = None
    if rank == 0 and world == 1 and not det and not args.no_probe:
        reductions = l2_reduction_ceiling(dev, n, R0, kernels["insert"]["ms"])

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "box": n, "slices_per_gpu": ns, "global_batch": ns * world,
                       "rotation_seed": ROT_SEED, "l2": "inputs larger than L2 (1.08 GB of targets per step)",
                       "parallelism": f"dp{world}" + (" (all_reduce of d/dvolume and inserted volume)"
                                                      if world > 1 else ""),
                       "deterministic": det},
            "roofline": roof, "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "fused_mse": fused, "torch_gpu_reference": torch_gpu, "l2_reductions": reductions,
            # extract (+ the pack of the bricked volume copy it gathers from), backward,
            # rotation-gradient finish, insert splat, insert finalize (+ absmax
            # pre-passes and the fixed-point add-back when deterministic)
            "gpu_launches": ((8 if det else 5) + copy_launches(ns * n * (n // 2 + 1), V)) * args.steps,
            "loss": float(loss.item()),
        }
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
