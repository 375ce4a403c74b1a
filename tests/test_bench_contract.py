"""The benchmark's host side, without a GPU: the command-line contract the
round-end runs use, and the reference legs' CTF (the reference's own
calculate_ctf_2d from baseline/_ref) against the oracle's restatement, so the
batched and full-scale reference legs weight by the same CTF as the kernels."""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench

    return bench


def test_command_line_contract(monkeypatch):
    b = _bench()
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "2", "--steps", "5", "--warmup", "3"])
    a = b.parse_args()
    assert (a.gpus, a.steps, a.warmup, a.impl, a.workload) == (2, 5, 3, "ours", "differentiation")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    assert b.parse_args().impl == "reference"
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = b.parse_args()
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1
    for flag in ("no_e2e", "no_fused", "no_torch_gpu", "no_cpu_baseline", "no_probe", "deterministic"):
        assert getattr(a, flag) is False
    assert set(b.KERNEL_CASES) >= {"extract", "backward", "insert", "insert_bwd", "batched_insert"}


def test_reference_ctf_matches_the_oracle(oracle):
    b = _bench()
    calc = b.reference_ctf()
    if calc is None:
        pytest.skip("baseline/_ref has no torch_ctf (run baseline/install_reference.py)")
    from teamtomo_b200 import batched

    box = 48
    rows = batched.ctf_params([0.8, 1.7, 2.5], astigmatism_um=[0.0, 0.1, 0.05],
                              astigmatism_angle_deg=[0.0, 30.0, 75.0], pixel_size_a=1.1)
    got = b.reference_ctf_images(calc, rows, box).numpy()
    ref = np.stack([oracle.ctf_2d(*[float(x) for x in r], image_shape=(box, box)) for r in rows.numpy()])
    assert got.shape == (3, box, box // 2 + 1)
    assert np.abs(got - ref).max() < 2e-4  # the reference computes in float32, the oracle in float64


def test_reference_ctf_insert_weights_are_ctf_squared_insertions(oracle):
    """The reference legs' CTF-weighted insertion (images x CTF, then CTF^2 for
    the weights) matches the oracle's two insertions on a small case."""
    b = _bench()
    mods, calc = b.reference_modules(), b.reference_ctf()
    if mods is None or calc is None:
        pytest.skip("baseline/_ref missing (run baseline/install_reference.py)")
    from helpers import rel_l2, rotations
    from teamtomo_b200 import batched

    n, k = 24, 6
    rng = np.random.default_rng(5)
    imgs = (rng.standard_normal((k, n, n // 2 + 1)) + 1j * rng.standard_normal((k, n, n // 2 + 1))).astype(
        np.complex64)
    R = rotations(k, seed=9)
    rows = batched.ctf_params(np.linspace(0.9, 2.2, k), pixel_size_a=1.0)
    v, w = b.reference_ctf_insert(mods, calc, torch.from_numpy(imgs), torch.from_numpy(R), rows, n)
    ctf = np.stack([oracle.ctf_2d(*[float(x) for x in r], image_shape=(n, n)) for r in rows.numpy()])
    rv, _ = oracle.insert((imgs * ctf).astype(np.complex64), (n, n, n), R)
    rw, _ = oracle.insert((ctf * ctf).astype(np.complex64), (n, n, n), R)
    # float32 CTF (reference) against float64 (oracle): the GPU CTF tests use the same 1e-4
    assert rel_l2(v.numpy(), rv) < 1e-4 and rel_l2(w.numpy(), rw.real) < 1e-4


def test_reference_arm_prints_its_line():
    """--impl reference runs the reference's own torch code on the host cores
    (here on a 32^3 box) and prints the contract's JSON line."""
    import json
    import subprocess

    if not os.path.isdir(os.path.join(ROOT, "baseline", "_ref", "torch_fourier_slice")):
        pytest.skip("baseline/_ref missing (run baseline/install_reference.py)")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--box", "32", "--steps", "1",
                        "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "slices/s"
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "slices/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
