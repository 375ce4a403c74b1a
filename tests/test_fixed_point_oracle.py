"""CPU checks of the fixed-point (deterministic) restatement in the oracle.

The reference has no deterministic mode, so the fixed-point oracle is pinned
through the reference's own float outputs: converted back, its volumes and
weights must match the golden insertions within float32 summation noise.  Its
integer sums must not depend on the slice order or on splitting the slices
into several accumulations.
"""

from __future__ import annotations

import numpy as np

from helpers import rel_l2, rotations


def _insert_kwargs(g, name):
    fmax = float(g[f"insert_{name}_fmax"])
    return dict(fftfreq_max=None if fmax < 0 else fmax, zyx_matrices=bool(int(g[f"insert_{name}_zyx"])))


def test_fixed_insert_matches_reference_golden(golden, oracle):
    for name in golden["insert_cases"]:
        name = str(name)
        imgs = golden[f"insert_{name}_images"]
        n = imgs.shape[-2]
        rot = golden[f"insert_{name}_rot"]
        k = rot.reshape(-1, 3, 3).shape[0]
        bits = oracle.fixed_absmax_bits(imgs)
        acc = oracle.insert_fixed(imgs, (n, n, n), rot, bits, k, **_insert_kwargs(golden, name))
        c128 = imgs.dtype == np.complex128
        vol, w = oracle.fixed_finalize(acc, bits, k, complex128=c128)
        tol = 1e-12 if c128 else 1e-6
        assert rel_l2(vol, golden[f"insert_{name}_volume"]) < tol, name
        assert rel_l2(w, golden[f"insert_{name}_weights"]) < tol, name
        # same support, except voxels whose total weight is below the fixed-point
        # quantum of the weights (a few products of near-zero corner fractions)
        gw = golden[f"insert_{name}_weights"]
        quantum = 1.0 / oracle.fixed_scales(bits, k)[1]
        differ = (w != 0) != (gw != 0)
        assert np.all(np.abs(gw[differ]) < quantum), name


def test_fixed_sums_are_order_and_split_invariant(oracle):
    rng = np.random.default_rng(5)
    n, k = 16, 24
    imgs = (rng.standard_normal((k, n, n // 2 + 1)) + 1j * rng.standard_normal((k, n, n // 2 + 1))).astype(
        np.complex64)
    rot = rotations(k, seed=8)
    bits = oracle.fixed_absmax_bits(imgs)
    whole = oracle.insert_fixed(imgs, (n, n, n), rot, bits, k)
    perm = rng.permutation(k)
    assert np.array_equal(oracle.insert_fixed(imgs[perm], (n, n, n), rot[perm], bits, k), whole)
    parts = sum(oracle.insert_fixed(imgs[s], (n, n, n), rot[s], bits, k)
                for s in (slice(0, 7), slice(7, 19), slice(19, k)))
    assert np.array_equal(parts, whole)


def test_fixed_scale_rule(oracle):
    one = int(np.array([1.0], np.float32).view(np.uint32)[0])  # 1.0 = 0.5 * 2^1
    assert oracle.fixed_scales(one, 4096) == (2.0 ** (62 - 8 - 12 - 1), 2.0 ** (62 - 8 - 12))
    assert oracle.fixed_scales(0, 1) == (2.0 ** 54, 2.0 ** 54)
    assert oracle.fixed_absmax_bits(np.array([1 + 3j, -4 - 1j], np.complex64)) == int(
        np.array([4.0], np.float32).view(np.uint32)[0])
    # float64 magnitudes are rounded up to float32
    v = 1.0 + 2.0 ** -40
    bits = oracle.fixed_absmax_bits(np.array([v]))
    assert float(np.array([bits], np.uint32).view(np.float32)[0]) >= v
