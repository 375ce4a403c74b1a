"""Seeded synthetic inputs shared by the tests."""

from __future__ import annotations

import numpy as np
from scipy.stats import special_ortho_group


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel().astype(np.complex128))
    num = np.linalg.norm((a.astype(np.complex128) - b.astype(np.complex128)).ravel())
    return float(num / den) if den > 0 else float(num)


def blob_volume(n: int, seed: int, n_blobs: int = 20) -> np.ndarray:
    """Sum of Gaussian blobs (sigma U(2,6) px * n/64, centres uniform in a
    ball of radius 0.375 n) plus N(0, 0.01^2) noise, float32."""
    rng = np.random.default_rng(seed)
    ax = np.arange(n, dtype=np.float32)
    vol = np.zeros((n, n, n), np.float32)
    for _ in range(n_blobs):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        c = n / 2 + u * 0.375 * n * rng.uniform() ** (1.0 / 3.0)
        s = rng.uniform(2, 6) * n / 64
        gz = np.exp(-((ax - c[0]) ** 2) / (2 * s * s))
        gy = np.exp(-((ax - c[1]) ** 2) / (2 * s * s))
        gx = np.exp(-((ax - c[2]) ** 2) / (2 * s * s))
        vol += gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    vol += rng.normal(0, 0.01, size=vol.shape).astype(np.float32)
    return vol


def rfft_volume_np(vol: np.ndarray) -> np.ndarray:
    """fftshift -> rfftn -> fftshift(z, y): the layout the slice functions take."""
    f = np.fft.rfftn(np.fft.fftshift(vol))
    return np.fft.fftshift(f, axes=(0, 1)).astype(np.complex64)


def rotations(n: int, seed: int) -> np.ndarray:
    return special_ortho_group.rvs(3, size=n, random_state=seed).reshape(n, 3, 3)


# ZYZ Euler pairs (degrees) 180 deg apart whose slices are complex conjugates,
# with ambiguous points around x=0 (test_extract_central_slices_rfft_3d.py:22-31)
PAIRS = [
    ([0, 0, 0], [0, 0, 180]), ([0, 0, 0], [180, 0, 0]), ([0, 20, 0], [0, 20, 180]),
    ([0, 20, 90], [0, 20, 270]), ([0, 60, 0], [0, 60, 180]), ([90, 90, 0], [90, 90, 180]),
    ([45, 0, 0], [45, 0, 180]), ([45, 90, 0], [45, 90, 180]),
]


def fsc(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Fourier shell correlation of two real cubes, shells of width 1/n
    (rfft, |k| rounded to the nearest shell index), DC shell first."""
    n = a.shape[0]
    fa, fb = np.fft.rfftn(a), np.fft.rfftn(b)
    k = np.fft.fftfreq(n)
    kx = np.fft.rfftfreq(n)
    r = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kx[None, None, :] ** 2) * n
    shell = np.rint(r).astype(int)
    out = []
    for s in range(n // 2 + 1):
        m = shell == s
        num = np.real(np.sum(fa[m] * np.conj(fb[m])))
        den = np.sqrt(np.sum(np.abs(fa[m]) ** 2) * np.sum(np.abs(fb[m]) ** 2))
        out.append(num / den if den > 0 else 1.0)
    return np.array(out)
