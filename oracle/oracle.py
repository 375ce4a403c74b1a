"""CPU oracle for the Fourier-slice path (TEST INFRASTRUCTURE ONLY).

Nothing in ``teamtomo_b200`` imports this module.  Only ``tests/``, the smoke
check and the CPU-baseline legs of ``bench.py`` use it, as the checker.

Two layers:

* ``liboracle.so`` (``fourier_slice_oracle.c``): float32 restatement of the
  reference's central-slice extraction, insertion (with its per-corner Friedel
  mirror) and the extraction's gradients.  Built by ``oracle/Makefile``.
* numpy restatements of ``torch_image_interpolation.sample_image_3d`` /
  ``insert_into_image_3d`` (image_interpolation_3d.py:11-101, 104-275) and of
  the real-space wrappers ``project_3d_to_2d`` (torch_fourier_slice/project.py:12-93)
  and ``backproject_2d_to_3d`` (torch_fourier_slice/backproject.py:11-92).

All arrays are numpy; complex arrays are complex64/complex128 C-contiguous.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i64 = ctypes.c_int64
_int = ctypes.c_int
_f32 = ctypes.c_float


def build() -> str:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "fourier_slice_oracle.c")
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_extract.argtypes = [_f32p, _i64, _i64, _i64, _f32p, _i64, _i64, _i64, _i64,
                                  _int, _f32, _int, _f32, _f32, _int, _f32, _f32p, _u8p,
                                  _f32p, _int]
        L.orc_extract_grad.argtypes = [_f32p, _i64, _i64, _i64, _f32p, _i64, _i64, _i64, _i64,
                                       _int, _f32, _int, _f32, _f32, _int, _f32, _f32p, _f32p,
                                       _f64p, _int]
        L.orc_slice_geometry.argtypes = [_f32p, _i64, _i64, _i64, _i64, _i64, _i64, _i64,
                                         _int, _f32, _int, _f32, _f32, _int, _f32, _int, _u8p,
                                         _f32p]
        for name, p in (("orc_insert_c64", _f32p), ("orc_insert_c128", _f64p),
                        ("orc_insert_c64_mt", _f32p)):
            getattr(L, name).argtypes = [p, _i64, _i64, _i64, _i64, _f32p, _int, _f32, _int,
                                         p, p, _int, _int]
        _lib = L
    return _lib


def _ptr(a, t):
    if a is None:
        return ctypes.cast(None, t)
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


def _rot_f32(rotation_matrices) -> np.ndarray:
    r = np.asarray(rotation_matrices)
    return np.ascontiguousarray(r.astype(np.float32).reshape(-1, 9))


def _f32_scalar(x: float) -> np.float32:
    return np.float32(x)


def extract(volume_rfft, image_shape, rotation_matrices, fftfreq_max=None, zyx_matrices=False,
            x_tolerance=1e-8, rot_tolerance=1e-8, return_aux=False, nthreads=1):
    """Restatement of extract_central_slices_rfft_3d (complex64 volumes)."""
    vol = np.ascontiguousarray(volume_rfft, dtype=np.complex64)
    D, H, W = vol.shape
    R = np.asarray(rotation_matrices)
    stack = R.shape[:-2]
    r = _rot_f32(R)
    n = r.shape[0]
    d, h, w = (int(s) for s in image_shape)
    wr = w // 2 + 1
    out = np.zeros((n, h, wr), np.complex64)
    conj = np.zeros((n, h, wr), np.uint8) if return_aux else None
    coords = np.zeros((n, h, wr, 3), np.float32) if return_aux else None
    lib().orc_extract(
        _ptr(vol.view(np.float32), _f32p), D, H, W, _ptr(r, _f32p), n, d, h, w,
        int(fftfreq_max is not None), _f32_scalar(fftfreq_max or 0.0), int(zyx_matrices),
        _f32_scalar(x_tolerance), _f32_scalar(x_tolerance * 10),
        int(rot_tolerance is not None), _f32_scalar(rot_tolerance or 0.0),
        _ptr(out.view(np.float32), _f32p), _ptr(conj, _u8p),
        _ptr(coords, _f32p), nthreads)
    out = out.reshape(*stack, h, wr)
    if return_aux:
        return out, conj.reshape(*stack, h, wr).astype(bool), coords.reshape(*stack, h, wr, 3)
    return out


def extract_grad(volume_rfft, image_shape, rotation_matrices, grad, fftfreq_max=None,
                 zyx_matrices=False, x_tolerance=1e-8, rot_tolerance=1e-8, want_dvol=True,
                 want_drot=True, nthreads=1):
    """Gradients of the extraction w.r.t. the volume and the rotation matrices."""
    vol = np.ascontiguousarray(volume_rfft, dtype=np.complex64)
    D, H, W = vol.shape
    R = np.asarray(rotation_matrices)
    r = _rot_f32(R)
    n = r.shape[0]
    d, h, w = (int(s) for s in image_shape)
    g = np.ascontiguousarray(np.asarray(grad, dtype=np.complex64).reshape(n, h, w // 2 + 1))
    dvol = np.zeros_like(vol) if want_dvol else None
    drot = np.zeros((n, 9), np.float64) if want_drot else None
    lib().orc_extract_grad(
        _ptr(vol.view(np.float32), _f32p), D, H, W, _ptr(r, _f32p), n, d, h, w,
        int(fftfreq_max is not None), _f32_scalar(fftfreq_max or 0.0), int(zyx_matrices),
        _f32_scalar(x_tolerance), _f32_scalar(x_tolerance * 10),
        int(rot_tolerance is not None), _f32_scalar(rot_tolerance or 0.0),
        _ptr(g.view(np.float32), _f32p),
        _ptr(dvol.view(np.float32) if dvol is not None else None, _f32p),
        _ptr(drot, _f64p), nthreads)
    if drot is not None:
        drot = drot.reshape(R.shape)
    return dvol, drot


def insert(image_rfft, volume_shape, rotation_matrices, fftfreq_max=None, zyx_matrices=False,
           nthreads=1, mirror=True):
    """Restatement of insert_central_slices_rfft_3d -> (volume, weights).

    ``mirror=False`` leaves out the per-corner Friedel mirror insertion (used
    to check the x=0 plane post-pass form against the reference)."""
    img = np.asarray(image_rfft)
    double = img.dtype == np.complex128
    img = np.ascontiguousarray(img, dtype=np.complex128 if double else np.complex64)
    vd, vh, vw = (int(s) for s in volume_shape)
    wr = vw // 2 + 1
    r = _rot_f32(rotation_matrices)
    n = r.shape[0]
    img = img.reshape(n, vh, wr)
    real = np.float64 if double else np.float32
    vol = np.zeros((vd, vh, wr), img.dtype)
    wts = np.zeros((vd, vh, wr), real)
    if double:
        fn, p = lib().orc_insert_c128, _f64p
    else:
        fn, p = (lib().orc_insert_c64_mt if nthreads != 1 else lib().orc_insert_c64), _f32p
    fn(_ptr(img.view(real), p), n, vd, vh, vw, _ptr(r, _f32p), int(fftfreq_max is not None),
       _f32_scalar(fftfreq_max or 0.0), int(zyx_matrices), _ptr(vol.view(real), p),
       _ptr(wts, p), int(mirror), nthreads)
    return vol, wts


def slice_geometry(rotation_matrices, image_shape, volume_dims, mode, fftfreq_max=None,
                   zyx_matrices=False, x_tolerance=1e-8, rot_tolerance=1e-8):
    """Per-pixel (flags, coords) of the extraction (mode 0) / insertion (mode 1)
    rule: flags bit0 kept, bit1 conjugated, bit2 inside the volume."""
    r = _rot_f32(rotation_matrices)
    n = r.shape[0]
    d, h, w = (int(s) for s in image_shape)
    D, H, W = (int(s) for s in volume_dims)
    wr = w // 2 + 1
    flags = np.zeros((n, h, wr), np.uint8)
    coords = np.zeros((n, h, wr, 3), np.float32)
    lib().orc_slice_geometry(
        _ptr(r, _f32p), n, d, h, w, D, H, W, int(fftfreq_max is not None),
        _f32_scalar(fftfreq_max or 0.0), int(zyx_matrices), _f32_scalar(x_tolerance),
        _f32_scalar(x_tolerance * 10), int(rot_tolerance is not None),
        _f32_scalar(rot_tolerance or 0.0), int(mode), _ptr(flags, _u8p), _ptr(coords, _f32p))
    return flags, coords


def extract_f64(volume_rfft, image_shape, rotation_matrices, zyx_matrices=False):
    """float64 restatement of the extraction for finite-difference checks.

    Same geometry as the reference (frequency grid, xyz->zyx flip, conjugate
    redirect, array coordinates, grid_sample trilinear, zero outside) but in
    float64 with the plain sign rule x' < 0 (no tolerances); finite
    differences use rotations with no pixel near the x' = 0 boundary."""
    vol = np.asarray(volume_rfft, np.complex128)
    D, H, W = vol.shape
    R = np.asarray(rotation_matrices, np.float64).reshape(-1, 3, 3)
    M = R if zyx_matrices else R[:, ::-1, ::-1]
    d, h, w = (int(s) for s in image_shape)
    k = np.arange(h)
    fy = np.fft.fftshift(np.where(k < (h + 1) // 2, k, k - h) / h)
    fx = np.arange(w // 2 + 1) / w
    q = np.stack(np.broadcast_arrays(np.zeros((h, 1)), fy[:, None], fx[None, :]), -1)  # (h, wr, 3)
    p = np.einsum("nij,hwj->nhwi", M, q)
    cj = p[..., 2] < -1e-8
    # near-zero tie-break of _determine_near_zero_conjugate_mask (:9-81)
    r11 = M[:, 2, 2][:, None, None]
    r12 = M[:, 2, 1][:, None, None]
    near = np.abs(p[..., 2]) < 1e-8
    cj |= near & np.where(np.abs(r11) <= 1e-7, r12 < 0, r11 < 0)
    p[cj] *= -1
    c = np.empty_like(p)
    c[..., 0] = (p[..., 0] + 0.5) / (1 - 1 / d) * (d - 1)
    c[..., 1] = (p[..., 1] + 0.5) / (1 - 1 / h) * (h - 1)
    c[..., 2] = p[..., 2] * 2 * (w // 2)
    inside = np.all((c >= 0) & (c <= np.array([D, H, W]) - 1), -1)
    cc = np.clip(c, 0, np.array([D, H, W]) - 1)
    f = np.floor(cc)
    t = cc - f
    f = f.astype(np.int64)
    out = np.zeros(c.shape[:-1], np.complex128)
    for bz in (0, 1):
        for by in (0, 1):
            for bx in (0, 1):
                zi, yi, xi = f[..., 0] + bz, f[..., 1] + by, f[..., 2] + bx
                ok = (zi < D) & (yi < H) & (xi < W)
                wgt = ((t[..., 0] if bz else 1 - t[..., 0]) * (t[..., 1] if by else 1 - t[..., 1])
                       * (t[..., 2] if bx else 1 - t[..., 2]))
                v = vol[np.minimum(zi, D - 1), np.minimum(yi, H - 1), np.minimum(xi, W - 1)]
                out += np.where(ok, v * wgt, 0)
    out[~inside] = 0
    out[cj] = np.conj(out[cj])
    return out


def ctf_2d(defocus_um, astigmatism_um, astigmatism_angle_deg, voltage_kv, spherical_aberration_mm,
           amplitude_contrast, phase_shift_deg, pixel_size_a, image_shape, rfft=True, fftshift=True):
    """Restatement of torch_ctf.calculate_ctf_2d (torch-ctf/src/torch_ctf/ctf_2d.py:12-131,
    ctf_utils.py:46-86, ctf_aberrations.py:9-81) for scalar parameters, without
    Zernike / beam-tilt / magnification terms, in float64:
    -sin(k1 s^2 df + k2 s^4 - phase - atan(A / sqrt(1 - A^2)))."""
    h, w = image_shape
    fy = np.fft.fftfreq(h)
    fx = np.fft.rfftfreq(w) if rfft else np.fft.fftfreq(w)
    if fftshift:
        fy = np.fft.fftshift(fy)
        if not rfft:
            fx = np.fft.fftshift(fx)
    y, x = np.meshgrid(fy / pixel_size_a, fx / pixel_size_a, indexing="ij")
    s2 = y * y + x * x
    nrm = np.sqrt(s2 + np.finfo(np.float32).eps)
    th = np.deg2rad(astigmatism_angle_deg)
    a = np.sqrt(astigmatism_um) * np.array([np.sin(th), np.cos(th)])
    df = defocus_um - astigmatism_um + 2 * ((y / nrm) * a[0] + (x / nrm) * a[1]) ** 2
    h_pl, c, m0, e = 6.62607015e-34, 299792458.0, 9.1093837015e-31, 1.602176634e-19
    ev = e * voltage_kv * 1e3
    lam = h_pl * c / np.sqrt(ev * (2 * m0 * c * c + ev)) * 1e10
    k1 = -np.pi * lam
    k2 = np.pi / 2 * spherical_aberration_mm * 1e7 * lam ** 3
    ac = amplitude_contrast
    chi = (k1 * s2 * df * 1e4 + k2 * s2 * s2 - np.deg2rad(phase_shift_deg)
           - np.arctan(ac / np.sqrt(1 - ac * ac)))
    return -np.sin(chi)


def mirror_x0_post_pass(vol, wts):
    """Friedel completion of the x=0 plane as one post-pass (numpy):
    out[v] = acc[v] + conj(acc[m v]) unless m v is the DC voxel,
    m(z, y) = ((d - z) % d, (h - y) % h); the same for the weights."""
    vol = np.array(vol, copy=True)
    wts = np.array(wts, copy=True)
    d, h = vol.shape[-3:-1]
    z = np.arange(d)[:, None]
    y = np.arange(h)[None, :]
    zm, ym = (d - z) % d, (h - y) % h
    keep = ~((zm == d // 2) & (ym == h // 2))
    p, pw = vol[..., 0].copy(), wts[..., 0].copy()
    vol[..., 0] = p + np.where(keep, np.conj(p[..., zm, ym]), 0)
    wts[..., 0] = pw + np.where(keep, pw[zm, ym], 0)
    return vol, wts


def insert_grad_images(grad_volume, volume_shape, rotation_matrices, fftfreq_max=None,
                       zyx_matrices=False, dtype=np.complex64):
    """Gradient of insert_central_slices_rfft_3d's volume w.r.t. its images
    (PyTorch's complex convention) for upstream gradient ``grad_volume``: the
    adjoint of the Friedel completion (G[v] + conj(G[m v]) on the x=0 plane
    unless v itself is DC: out[u] takes conj(acc[m u]) unless m u is DC, and m
    is its own inverse — for odd boxes m(DC) is not DC), then the insertion's own trilinear weights gathered back to
    each kept source pixel, conjugated where the point was redirected.  The
    weights output does not depend on the images.  (numpy, float64 sums)"""
    gv = np.asarray(grad_volume).astype(np.complex128)
    vd, vh, vw = (int(s) for s in volume_shape)
    wr = vw // 2 + 1
    z = np.arange(vd)[:, None]
    y = np.arange(vh)[None, :]
    zm, ym = (vd - z) % vd, (vh - y) % vh
    keep = ~((z == vd // 2) & (y == vh // 2))
    ga = gv.copy()
    ga[:, :, 0] = gv[:, :, 0] + np.where(keep, np.conj(gv[zm, ym, 0]), 0)
    r = _rot_f32(rotation_matrices)
    n = r.shape[0]
    flags, coords = slice_geometry(r, volume_shape, (vd, vh, wr), 1, fftfreq_max=fftfreq_max,
                                   zyx_matrices=zyx_matrices)
    sel = (flags & 5) == 5
    c = coords[sel]
    lo = np.floor(c)
    hi = np.ceil(c)
    t = (c - lo).astype(np.float32)
    one = np.float32(1)
    acc = np.zeros(len(c), np.complex128)
    flat = ga.reshape(-1)
    for k in range(8):
        b = ((k >> 2) & 1, (k >> 1) & 1, k & 1)
        f = [t[:, a] if b[a] else one - t[:, a] for a in range(3)]
        w = (f[0] * f[1]) * f[2]
        idx = [(hi if b[a] else lo)[:, a].astype(np.int64) for a in range(3)]
        vi = (idx[0] * vh + idx[1]) * wr + idx[2]
        acc += np.where(w != 0, w.astype(np.float64) * flat[vi], 0)
    acc = np.where((flags[sel] & 2) != 0, np.conj(acc), acc)
    out = np.zeros((n, vh, wr), dtype)
    out[sel] = acc.astype(dtype)
    return out


def affine_transform_image_3d(image, matrices, interpolation, output_shape=None, zyx_matrices=False):
    """Restatement of torch_transform_image.affine_transform_image_3d
    (transforms_3d.py:10-40): float32 homogeneous coordinates M (z, y, x, 1)
    with each product rounded and the sums taken left to right, then
    sample_image_3d."""
    f32 = np.float32
    img = np.asarray(image)
    d, h, w = (int(s) for s in (output_shape if output_shape else img.shape[-3:]))
    M = np.array(matrices, dtype=f32, copy=True)
    if not zyx_matrices:
        M[..., :3, :3] = M[..., :3, :3][..., ::-1, ::-1]
        M[..., :3, 3] = M[..., :3, 3][..., ::-1]
    z, y, x = (a.astype(f32) for a in np.indices((d, h, w)))
    cols = (z, y, x, np.ones_like(z))
    stack = M.shape[:-2]
    Mf = M.reshape(-1, 4, 4)
    outs = []
    for m in Mf:
        c = np.zeros((d, h, w, 3), f32)
        for i in range(3):
            acc = (m[i, 0] * cols[0]).astype(f32)
            for j in (1, 2, 3):
                acc = (acc + (m[i, j] * cols[j]).astype(f32)).astype(f32)
            c[..., i] = acc
        real = np.float64 if img.dtype in (np.float64, np.complex128) else f32
        outs.append(sample_image_3d(img, c.astype(real), interpolation))
    return np.stack(outs).reshape(*stack, *outs[0].shape)


# ----------------------------------------------------------------------------
# central lines of 2D images (numpy, float32 arithmetic)
# ----------------------------------------------------------------------------

def _source_index_np(c, n):
    """grid_sample's array -> grid -> array round trip (align_corners, border clip)."""
    f32 = np.float32
    half = f32(0.5) * f32(n) - f32(0.5)
    g = (c / half).astype(f32) - f32(1)
    ix = ((g + f32(1)) * f32(0.5)).astype(f32) * f32(n - 1)
    return np.clip(ix.astype(f32), f32(0), f32(n - 1))


def extract_lines_2d(image_rfft, image_shape, rotation_matrices, fftfreq_max=None, yx_matrices=False):
    """Restatement of extract_central_slices_rfft_2d
    (_extract_central_slices_rfft_2d.py:9-84): central lines (..., w//2+1) of
    an fftshifted (h, w//2+1) rfft, bilinear grid_sample sampling, strict
    x' < 0 redirect; samples with frequency > fftfreq_max are zero."""
    f32 = np.float32
    img = np.asarray(image_rfft).astype(np.complex64)
    H, W = img.shape
    h, w = (int(x) for x in image_shape)
    R = np.asarray(rotation_matrices)
    stack = R.shape[:-2]
    r = R.astype(f32).reshape(-1, 2, 2)
    if not yx_matrices:
        r = r[:, ::-1, ::-1]
    wr = w // 2 + 1
    qx = np.arange(wr, dtype=f32) * f32(1.0 / w)
    py = (r[:, 0, 1][:, None] * qx[None, :]).astype(f32)
    px = (r[:, 1, 1][:, None] * qx[None, :]).astype(f32)
    cj = px < 0
    py = np.where(cj, -py, py)
    px = np.where(cj, -px, px)
    iw0 = f32(1) - f32(1.0) / f32(h)
    cy = (((py + f32(0.5)).astype(f32) / iw0).astype(f32) * f32(h - 1)).astype(f32)
    cx = ((px * f32(2)).astype(f32) * f32(wr - 1)).astype(f32)
    inside = (cy >= 0) & (cy <= H - 1) & (cx >= 0) & (cx <= W - 1)
    if fftfreq_max is not None:
        inside &= (qx <= f32(fftfreq_max))[None, :]
    iy = _source_index_np(cy, H)
    ix = _source_index_np(cx, W)
    y0 = np.floor(iy).astype(np.int64)
    x0 = np.floor(ix).astype(np.int64)
    ay1 = (iy - y0).astype(np.float64)
    ax1 = (ix - x0).astype(np.float64)
    out = np.zeros(py.shape, np.complex128)
    for by in (0, 1):
        for bx in (0, 1):
            yy, xx = y0 + by, x0 + bx
            ok = inside & (yy < H) & (xx < W)
            wgt = (ay1 if by else 1 - ay1) * (ax1 if bx else 1 - ax1)
            out += np.where(ok, wgt * img[np.clip(yy, 0, H - 1), np.clip(xx, 0, W - 1)], 0)
    out = np.where(cj, np.conj(out), out)
    out = np.where(inside, out, 0)
    return out.astype(np.complex64).reshape(*stack, wr)


def project_2d_to_1d(image, rotation_matrices, pad_factor=2.0, fftfreq_max=None, yx_matrices=False):
    """Restatement of torch_fourier_slice.project_2d_to_1d (project.py): pad,
    premultiply by sinc^2, 2D rfft, central lines, 1D irfft without an output
    size, recentre, unpad."""
    img = np.asarray(image, np.float64)
    d = img.shape[-1]
    p = int((d * (pad_factor - 1.0)) // 2) if pad_factor > 1.0 else 0
    if p:
        img = np.pad(img, p)
    n = img.shape[-1]
    f = np.fft.fftshift(np.fft.fftfreq(n))
    img = img * np.sinc(np.sqrt(f[:, None] ** 2 + f[None, :] ** 2)) ** 2
    dft = np.fft.fftshift(np.fft.rfftn(np.fft.fftshift(img)), axes=(0,))
    lines = extract_lines_2d(dft, (n, n), rotation_matrices, fftfreq_max=fftfreq_max, yx_matrices=yx_matrices)
    proj = np.fft.ifftshift(np.fft.irfft(lines.astype(np.complex128), axis=-1), axes=-1)
    if p:
        proj = proj[..., p:-p]
    return proj.astype(np.float32)


# ----------------------------------------------------------------------------
# deterministic insertion: 64-bit fixed point (numpy, bit-exact restatement of
# the CUDA fixed-point mode; the reference has no such mode, so it is pinned
# through its float outputs)
# ----------------------------------------------------------------------------

FIXED_HEADROOM_BITS = 8


def _ceil_log2(n: int) -> int:
    l = 0
    while l < 62 and (1 << l) < n:
        l += 1
    return l


def fixed_absmax_bits(*arrays) -> int:
    """uint32 bit pattern of max |re|, |im| over the arrays, as float32
    (float64 magnitudes rounded up to float32)."""
    best = np.float32(0)
    for a in arrays:
        a = np.asarray(a)
        if a.size == 0:
            continue
        real = a.view(a.real.dtype) if np.iscomplexobj(a) else a
        v = np.abs(real).max()
        f = np.float32(v)
        if float(f) < float(v):
            f = np.nextafter(f, np.float32(np.inf))
        best = max(best, f)
    return int(np.array([best], np.float32).view(np.uint32)[0])


def fixed_scales(absmax_bits: int, max_slices: int) -> tuple[float, float]:
    """(data scale, weight scale): 2^(62 - 8 - ceil(log2 max_slices) - E) with
    |data| < 2^E, and 2^(62 - 8 - ceil(log2 max_slices))."""
    a = np.array([absmax_bits], np.uint32).view(np.float32)[0]
    e = 0
    if 0 < a <= np.finfo(np.float32).max:
        e = int(np.frexp(a)[1])
    l = _ceil_log2(int(max_slices))
    return 2.0 ** (62 - FIXED_HEADROOM_BITS - l - e), 2.0 ** (62 - FIXED_HEADROOM_BITS - l)


def insert_fixed(image_rfft, volume_shape, rotation_matrices, absmax_bits, max_slices,
                 fftfreq_max=None, zyx_matrices=False):
    """Fixed-point accumulator (d, h, w//2+1, 3) int64 (re, im, w) of the
    deterministic insertion, before the Friedel completion.  Same pixels,
    redirect, bounds and float32 corner weights ((1-t) / t products, left to
    right) as insert(); each term data*w rounded once (half to even)."""
    img = np.asarray(image_rfft)
    vd, vh, vw = (int(s) for s in volume_shape)
    wr = vw // 2 + 1
    r = _rot_f32(rotation_matrices)
    n = r.shape[0]
    img = img.reshape(n, vh, wr)
    flags, coords = slice_geometry(r, volume_shape, (vd, vh, wr), 1, fftfreq_max=fftfreq_max,
                                   zyx_matrices=zyx_matrices)
    sel = (flags & 5) == 5
    c = coords[sel]
    d = img[sel]
    re = d.real.astype(np.float64)
    im = np.where((flags[sel] & 2) != 0, -d.imag, d.imag).astype(np.float64)
    lo = np.floor(c)
    hi = np.ceil(c)
    t = (c - lo).astype(np.float32)
    one = np.float32(1)
    sd, sw = fixed_scales(absmax_bits, max_slices)
    acc = np.zeros((vd * vh * wr, 3), np.int64)
    for k in range(8):
        b = ((k >> 2) & 1, (k >> 1) & 1, k & 1)
        f = [t[:, a] if b[a] else one - t[:, a] for a in range(3)]
        w = (f[0] * f[1]) * f[2]
        idx = [(hi if b[a] else lo)[:, a].astype(np.int64) for a in range(3)]
        vi = (idx[0] * vh + idx[1]) * wr + idx[2]
        nz = w != 0
        w64 = w.astype(np.float64)
        for col, val in ((0, re * w64 * sd), (1, im * w64 * sd), (2, w64 * 1.0 * sw)):
            np.add.at(acc[:, col], vi[nz], np.rint(val[nz]).astype(np.int64))
    return acc.reshape(vd, vh, wr, 3)


def fixed_finalize(acc, absmax_bits, max_slices, complex128=False):
    """Fixed-point accumulator (d, h, w, 3) -> (volume, weights): Friedel
    completion of the x=0 plane on the integers, then one conversion."""
    a = np.array(acc, dtype=np.int64, copy=True)
    d, h = a.shape[:2]
    z = np.arange(d)[:, None]
    y = np.arange(h)[None, :]
    zm, ym = (d - z) % d, (h - y) % h
    keep = ~((zm == d // 2) & (ym == h // 2))
    p = np.array(acc[:, :, 0, :], dtype=np.int64)
    a[:, :, 0, 0] = p[..., 0] + np.where(keep, p[zm, ym, 0], 0)
    a[:, :, 0, 1] = p[..., 1] - np.where(keep, p[zm, ym, 1], 0)
    a[:, :, 0, 2] = p[..., 2] + np.where(keep, p[zm, ym, 2], 0)
    sd, sw = fixed_scales(absmax_bits, max_slices)
    real = np.float64 if complex128 else np.float32
    vol = np.empty(a.shape[:3], np.complex128 if complex128 else np.complex64)
    vol.real = (a[..., 0].astype(np.float64) * (1.0 / sd)).astype(real)
    vol.imag = (a[..., 1].astype(np.float64) * (1.0 / sd)).astype(real)
    wts = (a[..., 2].astype(np.float64) * (1.0 / sw)).astype(real)
    return vol, wts


# ----------------------------------------------------------------------------
# torch_image_interpolation restatements (numpy)
# ----------------------------------------------------------------------------

def _roundtrip(c, n, dt):
    """array coord -> grid_sample coord -> source index (align_corners=True)."""
    fn = dt.type(n)
    half = dt.type(0.5) * fn - dt.type(0.5)
    g = c / half - dt.type(1)
    ix = ((g + dt.type(1)) / dt.type(2)) * (fn - dt.type(1))
    return np.clip(ix, dt.type(0), fn - dt.type(1))


def sample_image_3d(image, coordinates, interpolation="trilinear"):
    """Restatement of sample_image_3d (image_interpolation_3d.py:11-101)."""
    image = np.asarray(image)
    if image.ndim not in (3, 4):
        raise ValueError("image should have shape (d, h, w) or (c, d, h, w)")
    multi = image.ndim == 4
    img = image if multi else image[None]
    coords = np.asarray(coordinates)
    batch = coords.shape[:-1]
    c = coords.reshape(-1, 3)
    rdt = np.dtype(np.float64) if img.dtype in (np.float64, np.complex128) else np.dtype(np.float32)
    c = c.astype(rdt)
    C, D, H, W = img.shape
    out = np.zeros((c.shape[0], C), img.dtype)
    iz, iy, ix = _roundtrip(c[:, 0], D, rdt), _roundtrip(c[:, 1], H, rdt), _roundtrip(c[:, 2], W, rdt)
    if interpolation == "nearest":
        z = np.rint(iz).astype(np.int64)
        y = np.rint(iy).astype(np.int64)
        x = np.rint(ix).astype(np.int64)
        ok = (z >= 0) & (z < D) & (y >= 0) & (y < H) & (x >= 0) & (x < W)
        out[ok] = img[:, z[ok], y[ok], x[ok]].T
    else:
        z0, y0, x0 = np.floor(iz), np.floor(iy), np.floor(ix)
        z1, y1, x1 = z0 + 1, y0 + 1, x0 + 1
        for bz in (0, 1):
            for by in (0, 1):
                for bx in (0, 1):
                    wz = (iz - z0) if bz else (z1 - iz)
                    wy = (iy - y0) if by else (y1 - iy)
                    wx = (ix - x0) if bx else (x1 - ix)
                    w = wx * wy * wz
                    zi = (z1 if bz else z0).astype(np.int64)
                    yi = (y1 if by else y0).astype(np.int64)
                    xi = (x1 if bx else x0).astype(np.int64)
                    ok = (zi < D) & (yi < H) & (xi < W)
                    v = np.zeros_like(out)
                    v[ok] = img[:, zi[ok], yi[ok], xi[ok]].T
                    out += v * w[:, None]
    shape = np.array([D, H, W], rdt)
    inside = np.all((c >= 0) & (c <= shape - 1), axis=-1)
    out[~inside] = 0
    out = out.reshape(*batch, C)
    return out if multi else out[..., 0]


def insert_into_image_3d(values, coordinates, image, weights=None, interpolation="trilinear"):
    """Restatement of insert_into_image_3d (image_interpolation_3d.py:104-275).

    Accumulates into copies of ``image`` / ``weights`` and returns them."""
    image = np.array(image, copy=True)
    multi = image.ndim == 4
    D, H, W = image.shape[-3:]
    values = np.asarray(values)
    coords = np.asarray(coordinates)
    vshape = values.shape[:-1] if multi else values.shape
    if vshape != coords.shape[:-1]:
        raise ValueError("One coordinate triplet is required for each value in data.")
    if coords.shape[-1] != 3:
        raise ValueError("Coordinates must be 3D with shape (..., 3).")
    if image.dtype != values.dtype:
        raise ValueError("Image and values must have the same dtype.")
    weights = np.zeros((D, H, W), np.float32) if weights is None else np.array(weights, copy=True)
    img = image if multi else image[None]
    vals = values.reshape(-1, img.shape[0]) if multi else values.reshape(-1, 1)
    c = coords.reshape(-1, 3).astype(np.float32)
    ub = np.array([D, H, W], np.float32) - 1
    ok = np.all((c >= 0) & (c <= ub), axis=-1)
    vals, c = vals[ok], c[ok]
    if interpolation == "nearest":
        idx = np.rint(c).astype(np.int64)
        for ch in range(img.shape[0]):
            np.add.at(img[ch], (idx[:, 0], idx[:, 1], idx[:, 2]), vals[:, ch])
        np.add.at(weights, (idx[:, 0], idx[:, 1], idx[:, 2]), np.ones(len(c), weights.dtype))
    elif interpolation == "trilinear":
        lo = np.floor(c)
        hi = np.ceil(c)
        t = c - lo
        one = np.float32(1)
        for bz in (0, 1):
            for by in (0, 1):
                for bx in (0, 1):
                    fz = t[:, 0] if bz else one - t[:, 0]
                    fy = t[:, 1] if by else one - t[:, 1]
                    fx = t[:, 2] if bx else one - t[:, 2]
                    w = ((fz * fy) * fx).astype(weights.dtype)
                    zi = (hi if bz else lo)[:, 0].astype(np.int64)
                    yi = (hi if by else lo)[:, 1].astype(np.int64)
                    xi = (hi if bx else lo)[:, 2].astype(np.int64)
                    for ch in range(img.shape[0]):
                        np.add.at(img[ch], (zi, yi, xi), vals[:, ch] * w.astype(vals.dtype))
                    np.add.at(weights, (zi, yi, xi), w)
    out = img if multi else img[0]
    return out, weights


# ----------------------------------------------------------------------------
# real-space wrappers (numpy FFTs around the C oracle)
# ----------------------------------------------------------------------------

def _fftfreq_norm_grid(shape):
    """|fftfreq| grid, fftshifted, float32 (torch_grid_utils fftfreq_grid norm=True)."""
    axes = []
    for n in shape:
        k = np.arange(n)
        kk = np.where(k < (n + 1) // 2, k, k - n).astype(np.float32) * np.float32(1.0 / n)
        axes.append(np.fft.fftshift(kk))
    g = np.meshgrid(*axes, indexing="ij")
    s = np.zeros(shape, np.float32)
    for a in g:
        s = s + a * a
    return np.sqrt(s)


def _sinc(x):
    return np.sinc(x.astype(np.float64)).astype(np.float32)


def _crop_pad(pad_factor, n):
    return int((n * (pad_factor - 1.0)) // 2)


def project_3d_to_2d(volume, rotation_matrices, pad_factor=2.0, fftfreq_max=None,
                     zyx_matrices=False):
    vol = np.asarray(volume, np.float32)
    d, h, w = vol.shape
    if len({d, h, w}) != 1:
        raise ValueError("all dimensions of volume must be equal.")
    if pad_factor < 1.0:
        raise ValueError("pad_factor must be >= 1.0")
    p = 0
    if pad_factor > 1.0:
        p = _crop_pad(pad_factor, w)
        vol = np.pad(vol, p)
    shape = vol.shape
    vol = vol * _sinc(_fftfreq_norm_grid(shape)) ** 2
    dft = np.fft.rfftn(np.fft.fftshift(vol), axes=(0, 1, 2))
    dft = np.fft.fftshift(dft, axes=(0, 1)).astype(np.complex64)
    sl = extract(dft, shape, rotation_matrices, fftfreq_max=fftfreq_max,
                 zyx_matrices=zyx_matrices)
    sl = np.fft.ifftshift(sl, axes=(-2,))
    im = np.fft.irfftn(sl, axes=(-2, -1))  # no output size, as the reference (odd: n-1 wide)
    im = np.fft.ifftshift(im, axes=(-2, -1)).astype(np.float32)
    if p:
        im = im[..., p:-p, p:-p]
    return im


def backproject_2d_to_3d(images, rotation_matrices, pad_factor=2.0, fftfreq_max=None,
                         zyx_matrices=False):
    imgs = np.asarray(images)
    h, w = imgs.shape[-2:]
    if h != w:
        raise ValueError("images must be square.")
    if pad_factor < 1.0:
        raise ValueError("pad_factor must be >= 1.0")
    double = imgs.dtype == np.float64
    p = 0
    if pad_factor > 1.0:
        p = _crop_pad(pad_factor, w)
        imgs = np.pad(imgs, [(0, 0)] * (imgs.ndim - 2) + [(p, p), (p, p)])
    w = imgs.shape[-1]
    shape = (w, w, w)
    f = np.fft.rfftn(np.fft.fftshift(imgs, axes=(-2, -1)), axes=(-2, -1))
    f = np.fft.fftshift(f, axes=(-2,)).astype(np.complex128 if double else np.complex64)
    vol, wts = insert(f, shape, rotation_matrices, fftfreq_max=fftfreq_max,
                      zyx_matrices=zyx_matrices)
    vol = vol / np.maximum(wts, 1.0)
    vol = np.fft.ifftshift(vol, axes=(0, 1))
    real = np.fft.irfftn(vol, axes=(0, 1, 2))  # no output size, as the reference
    real = np.fft.ifftshift(real)
    real = real / _sinc(_fftfreq_norm_grid(real.shape)).astype(real.dtype) ** 2
    if p:
        real = real[p:-p, p:-p, p:-p]
    return real.astype(np.float64 if double else np.float32)
