"""Generate the golden fixtures in this directory from the reference itself.

Imports the pure-Python reference (torch-fourier-slice, torch-image-interpolation,
torch-grid-utils) from its source tree and records inputs and outputs of
small, seeded cases into ``golden.npz``.  The fixtures are committed; the
reference does not need to exist where the tests run.

Usage:  python tests/golden/make_golden.py [/path/to/reference]

Cases (reference test each one mirrors):
  extract_*      extract_central_slices_rfft_3d: random SO(3) (seeded), the
                 ZYZ pairs 180 deg apart of test_extract_central_slices_rfft_3d.py:22-31,
                 axis-aligned 90 deg rotations, fftfreq_max, zyx_matrices,
                 inflated image_shape (:146-186), odd box size, float64 rotations
                 with rot_tolerance=None
  insert_*       insert_central_slices_rfft_3d incl. complex128 (weights f64)
  grad_*         reference autograd: d/drotation (float64 leaf) and d/dvolume
                 (tiny size: the reference expands the volume per sample)
  sample_*       sample_image_3d values (real / complex / multichannel, trilinear / nearest)
  insimg_*       insert_into_image_3d (trilinear / nearest, f32 / c64, f64 weights)
  project_*      project_3d_to_2d of the conftest cube (torch-fourier-slice/tests/conftest.py:5-10)
  backproject_*  backproject_2d_to_3d of those projections (float32 and float64)
  ctf_*          torch-ctf calculate_ctf_2d grids
  insgrad_*      reference autograd of insert_central_slices_rfft_3d w.r.t. the images
  bpgrad_*       reference autograd of backproject_2d_to_3d w.r.t. the images
  lines_*, linesgrad_*, proj1d_*   extract_central_slices_rfft_2d (+ its autograd), project_2d_to_1d
  affine_*       torch_transform_image.affine_transform_image_3d
  sgrad_*        sample_image_3d autograd w.r.t. the image and the coordinates
  igrad_*        insert_into_image_3d autograd w.r.t. the values
"""

from __future__ import annotations

import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TT_REFERENCE_ROOT")
if not REF:
    sys.exit("usage: make_golden.py REFERENCE_ROOT (or set TT_REFERENCE_ROOT): the reference checkout's root")
for pkg in ("torch-fourier-slice", "torch-image-interpolation", "torch-grid-utils"):
    sys.path.insert(0, os.path.join(REF, "packages", "primitives", pkg, "src"))

import torch  # noqa: E402
from scipy.spatial.transform import Rotation  # noqa: E402
from scipy.stats import special_ortho_group  # noqa: E402
from torch_fourier_slice import (  # noqa: E402
    backproject_2d_to_3d,
    extract_central_slices_rfft_3d,
    insert_central_slices_rfft_3d,
    project_3d_to_2d,
)
from torch_image_interpolation import insert_into_image_3d, sample_image_3d  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")
PAIRS = [  # ZYZ degrees, test_extract_central_slices_rfft_3d.py:22-31
    ([0, 0, 0], [0, 0, 180]), ([0, 0, 0], [180, 0, 0]), ([0, 20, 0], [0, 20, 180]),
    ([0, 20, 90], [0, 20, 270]), ([0, 60, 0], [0, 60, 180]), ([90, 90, 0], [90, 90, 180]),
    ([45, 0, 0], [45, 0, 180]), ([45, 90, 0], [45, 90, 180]),
]


def blob_volume(n: int, seed: int) -> np.ndarray:
    """Sum of 20 Gaussian blobs (sigma 2-6 px scaled by n/64) + N(0, 0.01^2)."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(*([np.arange(n)] * 3), indexing="ij")
    vol = np.zeros((n, n, n), np.float64)
    for _ in range(20):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        c = n / 2 + u * 0.375 * n * rng.uniform() ** (1.0 / 3.0)
        s = rng.uniform(2, 6) * n / 64
        vol += np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / (2 * s * s))
    vol += rng.normal(0, 0.01, size=vol.shape)
    return vol.astype(np.float32)


def rfft_volume(vol: np.ndarray) -> torch.Tensor:
    t = torch.tensor(vol)
    t = torch.fft.fftshift(t, dim=(-3, -2, -1))
    t = torch.fft.rfftn(t, dim=(-3, -2, -1))
    return torch.fft.fftshift(t, dim=(-3, -2))


def zyz(angles) -> np.ndarray:
    return Rotation.from_euler("ZYZ", np.asarray(angles, float), degrees=True).as_matrix()


def special_rotations() -> np.ndarray:
    mats = [zyz(a) for pair in PAIRS for a in pair]
    mats += [
        np.array([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], float),   # y 90 (test_torch_fourier_slice.py:196-203)
        np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1]], float),   # z 90 (:206-214)
        np.eye(3),
        np.diag([1.0, -1.0, -1.0]),
    ]
    return np.stack(mats)


def main():
    torch.manual_seed(0)
    g: dict[str, np.ndarray] = {}

    # ---------------- extraction ----------------
    cases = []
    for n in (16, 17):
        vol = rfft_volume(blob_volume(n, 100 + n))
        rnd = special_ortho_group.rvs(3, size=24, random_state=n)
        rots = np.concatenate([rnd, special_rotations()])
        cases += [
            (f"n{n}", vol, (n, n, n), rots, dict()),
            (f"n{n}_fmax", vol, (n, n, n), rots, dict(fftfreq_max=0.3)),
            (f"n{n}_zyx", vol, (n, n, n), rots, dict(zyx_matrices=True)),
        ]
    vol16 = rfft_volume(blob_volume(16, 116))
    rots16 = np.concatenate([special_ortho_group.rvs(3, size=8, random_state=5), special_rotations()])
    cases.append(("n16_big_image", vol16, (64, 64, 64), rots16, dict()))
    cases.append(("n16_nortol", vol16, (16, 16, 16), rots16, dict(rot_tolerance=None)))
    cases.append(("n16_xtol", vol16, (16, 16, 16), rots16, dict(x_tolerance=1e-3)))
    names = []
    for name, vol, shape, rots, kw in cases:
        out = extract_central_slices_rfft_3d(vol, shape, torch.tensor(rots), **kw)
        g[f"extract_{name}_volume"] = vol.numpy()
        g[f"extract_{name}_rot"] = rots
        g[f"extract_{name}_shape"] = np.array(shape)
        g[f"extract_{name}_fmax"] = np.array(kw.get("fftfreq_max", -1.0))
        g[f"extract_{name}_zyx"] = np.array(int(kw.get("zyx_matrices", False)))
        rtol = kw.get("rot_tolerance", 1e-8)
        g[f"extract_{name}_rtol"] = np.array(-1.0 if rtol is None else rtol)
        g[f"extract_{name}_xtol"] = np.array(kw.get("x_tolerance", 1e-8))
        g[f"extract_{name}_out"] = out.numpy()
        names.append(name)
    g["extract_cases"] = np.array(names)

    # ---------------- insertion ----------------
    names = []
    for n, dt, kw in ((16, torch.complex64, {}), (17, torch.complex64, {}),
                      (16, torch.complex64, dict(fftfreq_max=0.25)),
                      (16, torch.complex128, {}), (16, torch.complex64, dict(zyx_matrices=True))):
        rots = np.concatenate([special_ortho_group.rvs(3, size=12, random_state=n + 7),
                               special_rotations()])
        imgs = torch.randn(len(rots), n, n // 2 + 1, dtype=dt)
        vol, w = insert_central_slices_rfft_3d(imgs, (n, n, n), torch.tensor(rots), **kw)
        name = f"n{n}_{str(dt).split('.')[-1]}" + "".join(f"_{k}" for k in kw)
        g[f"insert_{name}_images"] = imgs.numpy()
        g[f"insert_{name}_rot"] = rots
        g[f"insert_{name}_fmax"] = np.array(kw.get("fftfreq_max", -1.0))
        g[f"insert_{name}_zyx"] = np.array(int(kw.get("zyx_matrices", False)))
        g[f"insert_{name}_volume"] = vol.numpy()
        g[f"insert_{name}_weights"] = w.numpy()
        names.append(name)
    g["insert_cases"] = np.array(names)

    # ---------------- gradients (reference autograd) ----------------
    n = 16
    vol = rfft_volume(blob_volume(n, 7))
    rots = special_ortho_group.rvs(3, size=8, random_state=11)
    G = torch.randn(8, n, n // 2 + 1, dtype=torch.complex64)
    R = torch.tensor(rots, requires_grad=True)
    s = extract_central_slices_rfft_3d(vol, (n, n, n), R)
    (s * G.conj()).real.sum().backward()
    g["grad_drot_volume"], g["grad_drot_rot"], g["grad_drot_G"] = vol.numpy(), rots, G.numpy()
    g["grad_drot_out"] = R.grad.numpy()
    n = 10
    vol = rfft_volume(blob_volume(n, 9)).requires_grad_(True)
    rots = special_ortho_group.rvs(3, size=6, random_state=13)
    G = torch.randn(6, n, n // 2 + 1, dtype=torch.complex64)
    s = extract_central_slices_rfft_3d(vol, (n, n, n), torch.tensor(rots))
    (s * G.conj()).real.sum().backward()
    g["grad_dvol_volume"], g["grad_dvol_rot"], g["grad_dvol_G"] = vol.detach().numpy(), rots, G.numpy()
    g["grad_dvol_out"] = vol.grad.numpy()

    # ---------------- sample_image_3d ----------------
    rng = np.random.default_rng(3)
    for name, shape, dt in (("real", (7, 8, 9), torch.float32), ("complex", (7, 8, 9), torch.complex64),
                            ("multi", (3, 7, 8, 9), torch.float32), ("f64", (7, 8, 9), torch.float64)):
        img = torch.randn(shape, dtype=dt)
        hi = np.array(shape[-3:]) - 1
        coords = rng.uniform(-0.7, hi + 0.7, size=(5, 11, 3))
        coords[0, :3] = np.array([[0, 0, 0], hi, [hi[0], 0.5, hi[2]]])
        rdt = torch.float64 if dt in (torch.float64, torch.complex128) else torch.float32
        c = torch.tensor(coords, dtype=rdt)
        for mode in ("trilinear", "nearest"):
            g[f"sample_{name}_{mode}_out"] = sample_image_3d(img, c, interpolation=mode).numpy()
        g[f"sample_{name}_image"], g[f"sample_{name}_coords"] = img.numpy(), c.numpy()

    # ---------------- insert_into_image_3d ----------------
    for name, dt, wdt in (("f32", torch.float32, torch.float32), ("c64", torch.complex64, torch.float32),
                          ("f32w64", torch.float32, torch.float64)):
        img = torch.zeros((9, 10, 11), dtype=dt)
        vals = torch.randn((4, 13), dtype=dt)
        coords = torch.tensor(rng.uniform(-0.5, 10.5, size=(4, 13, 3)), dtype=torch.float32)
        coords[0, 0] = torch.tensor([2.0, 3.0, 4.0])
        coords[0, 1] = torch.tensor([8.0, 9.0, 10.0])
        for mode in ("trilinear", "nearest"):
            i2, w2 = insert_into_image_3d(vals, coords, img.clone(), torch.zeros((9, 10, 11), dtype=wdt),
                                          interpolation=mode)
            g[f"insimg_{name}_{mode}_image"], g[f"insimg_{name}_{mode}_weights"] = i2.numpy(), w2.numpy()
        g[f"insimg_{name}_values"], g[f"insimg_{name}_coords"] = vals.numpy(), coords.numpy()
    img = torch.zeros((2, 9, 10, 11))
    vals = torch.randn((4, 13, 2))
    coords = torch.tensor(rng.uniform(0, 8, size=(4, 13, 3)), dtype=torch.float32)
    i2, w2 = insert_into_image_3d(vals, coords, img.clone())
    g["insimg_multi_values"], g["insimg_multi_coords"] = vals.numpy(), coords.numpy()
    g["insimg_multi_trilinear_image"], g["insimg_multi_trilinear_weights"] = i2.numpy(), w2.numpy()

    # ---------------- project / backproject ----------------
    cube = torch.zeros((32, 32, 32))
    cube[8:24, 8:24, 8:24] = 1
    cube[16, 16, 16] = 32
    rots = special_ortho_group.rvs(3, size=6, random_state=42)
    proj = project_3d_to_2d(cube, torch.tensor(rots))
    g["project_volume"], g["project_rot"], g["project_out"] = cube.numpy(), rots, proj.numpy()
    g["project_fmax_out"] = project_3d_to_2d(cube, torch.tensor(rots), fftfreq_max=0.25).numpy()
    g["project_pad1_out"] = project_3d_to_2d(cube, torch.tensor(rots), pad_factor=1.0).numpy()
    rec = backproject_2d_to_3d(proj, torch.tensor(rots))
    g["backproject_images"], g["backproject_rot"], g["backproject_out"] = proj.numpy(), rots, rec.numpy()
    rec64 = backproject_2d_to_3d(proj.double(), torch.tensor(rots))
    g["backproject_f64_out"] = rec64.numpy()
    # odd padded box: the reference's irfftn has no output size -> (d, d-1) images
    odd = torch.tensor(blob_volume(33, 33))
    proj_odd = project_3d_to_2d(odd, torch.tensor(rots), pad_factor=1.5)
    g["project_odd_volume"], g["project_odd_out"] = odd.numpy(), proj_odd.numpy()
    imgs_odd = torch.tensor(np.random.default_rng(4).standard_normal((6, 33, 33)).astype(np.float32))
    g["backproject_odd_images"] = imgs_odd.numpy()
    g["backproject_odd_out"] = backproject_2d_to_3d(imgs_odd, torch.tensor(rots), pad_factor=1.5).numpy()

    # ---------------- CTF (torch-ctf calculate_ctf_2d) ----------------
    sys.path.insert(0, os.path.join(REF, "packages", "primitives", "torch-ctf", "src"))
    from torch_ctf import calculate_ctf_2d

    ctf_cases = [  # defocus, astig, angle, kV, Cs, Ac, phase, px, shape, rfft, fftshift
        (1.5, 0.0, 0.0, 300.0, 2.7, 0.1, 0.0, 8.0, (10, 10), False, False),  # test_torch_ctf.py:376-392
        (2.5, 0.0, 0.0, 300.0, 2.7, 0.1, 0.0, 8.0, (10, 10), False, False),
        (2.0, 0.5, 30.0, 300.0, 2.7, 0.07, 0.0, 1.0, (64, 64), True, True),
        (0.8, 0.2, 75.0, 200.0, 2.0, 0.1, 20.0, 1.5, (33, 33), True, True),
        (3.0, 0.0, 0.0, 300.0, 2.7, 0.07, 0.0, 1.0, (128, 128), True, True),
    ]
    for i, (df, ast, ang, kv, cs, ac, ps, px, shape, rf, fs) in enumerate(ctf_cases):
        ctf = calculate_ctf_2d(defocus=df, astigmatism=ast, astigmatism_angle=ang, voltage=kv,
                               spherical_aberration=cs, amplitude_contrast=ac, phase_shift=ps,
                               pixel_size=px, image_shape=shape, rfft=rf, fftshift=fs)
        g[f"ctf_{i}_params"] = np.array([df, ast, ang, kv, cs, ac, ps, px], np.float64)
        g[f"ctf_{i}_shape"] = np.array(shape)
        g[f"ctf_{i}_flags"] = np.array([int(rf), int(fs)])
        g[f"ctf_{i}_out"] = ctf.numpy()
    g["ctf_cases"] = np.array(len(ctf_cases))

    # ---------------- insertion backward w.r.t. the images (reference autograd) ----------------
    gen = torch.Generator().manual_seed(21)
    names = []
    for n, dt, kw in ((16, torch.complex64, {}), (17, torch.complex64, {}), (16, torch.complex128, {}),
                      (16, torch.complex64, dict(fftfreq_max=0.3, zyx_matrices=True))):
        rots = np.concatenate([special_ortho_group.rvs(3, size=10, random_state=n + 31),
                               special_rotations()])
        imgs = torch.randn(len(rots), n, n // 2 + 1, dtype=dt, generator=gen).requires_grad_(True)
        gvol = torch.randn(n, n, n // 2 + 1, dtype=dt, generator=gen)
        vol, _ = insert_central_slices_rfft_3d(imgs, (n, n, n), torch.tensor(rots), **kw)
        (vol * gvol.conj()).real.sum().backward()
        name = f"n{n}_{str(dt).split('.')[-1]}" + "".join(f"_{k}" for k in kw)
        g[f"insgrad_{name}_images"] = imgs.detach().numpy()
        g[f"insgrad_{name}_rot"] = rots
        g[f"insgrad_{name}_gvol"] = gvol.numpy()
        g[f"insgrad_{name}_fmax"] = np.array(kw.get("fftfreq_max", -1.0))
        g[f"insgrad_{name}_zyx"] = np.array(int(kw.get("zyx_matrices", False)))
        g[f"insgrad_{name}_out"] = imgs.grad.numpy()
        names.append(name)
    g["insgrad_cases"] = np.array(names)

    # ---------------- backprojection backward w.r.t. the images (reference autograd) ----------------
    gen = torch.Generator().manual_seed(23)
    for name, d, pf in (("even", 16, 2.0), ("odd", 17, 1.5)):
        rots = special_ortho_group.rvs(3, size=5, random_state=d)
        imgs = torch.randn(5, d, d, generator=gen).requires_grad_(True)
        rec = backproject_2d_to_3d(imgs, torch.tensor(rots), pad_factor=pf)
        G = torch.randn(rec.shape, generator=gen)
        (rec * G).sum().backward()
        g[f"bpgrad_{name}_images"], g[f"bpgrad_{name}_rot"] = imgs.detach().numpy(), rots
        g[f"bpgrad_{name}_G"], g[f"bpgrad_{name}_pad"] = G.numpy(), np.array(pf)
        g[f"bpgrad_{name}_out"] = imgs.grad.numpy()

    # ---------------- d/drotation at axis-aligned rotations (points on the border) ----------------
    n = 16
    vol = rfft_volume(blob_volume(n, 31))
    rots = special_rotations()
    G = torch.randn(len(rots), n, n // 2 + 1, dtype=torch.complex64, generator=torch.Generator().manual_seed(31))
    R = torch.tensor(rots, requires_grad=True)
    (extract_central_slices_rfft_3d(vol, (n, n, n), R) * G.conj()).real.sum().backward()
    g["grad_axes_volume"], g["grad_axes_rot"], g["grad_axes_G"] = vol.numpy(), rots, G.numpy()
    g["grad_axes_out"] = R.grad.numpy()

    # ---------------- central lines of 2D images ----------------
    from torch_fourier_slice import extract_central_slices_rfft_2d, project_2d_to_1d

    gen = torch.Generator().manual_seed(29)
    th = torch.tensor(np.concatenate([np.linspace(0, 2 * np.pi, 13, endpoint=False), [np.pi / 2, np.pi]]))
    rot2 = torch.stack([torch.stack([torch.cos(th), -torch.sin(th)], -1),
                        torch.stack([torch.sin(th), torch.cos(th)], -1)], -2)  # (15, 2, 2) float64
    names = []
    for h, yx in ((16, False), (17, False), (16, True)):
        img = torch.randn(h, h // 2 + 1, dtype=torch.complex64, generator=gen)
        name = f"h{h}" + ("_yx" if yx else "")
        g[f"lines_{name}_image"], g[f"lines_{name}_rot"] = img.numpy(), rot2.numpy()
        g[f"lines_{name}_yx"] = np.array(int(yx))
        g[f"lines_{name}_out"] = extract_central_slices_rfft_2d(img, (h, h), rot2, yx_matrices=yx).numpy()
        names.append(name)
    g["lines_cases"] = np.array(names)
    R = rot2.clone().requires_grad_(True)
    img = torch.randn(16, 9, dtype=torch.complex64, generator=gen).requires_grad_(True)
    G = torch.randn(15, 9, dtype=torch.complex64, generator=gen)
    (extract_central_slices_rfft_2d(img, (16, 16), R) * G.conj()).real.sum().backward()
    g["linesgrad_image"], g["linesgrad_G"] = img.detach().numpy(), G.numpy()
    g["linesgrad_drot"], g["linesgrad_dimage"] = R.grad.numpy(), img.grad.numpy()
    for name, d, pf in (("even", 32, 2.0), ("odd", 17, 1.5)):
        im = torch.randn(d, d, generator=gen)
        g[f"proj1d_{name}_image"], g[f"proj1d_{name}_pad"] = im.numpy(), np.array(pf)
        g[f"proj1d_{name}_out"] = project_2d_to_1d(im, rot2.float(), pad_factor=pf).numpy()

    # ---------------- affine_transform_image_3d (torch-transform-image) ----------------
    for pkg in ("torch-transform-image", "torch-affine-utils"):
        sys.path.insert(0, os.path.join(REF, "packages", "primitives", pkg, "src"))
    from torch_transform_image import affine_transform_image_3d

    gen = torch.Generator().manual_seed(37)
    rot = torch.tensor(special_ortho_group.rvs(3, size=3, random_state=37), dtype=torch.float32)
    M = torch.eye(4).repeat(3, 1, 1)
    M[:, :3, :3] = rot
    M[:, :3, 3] = torch.tensor([[1.5, -2.0, 0.25], [0.0, 3.0, -1.0], [2.0, 2.0, 2.0]])
    for name, img in (("real", torch.randn(9, 10, 11, generator=gen)),
                      ("complex", torch.randn(9, 10, 11, dtype=torch.complex64, generator=gen)),
                      ("multi", torch.randn(2, 9, 10, 11, generator=gen))):
        g[f"affine_{name}_image"] = img.numpy()
        for mode in ("trilinear", "nearest"):  # the reference takes one (4, 4) matrix per call
            g[f"affine_{name}_{mode}_out"] = np.stack(
                [affine_transform_image_3d(img, M[i], interpolation=mode).numpy() for i in range(3)])
    g["affine_matrices"] = M.numpy()
    g["affine_shape_zyx_out"] = affine_transform_image_3d(g_img := torch.randn(8, 8, 8, generator=gen), M[0],
                                                          interpolation="trilinear", output_shape=(6, 7, 5),
                                                          zyx_matrices=True).numpy()
    g["affine_shape_zyx_image"] = g_img.numpy()

    # ---------------- sample_image_3d autograd (image and coordinates) ----------------
    gen = torch.Generator().manual_seed(41)
    rng2 = np.random.default_rng(41)
    for name, shape, dt in (("real", (7, 8, 9), torch.float32), ("complex", (7, 8, 9), torch.complex64),
                            ("multi", (3, 7, 8, 9), torch.float32)):
        img = torch.randn(shape, dtype=dt, generator=gen).requires_grad_(True)
        hi = np.array(shape[-3:]) - 1
        coords = rng2.uniform(-0.5, hi + 0.5, size=(6, 10, 3))
        coords[0, :4] = np.array([[0, 2.5, 3.5], [hi[0], 1.5, 2.5], [2.5, hi[1], 0], [3.25, 4.5, hi[2]]])
        c = torch.tensor(coords, dtype=torch.float32, requires_grad=True)
        out = sample_image_3d(img, c, interpolation="trilinear")
        G = torch.randn(out.shape, dtype=out.dtype, generator=gen)
        (out * G.conj()).real.sum().backward()
        g[f"sgrad_{name}_image"], g[f"sgrad_{name}_coords"], g[f"sgrad_{name}_G"] = (
            img.detach().numpy(), c.detach().numpy(), G.numpy())
        g[f"sgrad_{name}_dimage"], g[f"sgrad_{name}_dcoords"] = img.grad.numpy(), c.grad.numpy()

    # ---------------- insert_into_image_3d autograd w.r.t. the values ----------------
    for name, dt, mode in (("f32", torch.float32, "trilinear"), ("c64", torch.complex64, "trilinear"),
                           ("f32", torch.float32, "nearest")):
        vals = torch.randn((5, 12), dtype=dt, generator=gen).requires_grad_(True)
        coords = torch.tensor(rng2.uniform(-0.5, 9.5, size=(5, 12, 3)), dtype=torch.float32)
        img, _ = insert_into_image_3d(vals, coords, torch.zeros((9, 10, 11), dtype=dt), interpolation=mode)
        G = torch.randn(img.shape, dtype=dt, generator=gen)
        (img * G.conj()).real.sum().backward()
        key = f"igrad_{name}_{mode}"
        g[f"{key}_values"], g[f"{key}_coords"], g[f"{key}_G"] = vals.detach().numpy(), coords.numpy(), G.numpy()
        g[f"{key}_dvalues"] = vals.grad.numpy()

    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT}: {os.path.getsize(OUT) / 1e6:.2f} MB, {len(g)} arrays")


if __name__ == "__main__":
    main()
