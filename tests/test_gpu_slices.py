"""GPU parity of the central-slice kernels (through the C ABI) against the
reference's golden vectors and the CPU oracle.

Tolerances: bit-exact for the per-pixel masks (kept / conjugated / inside)
and the array coordinates; rel-L2 <= 1e-5 in fp32 for slices, volumes and
weights.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu
RTOL = 1e-5  # rel-L2, fp32


def tt():
    import teamtomo_b200

    return teamtomo_b200


def cuda(a):
    return torch.as_tensor(np.asarray(a)).cuda()


def _extract_kwargs(g, name):
    fmax = float(g[f"extract_{name}_fmax"])
    rtol = float(g[f"extract_{name}_rtol"])
    return dict(fftfreq_max=None if fmax < 0 else fmax, zyx_matrices=bool(int(g[f"extract_{name}_zyx"])),
                rot_tolerance=None if rtol < 0 else rtol, x_tolerance=float(g[f"extract_{name}_xtol"]))


def test_extract_matches_reference_golden(golden):
    for name in golden["extract_cases"]:
        name = str(name)
        out = tt().extract_central_slices_rfft_3d(
            cuda(golden[f"extract_{name}_volume"]), tuple(int(s) for s in golden[f"extract_{name}_shape"]),
            cuda(golden[f"extract_{name}_rot"]), **_extract_kwargs(golden, name))
        ref = golden[f"extract_{name}_out"]
        assert out.dtype == torch.complex64 and tuple(out.shape) == ref.shape, name
        assert rel_l2(out.cpu().numpy(), ref) < RTOL, name
        # zero pattern (outside fftfreq_max / outside the volume) is identical
        assert np.array_equal(out.cpu().numpy() == 0, ref == 0), name


@pytest.mark.parametrize("n", [64, 63])
@pytest.mark.parametrize("mode", ["extract", "insert"])
@pytest.mark.parametrize("kw", [dict(), dict(fftfreq_max=0.3), dict(zyx_matrices=True),
                                dict(rot_tolerance=None), dict(x_tolerance=1e-3)])
def test_geometry_bit_exact(oracle, golden, n, mode, kw):
    if mode == "insert" and ("rot_tolerance" in kw or "x_tolerance" in kw):
        pytest.skip("insertion has no tolerances")
    from teamtomo_b200.torch_fourier_slice.slice_extraction import central_slice_geometry

    rots = np.concatenate([rotations(300, seed=n), golden["extract_n16_rot"],
                           golden["extract_n16_rot"].astype(np.float32)])
    shape = (n, n, n)
    dims = (n, n, n // 2 + 1)
    f_gpu, c_gpu = central_slice_geometry(cuda(rots), shape, dims, mode=mode, **kw)
    f_ref, c_ref = oracle.slice_geometry(rots, shape, dims, 0 if mode == "extract" else 1, **kw)
    f_gpu, c_gpu = f_gpu.cpu().numpy(), c_gpu.cpu().numpy()
    assert np.array_equal(f_gpu, f_ref), f"{np.count_nonzero(f_gpu != f_ref)} flag mismatches"
    # exact float equality: identical values (the sign of a zero coordinate
    # may differ, the kernels drop the 0 * r0 term of the rotation)
    bad = np.count_nonzero(c_gpu != c_ref)
    assert bad == 0, f"{bad} coordinates differ"
    assert (f_ref & 2).any() and (f_ref & 4).any()


@pytest.mark.parametrize("n,nrot,kw", [(128, 200, {}), (96, 100, dict(fftfreq_max=0.4)),
                                       (65, 64, dict(zyx_matrices=True))])
def test_extract_matches_oracle(oracle, n, nrot, kw):
    vol = rfft_volume_np(blob_volume(n, seed=n))
    rots = rotations(nrot, seed=n + 1)
    out = tt().extract_central_slices_rfft_3d(cuda(vol), (n, n, n), cuda(rots), **kw)
    ref = oracle.extract(vol, (n, n, n), rots, **kw)
    assert rel_l2(out.cpu().numpy(), ref) < RTOL


def test_extract_leading_dims_and_empty():
    n = 32
    vol = cuda(rfft_volume_np(blob_volume(n, seed=1)))
    R = cuda(rotations(20, seed=2).reshape(4, 5, 3, 3))
    out = tt().extract_central_slices_rfft_3d(vol, (n, n, n), R)
    assert out.shape == (4, 5, n, n // 2 + 1)
    one = tt().extract_central_slices_rfft_3d(vol, (n, n, n), R[1, 2])
    assert one.shape == (n, n // 2 + 1)
    assert torch.equal(one, out[1, 2])
    empty = tt().extract_central_slices_rfft_3d(vol, (n, n, n), R[:0, 0])
    assert empty.shape == (0, n, n // 2 + 1)
    # every pixel outside the disc -> all zeros
    tiny = tt().extract_central_slices_rfft_3d(vol, (n, n, n), R[0], fftfreq_max=-1.0)
    assert torch.count_nonzero(tiny) == 0


def test_extract_does_not_mutate_rotations():
    n = 16
    vol = cuda(rfft_volume_np(blob_volume(n, seed=3)))
    R = torch.eye(3, device="cuda")[None].repeat(3, 1, 1)
    R[:, 0, 1] = 1e-9  # below rot_tolerance
    R0 = R.clone()
    R.requires_grad_(True)
    out = tt().extract_central_slices_rfft_3d(vol, (n, n, n), R)
    out.abs().sum().backward()
    assert torch.equal(R.detach(), R0)
    assert torch.all(R.grad[:, 0, 1] == 0)


def test_extract_conjugate_pairs(golden):
    """ZYZ pairs 180 deg apart give conjugate slices
    (test_extract_central_slices_rfft_3d.py:108-186, blob volume in place of
    the simulated map), at the true and a 4x inflated image_shape."""
    from scipy.spatial.transform import Rotation

    from helpers import PAIRS

    n = 64
    vol = cuda(rfft_volume_np(blob_volume(n, seed=64)))
    for shape in ((n, n, n), (4 * n, 4 * n, 4 * n)):
        for left, right in PAIRS:
            L = cuda(Rotation.from_euler("ZYZ", left, degrees=True).as_matrix())
            Rr = cuda(Rotation.from_euler("ZYZ", right, degrees=True).as_matrix())
            a = tt().extract_central_slices_rfft_3d(vol, shape, L)
            b = tt().extract_central_slices_rfft_3d(vol, shape, Rr)
            assert torch.allclose(a, torch.conj(b), atol=1e-6 * float(vol.abs().max())), (left, right)


def test_extract_random_conjugate_pairs():
    """test_extract_central_slices_rfft_3d.py:189-232: a +180 deg in-plane
    offset gives the conjugate slice."""
    from scipy.spatial.transform import Rotation

    n = 64
    vol = cuda(rfft_volume_np(blob_volume(n, seed=65)))
    rng = np.random.default_rng(0)
    ang = np.stack([rng.uniform(0, 360, 100), rng.uniform(0, 180, 100), rng.uniform(0, 360, 100)], 1)
    off = Rotation.from_euler("ZYZ", [0, 0, 180], degrees=True).as_matrix()
    left = Rotation.from_euler("ZYZ", ang, degrees=True).as_matrix()
    right = left @ off
    a = tt().extract_central_slices_rfft_3d(vol, (n, n, n), cuda(left))
    b = tt().extract_central_slices_rfft_3d(vol, (n, n, n), cuda(right))
    assert torch.allclose(a, torch.conj(b), atol=1e-6 * float(vol.abs().max()))


def test_extract_friedel_x0_line():
    """test_extract_central_slices_rfft_3d.py:72-105: the x=0 column of every
    extracted slice obeys Friedel symmetry."""
    n = 64
    vol = cuda(rfft_volume_np(blob_volume(n, seed=66)))
    s = tt().extract_central_slices_rfft_3d(vol, (n, n, n), cuda(rotations(10, seed=4)))
    x0 = s[:, :, 0]
    half = x0[:, 1: n // 2]
    conj_half = torch.flip(torch.conj(x0[:, -(n // 2 - 1):]), dims=[1])
    assert torch.allclose(half, conj_half, atol=1e-6 * float(vol.abs().max()))


def test_extract_complex128_rejected():
    n = 8
    vol = torch.zeros((n, n, n // 2 + 1), dtype=torch.complex128, device="cuda")
    with pytest.raises(RuntimeError):
        tt().extract_central_slices_rfft_3d(vol, (n, n, n), torch.eye(3, device="cuda"))


# ----------------------------------------------------------------------------
# insertion
# ----------------------------------------------------------------------------

def _insert_kwargs(g, name):
    fmax = float(g[f"insert_{name}_fmax"])
    return dict(fftfreq_max=None if fmax < 0 else fmax, zyx_matrices=bool(int(g[f"insert_{name}_zyx"])))


def test_insert_matches_reference_golden(golden):
    for name in golden["insert_cases"]:
        name = str(name)
        imgs = golden[f"insert_{name}_images"]
        n = imgs.shape[-2]
        vol, w = tt().insert_central_slices_rfft_3d(cuda(imgs), (n, n, n), cuda(golden[f"insert_{name}_rot"]),
                                                    **_insert_kwargs(golden, name))
        ref_v, ref_w = golden[f"insert_{name}_volume"], golden[f"insert_{name}_weights"]
        assert vol.cpu().numpy().dtype == ref_v.dtype and w.cpu().numpy().dtype == ref_w.dtype, name
        tol = 1e-12 if ref_v.dtype == np.complex128 else RTOL
        assert rel_l2(vol.cpu().numpy(), ref_v) < tol, name
        assert rel_l2(w.cpu().numpy(), ref_w) < tol, name
        assert np.array_equal(w.cpu().numpy() != 0, ref_w != 0), name


@pytest.mark.parametrize("n,nrot,kw", [(64, 300, {}), (63, 100, {}), (64, 100, dict(fftfreq_max=0.35)),
                                       (32, 64, dict(zyx_matrices=True)),
                                       (256, 40, {}),  # 4 z-slab passes
                                       (201, 30, dict(fftfreq_max=0.45))])  # odd box, 2 passes
def test_insert_matches_oracle(oracle, n, nrot, kw):
    rng = np.random.default_rng(n)
    imgs = (rng.standard_normal((nrot, n, n // 2 + 1)) + 1j * rng.standard_normal((nrot, n, n // 2 + 1)))
    imgs = imgs.astype(np.complex64)
    rots = rotations(nrot, seed=n + 2)
    vol, w = tt().insert_central_slices_rfft_3d(cuda(imgs), (n, n, n), cuda(rots), **kw)
    rv, rw = oracle.insert(imgs, (n, n, n), rots, **kw)
    assert rel_l2(vol.cpu().numpy(), rv) < RTOL
    assert rel_l2(w.cpu().numpy(), rw) < RTOL
    assert np.array_equal(w.cpu().numpy() != 0, rw != 0)


def test_insert_complex128(oracle):
    n, nrot = 32, 50
    rng = np.random.default_rng(5)
    imgs = (rng.standard_normal((nrot, n, n // 2 + 1)) + 1j * rng.standard_normal((nrot, n, n // 2 + 1)))
    rots = rotations(nrot, seed=6)
    vol, w = tt().insert_central_slices_rfft_3d(cuda(imgs), (n, n, n), cuda(rots))
    assert vol.dtype == torch.complex128 and w.dtype == torch.float64
    rv, rw = oracle.insert(imgs, (n, n, n), rots)
    assert rel_l2(vol.cpu().numpy(), rv) < 1e-12
    assert rel_l2(w.cpu().numpy(), rw) < 1e-12


def test_insert_friedel_symmetry_x0_plane():
    """test_torch_fourier_slice.py:174-291 on the kernels: the inserted x=0
    plane obeys F(z, y) = conj F(-z, -y)."""
    from scipy.spatial.transform import Rotation

    n = 32
    cube = torch.zeros((n, n, n), device="cuda")
    cube[8:24, 8:24, 8:24] = 1
    cube[16, 16, 16] = 32
    ang = np.array([[0.0, 0.0], [0.0, 0.0], [0.0, 180.0]]).T
    rx = Rotation.from_euler("ZYZ", ang, degrees=True).as_matrix()
    extra = np.stack([np.array([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], float),
                      np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1]], float)])
    rots = np.concatenate([rx, extra, rotations(4, seed=42)]).astype(np.float32)
    proj = tt().project_3d_to_2d(cube, cuda(rots))
    imgs = torch.fft.fftshift(torch.fft.rfftn(torch.fft.fftshift(proj, dim=(-2, -1)), dim=(-2, -1)), dim=(-2,))
    vol, _ = tt().insert_central_slices_rfft_3d(imgs, (n, n, n), cuda(rots))
    p = vol[:, :, 0].cpu().numpy()
    err, cnt = 0.0, 0
    for z in range(n // 2 + 1):
        for y in (range(n) if z < n // 2 else range(n // 2 + 1)):
            if z == n // 2 and y == n // 2:
                continue
            err += abs(p[z, y] - np.conj(p[(n - z) % n, (n - y) % n]))
            cnt += 1
    assert err / cnt < 1e-5


def test_insert_rejects_bad_shapes():
    with pytest.raises(ValueError):
        tt().insert_central_slices_rfft_3d(torch.zeros((2, 8, 4), dtype=torch.complex64, device="cuda"),
                                           (8, 8, 8), torch.eye(3, device="cuda")[None].repeat(2, 1, 1))
    with pytest.raises(ValueError):
        tt().insert_central_slices_rfft_3d(torch.zeros((2, 8, 5), dtype=torch.complex64, device="cuda"),
                                           (8, 8, 8), torch.eye(3, device="cuda")[None].repeat(3, 1, 1))


def test_multichannel_slices():
    n, c = 16, 3
    vols = cuda(np.stack([rfft_volume_np(blob_volume(n, seed=s)) for s in range(c)]))
    R = cuda(rotations(5, seed=7))
    out = tt().extract_central_slices_rfft_3d_multichannel(vols, (n, n, n), R)
    assert out.shape == (5, c, n, n // 2 + 1)
    for ch in range(c):
        assert torch.equal(out[:, ch], tt().extract_central_slices_rfft_3d(vols[ch], (n, n, n), R))
    v, w = tt().insert_central_slices_rfft_3d_multichannel(out, (n, n, n), R)
    assert v.shape == (c, n, n, n // 2 + 1) and w.shape == (n, n, n // 2 + 1)
    v1, w1 = tt().insert_central_slices_rfft_3d(out[:, 1].contiguous(), (n, n, n), R)
    assert rel_l2(v[1].cpu().numpy(), v1.cpu().numpy()) < RTOL
    assert rel_l2(w.cpu().numpy(), w1.cpu().numpy()) < RTOL
