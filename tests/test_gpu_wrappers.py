"""GPU parity of project_3d_to_2d / backproject_2d_to_3d and the
torch_image_interpolation primitives, mirroring the reference's own tests
(torch-fourier-slice/tests/test_torch_fourier_slice.py,
torch-image-interpolation/tests/test_image_interpolation_3d.py)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import blob_volume, fsc, rel_l2, rotations

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def tt():
    import teamtomo_b200

    return teamtomo_b200


def cuda(a):
    return torch.as_tensor(np.asarray(a)).cuda()


def cube(n=32):
    v = torch.zeros((n, n, n), device="cuda")
    v[8:24, 8:24, 8:24] = 1
    v[16, 16, 16] = 32
    return v


def test_project_matches_reference_golden(golden):
    vol, rot = cuda(golden["project_volume"]), cuda(golden["project_rot"])
    assert rel_l2(tt().project_3d_to_2d(vol, rot).cpu().numpy(), golden["project_out"]) < RTOL
    assert rel_l2(tt().project_3d_to_2d(vol, rot, fftfreq_max=0.25).cpu().numpy(),
                  golden["project_fmax_out"]) < RTOL
    assert rel_l2(tt().project_3d_to_2d(vol, rot, pad_factor=1.0).cpu().numpy(),
                  golden["project_pad1_out"]) < RTOL


def test_backproject_matches_reference_golden(golden):
    imgs, rot = cuda(golden["backproject_images"]), cuda(golden["backproject_rot"])
    rec = tt().backproject_2d_to_3d(imgs, rot)
    assert rec.dtype == torch.float32
    assert rel_l2(rec.cpu().numpy(), golden["backproject_out"]) < RTOL
    rec64 = tt().backproject_2d_to_3d(imgs.double(), rot)
    assert rec64.dtype == torch.float64
    assert rel_l2(rec64.cpu().numpy(), golden["backproject_f64_out"]) < RTOL
    # odd padded box (33 at pad 1.5 -> 49): (d, d-1) projections, (d, d, d-1) volumes
    po = tt().project_3d_to_2d(cuda(golden["project_odd_volume"]), cuda(golden["project_rot"]), pad_factor=1.5)
    assert tuple(po.shape) == golden["project_odd_out"].shape
    assert rel_l2(po.cpu().numpy(), golden["project_odd_out"]) < RTOL
    bo = tt().backproject_2d_to_3d(cuda(golden["backproject_odd_images"]), cuda(golden["project_rot"]),
                                   pad_factor=1.5)
    assert tuple(bo.shape) == golden["backproject_odd_out"].shape
    assert rel_l2(bo.cpu().numpy(), golden["backproject_odd_out"]) < RTOL


@pytest.mark.parametrize("n,pad", [(48, 2.0), (33, 1.5), (40, 1.0)])
def test_project_backproject_match_oracle(oracle, n, pad):
    vol = blob_volume(n, seed=n)
    rots = rotations(30, seed=n)
    p = tt().project_3d_to_2d(cuda(vol), cuda(rots), pad_factor=pad)
    ref = oracle.project_3d_to_2d(vol, rots, pad_factor=pad)
    assert p.shape == ref.shape  # (d, d-1) for odd padded boxes, as the reference
    assert rel_l2(p.cpu().numpy(), ref) < RTOL
    # square images (odd-box projections are not square and are rejected, as in the reference)
    imgs = np.random.default_rng(n).standard_normal((30, n, n)).astype(np.float32)
    r = tt().backproject_2d_to_3d(cuda(imgs), cuda(rots), pad_factor=pad)
    ref_r = oracle.backproject_2d_to_3d(imgs, rots, pad_factor=pad)
    assert r.shape == ref_r.shape
    assert rel_l2(r.cpu().numpy(), ref_r) < RTOL


def test_project_rotation_center():
    """test_torch_fourier_slice.py:22-46: a delta at the centre projects to the
    centre pixel for any rotation."""
    v = torch.zeros((32, 32, 32), device="cuda")
    v[16, 16, 16] = 1
    proj = tt().project_3d_to_2d(v, cuda(rotations(100, seed=0)))
    idx = proj.reshape(100, -1).argmax(-1).cpu().numpy()
    assert np.all(idx == 16 * 32 + 16)


def test_projection_backprojection_cycle():
    """test_torch_fourier_slice.py:75-102: 1500 rotations reconstruct the cube."""
    rots = cuda(rotations(1500, seed=1))
    c = cube()
    rec = tt().backproject_2d_to_3d(tt().project_3d_to_2d(c, rots), rots)
    f = fsc(c.cpu().numpy(), rec.cpu().numpy())
    assert np.all(f[1:] > 0.97), f
    assert np.all(f[-10:] > 0.99), f


def test_leading_dims():
    """test_torch_fourier_slice.py:105-128 (random, non-orthogonal matrices)."""
    R = torch.rand((4, 5, 3, 3), device="cuda")
    proj = tt().project_3d_to_2d(cube(), R)
    assert proj.shape == (4, 5, 32, 32)
    assert tt().backproject_2d_to_3d(proj, R).shape == (32, 32, 32)


def test_multichannel_shapes():
    """test_torch_fourier_slice.py:131-155."""
    vols = torch.rand((4, 10, 10, 10), device="cuda")
    R = cuda(rotations(8, seed=3))
    proj = tt().project_3d_to_2d_multichannel(vols, R)
    assert proj.shape == (8, 4, 10, 10)
    assert tt().backproject_2d_to_3d_multichannel(proj, R).shape == (4, 10, 10, 10)


def test_backproject_dtypes():
    """test_torch_fourier_slice.py:158-171."""
    for dt in (torch.float32, torch.float64):
        imgs = torch.rand((10, 28, 28), dtype=dt, device="cuda")
        R = cuda(rotations(10, seed=4)).to(dt)
        assert tt().backproject_2d_to_3d(imgs, R).dtype == dt


def test_wrapper_errors():
    with pytest.raises(ValueError):
        tt().project_3d_to_2d(torch.zeros((8, 8, 9), device="cuda"), torch.eye(3, device="cuda"))
    with pytest.raises(ValueError):
        tt().project_3d_to_2d(torch.zeros((8, 8, 8), device="cuda"), torch.eye(3, device="cuda"), pad_factor=0.5)
    with pytest.raises(ValueError):
        tt().backproject_2d_to_3d(torch.zeros((2, 8, 9), device="cuda"), torch.eye(3, device="cuda")[None])


def test_project_float64_volumes(oracle, monkeypatch):
    """float64 volumes project to float64 images (the reference raises
    RuntimeError for them), sampled in single precision: the float32
    projection of the same volume within rounding, the oracle within the
    float32 tolerance, and a float64 volume gradient."""
    vol = cuda(blob_volume(24, seed=7)).double()
    R = cuda(rotations(6, seed=8)).float()
    for graphs in ("1", "0"):  # the graph-replayed and the eager path
        monkeypatch.setenv("TT_PROJECT_GRAPHS", graphs)
        p64 = tt().project_3d_to_2d(vol, R)
        assert p64.dtype == torch.float64
        p32 = tt().project_3d_to_2d(vol.float(), R)
        assert rel_l2(p64.float().cpu().numpy(), p32.cpu().numpy()) < 1e-6
        ref = oracle.project_3d_to_2d(vol.cpu().numpy(), R.cpu().numpy())
        assert rel_l2(p64.cpu().numpy(), ref) < RTOL
    mc = tt().project_3d_to_2d_multichannel(torch.stack([vol, 2 * vol]), R)
    assert mc.dtype == torch.float64
    assert rel_l2(mc[:, 1].cpu().numpy(), 2 * mc[:, 0].cpu().numpy()) < 1e-6
    v = vol.clone().requires_grad_(True)
    tt().project_3d_to_2d(v, R).square().sum().backward()
    assert v.grad.dtype == torch.float64 and torch.isfinite(v.grad).all()
    with pytest.raises(RuntimeError):
        tt().extract_central_slices_rfft_3d(torch.zeros((8, 8, 5), dtype=torch.complex128, device="cuda"),
                                            (8, 8, 8), R)


def test_project_is_differentiable(oracle):
    n = 16
    vol = cuda(blob_volume(n, seed=2)).requires_grad_(True)
    R = cuda(rotations(4, seed=5)).float().requires_grad_(True)
    proj = tt().project_3d_to_2d(vol, R)
    proj.square().sum().backward()
    assert vol.grad is not None and R.grad is not None
    assert torch.isfinite(vol.grad).all() and torch.isfinite(R.grad).all()
    # directional derivative against a central difference of the GPU forward.
    # The loss is quadratic in the volume, so the central difference is exact
    # up to float32 rounding of lp - lm; a seeded direction keeps the
    # derivative large against that rounding (a direction nearly orthogonal to
    # the gradient would not).
    d = torch.randn(vol.shape, device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    eps = 1e-2
    with torch.no_grad():
        lp = tt().project_3d_to_2d(vol + eps * d, R).double().square().sum()
        lm = tt().project_3d_to_2d(vol - eps * d, R).double().square().sum()
    fd = ((lp - lm) / (2 * eps)).item()
    an = (vol.grad.double() * d.double()).sum().item()
    assert abs(an - fd) <= 1e-3 * abs(fd)


# ----------------------------------------------------------------------------
# torch_image_interpolation
# ----------------------------------------------------------------------------

@pytest.mark.parametrize("name", ["real", "complex", "multi", "f64"])
@pytest.mark.parametrize("mode", ["trilinear", "nearest"])
def test_sample_image_3d_golden(golden, name, mode):
    out = tt().sample_image_3d(cuda(golden[f"sample_{name}_image"]), cuda(golden[f"sample_{name}_coords"]),
                               interpolation=mode)
    ref = golden[f"sample_{name}_{mode}_out"]
    assert tuple(out.shape) == ref.shape and out.cpu().numpy().dtype == ref.dtype
    assert rel_l2(out.cpu().numpy(), ref) < (1e-12 if ref.dtype in (np.float64, np.complex128) else RTOL)


@pytest.mark.parametrize("name", ["f32", "c64", "f32w64"])
@pytest.mark.parametrize("mode", ["trilinear", "nearest"])
def test_insert_into_image_3d_golden(golden, name, mode):
    ref_i, ref_w = golden[f"insimg_{name}_{mode}_image"], golden[f"insimg_{name}_{mode}_weights"]
    img = torch.zeros(ref_i.shape, dtype=cuda(ref_i).dtype, device="cuda")
    w = torch.zeros(ref_w.shape, dtype=cuda(ref_w).dtype, device="cuda")
    img2, w2 = tt().insert_into_image_3d(cuda(golden[f"insimg_{name}_values"]), cuda(golden[f"insimg_{name}_coords"]),
                                         img, w, interpolation=mode)
    assert img2.data_ptr() == img.data_ptr()  # in place, as the reference
    assert w2.dtype == w.dtype
    assert rel_l2(img2.cpu().numpy(), ref_i) < RTOL and rel_l2(w2.cpu().numpy(), ref_w) < RTOL


def test_insert_into_image_3d_multichannel_golden(golden):
    ref = golden["insimg_multi_trilinear_image"]
    img, w = tt().insert_into_image_3d(cuda(golden["insimg_multi_values"]), cuda(golden["insimg_multi_coords"]),
                                       torch.zeros(ref.shape, device="cuda"))
    assert rel_l2(img.cpu().numpy(), ref) < RTOL
    assert rel_l2(w.cpu().numpy(), golden["insimg_multi_trilinear_weights"]) < RTOL


def test_insert_into_image_3d_known_answers():
    img, _ = tt().insert_into_image_3d(torch.tensor([5.0], device="cuda"),
                                       torch.tensor([[10.5, 14.5, 18.5]], device="cuda"),
                                       torch.zeros((28, 28, 28), device="cuda"))
    assert torch.allclose(img[10:12, 14:16, 18:20], torch.full((2, 2, 2), 5 / 8, device="cuda"))
    assert torch.allclose(img[:10, :14, :18], torch.zeros_like(img[:10, :14, :18]))
    img, _ = tt().insert_into_image_3d(torch.tensor([5.0], device="cuda"),
                                       torch.tensor([[10.7, 14.3, 18.9]], device="cuda"),
                                       torch.zeros((28, 28, 28), device="cuda"), interpolation="nearest")
    exp = torch.zeros((28, 28, 28), device="cuda")
    exp[11, 14, 19] = 5
    assert torch.equal(img, exp)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.complex64, torch.complex128])
def test_insert_into_image_3d_type_consistency(dtype):
    """test_image_interpolation_3d.py:160-191, including the reference's
    'bilinear' spelling, which inserts nothing."""
    image = torch.rand((4, 4, 4), dtype=dtype, device="cuda")
    before = image.clone()
    coords = cuda(np.random.uniform(low=0, high=3, size=(3, 4, 5, 3)))
    values = torch.rand(size=(3, 4, 5), dtype=dtype, device="cuda")
    weights = torch.zeros((4, 4, 4), dtype=torch.float64, device="cuda")
    for mode in ("bilinear", "nearest"):
        image, weights = tt().insert_into_image_3d(values, image=image, weights=weights, coordinates=coords,
                                                   interpolation=mode)
        assert image.dtype == dtype
        assert weights.dtype == torch.float64
    assert not torch.equal(image, before)
    assert weights.sum().item() == pytest.approx(60.0)


def test_insert_into_image_3d_errors():
    image = torch.rand((4, 4, 4), dtype=torch.complex64, device="cuda")
    coords = cuda(np.random.uniform(low=0, high=3, size=(3, 4, 5, 3)))
    with pytest.raises(ValueError):
        tt().insert_into_image_3d(torch.rand((3, 4, 5), dtype=torch.complex128, device="cuda"), coords, image)
    with pytest.raises(ValueError):
        tt().insert_into_image_3d(torch.rand((3, 4, 6), dtype=torch.complex64, device="cuda"), coords, image)
    with pytest.raises(ValueError):
        tt().sample_image_3d(torch.rand((4, 4), device="cuda"), coords)


def test_sample_image_3d_matches_oracle(oracle):
    rng = np.random.default_rng(0)
    img = (rng.standard_normal((2, 20, 21, 22)) + 1j * rng.standard_normal((2, 20, 21, 22))).astype(np.complex64)
    coords = rng.uniform(-1, 22, size=(1000, 3)).astype(np.float32)
    for mode in ("trilinear", "nearest"):
        out = tt().sample_image_3d(cuda(img), cuda(coords), interpolation=mode)
        assert rel_l2(out.cpu().numpy(), oracle.sample_image_3d(img, coords, mode)) < RTOL


@pytest.mark.parametrize("name", ["even", "odd"])
def test_backprojection_gradient_matches_reference_autograd(golden, name):
    imgs = torch.as_tensor(golden[f"bpgrad_{name}_images"]).cuda().requires_grad_(True)
    rot = torch.as_tensor(golden[f"bpgrad_{name}_rot"]).cuda()
    pf = float(golden[f"bpgrad_{name}_pad"])
    import teamtomo_b200 as tt

    rec = tt.backproject_2d_to_3d(imgs, rot, pad_factor=pf)
    # the differentiable composition computes the same reconstruction as the fused path
    with torch.no_grad():
        fused = tt.backproject_2d_to_3d(imgs, rot, pad_factor=pf)
    assert rel_l2(rec.detach().cpu().numpy(), fused.cpu().numpy()) < 1e-6
    (rec * torch.as_tensor(golden[f"bpgrad_{name}_G"]).cuda()).sum().backward()
    assert rel_l2(imgs.grad.cpu().numpy(), golden[f"bpgrad_{name}_out"]) < 1e-5


@pytest.mark.parametrize("name", ["real", "complex", "multi"])
def test_sample_image_3d_gradients_match_reference_autograd(golden, name):
    import teamtomo_b200 as tt

    img = torch.as_tensor(golden[f"sgrad_{name}_image"]).cuda().requires_grad_(True)
    c = torch.as_tensor(golden[f"sgrad_{name}_coords"]).cuda().requires_grad_(True)
    out = tt.sample_image_3d(img, c)
    (out * torch.as_tensor(golden[f"sgrad_{name}_G"]).cuda().conj()).real.sum().backward()
    assert rel_l2(img.grad.cpu().numpy(), golden[f"sgrad_{name}_dimage"]) < 1e-6
    assert rel_l2(c.grad.cpu().numpy(), golden[f"sgrad_{name}_dcoords"]) < 1e-5
    # border and outside points: same zeros as grid_sample's backward
    assert np.array_equal(c.grad.cpu().numpy() == 0, golden[f"sgrad_{name}_dcoords"] == 0)


@pytest.mark.parametrize("key", ["f32_trilinear", "c64_trilinear", "f32_nearest"])
def test_insert_into_image_3d_value_gradient_matches_reference(golden, key):
    import teamtomo_b200 as tt

    k = f"igrad_{key}"
    vals = torch.as_tensor(golden[f"{k}_values"]).cuda().requires_grad_(True)
    img = torch.zeros((9, 10, 11), dtype=vals.dtype, device="cuda")
    out, w = tt.insert_into_image_3d(vals, torch.as_tensor(golden[f"{k}_coords"]).cuda(), img,
                                     interpolation=key.split("_")[1])
    assert out is img and not w.requires_grad
    (out * torch.as_tensor(golden[f"{k}_G"]).cuda().conj()).real.sum().backward()
    assert rel_l2(vals.grad.cpu().numpy(), golden[f"{k}_dvalues"]) < 1e-6
