"""The CPU oracle pinned against golden vectors produced by the reference itself.

These run without a GPU.  They are what makes the oracle trustworthy as the
checker of the CUDA path: extraction must match the reference bit for bit,
everything accumulated (insertion, gradients) within float32 summation-order
noise.
"""

from __future__ import annotations

import numpy as np
import pytest

from helpers import rel_l2


def _extract_kwargs(g, name):
    fmax = float(g[f"extract_{name}_fmax"])
    rtol = float(g[f"extract_{name}_rtol"])
    return dict(
        fftfreq_max=None if fmax < 0 else fmax,
        zyx_matrices=bool(int(g[f"extract_{name}_zyx"])),
        rot_tolerance=None if rtol < 0 else rtol,
        x_tolerance=float(g[f"extract_{name}_xtol"]),
    )


def _insert_kwargs(g, name):
    fmax = float(g[f"insert_{name}_fmax"])
    return dict(fftfreq_max=None if fmax < 0 else fmax,
                zyx_matrices=bool(int(g[f"insert_{name}_zyx"])))


def test_extract_bit_exact(golden, oracle):
    for name in golden["extract_cases"]:
        name = str(name)
        out = oracle.extract(golden[f"extract_{name}_volume"], tuple(golden[f"extract_{name}_shape"]),
                             golden[f"extract_{name}_rot"], **_extract_kwargs(golden, name))
        ref = golden[f"extract_{name}_out"]
        assert out.shape == ref.shape, name
        assert np.array_equal(out, ref), f"{name}: max |diff| {np.abs(out - ref).max()}"


def test_insert_matches_reference(golden, oracle):
    for name in golden["insert_cases"]:
        name = str(name)
        imgs = golden[f"insert_{name}_images"]
        n = imgs.shape[-2]
        vol, w = oracle.insert(imgs, (n, n, n), golden[f"insert_{name}_rot"],
                               **_insert_kwargs(golden, name))
        assert vol.dtype == golden[f"insert_{name}_volume"].dtype
        assert w.dtype == golden[f"insert_{name}_weights"].dtype
        tol = 1e-12 if vol.dtype == np.complex128 else 1e-6
        assert rel_l2(vol, golden[f"insert_{name}_volume"]) < tol, name
        assert rel_l2(w, golden[f"insert_{name}_weights"]) < tol, name
        # whole-volume support is identical: no voxel touched by one and not the other
        assert np.array_equal(w != 0, golden[f"insert_{name}_weights"] != 0), name


def test_gradients_match_reference_autograd(golden, oracle):
    vol = golden["grad_drot_volume"]
    n = vol.shape[0]
    _, drot = oracle.extract_grad(vol, (n, n, n), golden["grad_drot_rot"], golden["grad_drot_G"],
                                  want_dvol=False)
    assert rel_l2(drot, golden["grad_drot_out"]) < 1e-5
    vol = golden["grad_dvol_volume"]
    n = vol.shape[0]
    dvol, _ = oracle.extract_grad(vol, (n, n, n), golden["grad_dvol_rot"], golden["grad_dvol_G"],
                                  want_drot=False)
    assert rel_l2(dvol, golden["grad_dvol_out"]) < 1e-5


@pytest.mark.parametrize("name", ["real", "complex", "multi", "f64"])
@pytest.mark.parametrize("mode", ["trilinear", "nearest"])
def test_sample_image_3d(golden, oracle, name, mode):
    out = oracle.sample_image_3d(golden[f"sample_{name}_image"], golden[f"sample_{name}_coords"], mode)
    ref = golden[f"sample_{name}_{mode}_out"]
    assert out.shape == ref.shape and out.dtype == ref.dtype
    tol = 1e-12 if ref.dtype in (np.float64, np.complex128) else 1e-6
    assert rel_l2(out, ref) < tol


@pytest.mark.parametrize("name", ["f32", "c64", "f32w64"])
@pytest.mark.parametrize("mode", ["trilinear", "nearest"])
def test_insert_into_image_3d(golden, oracle, name, mode):
    img_ref = golden[f"insimg_{name}_{mode}_image"]
    w_ref = golden[f"insimg_{name}_{mode}_weights"]
    img, w = oracle.insert_into_image_3d(golden[f"insimg_{name}_values"], golden[f"insimg_{name}_coords"],
                                         np.zeros_like(img_ref), np.zeros_like(w_ref), mode)
    assert rel_l2(img, img_ref) < 1e-6 and rel_l2(w, w_ref) < 1e-6
    assert w.dtype == w_ref.dtype


def test_insert_into_image_3d_multichannel(golden, oracle):
    ref = golden["insimg_multi_trilinear_image"]
    img, w = oracle.insert_into_image_3d(golden["insimg_multi_values"], golden["insimg_multi_coords"],
                                         np.zeros_like(ref))
    assert rel_l2(img, ref) < 1e-6
    assert rel_l2(w, golden["insimg_multi_trilinear_weights"]) < 1e-6


def test_insert_into_image_3d_known_answers(oracle):
    # test_image_interpolation_3d.py:66-81: 5 at (10.5, 14.5, 18.5) -> 5/8 on 8 voxels
    img, _ = oracle.insert_into_image_3d(np.array([5.0], np.float32),
                                         np.array([[10.5, 14.5, 18.5]], np.float32),
                                         np.zeros((28, 28, 28), np.float32))
    assert np.allclose(img[10:12, 14:16, 18:20], 5 / 8)
    assert img.sum() == pytest.approx(5.0)
    # :100-113: nearest at (10.7, 14.3, 18.9) -> 5 at [11, 14, 19]
    img, _ = oracle.insert_into_image_3d(np.array([5.0], np.float32),
                                         np.array([[10.7, 14.3, 18.9]], np.float32),
                                         np.zeros((28, 28, 28), np.float32), interpolation="nearest")
    exp = np.zeros((28, 28, 28), np.float32)
    exp[11, 14, 19] = 5
    assert np.array_equal(img, exp)


def test_project_backproject(golden, oracle):
    vol, rot = golden["project_volume"], golden["project_rot"]
    assert rel_l2(oracle.project_3d_to_2d(vol, rot), golden["project_out"]) < 1e-5
    assert rel_l2(oracle.project_3d_to_2d(vol, rot, fftfreq_max=0.25), golden["project_fmax_out"]) < 1e-5
    assert rel_l2(oracle.project_3d_to_2d(vol, rot, pad_factor=1.0), golden["project_pad1_out"]) < 1e-5
    imgs = golden["backproject_images"]
    rec = oracle.backproject_2d_to_3d(imgs, golden["backproject_rot"])
    assert rel_l2(rec, golden["backproject_out"]) < 1e-5
    rec64 = oracle.backproject_2d_to_3d(imgs.astype(np.float64), golden["backproject_rot"])
    assert rec64.dtype == np.float64
    assert rel_l2(rec64, golden["backproject_f64_out"]) < 1e-5
    # odd padded box: (d, d-1) outputs, as the reference
    po = oracle.project_3d_to_2d(golden["project_odd_volume"], rot, pad_factor=1.5)
    assert po.shape == golden["project_odd_out"].shape == (6, 33, 32)
    assert rel_l2(po, golden["project_odd_out"]) < 1e-5
    bo = oracle.backproject_2d_to_3d(golden["backproject_odd_images"], rot, pad_factor=1.5)
    assert bo.shape == golden["backproject_odd_out"].shape == (33, 33, 32)
    assert rel_l2(bo, golden["backproject_odd_out"]) < 1e-5


def test_ctf_matches_reference(golden, oracle):
    """torch-ctf calculate_ctf_2d golden grids (incl. the 10x10 case of
    test_torch_ctf.py:376-392), atol 1e-4 as the reference test."""
    for i in range(int(golden["ctf_cases"])):
        rf, fs = (bool(x) for x in golden[f"ctf_{i}_flags"])
        out = oracle.ctf_2d(*golden[f"ctf_{i}_params"], image_shape=tuple(golden[f"ctf_{i}_shape"]),
                            rfft=rf, fftshift=fs)
        assert out.shape == golden[f"ctf_{i}_out"].shape
        np.testing.assert_allclose(out, golden[f"ctf_{i}_out"], atol=1e-4)


def test_insert_mirror_is_plane_post_pass(golden, oracle):
    """The reference's per-corner Friedel mirror equals a splat without it
    followed by one post-pass over the x=0 plane (the form the CUDA path uses)."""
    for name in golden["insert_cases"]:
        name = str(name)
        imgs = golden[f"insert_{name}_images"]
        n = imgs.shape[-2]
        acc, accw = oracle.insert(imgs, (n, n, n), golden[f"insert_{name}_rot"], mirror=False,
                                  **_insert_kwargs(golden, name))
        vol, w = oracle.mirror_x0_post_pass(acc, accw)
        tol = 1e-12 if vol.dtype == np.complex128 else 1e-6
        assert rel_l2(vol, golden[f"insert_{name}_volume"]) < tol, name
        assert rel_l2(w, golden[f"insert_{name}_weights"]) < tol, name


def test_insert_image_gradient_matches_reference_autograd(golden, oracle):
    """The gather adjoint of the insertion (with the Friedel completion's
    adjoint) against the reference's autograd w.r.t. the images."""
    for name in golden["insgrad_cases"]:
        name = str(name)
        imgs = golden[f"insgrad_{name}_images"]
        n = imgs.shape[-2]
        fmax = float(golden[f"insgrad_{name}_fmax"])
        out = oracle.insert_grad_images(golden[f"insgrad_{name}_gvol"], (n, n, n), golden[f"insgrad_{name}_rot"],
                                        fftfreq_max=None if fmax < 0 else fmax,
                                        zyx_matrices=bool(int(golden[f"insgrad_{name}_zyx"])), dtype=imgs.dtype)
        ref = golden[f"insgrad_{name}_out"]
        tol = 1e-12 if imgs.dtype == np.complex128 else 1e-6
        assert rel_l2(out, ref) < tol, name
        assert np.array_equal(out == 0, ref == 0), name  # same pixels receive no gradient


def test_lines_2d_match_reference(golden, oracle):
    for name in golden["lines_cases"]:
        name = str(name)
        img = golden[f"lines_{name}_image"]
        h = img.shape[0]
        out = oracle.extract_lines_2d(img, (h, h), golden[f"lines_{name}_rot"],
                                      yx_matrices=bool(int(golden[f"lines_{name}_yx"])))
        ref = golden[f"lines_{name}_out"]
        assert out.shape == ref.shape
        assert rel_l2(out, ref) < 1e-6, name
    for name in ("even", "odd"):
        im = golden[f"proj1d_{name}_image"]
        out = oracle.project_2d_to_1d(im, golden["lines_h16_rot"], pad_factor=float(golden[f"proj1d_{name}_pad"]))
        ref = golden[f"proj1d_{name}_out"]
        assert out.shape == ref.shape, name
        assert rel_l2(out, ref) < 1e-5, name


def test_rotation_gradient_on_the_border_matches_reference(golden, oracle):
    """Axis-aligned rotations put whole pixel columns on the x = 0 border,
    where grid_sample's backward passes no coordinate gradient."""
    vol = golden["grad_axes_volume"]
    n = vol.shape[0]
    _, drot = oracle.extract_grad(vol, (n, n, n), golden["grad_axes_rot"], golden["grad_axes_G"], want_dvol=False)
    assert rel_l2(drot, golden["grad_axes_out"]) < 1e-5


@pytest.mark.parametrize("name", ["real", "complex", "multi"])
@pytest.mark.parametrize("mode", ["trilinear", "nearest"])
def test_affine_transform_matches_reference(golden, oracle, name, mode):
    out = oracle.affine_transform_image_3d(golden[f"affine_{name}_image"], golden["affine_matrices"], mode)
    ref = golden[f"affine_{name}_{mode}_out"]
    assert out.shape == ref.shape
    assert rel_l2(out, ref) < 1e-6
    if mode == "nearest":
        assert np.array_equal(out, ref)


def test_affine_transform_output_shape_zyx(golden, oracle):
    out = oracle.affine_transform_image_3d(golden["affine_shape_zyx_image"], golden["affine_matrices"][0],
                                           "trilinear", output_shape=(6, 7, 5), zyx_matrices=True)
    assert rel_l2(out, golden["affine_shape_zyx_out"]) < 1e-6
