"""affine_transform_image_3d (one kernel: coordinates in registers + sampling)
against the reference's golden vectors and the oracle."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.as_tensor(np.asarray(a)).cuda()


def tt():
    import teamtomo_b200

    return teamtomo_b200


@pytest.mark.parametrize("name", ["real", "complex", "multi"])
@pytest.mark.parametrize("mode", ["trilinear", "nearest"])
def test_matches_reference_golden(golden, name, mode):
    f = tt().torch_transform_image.affine_transform_image_3d
    img = cuda(golden[f"affine_{name}_image"])
    M = cuda(golden["affine_matrices"])
    ref = golden[f"affine_{name}_{mode}_out"]
    batched = f(img, M, mode).cpu().numpy()  # (3, ...) in one launch
    single = np.stack([f(img, M[i], mode).cpu().numpy() for i in range(3)])
    assert batched.shape == ref.shape and np.array_equal(batched, single)
    if mode == "nearest":
        assert np.array_equal(batched, ref)  # same coordinates, same voxels
    else:
        assert rel_l2(batched, ref) < 1e-6


def test_output_shape_and_zyx(golden):
    out = tt().torch_transform_image.affine_transform_image_3d(
        cuda(golden["affine_shape_zyx_image"]), cuda(golden["affine_matrices"][0]), "trilinear",
        output_shape=(6, 7, 5), zyx_matrices=True)
    assert rel_l2(out.cpu().numpy(), golden["affine_shape_zyx_out"]) < 1e-6


def test_float64_image_and_large_volume(oracle):
    rng = np.random.default_rng(4)
    img = rng.standard_normal((20, 24, 28))
    M = np.eye(4, dtype=np.float32)
    M[:3, :3] = np.linalg.qr(rng.standard_normal((3, 3)))[0]
    M[:3, 3] = [3.0, -2.0, 1.5]
    out = tt().torch_transform_image.affine_transform_image_3d(cuda(img), cuda(M), "trilinear")
    assert out.dtype == torch.float64
    ref = oracle.affine_transform_image_3d(img, M, "trilinear")
    assert rel_l2(out.cpu().numpy(), ref) < 1e-12
