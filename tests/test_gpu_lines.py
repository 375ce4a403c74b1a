"""Central lines of 2D images (extract_central_slices_rfft_2d, project_2d_to_1d)
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


def _rot2(th):
    th = np.asarray(th, np.float64)
    return np.stack([np.stack([np.cos(th), -np.sin(th)], -1), np.stack([np.sin(th), np.cos(th)], -1)], -2)


def test_lines_match_reference_golden(golden):
    for name in golden["lines_cases"]:
        name = str(name)
        img = golden[f"lines_{name}_image"]
        h = img.shape[0]
        out = tt().extract_central_slices_rfft_2d(cuda(img), (h, h), cuda(golden[f"lines_{name}_rot"]),
                                                  yx_matrices=bool(int(golden[f"lines_{name}_yx"])))
        assert rel_l2(out.cpu().numpy(), golden[f"lines_{name}_out"]) < 1e-6, name


def test_line_gradients_match_reference_autograd(golden):
    img = cuda(golden["linesgrad_image"]).requires_grad_(True)
    R = cuda(golden["lines_h16_rot"]).requires_grad_(True)  # float64 leaf, as the reference run
    out = tt().extract_central_slices_rfft_2d(img, (16, 16), R)
    (out * cuda(golden["linesgrad_G"]).conj()).real.sum().backward()
    assert R.grad.dtype == torch.float64
    assert rel_l2(R.grad.cpu().numpy(), golden["linesgrad_drot"]) < 1e-5
    assert rel_l2(img.grad.cpu().numpy(), golden["linesgrad_dimage"]) < 1e-6


@pytest.mark.parametrize("h,yx", [(64, False), (65, False), (128, True)])
def test_lines_match_oracle(oracle, h, yx):
    rng = np.random.default_rng(h)
    img = (rng.standard_normal((h, h // 2 + 1)) + 1j * rng.standard_normal((h, h // 2 + 1))).astype(np.complex64)
    rot = _rot2(rng.uniform(0, 2 * np.pi, 200))
    out = tt().extract_central_slices_rfft_2d(cuda(img), (h, h), cuda(rot), yx_matrices=yx)
    ref = oracle.extract_lines_2d(img, (h, h), rot, yx_matrices=yx)
    assert rel_l2(out.cpu().numpy(), ref) < 1e-6


def test_project_2d_to_1d_matches_reference(golden):
    for name in ("even", "odd"):
        im = golden[f"proj1d_{name}_image"]
        out = tt().project_2d_to_1d(cuda(im), cuda(golden["lines_h16_rot"]).float(),
                                    pad_factor=float(golden[f"proj1d_{name}_pad"]))
        ref = golden[f"proj1d_{name}_out"]
        assert tuple(out.shape) == ref.shape, name
        assert rel_l2(out.cpu().numpy(), ref) < 1e-5, name


def test_fftfreq_max_zeroes_high_frequencies(oracle):
    h = 48
    rng = np.random.default_rng(3)
    img = (rng.standard_normal((h, h // 2 + 1)) + 1j * rng.standard_normal((h, h // 2 + 1))).astype(np.complex64)
    rot = cuda(_rot2(rng.uniform(0, 2 * np.pi, 20)))
    full = tt().extract_central_slices_rfft_2d(cuda(img), (h, h), rot)
    cut = tt().extract_central_slices_rfft_2d(cuda(img), (h, h), rot, fftfreq_max=0.25)
    q = np.arange(h // 2 + 1) / h
    keep = torch.as_tensor(q <= 0.25).cuda()
    assert torch.equal(cut[:, keep], full[:, keep])
    assert torch.all(cut[:, ~keep] == 0)
    ref = oracle.extract_lines_2d(img, (h, h), rot.cpu().numpy(), fftfreq_max=0.25)
    assert rel_l2(cut.cpu().numpy(), ref) < 1e-6
