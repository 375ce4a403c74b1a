"""Graph replay of small projections (project_3d_to_2d without autograd).

Replays must equal the eager path bit for bit, for new inputs of the same
shape on every call, return tensors the next call does not touch, and leave
autograd calls on the eager path.
"""

from __future__ import annotations

import pytest
import torch

from helpers import blob_volume, rel_l2, rotations

pytestmark = pytest.mark.gpu


def tt():
    import teamtomo_b200

    return teamtomo_b200


def _inputs(seed, n=32, k=12):
    vol = torch.as_tensor(blob_volume(n, seed=seed)).cuda()
    R = torch.as_tensor(rotations(k, seed=seed + 1)).float().cuda()
    return vol, R


def test_replays_equal_eager_and_are_independent(monkeypatch, oracle):
    from teamtomo_b200.torch_fourier_slice import project as P

    monkeypatch.setenv("TT_PROJECT_GRAPHS", "1")
    P._graphs.clear()
    outs = []
    for seed in (11, 12, 13):
        vol, R = _inputs(seed)
        outs.append((vol, R, tt().project_3d_to_2d(vol, R)))
    assert len(P._graphs) == 1  # one shape: one captured graph, replayed
    first = outs[0][2].clone()
    monkeypatch.setenv("TT_PROJECT_GRAPHS", "0")
    for vol, R, out in outs:
        assert torch.equal(out, tt().project_3d_to_2d(vol, R))
    assert torch.equal(outs[0][2], first)  # later replays did not write into it
    ref = oracle.project_3d_to_2d(outs[1][0].cpu().numpy(), outs[1][1].cpu().numpy())
    assert rel_l2(outs[1][2].cpu().numpy(), ref) < 1e-5


def test_other_shapes_and_arguments_get_their_own_graphs(monkeypatch):
    from teamtomo_b200.torch_fourier_slice import project as P

    monkeypatch.setenv("TT_PROJECT_GRAPHS", "1")
    P._graphs.clear()
    vol, R = _inputs(21)
    a = tt().project_3d_to_2d(vol, R)
    b = tt().project_3d_to_2d(vol, R, pad_factor=1.0)
    c = tt().project_3d_to_2d(vol, R[:5], fftfreq_max=0.3)
    assert len(P._graphs) == 3
    monkeypatch.setenv("TT_PROJECT_GRAPHS", "0")
    assert torch.equal(a, tt().project_3d_to_2d(vol, R))
    assert torch.equal(b, tt().project_3d_to_2d(vol, R, pad_factor=1.0))
    assert torch.equal(c, tt().project_3d_to_2d(vol, R[:5], fftfreq_max=0.3))


def test_autograd_calls_stay_eager(monkeypatch):
    from teamtomo_b200.torch_fourier_slice import project as P

    monkeypatch.setenv("TT_PROJECT_GRAPHS", "1")
    P._graphs.clear()
    vol, R = _inputs(31)
    v = vol.clone().requires_grad_(True)
    out = tt().project_3d_to_2d(v, R)
    out.square().sum().backward()
    assert len(P._graphs) == 0 and v.grad is not None and torch.isfinite(v.grad).all()


def test_calls_from_two_streams(monkeypatch):
    """A replay on a second stream waits for the previous call's output copy."""
    from teamtomo_b200.torch_fourier_slice import project as P

    monkeypatch.setenv("TT_PROJECT_GRAPHS", "1")
    P._graphs.clear()
    (v1, R1), (v2, R2) = _inputs(41), _inputs(42)
    s = torch.cuda.Stream()
    a = tt().project_3d_to_2d(v1, R1)
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        b = tt().project_3d_to_2d(v2, R2)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    monkeypatch.setenv("TT_PROJECT_GRAPHS", "0")
    assert torch.equal(a, tt().project_3d_to_2d(v1, R1))
    assert torch.equal(b, tt().project_3d_to_2d(v2, R2))
