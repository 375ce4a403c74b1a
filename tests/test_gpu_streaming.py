"""Streaming host-resident stacks: chunked, copy-overlapped processing gives
the results of the one-shot calls."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import blob_volume, rel_l2, rfft_volume_np, rotations

pytestmark = pytest.mark.gpu


def tt():
    import teamtomo_b200

    return teamtomo_b200


def _host_stack(n, k, seed):
    rng = np.random.default_rng(seed)
    imgs = (rng.standard_normal((k, n, n // 2 + 1)) + 1j * rng.standard_normal((k, n, n // 2 + 1))).astype(
        np.complex64)
    return torch.from_numpy(imgs).pin_memory(), torch.from_numpy(rotations(k, seed=seed).astype(np.float32)).pin_memory()


@pytest.mark.parametrize("chunk,depth", [(7, 2), (16, 3), (100, 2), (1, 1)])
def test_prefetch_delivers_every_chunk_in_order(chunk, depth):
    h_img, h_rot = _host_stack(16, 37, seed=1)
    seen = []
    for s0, s1, (img, rot) in tt().streaming.prefetch_to_device([h_img, h_rot], chunk, "cuda", depth=depth):
        assert img.is_cuda and img.shape[0] == s1 - s0 <= chunk
        # keep a copy: the buffer is reused depth chunks later
        seen.append((s0, img.clone(), rot.clone()))
    assert [s for s, _, _ in seen] == list(range(0, 37, chunk))
    assert torch.equal(torch.cat([x for _, x, _ in seen]).cpu(), h_img)
    assert torch.equal(torch.cat([r for _, _, r in seen]).cpu(), h_rot)


def test_streamed_insertion_equals_one_shot():
    n, k = 48, 150
    h_img, h_rot = _host_stack(n, k, seed=2)
    acc = tt().streaming.InsertionAccumulator((n, n, n), "cuda")
    for _, _, (img, rot) in tt().streaming.prefetch_to_device([h_img, h_rot], 40, "cuda"):
        acc.add(img, rot)
    vol, w = acc.finalize()
    v1, w1 = tt().insert_central_slices_rfft_3d(h_img.cuda(), (n, n, n), h_rot.cuda())
    assert rel_l2(vol.cpu().numpy(), v1.cpu().numpy()) < 1e-6
    assert rel_l2(w.cpu().numpy(), w1.cpu().numpy()) < 1e-6


def test_streamed_deterministic_insertion_is_bit_exact():
    n, k = 32, 90
    h_img, h_rot = _host_stack(n, k, seed=3)
    bound = float(torch.view_as_real(h_img).abs().max())
    acc = tt().streaming.InsertionAccumulator((n, n, n), "cuda", deterministic=True, data_bound=bound,
                                              max_slices=k)
    for _, _, (img, rot) in tt().streaming.prefetch_to_device([h_img, h_rot], 25, "cuda"):
        acc.add(img, rot)
    vol, w = acc.finalize()
    # same scale as the one-shot call (bound = the data's max, max_slices = k)
    v1, w1 = tt().insert_central_slices_rfft_3d(h_img.cuda(), (n, n, n), h_rot.cuda(), deterministic=True)
    assert torch.equal(vol, v1) and torch.equal(w, w1)
    small = tt().streaming.InsertionAccumulator((n, n, n), "cuda", deterministic=True, data_bound=bound / 4,
                                                max_slices=k)
    small.add(h_img[:10].cuda(), h_rot[:10].cuda())
    with pytest.raises(ValueError, match="exceeded data_bound"):
        small.finalize()


def test_streamed_gradients_equal_one_shot():
    n, k = 40, 120
    vol = torch.as_tensor(rfft_volume_np(blob_volume(n, seed=5, n_blobs=8))).cuda()
    h_tgt, h_rot = _host_stack(n, k, seed=6)

    def loss_of(S, T):
        return (S - T).abs().square().sum()

    V = vol.clone().requires_grad_(True)
    R = h_rot.cuda().requires_grad_(True)
    loss_of(tt().extract_central_slices_rfft_3d(V, (n, n, n), R), h_tgt.cuda()).backward()
    Vs = vol.clone().requires_grad_(True)
    dR = torch.empty_like(h_rot)
    for s0, s1, (T, Rb) in tt().streaming.prefetch_to_device([h_tgt, h_rot], 32, "cuda"):
        Rc = Rb.clone().requires_grad_(True)
        loss_of(tt().extract_central_slices_rfft_3d(Vs, (n, n, n), Rc), T).backward()
        dR[s0:s1] = Rc.grad.cpu()
    assert rel_l2(Vs.grad.cpu().numpy(), V.grad.cpu().numpy()) < 1e-6
    assert rel_l2(dR.numpy(), R.grad.cpu().numpy()) < 1e-6
