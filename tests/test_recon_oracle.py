"""The reconstructor oracle pinned against an independent implementation:
torch's CPU float64 conv2d and its autograd gradients (no GPU)."""

import numpy as np
import pytest
import torch

from oracle import recon_oracle as R

CASES = [(2, 7, 6, 8, 16, 3, 1, 1), (1, 9, 8, 16, 8, 3, 2, 1), (2, 6, 7, 8, 8, 2, 2, 0), (1, 5, 5, 24, 8, 1, 1, 0)]


@pytest.mark.parametrize("case", CASES, ids=[str(c) for c in CASES])
def test_conv_oracle_matches_torch(case):
    B, H, W, Ci, Co, ks, s, pad = case
    rng = np.random.default_rng(3)
    x = rng.standard_normal((B, H, W, Ci))
    w = rng.standard_normal((Co, ks, ks, Ci))
    xt = torch.tensor(np.transpose(x, (0, 3, 1, 2)), requires_grad=True)
    wt = torch.tensor(np.transpose(w, (0, 3, 1, 2)), requires_grad=True)
    yt = torch.nn.functional.conv2d(xt, wt, stride=s, padding=pad)
    y = R.conv_forward(x, w, s, pad)
    np.testing.assert_allclose(y, np.transpose(yt.detach().numpy(), (0, 2, 3, 1)), rtol=1e-10, atol=1e-10)
    dy = rng.standard_normal(y.shape)
    yt.backward(torch.tensor(np.transpose(dy, (0, 3, 1, 2))))
    np.testing.assert_allclose(R.conv_dgrad(dy, w, (H, W), s, pad), np.transpose(xt.grad.numpy(), (0, 2, 3, 1)),
                               rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(R.conv_wgrad(x, dy, ks, s, pad), np.transpose(wt.grad.numpy(), (0, 2, 3, 1)),
                               rtol=1e-10, atol=1e-10)


def test_packing_layouts():
    w = np.arange(2 * 3 * 3 * 8, dtype=np.float32).reshape(2, 3, 3, 8)
    p = R.pack_weights(w)
    assert p.shape == (16, 128)
    assert p[1, 5 * 8 + 3] == w[1, 1, 2, 3]
    t = R.pack_weights_transposed(w)
    assert t.shape == (16, 64)
    assert t[3, 5 * 2 + 1] == w[1, 1, 2, 3]


def test_round_bf16_ties_to_even():
    v = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, -2.5, 3.140625], np.float32)
    r = R.round_bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2**-6 and r[3] == -2.5


def _he_params(seed=0):
    rng = np.random.default_rng(seed)
    parts = []
    for name, k, s, p, ci, co, relu, src in R.LAYERS:
        fan = k * k * ci
        parts.append(rng.standard_normal(co * fan) * np.sqrt(2.0 / fan))
        parts.append(rng.standard_normal(co) * 0.05)
    return np.concatenate(parts)


def test_unet_param_count():
    assert R.param_count() == 216464


def test_unet_gradients_match_finite_differences():
    """The oracle's backward pass (float64, no bf16 rounding) against central differences."""
    params = _he_params()
    rng = np.random.default_rng(1)
    low = rng.integers(0, 256, (1, 10, 12, 4)).astype(np.uint8)
    high = rng.integers(0, 256, (1, 20, 24, 4)).astype(np.uint8)
    _, g = R.UNet(params, bf16=False).loss_and_backward(low, high)
    offsets = np.cumsum([0] + [co * k * k * ci + co for _, k, _, _, ci, co, _, _ in R.LAYERS])
    eps = 1e-5
    checked = 0
    for li in range(len(R.LAYERS)):
        for i in (offsets[li] + 3, offsets[li + 1] - 1):  # a weight and the last bias of each layer
            pp = params.copy()
            pp[i] += eps
            l1, _ = R.UNet(pp, bf16=False).loss_and_backward(low, high)
            pp[i] -= 2 * eps
            l0, _ = R.UNet(pp, bf16=False).loss_and_backward(low, high)
            fd = (l1 - l0) / (2 * eps)
            assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-9, (R.LAYERS[li][0], i, fd, g[i])
            checked += g[i] != 0
    assert checked >= 10


def test_bilinear_alignment_and_shuffle():
    low = np.arange(2 * 3 * 4, dtype=np.float64).reshape(1, 2, 3, 4)
    up = R.upsample_bilinear2(low)
    assert up.shape == (1, 4, 6, 4)
    np.testing.assert_allclose(up[0, 0, 0], low[0, 0, 0])
    np.testing.assert_allclose(up[0, 0, 1], 0.5 * (low[0, 0, 0] + low[0, 0, 1]))
    np.testing.assert_allclose(up[0, 3, 5], low[0, 1, 2])
    r = np.arange(16, dtype=np.float64).reshape(1, 1, 1, 16)
    s = R.shuffle(r)
    assert s[0, 1, 0, 2] == r[0, 0, 0, 2 * 4 + 2]
    np.testing.assert_allclose(R.unshuffle(s), r)
