"""The scatter-surrogate U-Net's numpy oracle (CPU): parameter layout matches
the GPU network's, and its analytic gradients match finite differences."""

import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import unet_oracle as uo  # noqa: E402


def _random_params(seed):
    rng = np.random.default_rng(seed)
    n = uo.parameter_count()
    p = rng.normal(0.0, 0.08, n)
    layers, wo, bo, _ = uo.unpack(p)
    layers[0][0][:, :, uo.INPUT_CHANNELS:] = 0.0  # padded input channels
    for _, b in layers:
        b[:] = rng.uniform(0.01, 0.05, b.shape)  # keep units active
    return p


def test_parameter_count_matches_layout():
    n = uo.parameter_count()
    expect = sum(9 * ci * co + co for ci, co, _ in uo.SPEC) + 33
    assert n == expect


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    p = _random_params(2)
    inp = rng.uniform(0.0, 1.0, (2, 8, 8, 2))
    target = rng.uniform(0.0, 1.0, (2, 8, 8))
    loss, g = uo.loss_and_gradients(p, inp, target)
    assert np.isfinite(loss)
    layers, _, _, n = uo.unpack(np.arange(uo.parameter_count(), dtype=np.float64))
    # a few parameters from several layers (first, bottleneck, decoder, output)
    picks = [int(layers[0][0][4, 3, 1]), int(layers[7][0][2, 5, 9]), int(layers[8][0][6, 17, 300]),
             int(layers[12][1][5]), int(layers[13][0][0, 1, 2]), n - 2, n - 1]
    eps = 1e-6
    for k in picks:
        q = p.copy()
        q[k] += eps
        lp = uo.loss_and_gradients(q, inp, target)[0]
        q[k] -= 2 * eps
        lm = uo.loss_and_gradients(q, inp, target)[0]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(fd)), (k, fd, g[k])
