"""The FP64 U-Net oracle's gradient against central finite differences (CPU).

The warm-start network has no counterpart in the reference; its oracle
(oracle/unet_oracle.py) is pinned by differentiating it numerically. Away
from ReLU kinks and max-pooling ties the agreement is to ~1e-6 relative.
"""
import numpy as np

import unet_oracle as UO


def test_oracle_gradient_matches_finite_differences():
    c, shape = 4, (8, 8, 8)
    rng = np.random.default_rng(0)
    n = sum(27 * ci * co + co for ci, co in UO.layer_shapes(c)) + c + 1
    p = np.zeros(n)
    off = 0
    for ci, co in UO.layer_shapes(c):
        p[off:off + 27 * ci * co] = rng.normal(0, np.sqrt(2 / (27 * ci)), 27 * ci * co)
        off += 27 * ci * co + co
    p[off:off + c] = rng.normal(0, 0.3, c)
    p[-1] = 0.01
    x = 0.01 + 0.01 * rng.random(shape)
    t = x + 0.003 * rng.normal(size=shape)
    _, g = UO.forward_backward(p, c, x, t, bf16=False, scale=50.0)
    for i in [5, 200, 27 * c + 3, off - 3, off + 1, n - 1]:
        h = 1e-4 * max(1.0, abs(p[i]))
        pp = p.copy()
        pp[i] += h
        lp, _ = UO.forward_backward(pp, c, x, t, bf16=False, scale=50.0)
        pp[i] -= 2 * h
        lm, _ = UO.forward_backward(pp, c, x, t, bf16=False, scale=50.0)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-3 * max(abs(g[i]), 1e-9) + 1e-12, (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5e-3], np.float32)
    r = UO.to_bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] - (-2.5e-3)) <= 2.5e-3 * 2 ** -8
