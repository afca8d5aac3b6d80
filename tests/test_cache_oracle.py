"""CPU checks of the radiance cache's FP64 oracle: its backward pass
against finite differences of the loss (FP64, no BF16 rounding), and its
BF16 rounding against known values."""

import numpy as np

from oracle import cache_oracle


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 2.0 ** -7, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e-3])
    r = cache_oracle.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                     # tie to even
    assert r[2] == 1.0 + 2.0 ** -7
    assert r[3] == 1.0 + 2.0 ** -6         # tie to even (upwards)
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-3) <= 3.0e-3 * 2.0 ** -8


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    w = np.concatenate([rng.uniform(-0.3, 0.3, 4096) for _ in range(5)] + [rng.uniform(-0.3, 0.3, 1024)])
    x = rng.uniform(-1.0, 1.0, size=(16, 64))
    t = rng.uniform(0.0, 2.0, size=(16, 3))
    gw, gx, _ = cache_oracle.gradients(w, x, t, quantize=False)
    # The oracle's gradient holds the loss's denominator constant; finite
    # differences see it move. Compare against the held-denominator loss.
    y0 = cache_oracle.forward(w, x, quantize=False)[1][:, :3]
    denom = y0 * y0 + 0.01

    def held(weights, inputs):
        y = cache_oracle.forward(weights, inputs, quantize=False)[1][:, :3]
        return float(np.sum((y - t) ** 2 / denom))

    eps = 1e-6
    for i in rng.choice(cache_oracle.WEIGHTS, 40, replace=False):
        if i >= 20480 and (i - 20480) % 16 >= 3:
            continue
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (held(wp, x) - held(wm, x)) / (2 * eps)
        assert abs(fd - gw[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, gw[i])
    for (s, j) in [(0, 0), (3, 10), (7, 40), (15, 55)]:
        xp, xm = x.copy(), x.copy()
        xp[s, j] += eps
        xm[s, j] -= eps
        fd = (held(w, xp) - held(w, xm)) / (2 * eps)
        assert abs(fd - gx[s, j]) <= 1e-5 * max(1.0, abs(fd)), (s, j, fd, gx[s, j])
