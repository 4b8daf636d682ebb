"""The CPU network oracle: its analytic gradient against central differences
(rounding switched off, so the function is smooth)."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(M, "bf16", lambda x: np.asarray(x, np.float64))
    monkeypatch.setattr(M, "f32", lambda x: np.asarray(x, np.float64))
    rng = np.random.default_rng(0)
    sizes = M.layer_sizes(6, 8, 2, 2)
    n = sum(fi * fo + fo for fi, fo in sizes)
    p = rng.normal(0, 0.4, n)
    x = rng.normal(0, 1, (5, 6))
    t = rng.normal(0, 1, (5, 2))
    norm = (np.zeros(6), np.ones(6), np.zeros(2), np.ones(2))
    loss, g = M.backward(p, sizes, x, t, *norm)
    h = 1e-6
    for k in rng.choice(n, 25, replace=False):
        e = np.zeros(n)
        e[k] = h
        fd = (M.backward(p + e, sizes, x, t, *norm)[0] - M.backward(p - e, sizes, x, t, *norm)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5e-3, 3.0e38], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0          # halfway, rounds to even
    assert r[2] == 1.0078125                     # above halfway rounds up
    assert abs(r[3] + 2.5e-3) < 1e-5
