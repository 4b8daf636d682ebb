"""The surrogate network's CUDA kernels and the sweep screener.

Gradients of bes_mlp_backward are checked against the CPU FP64 oracle
(oracle/mlp_oracle.py, same BF16 rounding points); the last test shows what
the trained network buys on a small sweep: most points are served without
integration, at a bounded error against the plain full-grid map."""
import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import surrogate as SG
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _net(width=64, depth=3, seed=1):
    net = SG.MLP(width=width, depth=depth, max_batch=1024, seed=seed)
    rng = np.random.default_rng(seed)
    norm = (rng.normal(0, 1, 6), rng.uniform(0.5, 2, 6), rng.normal(0, 1, 2), rng.uniform(0.5, 2, 2))
    net.set_normalization(*norm)
    return net, [np.asarray(a, np.float32) for a in norm]


def test_forward_matches_oracle(gpu):
    net, norm = _net()
    rng = np.random.default_rng(2)
    x = rng.normal(0, 1.5, (300, 6)).astype(np.float32)
    y = net.predict(x)
    want, _, _ = M.forward(net.parameters(), net.sizes, x, *norm)
    np.testing.assert_allclose(y, want, rtol=2e-3, atol=2e-3 * np.abs(want).max())


def test_gradients_match_oracle(gpu):
    import torch
    net, norm = _net(width=96, depth=4, seed=3)
    rng = np.random.default_rng(4)
    x = rng.normal(0, 1.5, (257, 6)).astype(np.float32)
    t = rng.normal(0, 1.0, (257, 2)).astype(np.float32)
    loss = net.backward(torch.as_tensor(x, device="cuda"), torch.as_tensor(t, device="cuda"))
    g = net.gradients()
    want_loss, want = M.backward(net.parameters(), net.sizes, x, t, *norm)
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, want_loss)
    k = 0
    for fi, fo in net.sizes:
        for size in (fi * fo, fo):
            a, b = g[k:k + size].astype(np.float64), want[k:k + size]
            assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b) + 1e-9, (fi, fo, size)
            k += size


def test_training_fits_a_smooth_map(gpu):
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (4096, 6))
    Y = np.stack([np.sin(2 * X[:, 0]) * X[:, 1] + 0.3 * X[:, 2] ** 2, np.cos(X[:, 3] + X[:, 4]) - X[:, 5]], 1)
    net = SG.MLP(width=128, depth=3, max_batch=1024, seed=0)
    hist = net.fit(X, Y, steps=1500, batch=256, lr=3e-3, log_every=100)
    first, last = hist[0][1], np.mean([h[1] for h in hist[-3:]])
    assert last < 0.02 * first, hist
    pred = net.predict(X[:512])
    assert np.sqrt(np.mean((pred - Y[:512]) ** 2)) < 0.05


def test_screened_sweep_integrates_fewer_points_at_bounded_error(gpu):
    radii = np.random.default_rng(11).uniform(2.0, 8.0, 32)
    X, Y, status, _ = SG.generate_runs(768, seed=3, n_periods=2, reset_at=1)
    ok = (status & 4) == 0
    net = SG.MLP(max_batch=1024, seed=2)
    net.fit(X[ok], Y[ok], steps=2000, batch=256, lr=2e-3)
    pa = np.linspace(0.5, 2.0, 16)
    fr = np.logspace(np.log10(20.0), np.log10(200.0), 16)

    def solve(pa_pts, f_pts):
        ens = SG.line_ensemble(pa_pts, f_pts, np.broadcast_to(radii, (len(pa_pts), 32)), n_periods=2, reset_at=1)
        return SG.solve_ensemble(ens)[0]

    PA, FR = np.meshgrid(pa, fr, indexing="ij")
    plain = solve(PA.ravel(), FR.ravel()).reshape(16, 16, 2)
    res = SG.screen_sweep(net, pa, fr, radii, solve, grad_quantile=0.6, audit_fraction=0.05)
    frac = res.integrated.mean()
    assert frac < 0.6                                            # the gain: most points are not integrated
    np.testing.assert_array_equal(res.map[res.integrated], plain[res.integrated])
    served = ~res.integrated
    err = np.abs(res.map[served][:, 0] - plain[served][:, 0])
    print("integrated fraction", frac, "median log10 strength error of served points", float(np.median(err)))
    assert np.median(err) < 0.08                                 # log10 strength (20 % relative), served points


def test_lattice_screener_with_and_without_network(gpu):
    """The multi-fidelity sweep screener with the trained network and without it
    (bilinear interpolation of the solver lattice, the counterfactual): both
    reproduce the solver exactly where they integrate and serve the rest within a
    bounded error.  What the network adds, measured: on the benchmark's sweep
    (128 x 128 points, 8 periods) the two served maps came out equal (mean error
    1.68 % both); on this coarse 33 x 33 grid the network's served points are
    worse (mean 1.4 % against 0.65 % on the B200).  The test asserts that the
    network moves the served error by less than two percentage points either
    way -- it claims no gain, because there is none to show."""
    radii = np.random.default_rng(11).uniform(2.0, 8.0, 32)
    X, Y, status, _ = SG.generate_runs(768, seed=3, n_periods=2, reset_at=1)
    ok = (status & 4) == 0
    net = SG.MLP(max_batch=1024, seed=2)
    net.fit(X[ok], Y[ok], steps=2000, batch=256, lr=2e-3)
    n = 33
    pa = np.linspace(0.5, 2.0, n)
    fr = np.logspace(np.log10(20.0), np.log10(200.0), n)

    def solve(pa_pts, f_pts):
        ens = SG.line_ensemble(pa_pts, f_pts, np.broadcast_to(radii, (len(pa_pts), 32)), n_periods=2, reset_at=1)
        return SG.solve_ensemble(ens)[0]

    PA, FR = np.meshgrid(pa, fr, indexing="ij")
    plain = solve(PA.ravel(), FR.ravel()).reshape(n, n, 2)
    stats = {}
    for tag, m in (("network", net), ("interpolation", None)):
        res = SG.screen_sweep_lattice(m, pa, fr, radii, solve, stride=4, cell_spread=0.3, cell_disagreement=0.1,
                                      audit_fraction=0.02)
        np.testing.assert_array_equal(res.map[res.integrated], plain[res.integrated])
        served = ~res.integrated
        assert served.any(), tag
        e = np.abs(10.0 ** res.map[..., 0] - 10.0 ** plain[..., 0]) / 10.0 ** plain[..., 0]
        stats[tag] = (float(res.integrated.mean()), float(np.median(e[served])), float(e[served].mean()))
    print("integrated fraction, median and mean served strength error:", stats)
    net.close()
    for tag, (frac, med, mean) in stats.items():
        assert med < 0.05 and mean < 0.05, (tag, stats)      # collapse strength, relative
    assert abs(stats["network"][2] - stats["interpolation"][2]) < 0.02, stats
