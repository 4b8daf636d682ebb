"""Host logic of the multi-fidelity sweep screener (no GPU: a stand-in network
and an analytic map play the solver)."""
import numpy as np

from bubbleensemble_implicitextension_b200 import surrogate as SG


class _Net:
    """Stand-in network: a fixed smooth guess of log10 strength and R_max."""

    def predict(self, X):
        return np.stack([0.8 + 0.3 * X[:, 0], 2.0 + 0.0 * X[:, 0]], 1).astype(np.float32)


def _grid(n=33):
    return np.linspace(0.5, 2.0, n), np.logspace(np.log10(20.0), np.log10(200.0), n)


def _map(pa, f, rough=False):
    v = np.stack([1.0 + 0.4 * pa + 0.1 * np.log10(f), 1.5 + 0.2 * pa], 1)
    if rough:
        v[:, 0] += np.where(pa > 1.5, 0.3, 0.0)   # a jump, as at a bifurcation of the collapse pattern
    return v


def _run(rough, **kw):
    pa, f = _grid()
    calls = []

    def solve(pp, ff):
        calls.append(len(pp))
        return _map(pp, ff, rough)

    res = SG.screen_sweep_lattice(_Net(), pa, f, np.full(32, 5.0), solve, **kw)
    PA, FR = np.meshgrid(pa, f, indexing="ij")
    truth = _map(PA.ravel(), FR.ravel(), rough).reshape(len(pa), len(f), 2)
    return res, truth, calls


def test_smooth_map_is_served_from_the_lattice():
    res, truth, calls = _run(False, stride=4, cell_spread=0.5, cell_disagreement=0.05, audit_fraction=0.0)
    assert res.lattice[::4, ::4].all() and res.lattice[-1, -1]
    assert res.integrated.mean() < 0.15
    # integrated points carry the solver's values exactly, served points the corrected network
    assert np.array_equal(res.map[res.integrated], truth[res.integrated])
    served = ~res.integrated
    err = np.abs(10 ** res.map[served][:, 0] - 10 ** truth[served][:, 0]) / 10 ** truth[served][:, 0]
    assert err.max() < 0.01
    assert calls[0] == res.lattice.sum()


def test_cells_across_a_jump_are_integrated():
    res, truth, _ = _run(True, stride=4, cell_spread=0.5, cell_disagreement=0.05, audit_fraction=0.0)
    pa, _ = _grid()
    band = (pa > 1.45) & (pa < 1.55)          # the lattice cell rows that straddle the jump at 1.5 bar
    assert res.integrated[band].all()
    assert res.integrated.mean() < 0.4
    served = ~res.integrated
    err = np.abs(10 ** res.map[served][:, 0] - 10 ** truth[served][:, 0]) / 10 ** truth[served][:, 0]
    assert err.max() < 0.02


def test_audit_points_are_integrated_and_measured():
    res, truth, _ = _run(False, stride=4, cell_spread=0.5, cell_disagreement=0.05, audit_fraction=0.1, seed=3)
    assert res.audited.any()
    assert res.integrated[res.audited].all()
    assert np.array_equal(res.map[res.audited], truth[res.audited])
    assert 0.0 <= res.audit_max_rel_error < 0.01


def test_without_network_serves_the_lattice_interpolation():
    """mlp=None: the counterfactual screener (bilinear interpolation of the lattice,
    corner-spread criterion only) -- the baseline the network is measured against."""
    pa, f = _grid()
    PA, FR = np.meshgrid(pa, f, indexing="ij")
    truth = _map(PA.ravel(), FR.ravel(), False).reshape(len(pa), len(f), 2)
    res = SG.screen_sweep_lattice(None, pa, f, np.full(32, 5.0), lambda pp, ff: _map(pp, ff, False), stride=4,
                                  cell_spread=0.5, cell_disagreement=0.05, audit_fraction=0.0)
    assert np.array_equal(res.map[res.integrated], truth[res.integrated])
    # the analytic map is linear in pa and in log10 f but not in f itself: interpolation errs a little
    served = ~res.integrated
    err = np.abs(10 ** res.map[served][:, 0] - 10 ** truth[served][:, 0]) / 10 ** truth[served][:, 0]
    assert 0.0 < err.max() < 0.05


def test_verify_integrates_every_served_point():
    pa, f = _grid()
    calls = []

    def solve(pp, ff):
        calls.append(len(pp))
        return _map(pp, ff, True)

    res = SG.screen_sweep_lattice(_Net(), pa, f, np.full(32, 5.0), solve, stride=4, cell_spread=0.5,
                                  cell_disagreement=0.05, audit_fraction=0.0, verify=True)
    PA, FR = np.meshgrid(pa, f, indexing="ij")
    truth = _map(PA.ravel(), FR.ravel(), True).reshape(len(pa), len(f), 2)
    assert np.array_equal(res.map, truth)                       # the verified map is the solver's everywhere
    assert sum(calls) == len(pa) * len(f)                       # every point integrated exactly once
    served = ~res.integrated
    assert np.allclose(res.served_map[res.integrated], truth[res.integrated])
    assert (res.served_rel_error[res.integrated] == 0).all() and res.served_rel_error[served].max() < 0.02
