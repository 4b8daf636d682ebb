"""One geometry, per-system radii: the oracle's factored shared-matrix
association (a_i G_ij b_j, factors applied to the vectors) against the same
systems with each system's matrix written out (no sharing)."""
import dataclasses

import numpy as np

from bubbleensemble_implicitextension_b200 import workloads as W
from oracle import oracle as O


def test_factored_matches_explicit_matrices():
    ens = W.c3_radii_ensemble(n_systems=3, n_units=40, n_periods=1, cube_um=400.0 * (40 / 128) ** (1 / 3))
    ens.max_steps_per_period = 50_000
    a = O.run(ens, n_periods=1, reset_at=-1)
    b = O.run(W.explicit_matrices(ens), n_periods=1, reset_at=-1)
    rel = np.abs(a["state"] - b["state"]) / np.abs(b["state"])
    assert rel.max() < 1e-6                        # two associations of the same products, one period
    assert np.array_equal(a["iuacc"], b["iuacc"])  # the same collapse events
    assert (a["iuacc"] >= 0).any()


def test_unit_factors_reproduce_the_unscaled_association():
    ens = W.c3_ensemble(n_systems=2, n_units=40, n_periods=1, cube_um=300.0, factored=False)
    ens.max_steps_per_period = 50_000
    ones = dataclasses.replace(ens, coupling_row_scale=np.ones(ens.total_units),
                               coupling_col_scale=np.ones(ens.total_units))
    x = O.run(ens, n_periods=1, reset_at=-1)
    y = O.run(ones, n_periods=1, reset_at=-1)
    for k in ("state", "uacc", "iuacc", "n_accepted", "n_bicg_iter"):
        assert np.array_equal(x[k], y[k]), k


def test_symmetric_and_general_shared_associations_agree():
    """The same C3 systems given as the symmetric geometry with unit factors
    (both products as row sums) and as the reference-format matrix (transposed
    product as a column tree): equal physics, rounding-level differences."""
    kw = dict(n_systems=2, n_units=48, n_periods=1, cube_um=350.0, seed=4)
    a = O.run(W.c3_ensemble(factored=True, **kw), n_periods=1, reset_at=-1)
    b = O.run(W.c3_ensemble(factored=False, **kw), n_periods=1, reset_at=-1)
    rel = np.abs(a["state"] - b["state"]) / np.abs(b["state"])
    assert rel.max() < 1e-6
    assert np.array_equal(a["iuacc"], b["iuacc"])


def test_factored_line_matches_reference_format():
    """C1 as the symmetric line geometry with unit factors (shared association)
    against the reference-format matrix: one period, 1e-6 and equal events."""
    kw = dict(n_pa=2, n_f=2, n_periods=1, reset_at=-1)
    a = O.run(W.c1_ensemble(factored=True, **kw).subset([1, 2]), n_periods=1, reset_at=-1)
    b = O.run(W.c1_ensemble(factored=False, **kw).subset([1, 2]), n_periods=1, reset_at=-1)
    rel = np.abs(a["state"] - b["state"]) / np.abs(b["state"])
    assert rel.max() < 1e-6
    assert np.array_equal(a["iuacc"], b["iuacc"])
