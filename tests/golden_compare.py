"""Comparison of a run with a golden fixture from the reference's own solver.

Tolerances (the parity bar): radii within 1e-8 relative at the end of the run
and at the saved dense-output times, collapse strength Rmax/Rmin within
1e-6 relative, identical event counts.  Over several periods the recorded
maxima (located events) are held to 1e-8 and the strengths to 1e-6 for at
least 99.9 % of the records (2e-5 at most): see the comment in check().  Dense output stores accepted step
ends, whose times move with the step-size controller (its error estimate
is a cancelling difference, so rounding-level changes shift the steps by
~1e-7), so a saved radius is first moved to the reference's saved time with
its own dR/dtau:  R(t_ref) = R(t) + dR/dtau (t_ref - t)."""
import json
from pathlib import Path

import numpy as np

from bubbleensemble_implicitextension_b200 import workloads as W
from tests.golden import cases

GOLDEN = Path(__file__).resolve().parent / "golden"
R_TOL = 1e-8
STRENGTH_TOL = 1e-6
MULTI_PERIOD_STRENGTH_MAX = 2e-5


def load(name):
    g = np.load(GOLDEN / f"{name}.npz")
    return {k: g[k] for k in g.files if k != "case"}, json.loads(str(g["case"]))


def check(name, got, subset=None, multi_period_share=1e-3):
    """Compare a run with the fixture `name`; `subset` (a slice of the fixture's
    systems) when the run covered only those (whole systems of equal size);
    multi_period_share: the share of collapse strengths of a multi-period case
    allowed above 1e-6 (see below)."""
    g, _ = load(name)
    ens, run = cases.build(name, subset=subset)
    if subset is not None:
        n = int(ens.units[0])
        ns_all = len(cases.CASES[name]["systems"])
        keep = np.arange(ns_all)[subset]
        cols = np.concatenate([np.arange(k * n, (k + 1) * n) for k in keep])
        g = {k: (v[..., cols] if k in ("state", "uacc", "iuacc") else v) for k, v in g.items()}
    R, Rg = got["state"][0], g["state"][0]
    rel = np.abs(R - Rg) / np.abs(Rg)
    assert rel.max() <= R_TOL, f"{name}: final radius differs by {rel.max():.3e}"
    dR, dRg = got["state"][1], g["state"][1]
    assert np.all(np.abs(dR - dRg) <= R_TOL * np.maximum(np.abs(dRg), 1.0)), f"{name}: final dR/dtau"
    np.testing.assert_array_equal(got["iuacc"], g["iuacc"], err_msg=f"{name}: event counts")
    _, _, s, c = W.collapse_records(got["uacc"], got["iuacc"], ens.units)
    _, _, sg, cg = W.collapse_records(g["uacc"], g["iuacc"], ens.units)
    np.testing.assert_array_equal(c, cg)
    m = sg > 0
    np.testing.assert_array_equal(s > 0, m)
    if m.any():
        srel = np.abs(s[m] - sg[m]) / np.abs(sg[m])
        if run["n_periods"] == 1:
            assert srel.max() <= STRENGTH_TOL, f"{name}: collapse strength differs by {srel.max():.3e}"
        else:
            # The recorded maxima are located events and must match like the radii.  A
            # recorded minimum is the smallest radius at an accepted step end, not a
            # located extremum, so over several periods a rounding-level shift of the
            # step ends alone moves a few of them by more than 1e-6 (the oracle against
            # the reference: 3 of 36155 records over 4 periods, at most 8.5e-6, p99.9
            # 5e-8): the strength bar holds for at least 99.9 % of the records.
            rmax, _, _, _ = W.collapse_records(got["uacc"], got["iuacc"], ens.units)
            rmaxg, _, _, _ = W.collapse_records(g["uacc"], g["iuacc"], ens.units)
            mrel = np.abs(rmax[m] - rmaxg[m]) / np.abs(rmaxg[m])
            assert mrel.max() <= R_TOL, f"{name}: a recorded maximum differs by {mrel.max():.3e}"
            over = int((srel > STRENGTH_TOL).sum())
            assert over <= max(1, int(multi_period_share * srel.size)), \
                f"{name}: {over} of {srel.size} strengths differ by > 1e-6"
            assert srel.max() <= MULTI_PERIOD_STRENGTH_MAX, f"{name}: collapse strength differs by {srel.max():.3e}"
    if run.get("ndo"):
        np.testing.assert_array_equal(got["dense_index"], g["dense_index"])
        dt = g["dense_time"] - got["dense_time"]
        assert np.abs(dt).max() < 1e-4, f"{name}: saved times differ by {np.abs(dt).max():.3e}"
        dtu = np.repeat(dt, ens.units, axis=1)
        Rt = got["dense_state"][:, 0] + got["dense_state"][:, 1] * dtu
        drel = np.abs(Rt - g["dense_state"][:, 0]) / np.abs(g["dense_state"][:, 0])
        assert drel.max() <= R_TOL, f"{name}: radius at saved times differs by {drel.max():.3e}"
    return float(rel.max())
