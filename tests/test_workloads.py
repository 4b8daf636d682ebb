"""Host-side workload builders: the factored coupling inputs equal the
reference-format matrices, and the shard bounds cover every system once."""
import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import workloads as W


@pytest.mark.parametrize("build", [
    lambda f: W.c1_ensemble(n_pa=2, n_f=2, factored=f),
    lambda f: W.c3_ensemble(n_systems=2, n_units=40, cube_um=300.0, factored=f),
])
def test_factored_coupling_is_the_reference_matrix(build):
    fac, ref = build(True), build(False)
    assert fac.shared_matrices and fac.coupling_row_scale is not None
    G = fac.coupling[:fac.units[0] ** 2].reshape(fac.units[0], -1)
    assert np.array_equal(G, G.T)                         # the staged geometry is symmetric
    explicit = W.explicit_matrices(fac)
    n = int(ref.units[0])
    C_ref = ref.coupling[:n * n]
    for s in range(fac.n_systems):
        C_fac = explicit.coupling[s * n * n:(s + 1) * n * n]
        np.testing.assert_allclose(C_fac, C_ref, rtol=4e-16 * 8, atol=0.0)


@pytest.mark.parametrize("world", [1, 2, 3, 7, 400])
def test_shard_bounds_cover_every_system_once(world):
    units = np.random.default_rng(1).choice([4, 8, 16, 32, 48, 64], 300)
    b = W.shard_bounds(units, world)
    assert len(b) == world + 1 and b[0] == 0 and b[-1] == len(units)
    assert np.all(np.diff(b) >= 0)


def test_ring_ensemble_is_banded():
    from bubbleensemble_implicitextension_b200 import workloads as W
    ens = W.ring_ensemble(n_systems=3, n_units=40, band_width=2)
    n = 40
    for s in range(3):
        C = ens.coupling[s * n * n:(s + 1) * n * n].reshape(n, n).T
        off = (np.arange(n)[None, :] - np.arange(n)[:, None]) % n
        band = ((off <= 2) | (off >= n - 2)) & (off != 0)
        assert (C[band] > 0).all() and (C[~band] == 0).all()
    assert ens.band_width == 2


def test_oracle_banded_association_matches_full_matrix(oracle_lib):
    """The banded association (band products over the 2 CBW + 1 diagonals only)
    and the full-matrix association of the same banded matrix agree to rounding."""
    from bubbleensemble_implicitextension_b200 import workloads as W
    ens = W.ring_ensemble(n_systems=2, n_units=64, band_width=2)
    ens.max_steps_per_period = 50_000
    a = oracle_lib.run(ens, band_width=2)
    b = oracle_lib.run(ens, band_width=0)
    np.testing.assert_array_equal(a["iuacc"], b["iuacc"])
    assert (np.abs(a["state"][0] - b["state"][0]) / b["state"][0]).max() < 1e-10
