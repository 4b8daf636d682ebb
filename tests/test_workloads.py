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
