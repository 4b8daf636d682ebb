"""Parity of the sm_100a kernel with the CPU oracle (bit for bit).

Kernel and oracle follow the same arithmetic order with explicit fused
multiply-adds and the same elementary functions, so every output must be
identical: states, collapse records, event counts, step/BiCG counters,
status bits and dense output."""
import numpy as np
import pytest

from bubbleensemble_implicitextension_b200 import solver as S
from bubbleensemble_implicitextension_b200 import workloads as W
from tests.helpers import assert_bitwise, ragged_ensemble, run_gpu

pytestmark = pytest.mark.gpu

KEYS = ["state", "uacc", "iuacc", "n_accepted", "n_rejected", "n_bicg_iter", "n_rhs", "status"]


def bounded(ens, budget=50_000):
    """Cap the attempted steps per period so that no test can run long."""
    ens.max_steps_per_period = budget
    return ens


def test_c1_subset_two_periods_with_reset(gpu, oracle_lib):
    ens = bounded(W.c1_ensemble().subset([0, 3, 7, 64, 100, 128, 200, 240, 250, 255]))
    got = run_gpu(ens, n_periods=2, reset_at=1)
    want = oracle_lib.run(ens, n_periods=2, reset_at=1)
    assert_bitwise(got, want, KEYS)
    assert (got["iuacc"] >= 0).any(), "no collapse was recorded"


def test_ragged_sizes_one_launch_per_class(gpu, oracle_lib):
    ens = bounded(ragged_ensemble([4, 8, 16, 20, 32, 33, 48, 64, 5, 31]))
    got = run_gpu(ens, n_periods=1, reset_at=-1)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1)
    assert_bitwise(got, want, KEYS)


def test_n128(gpu, oracle_lib):
    ens = bounded(ragged_ensemble([128, 100], seed=5))
    got = run_gpu(ens, n_periods=1, reset_at=-1)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1)
    assert_bitwise(got, want, KEYS)


def test_solve_loop_equals_persistent_launch(gpu):
    ens = bounded(W.c1_ensemble().subset([5, 77, 190]))
    a = run_gpu(ens, n_periods=3, reset_at=2, per_period_solve=True)
    b = run_gpu(ens, n_periods=3, reset_at=2)
    assert_bitwise(a, b, KEYS)


def test_rk4(gpu, oracle_lib):
    ens = bounded(W.c1_ensemble().subset([20, 130]))
    ens.dt0 = 2e-3
    got = run_gpu(ens, n_periods=1, reset_at=-1, algorithm=S.Algorithms.RK4)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, algorithm=0)
    assert_bitwise(got, want, KEYS)


def test_dense_output(gpu, oracle_lib):
    ens = bounded(W.c1_ensemble().subset([40, 41]))
    got = run_gpu(ens, n_periods=2, reset_at=-1, ndo=24, do_min_dt=0.05, do_save_frequency=2)
    want = oracle_lib.run(ens, n_periods=2, reset_at=-1, ndo=24, do_min_dt=0.05, do_save_frequency=2)
    assert_bitwise(got, want, KEYS + ["dense_index", "dense_time", "dense_state"])
    assert (got["dense_index"] == 24).all()


def test_warps_per_block_does_not_change_results(gpu):
    ens = bounded(W.c1_ensemble().subset(list(range(0, 256, 37))))
    a = run_gpu(ens, n_periods=1, reset_at=-1, warps_per_block=1)
    b = run_gpu(ens, n_periods=1, reset_at=-1, warps_per_block=4)
    assert_bitwise(a, b, KEYS)


def test_graph_replay_equals_direct_launches(gpu):
    ens = bounded(ragged_ensemble([32, 16, 64, 48, 8, 32, 100], seed=9))
    direct = run_gpu(ens, n_periods=1, reset_at=-1, use_graph=False)
    replay = run_gpu(ens, n_periods=1, reset_at=-1, repeat=3)
    assert_bitwise(replay, direct, KEYS)


@pytest.mark.parametrize("n,seed,wps,wpb,factored", [(128, 31, 0, 8, True), (100, 32, 1, 4, True),
                                                     (64, 33, 0, 8, True), (48, 34, 1, 4, True), (72, 35, 0, 4, True),
                                                     (40, 36, 0, 2, True), (128, 37, 0, 8, False),
                                                     (100, 38, 1, 4, False), (64, 39, 0, 4, False)])
def test_shared_matrix_staged_per_cta(n, seed, wps, wpb, factored, gpu, oracle_lib):
    """SharedCouplingMatrices on: one matrix for the whole launch, staged once per
    CTA; the products follow the oracle's shared-matrix association (on 2 or 4
    warps per system, or one warp with 2 or 4 units per lane).  factored: a
    symmetric geometry with unit factors, both products as row sums from one
    read; otherwise the reference-format (unsymmetric) matrix."""
    ens = bounded(W.c3_ensemble(n_systems=6, n_units=n, seed=seed, pa_bar=1.0, f_khz=150.0, n_periods=1,
                                reset_at=-1, cube_um=400.0 * (n / 32) ** (1 / 3), factored=factored))
    got = run_gpu(ens, n_periods=1, reset_at=-1, shared_matrices=True, warps_per_block=wpb, warps_per_system=wps)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, shared_assoc=True)
    assert_bitwise(got, want, KEYS)


def test_single_warp_systems_match_oracle(gpu, oracle_lib):
    """WarpsPerSystem = 1: systems above 32 units on one warp (2 or 4 units per lane)."""
    ens = bounded(ragged_ensemble([33, 64, 65, 128, 90, 47], seed=21))
    got = run_gpu(ens, n_periods=1, reset_at=-1, warps_per_system=1)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1)
    assert_bitwise(got, want, KEYS)


def test_multi_warp_dense_output_and_rk4(gpu, oracle_lib):
    """Multi-warp systems with dense output (the group's first warp stores the
    time) and with the RK4 stepper."""
    ens = bounded(ragged_ensemble([40, 120], seed=23))
    got = run_gpu(ens, n_periods=1, reset_at=-1, ndo=16, do_min_dt=0.05)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, ndo=16, do_min_dt=0.05)
    assert_bitwise(got, want, KEYS + ["dense_index", "dense_time", "dense_state"])
    ens.dt0 = 2e-3
    got = run_gpu(ens, n_periods=1, reset_at=-1, algorithm=S.Algorithms.RK4)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1, algorithm=0)
    assert_bitwise(got, want, KEYS)


def test_multi_warp_groups_pull_many_systems(gpu):
    """Many more systems than resident groups, several groups per CTA: the
    multi-warp and single-warp layouts give identical results."""
    rng = np.random.default_rng(41)
    ens = bounded(ragged_ensemble(list(rng.integers(33, 129, 700)), seed=42), budget=400)
    a = run_gpu(ens, n_periods=1, reset_at=-1, warps_per_system=1)
    b = run_gpu(ens, n_periods=1, reset_at=-1)
    c = run_gpu(ens, n_periods=1, reset_at=-1, warps_per_block=2)
    assert_bitwise(b, a, KEYS)
    assert_bitwise(c, a, KEYS)


@pytest.mark.parametrize("n,wps", [(128, 0), (100, 1), (64, 0)])
def test_shared_geometry_with_per_system_radii(n, wps, gpu, oracle_lib):
    """One staged geometry G for the launch, each system's own radii through the
    unit factors a_i = R_i^-2, b_j = R_j^3 (C_ij = a_i G_ij b_j)."""
    ens = bounded(W.c3_radii_ensemble(n_systems=5, n_units=n, seed=40 + n, n_periods=1,
                                      cube_um=400.0 * (n / 32) ** (1 / 3)))
    got = run_gpu(ens, n_periods=1, reset_at=-1, warps_per_block=8, warps_per_system=wps)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1)
    assert_bitwise(got, want, KEYS)


def test_coupling_factors_need_the_shared_matrix_kernels(gpu):
    """Factors other than 1 on a launch without the shared-matrix kernels are refused."""
    ens = W.c3_radii_ensemble(n_systems=2, n_units=40, n_periods=1)
    ens.shared_matrices = False
    ps = ens.make_solver()
    try:
        ps.SynchroniseFromHostToDevice(S.ListOfVariables.All)
        with pytest.raises(S.BesError, match="CouplingRowScale"):
            ps.solve_periods(1, -1)
    finally:
        ps.close()


def test_autotuned_shapes_give_identical_results(gpu):
    """bes_autotune times every launch shape of every class, restores the device
    state and keeps the fastest: the following solve equals a plain one."""
    ens = bounded(ragged_ensemble([16, 32, 48, 64, 100, 128, 8, 40, 90, 20], seed=51))
    a = run_gpu(ens, n_periods=1, reset_at=-1)
    b = run_gpu(ens, n_periods=1, reset_at=-1, autotune=True)
    assert_bitwise(b, a, KEYS)


def test_shared_symmetric_geometry_n32_row_in_registers(gpu, oracle_lib):
    """C1 given as the shared symmetric line geometry with unit factors: the
    N <= 32 kernel keeps a row of G in registers (RHS 6, and RHS 5 with ragged
    sizes below), bit-identical to the oracle's shared association."""
    ens = bounded(W.c1_ensemble(factored=True).subset([0, 3, 7, 64, 100, 128, 200, 250]))
    got = run_gpu(ens, n_periods=2, reset_at=1)
    want = oracle_lib.run(ens, n_periods=2, reset_at=1)
    assert_bitwise(got, want, KEYS)
    assert (got["iuacc"] >= 0).any()


def test_shared_symmetric_geometry_ragged_n_le_32(gpu, oracle_lib):
    full = W.c1_ensemble(factored=True, n_units=24, n_pa=4, n_f=2)
    ens = bounded(full)
    got = run_gpu(ens, n_periods=1, reset_at=-1)
    want = oracle_lib.run(ens, n_periods=1, reset_at=-1)
    assert_bitwise(got, want, KEYS)
