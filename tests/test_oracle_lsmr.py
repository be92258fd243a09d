"""Pins the CPU LSMR oracle to fagra's own LSMR unit tests (src/lsmr.rs:607-1118)."""
import numpy as np
import pytest

import oracle
from tests import cases

OK, INVALID_OPTIONS, LINEAR_SOLVE_FAILED = 0, 6, 8


def test_damped_products_match_dense_with_shared_columns():
    # src/lsmr.rs:617-727 (f64, 1e-12): two emissions share all three columns.
    J, rows = cases.lsmr_shared_columns()
    b = oracle.Lsmr()
    assert b.prepare(3) == OK
    for row in rows:
        assert b.accumulate([0.0, 0.0], [(0, J[row:row + 2])]) == OK
    assert b.prepare_damping(0.1) == OK
    s = b.scales()
    x, y = cases.lsmr_product_vectors(3, 7)
    for scaled in (False, True):
        for lam in (0.0, 0.01, 1e8):
            dense = cases.damped_dense(J, s, lam, scaled)
            for k in range(2):
                fwd, tr = b.damped_products(lam, scaled, x[:, k], y[:, k])
                ef, et = dense @ x[:, k], dense.T @ y[:, k]
                assert np.all(np.abs(fwd - ef) < 1e-12 * np.maximum(np.abs(ef), 1.0))
                assert np.all(np.abs(tr - et) < 1e-12 * np.maximum(np.abs(et), 1.0))


def test_prepared_modes_reject_stale_configuration():
    # src/lsmr.rs:729-778
    b = oracle.Lsmr()
    b.block_preconditioning = True
    assert b.prepare(2) == OK
    assert b.accumulate([-1.0, -1.0], [(0, np.array([[1.0, 0.0], [0.0, 3.0]]))]) == OK
    assert b.prepare_damping(0.1) == OK
    b.block_preconditioning = False
    assert b.solve_damped(1.0)[0] == INVALID_OPTIONS
    assert b.prepare_damping(0.1) == OK
    st, step, _ = b.solve_damped(1.0)
    assert st == OK and abs(step[0] - 0.5) < 1e-12 and abs(step[1] - 1 / 6) < 1e-12
    b.diagonal_preconditioning = False
    assert b.solve_damped(1.0)[0] == INVALID_OPTIONS
    assert b.prepare_damping(0.1) == OK
    b.max_iterations = 1
    assert b.solve_damped(1.0)[0] == LINEAR_SOLVE_FAILED
    assert b.diagnostics()["termination"] == "IterationLimit"
    b.clear()
    assert b.solve_damped(1.0)[0] == INVALID_OPTIONS


@pytest.mark.parametrize("block", [False, True])
def test_mixed_scale_damping_matches_svd(block):
    # src/lsmr.rs:780-855 (f64 1e-7)
    tol = 1e-7
    J, r = cases.lsmr_mixed_scale()
    b = oracle.Lsmr()
    b.block_preconditioning = block
    assert b.prepare(4) == OK
    assert b.accumulate(r, [(0, J)]) == OK
    assert b.prepare_damping(1e-3) == OK
    s = b.scales()
    for lam in (0.1, 10.0, 1e-3, 1e6):
        expected = cases.augmented_solution(J, r, s, lam)
        st, actual, pred = b.solve_damped(lam)
        assert st == OK
        assert np.all(np.abs(actual - expected) < tol * np.maximum(np.abs(expected), 1.0)), lam
        assert actual[3] == 0.0
        assert abs(pred - 0.5 * (r @ r - np.sum((J @ actual + r) ** 2))) < tol
        d = b.diagnostics()
        assert d["termination"] == "Converged" and d["finite_step"]
        assert d["scaled_relative"] < tol
        assert abs(d["scaled_relative"] - d["estimated_relative"]) < tol
        assert d["original_relative"] < tol
    b.block_preconditioning = False
    assert b.prepare_damping(1e-3) == OK
    b.max_iterations = 1
    assert b.solve_damped(1e-3)[0] == LINEAR_SOLVE_FAILED
    d = b.diagnostics()
    assert d["termination"] == "IterationLimit" and d["iterations"] == 1
    assert d["finite_step"] and np.isfinite(d["original_relative"])
    assert d["scaled_relative"] > b.relative_tolerance
    assert b.prepare(4) == OK
    assert b.diagnostics()["termination"] is None


@pytest.mark.parametrize("precondition,block", [(False, False), (True, False), (True, True)])
def test_damped_retries_match_augmented_svd(precondition, block):
    # src/lsmr.rs:857-903 (f64 1e-9)
    tol = 1e-9
    J, r = cases.lsmr_retry_system()
    b = oracle.Lsmr()
    b.diagonal_preconditioning = precondition
    b.block_preconditioning = block
    assert b.prepare(3) == OK
    assert b.accumulate(r, [(0, J)]) == OK
    assert b.prepare_damping(1.0) == OK
    st, plain = b.solve()
    assert st == OK
    for lam in (1e-8, 0.01, 1.0, 100.0, 1e-4, 0.0):
        scales = np.maximum(np.linalg.norm(J, axis=0), 1.0)
        expected = cases.augmented_solution(J, r, scales, lam)
        st, actual, pred = b.solve_damped(lam)
        assert st == OK
        assert np.linalg.norm(actual - expected) < tol, (lam, actual, expected)
        assert abs(pred - 0.5 * (r @ r - np.sum((J @ actual + r) ** 2))) < tol
    st, again = b.solve()
    assert st == OK and np.all(np.abs(again - plain) < tol)
    solves, iterations = b.work()
    assert solves == 8 and iterations > 0


def test_block_preconditioning_handles_coupling_gaps_and_adjoint():
    # src/lsmr.rs:905-964
    J, r = cases.lsmr_coupling_gap()
    b = oracle.Lsmr()
    b.block_preconditioning = True
    assert b.prepare(5) == OK
    assert b.accumulate(r, [(3, J[:, 3:5]), (0, J[:, 0:2])]) == OK
    assert b.prepare_damping(0.1) == OK
    s = b.scales()
    for lam in (0.01, 1.0, 100.0):
        expected = cases.augmented_solution(J, r, s, lam)
        st, actual, _ = b.solve_damped(lam)
        assert st == OK
        assert np.linalg.norm(actual - expected) < 1e-8
        assert actual[2] == 0.0
        d = b.diagnostics()
        assert d["block_fallbacks"] == 0 and d["scaled_relative"] < 1e-8
        for k in range(2):
            x = np.array([i + 2 * k - 2.0 for i in range(5)])
            y = np.array([2 * i + k + 1.0 for i in range(5)])
            px, pty = b.precond(x, y)
            assert abs(px @ y - x @ pty) < 1e-10


def test_large_coordinate_vectors():
    # src/lsmr.rs:966-988
    b = oracle.Lsmr()
    for n in (300, 1024):
        assert b.prepare(n) == OK
        b.clear()
        for col in range(0, n, 2):
            assert b.accumulate([-float(col), -(col + 1.0)], [(col, np.eye(2))]) == OK
        st, step = b.solve()
        assert st == OK
        assert np.all(np.abs(step - np.arange(n)) < 1e-8)


def test_rectangular_solve_matches_dense_normal_equations():
    # src/lsmr.rs:990-1118: noncontiguous views, dense normal solution, one-iteration failure.
    b = oracle.Lsmr()
    assert b.prepare(0) == OK
    st, step = b.solve()
    assert st == OK and len(step) == 0
    assert b.prepare(4) == OK
    b.clear()
    st, step = b.solve()
    assert st == OK and list(step) == [0.0] * 4
    emissions, J, r = cases.lsmr_rectangular()
    for _ in range(2):
        b.clear()
        for res, blocks in emissions:
            assert b.accumulate(res, blocks) == OK
        st, g = b.gradient_norm()
        assert st == OK and g == np.max(np.abs(J.T @ r))
        b.max_iterations = 1
        assert b.solve()[0] == LINEAR_SOLVE_FAILED
        b.max_iterations = 1000
        expected = np.linalg.solve(J.T @ J, -J.T @ r)
        for _ in range(2):
            st, step = b.solve()
            assert st == OK and np.all(np.abs(step - expected) < 1e-8)
    for tol in (float("nan"), float("inf"), -1.0, 1.0):
        b.relative_tolerance = tol
        assert b.prepare(4) == INVALID_OPTIONS
