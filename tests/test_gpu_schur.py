"""Device Schur backend against the oracle and fagra's own Schur unit tests."""
import numpy as np
import pytest

import fagra_b200 as fg
import oracle
from tests import cases

pytestmark = pytest.mark.gpu


def _filled(backend, emissions):
    backend.prepare(12)
    backend.clear()
    for res, blocks in emissions:
        backend.accumulate(res, blocks)
    backend.prepare_damping(0.1)


@pytest.mark.parametrize("precision,tol", [("f64", 1e-7), ("f32", 3e-3)])
def test_schur_matches_augmented_svd_with_retries_unaries_and_unused_blocks(precision, tol):
    # src/schur.rs:690-789 (f64 1e-7, f32 3e-3)
    emissions, J, r = cases.twelve_column_schur_emissions()
    b = fg.Schur(6, 2, 2, precision=precision)
    b.collect_timings = True
    if precision == "f32":
        b.relative_tolerance = 1e-6
    _filled(b, emissions)
    scales = b.model()["scales"]
    for lam in [0.001, 1.0, 100.0, 0.01]:
        expected = cases.augmented_solution(J, r, scales, lam)
        step = b.solve_damped(lam)
        actual = step.delta
        assert np.linalg.norm(actual - expected) < tol * max(np.linalg.norm(expected), 1.0), (lam, actual, expected)
        assert abs(step.predicted_reduction - 0.5 * (r @ r - np.sum((J @ actual + r) ** 2))) < tol
        for k in (4, 5, 10, 11):
            assert actual[k] == 0.0
        d = b.diagnostics()
        assert d.termination == "Converged"
        assert d.reduced_relative_residual < tol and d.scaled_relative_residual < tol
    b.max_iterations = 1
    with pytest.raises(fg.LinearSolveFailed):
        b.solve_damped(0.001)
    d = b.diagnostics()
    assert d.termination == "IterationLimit"
    assert d.iterations == 1
    assert d.estimated_relative_residual is None
    assert np.isfinite(d.reduced_relative_residual) and d.reduced_relative_residual > b.relative_tolerance
    assert b.timings().linear_solve > 0
    b.prepare(12)
    assert b.statistics().solves == 0
    assert b.timings().linear_solve == 0


def test_schur_partition_structure_and_singular_elimination():
    # src/schur.rs:792-870
    j = np.array([[1.0, 1.0]])
    b = fg.Schur(2, 2, 2)
    with pytest.raises(fg.InvalidOptions):
        b.prepare(5)
    b.prepare(6)
    b.clear()
    with pytest.raises(fg.UnsupportedStructure):
        b.accumulate([1.0], [(2, j), (4, j)])
    with pytest.raises(fg.UnsupportedStructure):
        b.accumulate([1.0], [(1, j)])
    with pytest.raises(fg.SolverError):
        b.solve_damped(0.1)
    b.accumulate([1.0], [(0, j), (2, j)])
    b.prepare_damping(0.1)
    with pytest.raises(fg.SolverError):
        b.solve_damped(0.0)
    assert b.diagnostics().termination == "NotPositiveDefinite"
    b.solve_damped(0.1)
    with pytest.raises(fg.SolverError):
        b.solve_damped(float("nan"))
    coupled = fg.Schur(4, 2, 2)
    coupled.prepare(6)
    with pytest.raises(fg.UnsupportedStructure):
        coupled.accumulate([1.0], [(0, j), (2, j)])
    undamped = fg.Schur(2, 2, 2)
    undamped.prepare(4)
    for col in (0, 2):
        undamped.accumulate([1.0, 2.0], [(col, np.eye(2))])
    for _ in range(2):
        np.testing.assert_allclose(undamped.solve(), [-1, -2, -1, -2], atol=1e-10)
    for retained, n in [(0, 0), (0, 2), (2, 2)]:
        e = fg.Schur(retained, 2, 2)
        e.prepare(n)
        e.clear()
        if n:
            e.accumulate([1.0], [(0, j)])
        e.prepare_damping(0.1)
        e.solve_damped(0.1)


def test_index_maps_are_bit_exact_and_values_match_oracle():
    """Jacobian blocks, edges, owner map and variable blocks equal the oracle's
    bit for bit; packed values, -r, gradient, scales, Gram and cross blocks
    agree to f64 rounding."""
    emissions, _, _ = cases.twelve_column_schur_emissions()
    b = fg.Schur(6, 2, 2)
    _filled(b, emissions)
    o = oracle.Schur(6, 2, 2)
    o.prepare(12)
    o.clear()
    for res, blocks in emissions:
        o.accumulate(res, blocks)
    o.prepare_damping(0.1)
    ref = o.export()
    s = b.structure()
    m = b.model()
    owners_ref = np.where(ref["owners"] == np.iinfo(np.uint64).max, np.iinfo(np.uint64).max, ref["owners"])
    assert np.array_equal(s["blocks"], ref["blocks"])
    assert np.array_equal(s["edges"], ref["edges"])
    assert np.array_equal(s["owners"], owners_ref)
    assert np.array_equal(s["variables"], ref["variables"])
    for key in ("values", "negative_residual", "gradient", "scales", "gram", "cross"):
        np.testing.assert_allclose(m[key], ref[key], rtol=1e-13, atol=1e-13, err_msg=key)


@pytest.mark.parametrize("lam", [0.0, 1e-3, 1.0])
def test_reduced_operator_matches_oracle(lam):
    emissions, _, _ = cases.twelve_column_schur_emissions()
    if lam == 0.0:
        lam = 1e-9
    b = fg.Schur(6, 2, 2)
    _filled(b, emissions)
    o = oracle.Schur(6, 2, 2)
    o.prepare(12)
    o.clear()
    for res, blocks in emissions:
        o.accumulate(res, blocks)
    o.prepare_damping(0.1)
    x = np.linspace(-1, 2, 6)
    np.testing.assert_allclose(b.reduced_apply(lam, x), o.reduced_apply(lam, x), rtol=1e-12, atol=1e-12)


def test_lm_with_schur_converges_on_scalar_curves():
    # tests/levenberg_marquardt.rs:661-703
    x0, cost, lin = cases.scalar_curve_link_problem()
    p = fg.CallbackProblem(x0, cost, lin)
    lm = fg.LevenbergMarquardt(fg.Schur(1, 1, 1))
    for _ in range(2):  # warm workspace reuse on a fresh start
        p.x[:] = x0
        report = lm.solve_batch(p)
        assert report.final_cost < 1e-12
        assert abs(p.x[0] - 1) < 1e-8 and abs(p.x[1] - 2) < 1e-8


def test_gauss_newton_with_schur_matches_oracle():
    x0, cost, lin = cases.scalar_curve_link_problem()
    p = fg.CallbackProblem(x0, cost, lin)
    rep = fg.GaussNewton(fg.Schur(1, 1, 1)).solve_batch(p)
    q = oracle.CallbackProblem(x0, cost, lin)
    code, orep = q.gn(oracle.Schur(1, 1, 1))
    assert code == 0
    assert rep.iterations == orep.iterations
    np.testing.assert_allclose(p.x, q.x, rtol=1e-10, atol=1e-12)
