"""Device LSMR backend against the oracle and fagra's own LSMR unit tests
(src/lsmr.rs:607-1118)."""
import numpy as np
import pytest

import fagra_b200 as fg
import oracle
from fagra_b200 import synthetic
from tests import cases

pytestmark = pytest.mark.gpu

def test_damped_products_match_dense_with_shared_columns():
    # src/lsmr.rs:617-727 (f64 1e-12, f32 1e-5)
    J, rows = cases.lsmr_shared_columns()
    for precision, tol in (("f64", 1e-12), ("f32", 1e-5)):
        b = fg.Lsmr(precision=precision)
        b.prepare(3)
        for row in rows:
            b.accumulate([0.0, 0.0], [(0, J[row:row + 2])])
        b.prepare_damping(0.1)
        s = np.maximum(np.linalg.norm(J, axis=0), 0.1)
        x, y = cases.lsmr_product_vectors(3, 7)
        for scaled in (False, True):
            for lam in (0.0, 0.01, 1e8):
                dense = cases.damped_dense(J, s, lam, scaled)
                for k in range(2):
                    fwd, tr = b.damped_products(lam, scaled, x[:, k], y[:, k])
                    ef, et = dense @ x[:, k], dense.T @ y[:, k]
                    assert np.all(np.abs(fwd - ef) < tol * np.maximum(np.abs(ef), 1.0)), (precision, scaled, lam)
                    assert np.all(np.abs(tr - et) < tol * np.maximum(np.abs(et), 1.0)), (precision, scaled, lam)


def test_prepared_modes_reject_stale_configuration():
    # src/lsmr.rs:729-778
    b = fg.Lsmr()
    b.block_preconditioning = True
    b.prepare(2)
    b.accumulate([-1.0, -1.0], [(0, np.array([[1.0, 0.0], [0.0, 3.0]]))])
    b.prepare_damping(0.1)
    b.block_preconditioning = False
    with pytest.raises(fg.InvalidOptions):
        b.solve_damped(1.0)
    b.prepare_damping(0.1)
    step = b.solve_damped(1.0).delta
    assert abs(step[0] - 0.5) < 1e-12 and abs(step[1] - 1 / 6) < 1e-12
    b.diagonal_preconditioning = False
    with pytest.raises(fg.InvalidOptions):
        b.solve_damped(1.0)
    b.prepare_damping(0.1)
    b.max_iterations = 1
    with pytest.raises(fg.LinearSolveFailed):
        b.solve_damped(1.0)
    assert b.diagnostics().termination == "IterationLimit"
    b.clear()
    with pytest.raises(fg.InvalidOptions):
        b.solve_damped(1.0)


@pytest.mark.parametrize("precision,tol", [("f64", 1e-7), ("f32", 2e-3)])
@pytest.mark.parametrize("block", [False, True])
def test_mixed_scale_damping_matches_svd(precision, tol, block):
    # src/lsmr.rs:780-855 (f64 1e-7, f32 2e-3)
    J, r = cases.lsmr_mixed_scale()
    b = fg.Lsmr(precision=precision)
    b.block_preconditioning = block
    b.prepare(4)
    b.accumulate(r, [(0, J)])
    b.prepare_damping(1e-3)
    s = np.maximum(np.linalg.norm(J, axis=0), 1e-3)
    for lam in (0.1, 10.0, 1e-3, 1e6):
        expected = cases.augmented_solution(J, r, s, lam)
        step = b.solve_damped(lam)
        actual = step.delta
        assert np.all(np.abs(actual - expected) < tol * np.maximum(np.abs(expected), 1.0)), (lam, actual, expected)
        assert actual[3] == 0.0
        assert abs(step.predicted_reduction - 0.5 * (r @ r - np.sum((J @ actual + r) ** 2))) < tol
        d = b.diagnostics()
        assert d.termination == "Converged" and d.finite_step
        assert d.scaled_relative_residual < tol
        assert abs(d.scaled_relative_residual - d.estimated_relative_residual) < tol
        assert d.original_relative_residual < tol
        assert d.min_scale == pytest.approx(s.min()) and d.max_scale == pytest.approx(s.max())
    b.block_preconditioning = False
    b.prepare_damping(1e-3)
    b.max_iterations = 1
    with pytest.raises(fg.LinearSolveFailed):
        b.solve_damped(1e-3)
    d = b.diagnostics()
    assert d.termination == "IterationLimit" and d.iterations == 1
    assert d.finite_step and np.isfinite(d.original_relative_residual)
    assert d.scaled_relative_residual > b.relative_tolerance
    b.prepare(4)
    assert b.diagnostics().termination is None


@pytest.mark.parametrize("precision,tol", [("f64", 1e-9), ("f32", 3e-4)])
@pytest.mark.parametrize("precondition,block", [(False, False), (True, False), (True, True)])
def test_damped_retries_match_augmented_svd(precision, tol, precondition, block):
    # src/lsmr.rs:857-903 (f64 1e-9, f32 3e-4); 6 damped + 2 undamped solves
    J, r = cases.lsmr_retry_system()
    b = fg.Lsmr(precision=precision)
    b.diagonal_preconditioning = precondition
    b.block_preconditioning = block
    b.prepare(3)
    b.accumulate(r, [(0, J)])
    b.prepare_damping(1.0)
    plain = b.solve()
    for lam in (1e-8, 0.01, 1.0, 100.0, 1e-4, 0.0):
        scales = np.maximum(np.linalg.norm(J, axis=0), 1.0)
        expected = cases.augmented_solution(J, r, scales, lam)
        step = b.solve_damped(lam)
        assert np.linalg.norm(step.delta - expected) < tol, (lam, step.delta, expected)
        pred = 0.5 * (r @ r - np.sum((J @ step.delta + r) ** 2))
        assert abs(step.predicted_reduction - pred) < tol
    assert np.all(np.abs(b.solve() - plain) < tol)
    w = b.statistics()
    assert w.solves == 8 and w.iterations > 0


def test_block_preconditioning_handles_coupling_gaps():
    # src/lsmr.rs:905-964 (the adjoint identity of the factors is an oracle test)
    J, r = cases.lsmr_coupling_gap()
    b = fg.Lsmr()
    b.block_preconditioning = True
    b.collect_timings = True
    b.prepare(5)
    b.accumulate(r, [(3, J[:, 3:5]), (0, J[:, 0:2])])
    b.prepare_damping(0.1)
    s = np.maximum(np.linalg.norm(J, axis=0), 0.1)
    for lam in (0.01, 1.0, 100.0):
        expected = cases.augmented_solution(J, r, s, lam)
        actual = b.solve_damped(lam).delta
        assert np.linalg.norm(actual - expected) < 1e-8
        assert actual[2] == 0.0
        d = b.diagnostics()
        assert d.block_fallbacks == 0 and d.scaled_relative_residual < 1e-8
    t = b.timings()
    assert t.linear_solve > 0 and t.preconditioner > 0
    b.prepare(0)
    assert b.timings().linear_solve == 0


def test_large_coordinate_vectors():
    # src/lsmr.rs:966-988
    b = fg.Lsmr()
    for n in (300, 1024):
        b.prepare(n)
        b.clear()
        for col in range(0, n, 2):
            b.accumulate([-float(col), -(col + 1.0)], [(col, np.eye(2))])
        assert np.all(np.abs(b.solve() - np.arange(n)) < 1e-8)


def test_rectangular_solve_matches_dense_normal_equations():
    # src/lsmr.rs:990-1118
    b = fg.Lsmr()
    b.prepare(0)
    assert len(b.solve()) == 0
    b.prepare(4)
    b.clear()
    assert list(b.solve()) == [0.0] * 4
    emissions, J, r = cases.lsmr_rectangular()
    for _ in range(2):
        b.clear()
        for res, blocks in emissions:
            b.accumulate(res, blocks)
        assert b.gradient_norm() == np.max(np.abs(J.T @ r))
        b.max_iterations = 1
        with pytest.raises(fg.LinearSolveFailed):
            b.solve()
        b.max_iterations = 1000
        expected = np.linalg.solve(J.T @ J, -J.T @ r)
        for _ in range(2):
            assert np.all(np.abs(b.solve() - expected) < 1e-8)
    for tol in (float("nan"), float("inf"), -1.0, 1.0):
        b.relative_tolerance = tol
        with pytest.raises(fg.InvalidOptions):
            b.prepare(4)


def test_inconsistent_variable_blocks_rejected_only_with_block_preconditioning():
    # src/linear_model/block_factors.rs:52-87: overlapping ranges are a DimensionMismatch
    b = fg.Lsmr()
    b.prepare(4)
    b.accumulate([1.0], [(0, np.array([[1.0, 2.0]]))])
    b.accumulate([2.0], [(1, np.array([[3.0, 1.0]]))])
    b.prepare_damping(0.1)
    o = oracle.Lsmr()
    assert o.prepare(4) == 0
    assert o.accumulate([1.0], [(0, np.array([[1.0, 2.0]]))]) == 0
    assert o.accumulate([2.0], [(1, np.array([[3.0, 1.0]]))]) == 0
    assert o.prepare_damping(0.1) == 0
    st, expected, pred = o.solve_damped(0.5)
    assert st == 0
    step = b.solve_damped(0.5)
    assert np.allclose(step.delta, expected, atol=1e-12)
    b.block_preconditioning = True
    with pytest.raises(fg.DimensionMismatch):
        b.prepare_damping(0.1)


def _random_system(seed, variables=40, width=3, emissions=160):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(emissions):
        rows = int(rng.integers(1, 4))
        k = int(rng.integers(1, 3))
        vars_ = rng.choice(variables, size=k, replace=False)
        blocks = [(int(v) * width, rng.normal(size=(rows, width)) * 10.0 ** rng.uniform(-2, 2)) for v in vars_]
        out.append((rng.normal(size=rows), blocks))
    return out, variables * width


@pytest.mark.parametrize("mode", ["identity", "diagonal", "block"])
def test_random_block_system_matches_oracle(mode):
    # Column scales over four decades: the unpreconditioned runs exhaust the
    # 1000-iteration budget at small damping in both implementations.
    emissions, n = _random_system(7)
    o = oracle.Lsmr()
    b = fg.Lsmr()
    for be in (o, b):
        be.diagonal_preconditioning = mode != "identity"
        be.block_preconditioning = mode == "block"
    assert o.prepare(n) == 0
    b.prepare(n)
    for res, blocks in emissions:
        assert o.accumulate(res, blocks) == 0
        b.accumulate(res, blocks)
    st, g = o.gradient_norm()
    assert b.gradient_norm() == g
    assert o.prepare_damping(1e-6) == 0
    b.prepare_damping(1e-6)
    for lam in (1e-4, 1e-2, 1.0):
        st, expected, pred = o.solve_damped(lam)
        od = o.diagnostics()
        if st != 0:
            assert st == 8 and od["termination"] == "IterationLimit"
            with pytest.raises(fg.LinearSolveFailed):
                b.solve_damped(lam)
            dd = b.diagnostics()
            assert dd.termination == "IterationLimit" and dd.iterations == od["iterations"] == 1000
            continue
        step = b.solve_damped(lam)
        assert np.linalg.norm(step.delta - expected) <= 1e-8 * max(np.linalg.norm(expected), 1.0)
        assert abs(step.predicted_reduction - pred) <= 1e-8 * max(abs(pred), 1.0)
        dd = b.diagnostics()
        # faer's counts are unpinned; the device and the oracle round differently, which
        # only matters once an ill-conditioned run has lost Krylov orthogonality
        if od["iterations"] < 200:
            assert abs(dd.iterations - od["iterations"]) <= 2, (dd.iterations, od)
        assert dd.termination == "Converged"
        assert dd.scaled_relative_residual <= 10 * b.relative_tolerance


def test_gauss_newton_and_lm_with_lsmr_match_oracle():
    # tests/levenberg_marquardt.rs:661-703 problem through the LSMR backend;
    # GN uses Lsmr::solve (src/lsmr.rs:500-520), the undamped identity solve.
    x0, cost, lin = cases.scalar_curve_link_problem()
    p = fg.CallbackProblem(x0, cost, lin)
    report = fg.LevenbergMarquardt(fg.Lsmr()).solve_batch(p)
    assert report.final_cost < 1e-12
    assert abs(p.x[0] - 1) < 1e-8 and abs(p.x[1] - 2) < 1e-8
    p2 = fg.CallbackProblem(x0, cost, lin)
    rep = fg.GaussNewton(fg.Lsmr()).solve_batch(p2)
    q = oracle.CallbackProblem(x0, cost, lin)
    code, orep = q.gn(oracle.Lsmr())
    assert code == 0
    assert rep.iterations == orep.iterations
    np.testing.assert_allclose(p2.x, q.x, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("precision,tol,ptol", [("f64", 1e-6, 1e-9), ("f32", 1e-2, 1e-3)])
def test_bal16_damped_step_matches_oracle(precision, tol, ptol):
    """One block-Jacobi LSMR step on the linearized bal16 system; the oracle's
    own step is within 2e-8 of the exact damped solution."""
    d = synthetic.generate("bal16")
    ob = oracle.Bal.from_data(d)
    os_ = oracle.Lsmr()
    os_.block_preconditioning = True
    assert os_.prepare(ob.dimension()) == 0
    assert ob.linearize(os_) == 0
    assert os_.prepare_damping(1e-6) == 0
    st, expected, pred = os_.solve_damped(1e-3)
    assert st == 0
    problem = fg.BalProblem.from_data(d)
    b = fg.Lsmr(precision=precision)
    b.block_preconditioning = True
    b.prepare(problem.dimension())
    problem.linearize(b)
    b.prepare_damping(1e-6)
    step = b.solve_damped(1e-3)
    assert np.linalg.norm(step.delta - expected) <= tol * np.linalg.norm(expected)
    assert abs(step.predicted_reduction - pred) <= ptol * abs(pred)
    assert b.diagnostics().termination == "Converged"


def test_bal16_lm_with_lsmr_reaches_the_oracle_cost():
    """LM over the device BAL linearization with the LSMR backend: every
    accepted cost of the first five steps and the final cost match the
    oracle's LM over its LSMR restatement within 1e-6 relative."""
    d = synthetic.generate("bal16")
    ob = oracle.Bal.from_data(d)
    os_ = oracle.Lsmr()
    os_.block_preconditioning = True
    gold = []
    code, rep, ost = ob.lm(os_, max_iterations=20, on_accept=lambda s: gold.append(s.cost))
    assert code in (0, 9, 10) and gold
    b = fg.Lsmr()
    b.block_preconditioning = True
    lm = fg.LevenbergMarquardt(b)
    costs = []
    lm.on_accept = lambda s: costs.append(s.cost)
    out = lm.solve_batch_with_outcome(fg.BalProblem.from_data(d), fg.OptimizeOptions(20, 1e-8, 0.0, 0.0))
    assert type(out.result).__name__ in ("NoProgress", "NoConvergence", "OptimizeReport")
    n = min(len(costs), len(gold), 5)
    np.testing.assert_allclose(costs[:n], gold[:n], rtol=1e-6)
    assert abs(out.statistics.cost - ost.cost) <= 1e-6 * ost.cost
    assert out.work.linear_solve.iterations > 0


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_single_launch_and_polled_lsmr_take_the_same_steps(precision, monkeypatch):
    """An LSMR solve runs as one conditional-graph launch (the device decides
    when to stop); FAGRA_B200_POLLED_GRAPHS at backend creation selects the
    fallback, graphs of 8 iterations polled from the host in doubling
    batches. Same kernels in the same order: the same iterations and the same
    step, with different launch counts showing that the two paths ran."""
    d = synthetic.generate("bal1k", cameras=60, points=6000, seed=5)

    def backend():
        problem = fg.BalProblem.from_data(d)
        b = fg.Lsmr(precision=precision)
        b.block_preconditioning = True
        b.prepare(problem.dimension())
        problem.linearize(b)
        b.prepare_damping(1e-6)
        return b

    one = backend()
    monkeypatch.setenv("FAGRA_B200_POLLED_GRAPHS", "1")
    two = backend()
    monkeypatch.delenv("FAGRA_B200_POLLED_GRAPHS")
    for lam in (1e-4, 1e-2):
        l0 = fg.kernel_launches()
        a = one.solve_damped(lam)
        l1 = fg.kernel_launches()
        b = two.solve_damped(lam)
        l2 = fg.kernel_launches()
        da, db = one.diagnostics(), two.diagnostics()
        assert da.termination == db.termination == "Converged"
        assert da.iterations == db.iterations, lam
        tol = 1e-9 if precision == "f64" else 1e-6
        assert np.linalg.norm(b.delta - a.delta) <= tol * np.linalg.norm(a.delta), lam
        assert l1 - l0 != l2 - l1, lam
