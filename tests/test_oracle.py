"""Pins the CPU oracle to fagra's own known-answer tests (no GPU needed)."""
import numpy as np
import pytest

import oracle
from tests import cases

OK, INVALID_OPTIONS, LINEAR_SOLVE_FAILED = 0, 6, 8
INVALID_EVALUATION, DIMENSION_MISMATCH, UNSUPPORTED_STRUCTURE = 20, 21, 23


def test_projection_known_answer():
    # tests/bal.rs:104-112
    cam, X, expected = cases.bal_known_answer()
    pix, st = oracle.project(cam, X)
    assert st == OK
    assert abs(pix[0] - expected[0]) < 1e-12
    assert pix[1] == 2 * pix[0]
    _, st = oracle.project(cam, np.zeros(3))
    assert st == INVALID_EVALUATION


@pytest.mark.parametrize("rotation", cases.BAL_JACOBIAN_ROTATIONS)
def test_jacobians_match_central_differences(rotation):
    # tests/bal.rs:63-103
    cam, X = cases.bal_jacobian_case(rotation)
    jc, jp = oracle.jacobians(cam, X)
    h = 1e-6
    for k in range(12):
        cp, cm, xp, xm = cam.copy(), cam.copy(), X.copy(), X.copy()
        if k < 9:
            cp[k] += h
            cm[k] -= h
        else:
            xp[k - 9] += h
            xm[k - 9] -= h
        num = (oracle.project(cp, xp)[0] - oracle.project(cm, xm)[0]) / (2 * h)
        ana = jc[:, k] if k < 9 else jp[:, k - 9]
        assert np.linalg.norm(num - ana) < 1e-5 * max(np.linalg.norm(ana), 1.0), k


def test_linear_model_verification_known_answer():
    # src/linear_model.rs:344-367
    m = oracle.Model(3)
    j = np.array([[1.0, 2.0, 0.0], [3.0, -1.0, 0.0]])
    assert m.accumulate([-2.0, 5.0], [(0, j)]) == OK
    assert m.prepare_scales(0.5) == OK
    v = m.verify(np.array([0.2, -0.3, 0.4]), 0.7)
    assert abs(v["predicted"] + 5.785) < 1e-12
    np.testing.assert_allclose(v["normal_residual"], [16.7, -11.75, 0.07], atol=1e-12)
    assert list(v["reference"]) == [13.0, -9.0, 0.0]
    assert v["finite_step"] and v["residual_norm"] > 20
    g, neg = m.state()
    assert list(g) == [13.0, -9.0, 0.0]
    assert list(neg) == [2.0, -5.0]


def test_block_factors_fallback_and_overlap():
    # src/linear_model/block_factors.rs:211-245
    blocks = [[0, 0, 1, 2, 0]]
    st, fb = oracle.block_factors_fallbacks(1, 3, blocks, [1.0, 1.0], [1.0, 1.0, 1.0], [0.0, 0.01, 0.1])
    assert st == OK and fb == [1, 0, 0]
    st, fb = oracle.block_factors_fallbacks(1, 3, blocks, [np.inf, 1.0], [1.0, 1.0, 1.0], [0.01])
    assert st == OK and fb == [1]
    st, _ = oracle.block_factors_fallbacks(1, 3, blocks + [[0, 1, 1, 2, 0]], [1.0, 1.0], [1.0, 1.0, 1.0], [0.1])
    assert st == DIMENSION_MISMATCH


def test_schur_matches_augmented_svd_with_retries_unaries_and_unused_blocks():
    # src/schur.rs:690-789 (f64, tolerance 1e-7)
    tol = 1e-7
    emissions, J, r = cases.twelve_column_schur_emissions()
    s = oracle.Schur(6, 2, 2)
    assert s.prepare(12) == OK
    s.clear()
    for res, blocks in emissions:
        assert s.accumulate(res, blocks) == OK
    assert s.prepare_damping(0.1) == OK
    scales = s.export()["scales"]
    for lam in [0.001, 1.0, 100.0, 0.01]:
        expected = cases.augmented_solution(J, r, scales, lam)
        st, actual, pred = s.solve_damped(lam)
        assert st == OK
        assert np.linalg.norm(actual - expected) < tol * max(np.linalg.norm(expected), 1.0)
        assert abs(pred - 0.5 * (r @ r - np.sum((J @ actual + r) ** 2))) < tol
        for k in (4, 5, 10, 11):
            assert actual[k] == 0.0
        d = s.diagnostics()
        assert d["termination"] == "Converged"
        assert d["reduced"] < tol and d["scaled"] < tol
    s.max_iterations = 1
    st, _, _ = s.solve_damped(0.001)
    assert st == LINEAR_SOLVE_FAILED
    d = s.diagnostics()
    assert d["termination"] == "IterationLimit" and d["iterations"] == 1
    assert d["estimated"] is None
    assert np.isfinite(d["reduced"]) and d["reduced"] > s.relative_tolerance
    assert s.prepare(12) == OK
    assert s.work() == (0, 0)


def test_schur_partition_structure_and_singular_elimination():
    # src/schur.rs:792-870
    j = np.array([[1.0, 1.0]])
    s = oracle.Schur(2, 2, 2)
    assert s.prepare(5) == INVALID_OPTIONS
    assert s.prepare(6) == OK
    s.clear()
    assert s.accumulate([1.0], [(2, j), (4, j)]) == UNSUPPORTED_STRUCTURE
    assert s.accumulate([1.0], [(1, j)]) == UNSUPPORTED_STRUCTURE
    assert s.solve_damped(0.1)[0] != OK
    assert s.accumulate([1.0], [(0, j), (2, j)]) == OK
    assert s.prepare_damping(0.1) == OK
    assert s.solve_damped(0.0)[0] != OK
    assert s.diagnostics()["termination"] == "NotPositiveDefinite"
    assert s.solve_damped(0.1)[0] == OK
    assert s.solve_damped(float("nan"))[0] != OK
    coupled = oracle.Schur(4, 2, 2)
    assert coupled.prepare(6) == OK
    assert coupled.accumulate([1.0], [(0, j), (2, j)]) == UNSUPPORTED_STRUCTURE
    undamped = oracle.Schur(2, 2, 2)
    assert undamped.prepare(4) == OK
    for col in (0, 2):
        assert undamped.accumulate([1.0, 2.0], [(col, np.eye(2))]) == OK
    for _ in range(2):
        st, d = undamped.solve()
        assert st == OK
        np.testing.assert_allclose(d, [-1, -2, -1, -2], atol=1e-10)
    for retained, n in [(0, 0), (0, 2), (2, 2)]:
        b = oracle.Schur(retained, 2, 2)
        assert b.prepare(n) == OK
        b.clear()
        if n:
            assert b.accumulate([1.0], [(0, j)]) == OK
        assert b.prepare_damping(0.1) == OK
        assert b.solve_damped(0.1)[0] == OK


def test_schur_lm_converges_on_scalar_curves():
    # tests/levenberg_marquardt.rs:661-703
    x0, cost, lin = cases.scalar_curve_link_problem()
    p = oracle.CallbackProblem(x0, cost, lin)
    code, rep, st = p.lm(oracle.Schur(1, 1, 1))
    assert code == OK, code
    assert rep.final_cost < 1e-12
    a, b = p.x
    assert abs(a - 1) < 1e-8 and abs(b - 2) < 1e-8


def test_twelve_point_bal_reduces_reprojection_error():
    # tests/bal.rs:7-41 with the Schur backend (retained = the single camera)
    cams, pts, oc, op, px = cases.twelve_point_bal()
    bal = oracle.Bal(cams, pts, oc, op, px)
    _, initial = bal.cost()
    code, rep, st = bal.lm(oracle.Schur(9, 9, 3), max_iterations=50, gradient_tolerance=1e-8,
                           step_tolerance=1e-10, cost_tolerance=1e-12)
    assert code == OK, code
    _, final = bal.cost()
    assert final < initial * 1e-6
    assert abs(rep.final_cost - final) < 1e-12
    assert st.accepted_steps > 0


def test_bal16_oracle_lm_matches_golden():
    """Config bal16 (16 cameras, 1,000 points): the oracle's 20-step LM run
    reproduces the committed golden trace (tests/golden/make_golden.py)."""
    import json
    from pathlib import Path
    from fagra_b200 import synthetic
    gold = json.loads((Path(__file__).parent / "golden" / "bal16_oracle.json").read_text())
    d = synthetic.generate("bal16")
    assert d.num_observations == gold["observations"]
    bal = oracle.Bal.from_data(d)
    costs = []
    code, rep, st = bal.lm(oracle.Schur(9 * d.num_cameras, 9, 3), max_iterations=20,
                           on_accept=lambda s: costs.append(s.cost))
    assert code == gold["status"]
    assert abs(rep.initial_cost - gold["initial_cost"]) <= 1e-12 * gold["initial_cost"]
    assert abs(st.cost - gold["final_cost"]) <= 1e-9 * gold["final_cost"]
    np.testing.assert_allclose(costs, gold["accepted_costs"], rtol=1e-9)
