"""Device dense backends (DenseNormalCholesky, DenseSchur, DenseQr) and the
selected covariance against fagra's own tests and the oracle:
src/normal.rs:558-626, tests/direct_backends.rs, src/dense_schur/tests.rs,
src/covariance.rs:400-470."""
import numpy as np
import pytest

import fagra_b200 as fg
import oracle

pytestmark = pytest.mark.gpu
EPS = np.finfo(float).eps


def test_normal_known_answer_and_destructive_solve():
    # src/normal.rs:598-626: H = [[10],[14,20]], rhs [38, 54], step [1, 2]
    b = fg.DenseNormalCholesky()
    for _ in range(2):
        b.prepare(2)
        b.clear()
        b.accumulate([-5.0, -11.0], [(0, np.array([[1.0, 2.0], [3.0, 4.0]]))])
        assert b.gradient_norm() == 54.0
        step = b.solve()
        assert abs(step[0] - 1) < 1e-12 and abs(step[1] - 2) < 1e-12
        with pytest.raises(fg.InvalidOptions):
            b.prepare_damping(0.1)  # normal.rs:154-160: factored in place


def test_normal_information_rank_screen():
    # src/normal.rs:558-596
    for scale in (1e-6, 1.0, 1e6):
        b = fg.DenseNormalCholesky()
        b.prepare(2)
        b.clear()
        b.accumulate([0.0, 0.0], [(0, np.array([[scale, 1.0], [0.0, 1e-5]]))])
        with pytest.raises(fg.SingularInformation):
            b.covariance([0], 1e-8)
        b.covariance([0], 1e-12)
    b = fg.DenseNormalCholesky()
    b.prepare(1)
    b.clear()
    b.accumulate([0.0], [(0, np.array([[1e200]]))])
    with pytest.raises(fg.InvalidInformation):
        b.covariance([0], 0.0)


@pytest.mark.parametrize("make", [fg.DenseQr, fg.DenseNormalCholesky], ids=["qr", "normal"])
def test_direct_backends_match_reference_steps(make):
    # tests/direct_backends.rs:4-98 (f64)
    b = make()
    for m, n in [(7, 3), (43, 35), (1, 3), (0, 2), (0, 0), (7, 3)]:
        j = np.array([[(k + 1.0) if m == 1 else ((i * 7 + k * 13) % 17) / 5.0 - 1.0 + (4.0 if i == k else 0.0)
                       for k in range(n)] for i in range(m)]).reshape(m, n)
        r = np.array([i / 3.0 - 0.7 for i in range(m)])
        b.prepare(n)
        b.clear()
        with pytest.raises(fg.InvalidOptions):
            b.solve_damped(1.0)
        for row in range(m):
            b.accumulate(r[row:row + 1], [(c, j[row:row + 1, c:c + 1]) for c in reversed(range(n))])
        h, g = j.T @ j, j.T @ r
        if m >= n:
            expected = np.linalg.solve(h, -g) if n else np.zeros(0)
            actual = b.solve()
            assert np.all(np.abs(actual - expected) < 2e-5)
            b.clear()
            b.accumulate(r, [(0, j)])
        for floor in (0.0, -1.0, float("nan"), float("inf")):
            with pytest.raises(fg.InvalidOptions):
                b.prepare_damping(floor)
        b.prepare_damping(0.25)
        for lam in (-1.0, float("nan"), float("inf")):
            with pytest.raises(fg.InvalidOptions):
                b.solve_damped(lam)
        if m < n:
            with pytest.raises(fg.LinearSolveFailed):
                b.solve_damped(0.0)
        for lam in (0.1, 10.0, 0.01, 0.1):
            damped = h + np.diag(lam * np.maximum(np.diag(h), 0.25 ** 2))
            expected = np.linalg.solve(damped, -g) if n else np.zeros(0)
            step = b.solve_damped(lam)
            assert np.all(np.abs(step.delta - expected) < 2e-4)
            prediction = -g @ step.delta - 0.5 * np.sum((j @ step.delta) ** 2)
            assert abs(step.predicted_reduction - prediction) < 2e-4 * (1 + abs(prediction))
        b.clear()
        with pytest.raises(fg.InvalidOptions):
            b.solve_damped(1.0)


def test_qr_unused_coordinates_mixed_units_and_lost_direction():
    # tests/direct_backends.rs:108-178
    qr = fg.DenseQr()
    qr.prepare(3)
    qr.accumulate([-1.0, -1.0], [(0, np.array([[0.0, 1e9, 0.0], [0.0, 0.0, 1e-3]]))])
    qr.prepare_damping(1e-6)
    for lam in (1e-3, 1.0, 10.0, 1e-3):
        step = qr.solve_damped(lam)
        t = 1.0 / (1.0 + lam)
        assert step.delta[0] == 0.0
        assert abs(step.delta[1] * 1e9 / t - 1) < 1e-5 and abs(step.delta[2] * 1e-3 / t - 1) < 1e-5
        assert abs(step.predicted_reduction / (2 * t - t * t) - 1) < 1e-5
    j = np.array([[1.0, 1.0], [1e-10, 0.0], [0.0, 1e-10]])
    r = np.array([-3.0, -1e-10, -2e-10])
    qr, normal = fg.DenseQr(), fg.DenseNormalCholesky()
    for be in (qr, normal):
        be.prepare(2)
        be.accumulate(r, [(0, j)])
    step = qr.solve()
    assert abs(step[0] - 1) < 1e-6 and abs(step[1] - 2) < 1e-6
    with pytest.raises(fg.LinearSolveFailed):
        normal.solve()
    qr.relative_rank_tolerance = 1e-8
    with pytest.raises(fg.LinearSolveFailed):
        qr.solve()
    qr.prepare_damping(0.1)
    qr.solve_damped(0.01)


def _mixed_schur_emissions():
    # src/dense_schur/tests.rs:8-38
    out = []
    for count, columns in [(9, [(3, 3), (6, 2), (0, 2), (2, 1)]), (10, [(8, 3), (2, 1), (0, 2), (3, 3)]),
                           (8, [(2, 1), (3, 3), (0, 2)])]:
        storage = np.array([[3.0 if i // 2 == j else ((i * 7 + j * 3) % 13) / 11.0 for j in range(11)]
                            for i in range(2 * count)])
        view = storage[0::2]
        r = np.array([i * 0.17 - 0.5 for i in range(count)])
        out.append((r, [(o, view[:, o:o + w]) for o, w in columns]))
    return out


def test_dense_schur_matches_dense_normal_and_oracle_across_damping():
    # src/dense_schur/tests.rs:8-60 (f64 1e-11)
    schur, dense = fg.DenseSchur(6, [2, 3]), fg.DenseNormalCholesky()
    ref = oracle.DenseSchur(6, [2, 3])
    assert ref.prepare(11) == 0
    for be in (schur, dense):
        be.prepare(11)
        be.clear()
    for r, blocks in _mixed_schur_emissions():
        schur.accumulate(r, blocks)
        dense.accumulate(r, blocks)
        assert ref.accumulate(r, blocks) == 0
    schur.prepare_damping(1e-6)
    dense.prepare_damping(1e-6)
    assert ref.prepare_damping(1e-6) == 0
    for lam in (0.0, 0.001, 10.0, 0.01, 0.0):
        a, b = schur.solve_damped(lam), dense.solve_damped(lam)
        st, expected, pred = ref.solve_damped(lam)
        assert st == 0
        assert np.all(np.abs(a.delta - b.delta) < 1e-11)
        assert np.all(np.abs(a.delta - expected) < 1e-11)
        assert abs(a.predicted_reduction - pred) < 1e-10


def test_dense_schur_topology_and_singular_landmarks():
    # src/dense_schur/tests.rs:117-170
    b = fg.DenseSchur(3, [2, 1])
    with pytest.raises(fg.InvalidOptions):
        b.prepare(5)
    b.prepare(6)
    b.clear()
    j, k, r = np.ones((1, 2)), np.ones((1, 1)), np.ones(1)
    for blocks in ([(3, j), (5, k)], [(4, k)], [(2, j)]):
        with pytest.raises(fg.UnsupportedStructure):
            b.accumulate(r, blocks)
    b.accumulate(r, [(3, j)])
    b.prepare_damping(1e-6)
    with pytest.raises(fg.SolverError):
        b.solve_damped(0.0)
    b.solve_damped(0.1)
    with pytest.raises(fg.SolverError):
        b.solve_damped(float("nan"))


def test_dense_schur_covariance_rank_screen_and_match():
    # src/dense_schur/tests.rs:197-249 and 62-115
    for retained, widths in [(0, [2]), (2, [])]:
        b = fg.DenseSchur(retained, widths)
        b.prepare(2)
        b.clear()
        b.accumulate(np.zeros(2), [(0, np.array([[1.0, 1.0], [0.0, 1e-4]]))])
        with pytest.raises(fg.SingularInformation):
            b.covariance([], 1e-6)
        b.covariance([], 1e-12)
    schur, dense = fg.DenseSchur(3, [2, 3]), fg.DenseNormalCholesky()
    for be in (schur, dense):
        be.prepare(8)
        be.clear()
    j = np.array([[2.0 + c if r == c else ((r * 7 + c * 11) % 17) / 13.0 for c in range(8)] for r in range(9)])
    for landmark, width in [(3, 2), (5, 3)]:
        blocks = [(c, j[:, c:c + w]) for c, w in [(2, 1), (landmark, width), (0, 2)]]
        for be in (schur, dense):
            be.accumulate(np.zeros(9), blocks)
    a = schur.covariance([2, 0, 1])
    b = dense.covariance([2, 0, 1])
    assert np.all(np.abs(a - b) < 1e-12)


def test_covariance_matches_inverse_information_in_selection_order():
    # src/covariance.rs:400-470
    j = np.array([[4.0 if i == k else ((i * 7 + k * 11) % 13) / 30.0 for k in range(24)] for i in range(24)])
    reference = np.linalg.inv(j.T @ j)
    cols = list(range(9, 18)) + list(range(0, 9)) + list(range(18, 21))
    b = fg.DenseNormalCholesky()
    b.prepare(24)
    b.clear()
    b.accumulate(np.zeros(24), [(0, j[:, 0:9]), (9, j[:, 9:18]), (18, j[:, 18:21]), (21, j[:, 21:24])])
    cov = b.covariance(cols)
    assert cov.shape == (21, 21)
    assert np.all(np.abs(cov - reference[np.ix_(cols, cols)]) < 1e-12)
    with pytest.raises(fg.DuplicateCovarianceBlock):
        b.covariance([0, 0])
    with pytest.raises(fg.InvalidRankTolerance):
        b.covariance([0], 1.0)


def test_lm_and_gn_over_dense_backends():
    # tests/levenberg_marquardt.rs:661-703 problem through each dense backend;
    # GN steps match the oracle's DenseNormalCholesky GN.
    from tests import cases
    x0, cost, lin = cases.scalar_curve_link_problem()
    for make in (lambda: fg.DenseSchur(1, [1]), lambda: fg.DenseSchur(2, []), fg.DenseNormalCholesky,
                 fg.DenseQr):
        p = fg.CallbackProblem(x0, cost, lin)
        report = fg.LevenbergMarquardt(make()).solve_batch(p)
        assert report.final_cost < 1e-12
        assert abs(p.x[0] - 1) < 1e-8 and abs(p.x[1] - 2) < 1e-8
    p = fg.CallbackProblem(x0, cost, lin)
    rep = fg.GaussNewton(fg.DenseNormalCholesky()).solve_batch(p)
    q = oracle.CallbackProblem(x0, cost, lin)
    code, orep = q.gn(oracle.DenseNormal())
    assert code == 0 and rep.iterations == orep.iterations
    np.testing.assert_allclose(p.x, q.x, rtol=1e-10, atol=1e-12)
