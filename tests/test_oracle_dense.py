"""Pins the CPU oracle's dense backends, square-root elimination, selected
covariance and SE(3) geometry to fagra's own tests:
src/normal.rs:401-626, tests/direct_backends.rs, src/dense_schur/tests.rs,
src/marginalization/tests.rs, src/covariance.rs:329-470 and
tests/pose_geometry.rs."""
import numpy as np
import pytest
from scipy.linalg import expm

import oracle

OK, SINGULAR_INFORMATION, INVALID_INFORMATION = 0, 2, 3
INVALID_OPTIONS, LINEAR_SOLVE_FAILED = 6, 8
INVALID_EVALUATION, DIMENSION_MISMATCH, UNSUPPORTED_STRUCTURE = 20, 21, 23
EPS = np.finfo(float).eps


def test_normal_lower_triangle_rhs_and_solve():
    # src/normal.rs:598-626
    b = oracle.DenseNormal()
    for _ in range(2):
        assert b.prepare(2) == OK
        b.clear()
        assert b.accumulate([-5.0, -11.0], [(0, np.array([[1.0, 2.0], [3.0, 4.0]]))]) == OK
        normal, rhs = b.state()
        assert normal[0, 0] == 10 and normal[1, 0] == 14 and normal[1, 1] == 20
        assert list(rhs) == [38.0, 54.0]
        assert b.gradient_norm() == (OK, 54.0)
        st, step = b.solve()
        assert st == OK and abs(step[0] - 1) < 1e-12 and abs(step[1] - 2) < 1e-12


@pytest.mark.parametrize("rows", [0, 1, 2, 3, 4, 5, 8, 16, 32])
def test_normal_accumulation_matches_dense_reference(rows):
    # src/normal.rs:407-478: shuffled blocks, zero-stride views, an empty block
    b = oracle.DenseNormal()
    assert b.prepare(31) == OK
    b.clear()
    normal = np.zeros((31, 31))
    rhs = np.zeros(31)
    for weight in (1.0, 0.13, 0.0):
        storage = np.array([[weight * (((r * 7 + c * 11) % 23) - 11.0) / 13.0 for c in range(31)]
                            for r in range(2 * rows)]) if rows else np.zeros((0, 31))
        j = storage[0::2]  # view_with_steps(.., (1, 0)): every other row
        residual = np.array([weight * (r - 1.3) for r in range(rows)])
        blocks = [(o, j[:, o:o + w]) for o, w in [(24, 3), (6, 6), (31, 0), (18, 6), (0, 6), (27, 4), (12, 6)]]
        assert b.accumulate(residual, blocks) == OK
        normal += j.T @ j
        rhs -= j.T @ residual
    got, got_rhs = b.state()
    tol = 256 * EPS
    assert np.all(np.abs(got_rhs - rhs) <= tol * (1 + np.abs(rhs)))
    low = np.tril_indices(31)
    assert np.all(np.abs(got[low] - normal[low]) <= tol * (1 + np.abs(normal[low])))


def test_normal_information_rank_screen():
    # src/normal.rs:558-596
    for scale in (1e-6, 1.0, 1e6):
        b = oracle.DenseNormal()
        assert b.prepare(2) == OK
        b.clear()
        assert b.accumulate([0.0, 0.0], [(0, np.array([[scale, 1.0], [0.0, 1e-5]]))]) == OK
        assert b.information(1e-8) == SINGULAR_INFORMATION
        assert b.information(1e-12) == OK
    b = oracle.DenseNormal()
    assert b.prepare(1) == OK
    b.clear()
    assert b.accumulate([0.0], [(0, np.array([[1e200]]))]) == OK
    assert b.information(0.0) == INVALID_INFORMATION


def _direct_check(make):
    # tests/direct_backends.rs:4-98
    b = make()
    for m, n in [(7, 3), (43, 35), (1, 3), (0, 2), (0, 0), (7, 3)]:
        j = np.array([[(k + 1.0) if m == 1 else ((i * 7 + k * 13) % 17) / 5.0 - 1.0 + (4.0 if i == k else 0.0)
                       for k in range(n)] for i in range(m)]).reshape(m, n)
        r = np.array([i / 3.0 - 0.7 for i in range(m)])
        assert b.prepare(n) == OK
        b.clear()
        assert b.solve_damped(1.0)[0] == INVALID_OPTIONS
        for row in range(m):
            assert b.accumulate(r[row:row + 1], [(c, j[row:row + 1, c:c + 1]) for c in reversed(range(n))]) == OK
        h, g = j.T @ j, j.T @ r
        if m >= n:
            expected = np.linalg.solve(h, -g) if n else np.zeros(0)
            st, actual = b.solve()
            assert st == OK and np.all(np.abs(actual - expected) < 2e-5)
            b.clear()
            assert b.accumulate(r, [(0, j)]) == OK
        for floor in (0.0, -1.0, float("nan"), float("inf")):
            assert b.prepare_damping(floor) == INVALID_OPTIONS
        assert b.prepare_damping(0.25) == OK
        for lam in (-1.0, float("nan"), float("inf")):
            assert b.solve_damped(lam)[0] == INVALID_OPTIONS
        if m < n:
            assert b.solve_damped(0.0)[0] == LINEAR_SOLVE_FAILED
        for lam in (0.1, 10.0, 0.01, 0.1):
            damped = h + np.diag(lam * np.maximum(np.diag(h), 0.25 ** 2))
            expected = np.linalg.solve(damped, -g) if n else np.zeros(0)
            st, actual, pred = b.solve_damped(lam)
            assert st == OK and np.all(np.abs(actual - expected) < 2e-4)
            prediction = -g @ actual - 0.5 * np.sum((j @ actual) ** 2)
            assert abs(pred - prediction) < 2e-4 * (1 + abs(prediction))
        b.clear()
        assert b.solve_damped(1.0)[0] == INVALID_OPTIONS


def test_direct_backends_match_reference_steps_and_predictions():
    _direct_check(oracle.DenseQr)
    _direct_check(oracle.DenseNormal)


def test_qr_damping_unused_coordinates_and_mixed_units():
    # tests/direct_backends.rs:108-143
    qr = oracle.DenseQr()
    assert qr.prepare(3) == OK
    j = np.array([[0.0, 1e9, 0.0], [0.0, 0.0, 1e-3]])
    assert qr.accumulate([-1.0, -1.0], [(0, j)]) == OK
    assert qr.prepare_damping(1e-6) == OK
    for lam in (1e-3, 1.0, 10.0, 1e-3):
        st, d, pred = qr.solve_damped(lam)
        t = 1.0 / (1.0 + lam)
        assert st == OK and d[0] == 0.0
        for index, scale in ((1, 1e9), (2, 1e-3)):
            assert abs(d[index] * scale / t - 1) < 1e-5
        assert abs(pred / (2 * t - t * t) - 1) < 1e-5


def test_qr_keeps_a_direction_lost_by_normal_equations():
    # tests/direct_backends.rs:145-178
    j = np.array([[1.0, 1.0], [1e-10, 0.0], [0.0, 1e-10]])
    r = np.array([-3.0, -1e-10, -2e-10])
    qr, normal = oracle.DenseQr(), oracle.DenseNormal()
    assert qr.prepare(2) == OK and normal.prepare(2) == OK
    assert qr.accumulate(r, [(0, j)]) == OK and normal.accumulate(r, [(0, j)]) == OK
    st, step = qr.solve()
    assert st == OK and abs(step[0] - 1) < 1e-6 and abs(step[1] - 2) < 1e-6
    assert normal.solve()[0] == LINEAR_SOLVE_FAILED
    qr.set_tolerance(1e-8)
    assert qr.solve()[0] == LINEAR_SOLVE_FAILED
    assert qr.prepare_damping(0.1) == OK
    assert qr.solve_damped(0.01)[0] == OK


def test_dense_schur_mixed_blocks_match_dense_damping_retries():
    # src/dense_schur/tests.rs:8-60 (f64 1e-11)
    schur, dense = oracle.DenseSchur(6, [2, 3]), oracle.DenseNormal()
    assert schur.prepare(11) == OK and dense.prepare(11) == OK
    schur.clear()
    dense.clear()
    for count, columns in [(9, [(3, 3), (6, 2), (0, 2), (2, 1)]), (10, [(8, 3), (2, 1), (0, 2), (3, 3)]),
                           (8, [(2, 1), (3, 3), (0, 2)])]:
        storage = np.array([[3.0 if i // 2 == j else ((i * 7 + j * 3) % 13) / 11.0 for j in range(11)]
                            for i in range(2 * count)])
        view = storage[0::2]  # view_with_steps((0,0),(count,..),(1,0)): every other row
        r = np.array([i * 0.17 - 0.5 for i in range(count)])
        blocks = [(o, view[:, o:o + w]) for o, w in columns]
        assert schur.accumulate(r, blocks) == OK
        assert dense.accumulate(r, blocks) == OK
    assert schur.prepare_damping(1e-6) == OK and dense.prepare_damping(1e-6) == OK
    for lam in (0.0, 0.001, 10.0, 0.01, 0.0):
        sa, a, pa = schur.solve_damped(lam)
        sb, b, pb = dense.solve_damped(lam)
        assert sa == OK and sb == OK
        assert np.all(np.abs(a - b) < 1e-11)
        assert abs(pa - pb) < 1e-10


def test_dense_schur_topology_and_singular_landmarks():
    # src/dense_schur/tests.rs:117-170
    b = oracle.DenseSchur(3, [2, 1])
    assert b.prepare(5) != OK
    assert b.prepare(6) == OK
    b.clear()
    assert b.accumulate(np.zeros(0), [(3, np.zeros((0, 2)))]) == OK
    assert b.accumulate(np.zeros(0), [(5, np.zeros((0, 1)))]) == OK
    assert b.prepare_damping(1e-6) == OK
    assert b.solve_damped(0.1)[0] == OK
    b.clear()
    j, k, r = np.ones((1, 2)), np.ones((1, 1)), np.ones(1)
    for blocks in ([(3, j), (5, k)], [(4, k)], [(2, j)]):
        assert b.accumulate(r, blocks) == UNSUPPORTED_STRUCTURE
    assert b.accumulate(r, [(3, j)]) == OK
    assert b.prepare_damping(1e-6) == OK
    assert b.solve_damped(0.0)[0] != OK
    assert b.solve_damped(0.1)[0] == OK
    assert b.solve_damped(float("nan"))[0] != OK


def test_dense_schur_empty_partitions_and_unobserved_coordinates():
    # src/dense_schur/tests.rs:172-195
    for retained, widths, dim in [(0, [], 0), (2, [], 2), (0, [2], 2)]:
        b = oracle.DenseSchur(retained, widths)
        assert b.prepare(dim) == OK
        b.clear()
        if dim:
            assert b.accumulate(np.full(dim, 0.5), [(0, np.eye(dim))]) == OK
        assert b.solve()[0] == OK
    b = oracle.DenseSchur(1, [1])
    assert b.prepare(2) == OK
    b.clear()
    assert b.accumulate([0.0], []) == OK
    assert b.prepare_damping(1e-6) == OK
    assert b.solve_damped(0.0)[0] != OK
    assert b.solve_damped(1.0)[0] == OK


def test_dense_schur_covariance_rank_screen():
    # src/dense_schur/tests.rs:197-249
    for retained, widths in [(0, [2]), (2, [])]:
        b = oracle.DenseSchur(retained, widths)
        assert b.prepare(2) == OK
        b.clear()
        assert b.accumulate(np.zeros(2), [(0, np.array([[1.0, 1.0], [0.0, 1e-4]]))]) == OK
        assert b.covariance([], 1e-6)[0] == SINGULAR_INFORMATION
        assert b.covariance([], 1e-12)[0] == OK
    b = oracle.DenseSchur(1, [2])
    assert b.prepare(3) == OK
    b.clear()
    assert b.accumulate(np.zeros(1), [(0, np.eye(1))]) == OK
    assert b.covariance([], 64 * EPS)[0] == SINGULAR_INFORMATION


def test_dense_schur_covariance_matches_dense_normal():
    # src/dense_schur/tests.rs:62-115: retained selection (one, two) = columns [2, 0, 1]
    schur, dense = oracle.DenseSchur(3, [2, 3]), oracle.DenseNormal()
    assert schur.prepare(8) == OK and dense.prepare(8) == OK
    schur.clear()
    dense.clear()
    j = np.array([[2.0 + c if r == c else ((r * 7 + c * 11) % 17) / 13.0 for c in range(8)] for r in range(9)])
    for landmark, width in [(3, 2), (5, 3)]:
        blocks = [(c, j[:, c:c + w]) for c, w in [(2, 1), (landmark, width), (0, 2)]]
        assert schur.accumulate(np.zeros(9), blocks) == OK
        assert dense.accumulate(np.zeros(9), blocks) == OK
    cols = [2, 0, 1]
    sa, a = schur.covariance(cols, 64 * EPS)
    sb, b = dense.covariance(cols, 64 * EPS)
    assert sa == sb
    if sa == OK:
        assert np.all(np.abs(a - b) < 1e-12)


MARGINAL_CASES = [
    (4, 4, 2, [1., 2., 1., 0., 3., 2., 4., 0., 2., -1., 0., 0., 1., 1., 2., 3., 6., -1., 0., 1.]),
    (2, 4, 3, [1., 0., 2., 3., 4., 0., 1., 1., 2., 3.]),
    (3, 2, 1, [0., 1., 2., 0., 2., 3., 0., -1., 1.]),
    (4, 3, 1, [1., 2., 0., 1., 2., -1., 1., 3., -1., 0., 2., 4., 0., 1., -1., 2.]),
    (3, 2, 0, [1., 0., 2., 0., 1., 3., 0., 0., 4.]),
    (3, 1, 1, [1., 1., 2., 3., -1., 2.]),
]


@pytest.mark.parametrize("m,n,removed,values", MARGINAL_CASES)
def test_elimination_reduced_objective_matches_svd(m, n, removed, values):
    # src/marginalization/tests.rs:30-97 (f64 1e-11)
    rows = np.array(values).reshape(m, n + 1)
    st, a, b, constant, _ = oracle.eliminate(rows, removed)
    assert st == OK
    for shift in (-2.0, 0.0, 0.5, 3.0):
        delta = shift + 0.3 * np.arange(n - removed)
        rhs = rows[:, removed:n] @ delta + rows[:, n]
        if removed:
            e = rows[:, :removed]
            step = np.linalg.lstsq(e, -rhs, rcond=1e-10)[0]
            residual = e @ step + rhs
        else:
            residual = rhs
        expected = 0.5 * residual @ residual
        reduced = a @ delta + b
        actual = 0.5 * reduced @ reduced + constant
        assert abs(actual - expected) <= 1e-11 * (1 + abs(expected))


def test_elimination_keeps_directions_lost_by_normal_equations():
    # src/marginalization/tests.rs:99-120
    eps = 1e-10
    rows = np.array([1., 1., 1., 2., eps, -eps, 2., -1., 0., 0., 3., 4.]).reshape(3, 4)
    st, a, b, constant, rank = oracle.eliminate(rows, 2)
    assert st == OK and rank == 2
    for y in (-2.0, 0.0, 1.0, 5.0):
        r = a[0, 0] * y + b[0]
        expected = 0.5 * (3 * y + 4) ** 2
        assert abs(0.5 * r * r + constant - expected) <= 1e-11 * (1 + expected)


def test_selected_covariance_preserves_order_cross_terms_and_marginalization():
    # src/covariance.rs:400-470: 24x24 J over knots (9, 9), alignment (3), nuisance (3)
    j = np.array([[4.0 if i == k else ((i * 7 + k * 11) % 13) / 30.0 for k in range(24)] for i in range(24)])
    reference = np.linalg.inv(j.T @ j)
    cols = list(range(9, 18)) + list(range(0, 9)) + list(range(18, 21))
    b = oracle.DenseNormal()
    assert b.prepare(24) == OK
    b.clear()
    blocks = [(0, j[:, 0:9]), (9, j[:, 9:18]), (18, j[:, 18:21]), (21, j[:, 21:24])]
    assert b.accumulate(np.zeros(24), blocks) == OK
    st, cov = b.covariance(cols, 64 * EPS)
    assert st == OK and cov.shape == (21, 21)
    assert np.all(np.abs(cov - reference[np.ix_(cols, cols)]) < 1e-12)
    # Marginalize the nuisance by square-root elimination; the prior keeps the
    # marginal covariance of the other 21 coordinates.
    rows = np.hstack([j[:, 21:24], j[:, 0:21], np.zeros((24, 1))])
    st, a, prior_b, constant, rank = oracle.eliminate(rows, 3)
    assert st == OK and rank == 3
    p = oracle.DenseNormal()
    assert p.prepare(21) == OK
    p.clear()
    assert p.accumulate(prior_b, [(0, a)]) == OK
    st, cov2 = p.covariance(cols, 64 * EPS)
    assert st == OK
    assert np.all(np.abs(cov2 - reference[np.ix_(cols, cols)]) < 1e-12)


def _skew(v):
    return np.array([[0, -v[2], v[1]], [v[2], 0, -v[0]], [-v[1], v[0], 0]])


def _reference_right_jacobian(delta):
    # tests/pose_geometry.rs:10-24: Jr = integral exp(-s ad(delta)) ds via a 12x12 generator
    g = np.zeros((12, 12))
    w, v = _skew(delta[3:]), _skew(delta[:3])
    g[0:3, 0:3] = -w
    g[3:6, 3:6] = -w
    g[0:3, 3:6] = -v
    g[0:6, 6:12] = np.eye(6)
    return expm(g)[0:6, 6:12]


def _rotation(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def test_pose_geometry_matches_matrix_exponentials():
    # tests/pose_geometry.rs:40-104 (f64 2e-11)
    tol = 2e-11
    axis = np.array([2.0, -3.0, 1.0])
    axis /= np.linalg.norm(axis)
    for angle in (0.0, 1e-9, 0.019999, 0.020001, 0.099999, 0.100001, 0.499999, 0.5, 0.500001, 0.9,
                  np.pi - 1e-7, 4.0, 6.0):
        for scale in (0.0, 1.0, 100.0):
            delta = np.concatenate([np.array([0.7, 0.2, -0.4]) * scale, axis * angle])
            ref = _reference_right_jacobian(delta)
            jr = oracle.pose_right_jacobian(delta)
            assert np.all(np.abs(jr - ref) <= tol * (1 + np.abs(ref)))
            st, jinv = oracle.pose_log_jacobian(delta)
            assert st == OK
            inv = np.linalg.inv(ref)
            assert np.all(np.abs(jinv - inv) <= 10 * tol * (1 + np.abs(inv)))
            hat = np.zeros((4, 4))
            hat[0:3, 0:3] = _skew(axis * angle)
            hat[0:3, 3] = delta[:3]
            expected = expm(hat)
            pose = oracle.pose_exp(delta)
            assert np.all(np.abs(_rotation(pose[:4]) - expected[:3, :3]) <= tol * (1 + np.abs(expected[:3, :3])))
            assert np.all(np.abs(pose[4:] - expected[:3, 3]) <= tol * (1 + np.abs(expected[:3, 3])))
    for value in (float("nan"), float("inf"), np.finfo(float).max):
        assert oracle.pose_log_jacobian(np.full(6, value))[0] != OK


def test_pose_log_inverts_exp_and_adjoint_transports_tangents():
    rng = np.random.default_rng(3)
    for _ in range(20):
        d = rng.normal(size=6) * np.array([1, 1, 1, 0.5, 0.5, 0.5])
        assert np.allclose(oracle.pose_log(oracle.pose_exp(d)), d, atol=1e-12)
        x = oracle.pose_exp(rng.normal(size=6))
        # x Exp(d) = Exp(Ad(x) d) x
        lhs = oracle.pose_compose(x, oracle.pose_exp(d * 1e-3))
        rhs = oracle.pose_compose(oracle.pose_exp(oracle.pose_adjoint(x) @ (d * 1e-3)), x)
        assert np.allclose(lhs, rhs, atol=1e-12) or np.allclose(lhs, np.concatenate([-rhs[:4], rhs[4:]]), atol=1e-12)


def _se3_log_rel(ref, x):
    """Log(ref^-1 x) through the oracle's own pose primitives."""
    import ctypes as C
    dp = C.POINTER(C.c_double)
    inv, rel, out = np.zeros(7), np.zeros(7), np.zeros(6)
    a = np.ascontiguousarray(ref, np.float64)
    b = np.ascontiguousarray(x, np.float64)
    oracle.lib.or_pose_inverse(a.ctypes.data_as(dp), inv.ctypes.data_as(dp))
    oracle.lib.or_pose_compose(inv.ctypes.data_as(dp), b.ctypes.data_as(dp), rel.ctypes.data_as(dp))
    oracle.lib.or_pose_log(rel.ctypes.data_as(dp), out.ctypes.data_as(dp))
    return out


def test_window_prior_generalizes_the_anchor_and_follows_priors_update():
    """The window prior r = b + sum_i A_i Log(ref_i^-1 x_i) (src/marginalization.rs
    157-231): with s = 1, A = I, b = 0, ref = z it is the anchor PosePrior and
    the window solve is bit-identical; a two-pose prior's cost is the numpy
    restatement's."""
    from fagra_b200 import posegraph
    batch = posegraph.generate(2, min_poses=24, max_poses=30)
    poses, prior, ij, z = batch.window(0)
    a = oracle.window_solve(poses, prior, ij, z, removed=10)
    b = oracle.window_solve(poses, prior, ij, z, removed=10, marginal=(np.eye(6), np.zeros(6), prior[None, :]))
    assert np.array_equal(a["poses"], b["poses"])
    assert np.array_equal(a["prior_a"], b["prior_a"]) and np.array_equal(a["prior_b"], b["prior_b"])
    rng = np.random.default_rng(4)
    A = rng.normal(size=(9, 12))
    bb = rng.normal(size=9)
    refs = poses[:2] + 0.0
    refs[:, 4:] += 0.01 * rng.normal(size=(2, 3))
    st, c = oracle.window_cost(poses, prior, ij, z, marginal=(A, bb, refs))
    assert st == 0
    r = bb + A[:, :6] @ _se3_log_rel(refs[0], poses[0]) + A[:, 6:] @ _se3_log_rel(refs[1], poses[1])
    st0, c_rel = oracle.window_cost(poses, prior, ij, z, marginal=(np.zeros((1, 6)), np.zeros(1), prior[None, :]))
    assert st0 == 0
    assert abs(c - (c_rel + 0.5 * r @ r)) <= 1e-12 * c


def test_sliding_window_chain_on_the_oracle():
    """One sliding-window step on the oracle: the retained poses with the
    marginal prior (separators first) solve to a finite cost no worse than the
    prior-free restart's prior term, and the elimination of the next window
    succeeds with its separator inside the window."""
    from fagra_b200 import posegraph
    batch = posegraph.generate(3, min_poses=32, max_poses=44, seed=23)
    poses = batch.poses.copy()
    seps, elims = [], []
    for w in range(batch.windows):
        x, pr, ij, z = batch.window(w)
        r = oracle.window_solve(x, pr, ij, z, removed=10)
        assert r["code"] in (0, 9, 10)
        poses[batch.pose_offset[w]:batch.pose_offset[w + 1]] = r["poses"]
        seps.append(list(r["separator"]))
        elims.append((r["prior_a"], r["prior_b"]))
    nb, priors = posegraph.slide_windows(batch, 10, poses, seps, elims)
    for w in range(nb.windows):
        x, pr, ij, z = nb.window(w)
        assert len(x) == batch.sizes[w] - 10
        # at the linearization point the marginal prior's residual is b
        st, c = oracle.window_cost(x, pr, ij, z, marginal=priors[w])
        A, bv, refs = priors[w]
        st0, c0 = oracle.window_cost(x, pr, ij, z, marginal=(np.zeros((1, A.shape[1])), np.zeros(1), refs))
        assert st == 0 and st0 == 0
        assert abs(c - (c0 + 0.5 * bv @ bv)) <= 1e-10 * max(c, 1.0)
        r = oracle.window_solve(x, pr, ij, z, removed=10, marginal=priors[w])
        assert r["code"] in (0, 9, 10) and r["rank"] > 0
        assert r["stats"].cost <= c + 1e-12
