"""Batched pose-graph windows on the device against the oracle's per-window
LevenbergMarquardt over DenseSchur (src/dense_schur.rs) followed by the
square-root elimination of src/marginalization.rs:458-513."""
import numpy as np
import pytest

import oracle
from fagra_b200 import posegraph as pg

pytestmark = pytest.mark.gpu

OPTS = pg.WINDOW_OPTIONS


def _oracle(batch, w, removed=10):
    poses, prior, ij, z = batch.window(w)
    return oracle.window_solve(poses, prior, ij, z, removed=removed, **OPTS)


def _prior_objective(A, b, c, delta):
    r = A @ delta + b
    return 0.5 * r @ r + c


@pytest.fixture(scope="module")
def small_batch():
    return pg.generate(6, min_poses=20, max_poses=60, seed=11)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_windows_match_oracle_lm_and_prior(small_batch, precision):
    b = small_batch
    solver = pg.WindowSolver(b, removed=10, precision=precision)
    poses, reps, a, bb = solver.solve()
    rng = np.random.default_rng(4)
    for w in range(b.windows):
        ref = _oracle(b, w)
        rep = reps[w]
        assert rep.status in (0, 9, 10)
        assert ref["code"] == rep.status or (ref["code"] in (9, 10) and rep.status in (9, 10)), (w, ref["code"])
        # final cost within 1e-6 relative of the f64 oracle
        rcost = ref["stats"].cost
        assert abs(rep.final_cost - rcost) <= 1e-6 * max(rcost, 1e-12), (w, rep.final_cost, rcost)
        if precision == "f64":
            assert rep.iterations == ref["stats"].accepted_steps
        p0, p1 = b.pose_offset[w], b.pose_offset[w + 1]
        assert np.allclose(poses[p0:p1], ref["poses"], atol=1e-6 if precision == "f64" else 1e-5)
        # separator poses: identical index lists
        s0, s1 = solver.separator_offset[w], solver.separator_offset[w + 1]
        assert list(solver.separators[s0:s1]) == list(ref["separator"])
        # prior: same reduced objective on random separator increments
        assert rep.prior_status == 0 and rep.eliminated_rank == ref["rank"]
        A, bvec, c = solver.prior(w, rep, a, bb)
        for _ in range(3):
            d = rng.normal(size=A.shape[1]) * 0.1
            e = _prior_objective(A, bvec, c, d)
            r = _prior_objective(ref["prior_a"], ref["prior_b"], ref["prior_constant"], d)
            tol = 1e-6 if precision == "f64" else 1e-4
            assert abs(e - r) <= tol * max(abs(r), 1.0), (w, e, r)


def test_windows_second_run_reuses_the_tuned_graph(small_batch):
    b = small_batch
    solver = pg.WindowSolver(b, removed=10)
    first = solver.solve()
    panel, per, ms = solver.tuning()
    assert panel in (16, 32) and per in (1, 2) and ms.max() > 0
    second = solver.solve()
    assert np.array_equal(first[0], second[0])
    assert [r.final_cost for r in first[1]] == [r.final_cost for r in second[1]]


def test_windows_reject_bad_structure():
    import fagra_b200 as fg
    b = pg.generate(2, min_poses=20, max_poses=20, seed=3)
    bad = pg.WindowBatch(b.sizes, b.pose_offset, b.poses, b.truth, b.prior, b.rel_offset, b.rel_ij.copy(), b.rel_z)
    bad.rel_ij[0, 1] = 25  # outside window 0
    with pytest.raises(fg.DimensionMismatch):
        pg.WindowSolver(bad)
    bad.rel_ij[0, 1] = bad.rel_ij[0, 0]
    with pytest.raises(fg.UnsupportedStructure):
        pg.WindowSolver(bad)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_anchor_through_set_priors_is_bit_identical(small_batch, precision):
    """The anchor PosePrior is the window prior with s = 1, A = I, b = 0,
    ref = the anchor pose: the same solve bit for bit."""
    b = small_batch
    first = pg.WindowSolver(b, removed=10, precision=precision).solve()
    solver = pg.WindowSolver(b, removed=10, precision=precision)
    solver.set_priors([(np.eye(6), np.zeros(6), b.prior[w][None, :]) for w in range(b.windows)])
    second = solver.solve()
    assert np.array_equal(first[0], second[0])
    assert [r.final_cost for r in first[1]] == [r.final_cost for r in second[1]]
    assert [r.iterations for r in first[1]] == [r.iterations for r in second[1]]
    assert np.array_equal(first[2], second[2]) and np.array_equal(first[3], second[3])


@pytest.fixture(scope="module")
def chained():
    """One sliding-window step: solve, eliminate the oldest 10 poses, and
    hand the retained poses with the marginal prior to the next solve."""
    b = pg.generate(5, min_poses=32, max_poses=56, seed=23)
    solver = pg.WindowSolver(b, removed=10)
    poses, reps, a, bb = solver.solve()
    assert all(r.prior_status == 0 for r in reps)
    nb, priors = solver.slide(poses, reps, a, bb)
    # move the next window's estimates off the linearization point a little
    rng = np.random.default_rng(8)
    nb.poses[:, 4:] += 0.02 * rng.normal(size=(len(nb.poses), 3))
    return nb, priors


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_marginal_prior_windows_match_the_oracle(chained, precision):
    """Windows whose prior is the previous elimination's (Priors::update,
    src/marginalization.rs:157-231) against the oracle's window solve with the
    same prior: LM result, separator and the next elimination."""
    nb, priors = chained
    solver = pg.WindowSolver(nb, removed=10, precision=precision)
    solver.set_priors(priors)
    poses, reps, a, bb = solver.solve()
    rng = np.random.default_rng(5)
    for w in range(nb.windows):
        x, pr, ij, z = nb.window(w)
        ref = oracle.window_solve(x, pr, ij, z, removed=10, marginal=priors[w], **OPTS)
        rep = reps[w]
        assert ref["code"] == rep.status or (ref["code"] in (9, 10) and rep.status in (9, 10)), (w, ref["code"])
        rcost = ref["stats"].cost
        assert abs(rep.final_cost - rcost) <= 1e-6 * max(rcost, 1e-12), (w, rep.final_cost, rcost)
        if precision == "f64":
            assert rep.iterations == ref["stats"].accepted_steps
        p0, p1 = nb.pose_offset[w], nb.pose_offset[w + 1]
        assert np.allclose(poses[p0:p1], ref["poses"], atol=1e-6 if precision == "f64" else 1e-5)
        s0, s1 = solver.separator_offset[w], solver.separator_offset[w + 1]
        assert list(solver.separators[s0:s1]) == list(ref["separator"])
        assert rep.prior_status == 0 and rep.eliminated_rank == ref["rank"]
        A, bvec, c = solver.prior(w, rep, a, bb)
        for _ in range(3):
            d = rng.normal(size=A.shape[1]) * 0.1
            e = _prior_objective(A, bvec, c, d)
            r = _prior_objective(ref["prior_a"], ref["prior_b"], ref["prior_constant"], d)
            tol = 1e-6 if precision == "f64" else 1e-4
            assert abs(e - r) <= tol * max(abs(r), 1.0), (w, e, r)


def test_set_priors_rejects_bad_shapes_and_keeps_the_old_priors(small_batch):
    import fagra_b200 as fg
    b = small_batch
    solver = pg.WindowSolver(b, removed=10)
    first = solver.solve()
    bad = [(np.eye(6), np.zeros(6), b.prior[w][None, :]) for w in range(b.windows)]
    bad[1] = (np.zeros((6, 6 * 65)), np.zeros(6), np.tile(b.prior[1], (65, 1)))
    with pytest.raises(fg.DimensionMismatch):
        solver.set_priors(bad)
    bad[1] = (np.full((6, 6), np.nan), np.zeros(6), b.prior[1][None, :])
    with pytest.raises(fg.InvalidEvaluation):
        solver.set_priors(bad)
    second = solver.solve()
    assert np.array_equal(first[0], second[0])
