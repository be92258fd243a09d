"""Selected covariance through the sparse backends: Schur and Lsmr delegate to
LinearizedModel::covariance (src/schur.rs:548-556, src/lsmr.rs:598-604,
src/linear_model.rs:122-167), checked against fagra's own covariance test
(tests/levenberg_marquardt.rs:705-766) and against the oracle on bal16."""
import numpy as np
import pytest

import fagra_b200 as fg
import oracle
from fagra_b200 import synthetic

pytestmark = pytest.mark.gpu


def _covariance_problem():
    # tests/levenberg_marquardt.rs:705-766: Square curves toward 1 and 2 from (0.5, 1) plus a 0.1 link
    def residuals(x):
        a, b = x
        return [(a * a - 1.0, [(0, np.array([[2 * a]]))]),
                (b * b - 4.0, [(1, np.array([[2 * b]]))]),
                (0.1 * (b - a - 1.0), [(0, np.array([[-0.1]])), (1, np.array([[0.1]]))])]

    def cost(x):
        return sum(0.5 * r * r for r, _ in residuals(x))

    def linearize(x, emit):
        for r, blocks in residuals(x):
            emit(np.array([r]), blocks)

    return fg.CallbackProblem(np.array([0.5, 1.0]), cost, linearize)


@pytest.mark.parametrize("make,method", [(lambda: fg.Schur(1, 1, 1), fg.LevenbergMarquardt),
                                         (lambda: fg.Schur(1, 1, 1, precision="f32"), fg.LevenbergMarquardt),
                                         (fg.Lsmr, fg.GaussNewton), (fg.Lsmr, fg.LevenbergMarquardt)],
                         ids=["schur-lm", "schur-f32-lm", "lsmr-gn", "lsmr-lm"])
def test_scoped_covariance_matches_the_reference_values(make, method):
    solver = method(make())
    for sample in range(4):
        cols = [1, 0] if sample % 2 == 0 else [1]
        _, cov = solver.solve_batch_with_covariance(_covariance_problem(), columns=cols)
        tol = 1e-8 if "f32" not in repr(getattr(solver.backend(), "precision", "")) else 1e-6
        assert abs(cov[0, 0] - 4.01 / 64.2) < tol
        if len(cols) == 2:
            assert abs(cov[0, 1] - 0.01 / 64.2) < tol
            assert abs(cov[1, 1] - 16.01 / 64.2) < tol


def _random_bipartite(rng, cams=4, pts=10, cw=2, pw=1):
    """Emissions of a full-rank bipartite problem: every point seen by three
    cameras, each observation a (camera, point) Jacobian pair plus a camera prior row."""
    em = []
    for p in range(pts):
        for c in rng.choice(cams, size=3, replace=False):
            em.append((rng.normal(size=2), [(cw * c, rng.normal(size=(2, cw))),
                                             (cw * cams + pw * p, rng.normal(size=(2, pw)))]))
    for c in range(cams):
        em.append((rng.normal(size=cw), [(cw * c, np.eye(cw))]))
    return em, cw * cams + pw * pts


@pytest.mark.parametrize("make", [lambda: fg.Schur(8, 2, 1), fg.Lsmr], ids=["schur", "lsmr"])
def test_sparse_backend_covariance_matches_the_oracle(make):
    rng = np.random.default_rng(8)
    em, dim = _random_bipartite(rng)
    o = oracle.Schur(8, 2, 1)
    o.prepare(dim)
    o.clear()
    b = make()
    b.prepare(dim)
    b.clear()
    for r, blocks in em:
        assert o.accumulate(r, blocks) == 0
        b.accumulate(r, blocks)
    cols = [9, 0, 3, 12, 1]
    st, ref = o.covariance(cols)
    assert st == 0
    got = b.covariance(cols)
    assert np.max(np.abs(got - ref)) <= 1e-10 * np.max(np.abs(ref))
    with pytest.raises(fg.DuplicateCovarianceBlock):
        b.covariance([3, 3])
    with pytest.raises(fg.InvalidRankTolerance):
        b.covariance([3], 1.0)


def test_schur_covariance_of_a_bal_model_screens_the_gauge_like_the_oracle():
    # bundle adjustment without priors has a similarity gauge: the information
    # matrix is singular and both the oracle and the device refuse it
    d = synthetic.generate("bal16", points=120)
    o = oracle.Schur(9 * d.num_cameras, 9, 3)
    ob = oracle.Bal.from_data(d)
    o.prepare(ob.dimension())
    assert ob.linearize(o) == 0
    b = fg.Schur(9 * d.num_cameras, 9, 3)
    p = fg.BalProblem.from_data(d)
    b.prepare(p.dimension())
    p.linearize(b)
    cols = list(range(9, 18))
    st, ref = o.covariance(cols)
    if st == 0:
        got = b.covariance(cols)
        assert np.max(np.abs(got - ref)) <= 1e-8 * np.max(np.abs(ref))
    else:
        assert st == 2  # SingularInformation
        with pytest.raises(fg.SingularInformation):
            b.covariance(cols)
