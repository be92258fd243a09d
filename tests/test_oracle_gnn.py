"""The learned-preconditioner oracle (oracle/gnn.py) against central finite
differences, and its head against the block-Jacobi identity it starts from."""
import numpy as np
import pytest

from oracle import gnn


def _system(seed=3, C=12, cw=9, K=4):
    rng = np.random.default_rng(seed)
    X0 = rng.normal(size=(C, gnn.FEATURES)) * 0.5
    W = np.abs(rng.normal(size=(C, C)))
    W = W + W.T
    np.fill_diagonal(W, 0.0)
    W[W < 0.6] = 0.0
    rows = W.sum(1)
    A = np.where(rows[:, None] > 0, W / np.where(rows > 0, rows, 1)[:, None], 0.0)
    X = rng.normal(size=(K, C, cw))
    Y = rng.normal(size=(K, C, cw))
    mask = np.ones(C, bool)
    mask[1] = False
    return X0, A, X, Y, mask


def _params(seed=5):
    rng = np.random.default_rng(seed)
    return rng.normal(size=gnn.parameter_count()) * 0.2


def test_parameter_layout():
    assert gnn.parameter_count() == 64 * 64 + 64 + 3 * (128 * 64 + 64) + 64 * 64 + 64
    flat = _params()
    assert np.array_equal(gnn.pack(gnn.unpack(flat)), flat)


def test_gradient_matches_central_differences():
    X0, A, X, Y, mask = _system()
    flat = _params()
    loss, g, _ = gnn.loss_and_gradient(flat, X0, A, X, Y, mask, 9)
    rng = np.random.default_rng(7)
    names = [n for n, _ in gnn.layout()]
    offsets = np.cumsum([0] + [int(np.prod(s)) for _, s in gnn.layout()])
    h = 1e-6
    for k, name in enumerate(names):
        for idx in rng.choice(np.arange(offsets[k], offsets[k + 1]), size=4, replace=False):
            fp, fm = flat.copy(), flat.copy()
            fp[idx] += h
            fm[idx] -= h
            lp = gnn.loss_and_gradient(fp, X0, A, X, Y, mask, 9)[0]
            lm = gnn.loss_and_gradient(fm, X0, A, X, Y, mask, 9)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7, (name, idx, fd, g[idx])


def test_directional_derivative_and_rounded_gradient():
    X0, A, X, Y, mask = _system(seed=8, C=20)
    flat = _params(9)
    loss, g, _ = gnn.loss_and_gradient(flat, X0, A, X, Y, mask, 9)
    d = np.random.default_rng(1).normal(size=flat.shape)
    h = 1e-6
    fd = (gnn.loss_and_gradient(flat + h * d, X0, A, X, Y, mask, 9)[0]
          - gnn.loss_and_gradient(flat - h * d, X0, A, X, Y, mask, 9)[0]) / (2 * h)
    assert abs(fd - g @ d) <= 1e-6 * abs(fd)
    # bfloat16 operands perturb the gradient by about the bf16 unit roundoff
    _, gr, _ = gnn.loss_and_gradient(flat, X0, A, X, Y, mask, 9, rounded=True)
    assert np.linalg.norm(gr - g) <= 3e-2 * np.linalg.norm(g)


def test_zero_output_is_block_jacobi():
    C, cw = 5, 9
    rng = np.random.default_rng(2)
    L = np.tril(rng.normal(size=(C, cw, cw))) + 3 * np.eye(cw)[None]
    M = gnn.preconditioner_blocks(np.zeros((C, 64)), L, cw)
    for i in range(C):
        bj = np.linalg.inv(L[i] @ L[i].T)
        np.testing.assert_allclose(M[i], (1 + gnn.EPSILON) * bj, rtol=1e-10, atol=1e-12)


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3], np.float32)
    r = gnn.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 4 * 2 ** -8 and r[3] == -2.5
    assert abs(r[4] - 1e-3) <= 2 ** -9 * 1e-3


@pytest.mark.parametrize("lam", [1e-4, 1.0])
def test_features_of_a_two_camera_system(lam):
    # two cameras sharing one point: the covisibility is symmetric and each row sums to one
    rng = np.random.default_rng(4)
    cw, pw = 9, 3
    E = rng.normal(size=(2, cw, pw))
    cam_gram = np.stack([e @ e.T + np.eye(cw) for e in E])
    pt_gram = (E[0].T @ E[0] + E[1].T @ E[1])[None] + np.eye(pw)[None]
    X0, A, Lc = gnn.system_features(cam_gram, pt_gram, np.array([[0, 0], [1, 0]]), E, [1, 1], [1], lam)
    assert A[0, 1] == 1.0 and A[1, 0] == 1.0 and A[0, 0] == 0.0
    assert X0[0, 49] == 1.0 and abs(X0[0, 45] - np.log1p(1) / 4) < 1e-15
    Li = np.linalg.inv(Lc[0])
    Cinv = np.linalg.inv(pt_gram[0] + lam * np.eye(pw))
    P = Li @ E[0] @ Cinv @ E[0].T @ Li.T
    assert abs(X0[0, 0] - P[0, 0]) < 1e-12 and abs(X0[0, 1] - P[1, 0]) < 1e-12
