"""Scenarios ported from fagra's own tests, written once and run against both
the oracle (CPU) and the device backend (GPU) through the same calls.

Every scenario cites the fagra test it restates.
"""
from __future__ import annotations

import numpy as np


def twelve_column_schur_emissions():
    """src/schur.rs:690-728: five camera-point observations emitted in reverse
    block order (including a repeated pair) plus two unary rows; Schur(6, 2, 2)
    on 12 coordinates. Returns (emissions, J, r)."""
    observations = [(0, 6), (2, 6), (0, 8), (2, 8), (0, 6)]
    J = np.zeros((12, 12))
    r = np.zeros(12)
    emissions = []
    for i, (cam, point) in enumerate(observations):
        a = np.array([[0.01, 2.0], [-0.03, 1.0 + i]])
        b = np.array([[10.0, -0.3], [20.0 + i, 1.0]])
        res = np.array([i - 2.0, 1.0])
        emissions.append((res, [(point, b), (cam, a)]))
        J[2 * i:2 * i + 2, cam:cam + 2] = a
        J[2 * i:2 * i + 2, point:point + 2] = b
        r[2 * i:2 * i + 2] = res
    for i, col in enumerate([0, 8]):
        a = np.array([[0.5, -1.0]])
        emissions.append((np.array([0.7]), [(col, a)]))
        J[10 + i, col:col + 2] = a
        r[10 + i] = 0.7
    return emissions, J, r


def augmented_solution(J, r, scales, lam):
    """Minimum-norm solution of ||J d + r||^2 + lam ||D d||^2 by SVD."""
    n = J.shape[1]
    A = np.vstack([J, np.sqrt(lam) * np.diag(scales)])
    rhs = np.concatenate([-r, np.zeros(n)])
    return np.linalg.lstsq(A, rhs, rcond=1e-13)[0]


def scalar_curve_link_problem():
    """tests/levenberg_marquardt.rs:661-703: two scalars a, b (a retained,
    b eliminated by Schur(1, 1, 1)) with Square curves toward 1 and 2 and a
    0.1-weighted link b - a - 1, started from the reset solution (0.5, 3).
    Returns (x0, cost(x), linearize(x, emit))."""
    targets = (1.0, 2.0)

    def residuals(x):
        a, b = x
        return [(a * a - targets[0] ** 2, [(0, np.array([[2 * a]]))]),
                (b * b - targets[1] ** 2, [(1, np.array([[2 * b]]))]),
                (0.1 * (b - a - 1.0), [(0, np.array([[-0.1]])), (1, np.array([[0.1]]))])]

    def cost(x):
        return sum(0.5 * r * r for r, _ in residuals(x))

    def linearize(x, emit):
        for r, blocks in residuals(x):
            emit(np.array([r]), blocks)

    return np.array([0.5, 3.0]), cost, linearize


def bal_known_answer():
    """tests/bal.rs:104-112: camera [0,0,0, 0,0,0, 100, 0.1, 0.01] and point
    (1, 2, -2) project to x = 50 (1 + 0.1 * 1.25 + 0.01 * 1.25^2), y = 2x."""
    cam = np.array([0, 0, 0, 0, 0, 0, 100.0, 0.1, 0.01])
    X = np.array([1.0, 2.0, -2.0])
    x = 50.0 * (1.0 + 0.1 * 1.25 + 0.01 * 1.25 * 1.25)
    return cam, X, np.array([x, 2 * x])


BAL_JACOBIAN_ROTATIONS = [np.zeros(3), np.array([1e-10, -2e-10, 3e-10]), np.array([0.4, -0.2, 0.1]),
                          np.array([3.1, 0.1, -0.1])]  # tests/bal.rs:65-70


def bal_jacobian_case(rotation):
    """tests/bal.rs:71-76 camera/point for one rotation."""
    cam = np.array([rotation[0], rotation[1], rotation[2], 0.2, -0.1, 0.3, 500.0, 0.01, -0.001])
    X = np.array([0.8, -0.4, -5.0])
    return cam, X


def twelve_point_bal():
    """tests/bal.rs:7-41: one identity camera (f = 1), 12 points on a grid at
    depth 3..4.1, observed exactly, initial points offset by (0.02, -0.03, 0.01)."""
    from oracle import project
    cam = np.array([0, 0, 0, 0, 0, 0, 1.0, 0, 0])
    truth, init, pix = [], [], []
    for i in range(12):
        t = np.array([(i % 4) * 0.2 - 0.3, (i // 4) * 0.3 - 0.2, -3.0 - i * 0.1])
        p, st = project(cam, t)
        assert st == 0
        truth.append(t)
        init.append(t + np.array([0.02, -0.03, 0.01]))
        pix.append(p)
    return cam[None, :], np.array(init), np.zeros(12, np.uint32), np.arange(12, dtype=np.uint32), np.array(pix)


# ---------------------------------------------------------------- LSMR
def lsmr_shared_columns():
    """src/lsmr.rs:619-641: a 4x3 Jacobian whose rows 0-1 and 2-3 are emitted
    as two 2-row residuals on the same three columns."""
    J = np.array([[0.001, 2.0, 3.0], [0.002, -1.0, 4.0], [-0.001, 3.0, -2.0], [0.003, 1.0, 2.0]])
    return J, [0, 2]


def lsmr_product_vectors(n, m):
    """src/lsmr.rs:642-643: x(i,k) = i + k - 1.25 and y(i,k) = 2i + k - 2.5."""
    x = np.array([[i + k - 1.25 for k in range(2)] for i in range(n)])
    y = np.array([[2 * i + k - 2.5 for k in range(2)] for i in range(m)])
    return x, y


def damped_dense(J, scales, lam, scaled):
    """Dense Damped operator (src/lsmr.rs:128-224): [J D^-1; sqrt(lam) I] when
    scaled, else [J; sqrt(lam) D]."""
    n = J.shape[1]
    top = J / scales[None, :] if scaled else J
    diag = np.full(n, np.sqrt(lam)) if scaled else np.sqrt(lam) * scales
    return np.vstack([top, np.diag(diag)])


def lsmr_mixed_scale():
    """src/lsmr.rs:783-788: columns spanning eight orders of magnitude and an
    unused fourth column."""
    J = np.array([[1e-4, 2.0, 0.0, 0.0], [2e-4, -1.0, 3e4, 0.0], [0.0, 1.0, -1e4, 0.0]])
    return J, np.array([1.0, -2.0, 3.0])


def lsmr_retry_system():
    """src/lsmr.rs:860-863: a rank-deficient 3x3 system (third column zero)."""
    J = np.array([[1.0, 2.0, 0.0], [3.0, -1.0, 0.0], [0.0, 1.0, 0.0]])
    return J, np.array([-3.0, 2.0, 1.0])


def lsmr_coupling_gap():
    """src/lsmr.rs:907-910: a 4x5 Jacobian emitted as blocks (3, cols 3..5) and
    (0, cols 0..2); column 2 is never touched."""
    J = np.array([[1.0, 2.0, 0.0, 4.0, 2.0], [3.0, 1.0, 0.0, 2.0, 1.0], [2.0, 1.0, 0.0, 1.0, 3.0],
                  [1.0, 1.0, 0.0, 3.0, 2.0]])
    return J, np.array([1.0, -2.0, 3.0, -1.0])


def lsmr_rectangular():
    """src/lsmr.rs:1006-1041: a 3-row emission with a strided 3x2 view at
    column 2 and a 3x2 block at column 0, then a 2-row emission at column 0.
    Returns (emissions, dense J, r)."""
    storage = np.arange(20, dtype=np.float64).reshape(5, 4)
    ja = storage[1:4, 1:3]  # noncontiguous view
    jb = np.array([[1.0, 0.0], [0.0, 2.0], [3.0, -1.0]])
    jc = np.array([[2.0, 0.0], [0.0, 1.0]])
    emissions = [(np.array([1.0, -2.0, 3.0]), [(2, ja), (0, jb)]), (np.array([-4.0, 5.0]), [(0, jc)])]
    J = np.array([[1.0, 0.0, 5.0, 6.0], [0.0, 2.0, 9.0, 10.0], [3.0, -1.0, 13.0, 14.0], [2.0, 0.0, 0.0, 0.0],
                  [0.0, 1.0, 0.0, 0.0]])
    r = np.array([1.0, -2.0, 3.0, -4.0, 5.0])
    return emissions, J, r
