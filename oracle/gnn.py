"""ORACLE — test infrastructure only.

f64 numpy restatement of the learned block preconditioner of the device Schur
backend (fagra_b200/csrc/gnn.cu). fagra has no learned preconditioner: its
Schur backend preconditions the reduced camera system with the retained
block-Jacobi factors (src/schur.rs:658-682, src/linear_model/block_factors.rs:
113-138), and this network only reshapes those blocks. Nothing here is pinned
by a reference test; the backward pass is pinned by central finite differences
(tests/test_oracle_gnn.py) and the device kernels are checked against this
module (tests/test_gpu_gnn.py).

Inputs of one system, all in the whitened coordinates of block-Jacobi
(x = L_c^-T x_hat per camera, L_c L_c^T = B_c + lambda I):
* node features X0 (C x 64): the 45 lower-triangle entries (column-major
  order) of P_c = L_c^-1 U_c L_c^-T with U_c = sum_e E_e C_p^-1 E_e^T over the
  camera's edges, then log1p(degree)/4, log1p(coupling), log10(lambda)/12,
  trace(P_c)/cw and a constant 1;
* a row-normalized covisibility matrix A (C x C): a_ij = s_ij / sum_k s_ik with
  s_ij = sqrt(sum over shared points p of <K_ip, K_jp>_F) and
  K_e = G_e^T G_e, G_e = L_c^-1 E_e L_p^-T (so <K_ip, K_jp> = ||G_ip G_jp^T||_F^2);
* probes X (K x C x cw) and Y = S_hat X with S_hat = L^-1 S L^-T.

Network: h0 = relu(X0 W_in + b_in); three layers
h_l = h_{l-1} + relu([h_{l-1}, A h_{l-1}] W_l + b_l); O = h_3 W_out + b_out.
Head: A_c = I + 0.1 tril(O_c) (first cw(cw+1)/2 outputs, column-major lower),
M_hat_c = A_c A_c^T + 1e-3 I, so M = L_c^-T M_hat_c L_c^-1 is SPD and equals
block-Jacobi (up to the factor 1.001) when O = 0.
Loss: mean over probes and included coordinates of ||x - M_hat y||^2.
"""
from __future__ import annotations

import numpy as np

FEATURES = 64
HIDDEN = 64
LAYERS = 3
OUT_SCALE = 0.1
EPSILON = 1e-3


def layout():
    """[(name, shape)] in the flat parameter order the device uses."""
    out = [("W_in", (FEATURES, HIDDEN)), ("b_in", (HIDDEN,))]
    for l in range(1, LAYERS + 1):
        out += [(f"W_{l}", (2 * HIDDEN, HIDDEN)), (f"b_{l}", (HIDDEN,))]
    out += [("W_out", (HIDDEN, HIDDEN)), ("b_out", (HIDDEN,))]
    return out


def parameter_count():
    return sum(int(np.prod(s)) for _, s in layout())


def unpack(flat):
    p, o = {}, 0
    for name, shape in layout():
        n = int(np.prod(shape))
        p[name] = np.asarray(flat[o:o + n], np.float64).reshape(shape)
        o += n
    return p


def pack(p):
    return np.concatenate([np.asarray(p[name], np.float64).ravel() for name, _ in layout()])


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) and back, as the tensor-core
    operands are rounded."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _relu(x):
    return np.maximum(x, 0.0)


def forward(flat, X0, A, rounded=False):
    """Returns (O, cache). With rounded=True every GEMM operand is rounded to
    bfloat16 as on the device (accumulation stays f64 here)."""
    r = bf16 if rounded else (lambda v: np.asarray(v, np.float64))
    p = unpack(flat)
    Z0 = r(X0) @ r(p["W_in"]) + p["b_in"]
    H = _relu(Z0)
    cache = dict(X0=X0, Z=[Z0], HA=[])
    for l in range(1, LAYERS + 1):
        Ag = r(A) @ r(H)
        HA = np.concatenate([H, Ag], axis=1)
        Z = r(HA) @ r(p[f"W_{l}"]) + p[f"b_{l}"]
        cache["HA"].append(HA)
        cache["Z"].append(Z)
        H = H + _relu(Z)
    cache["H3"] = H
    O = r(H) @ r(p["W_out"]) + p["b_out"]
    return O, cache


def _lower_index(cw):
    return [(rr, c) for c in range(cw) for rr in range(c, cw)]


def head_matrices(O, cw):
    C = O.shape[0]
    T = np.zeros((C, cw, cw))
    for k, (rr, c) in enumerate(_lower_index(cw)):
        T[:, rr, c] = OUT_SCALE * O[:, k]
    A = np.eye(cw)[None] + T
    M = A @ A.transpose(0, 2, 1) + EPSILON * np.eye(cw)[None]
    return A, M


def head_loss(O, X, Y, mask, cw):
    """Loss and dL/dO for probes X, Y of shape (K, C, cw)."""
    K = X.shape[0]
    A, M = head_matrices(O, cw)
    m = mask.astype(np.float64)
    n = max(m.sum() * cw, 1.0)
    R = X - np.einsum("irc,kic->kir", M, Y)
    loss = float(np.sum(m[None, :, None] * R * R) / (K * n))
    G = -(2.0 / (K * n)) * np.einsum("kir,kic->irc", R, Y) * m[:, None, None]
    dA = (G + G.transpose(0, 2, 1)) @ A
    dO = np.zeros_like(O)
    for k, (rr, c) in enumerate(_lower_index(cw)):
        dO[:, k] = OUT_SCALE * dA[:, rr, c]
    return loss, dO


def loss_and_gradient(flat, X0, A, X, Y, mask, cw, rounded=False):
    r = bf16 if rounded else (lambda v: np.asarray(v, np.float64))
    p = unpack(flat)
    O, cache = forward(flat, X0, A, rounded)
    loss, dO = head_loss(O, X, Y, mask, cw)
    g = {}
    H3 = cache["H3"]
    g["W_out"] = r(H3).T @ r(dO)
    g["b_out"] = dO.sum(0)
    dH = r(dO) @ r(p["W_out"]).T
    for l in range(LAYERS, 0, -1):
        Z, HA = cache["Z"][l], cache["HA"][l - 1]
        dZ = dH * (Z > 0)
        g[f"W_{l}"] = r(HA).T @ r(dZ)
        g[f"b_{l}"] = dZ.sum(0)
        dHA = r(dZ) @ r(p[f"W_{l}"]).T
        dH = dH + dHA[:, :HIDDEN] + r(A).T @ r(dHA[:, HIDDEN:])
    dZ0 = dH * (cache["Z"][0] > 0)
    g["W_in"] = r(X0).T @ r(dZ0)
    g["b_in"] = dZ0.sum(0)
    return loss, pack(g), O


def preconditioner_blocks(O, Lc, cw):
    """Explicit M_c = L_c^-T M_hat_c L_c^-1 from the network output and the
    block-Jacobi factors Lc (C x cw x cw lower)."""
    _, M = head_matrices(O, cw)
    out = np.zeros_like(M)
    for i in range(O.shape[0]):
        Li = np.linalg.inv(Lc[i])
        out[i] = Li.T @ M[i] @ Li
    return out


def system_features(cam_gram, pt_gram, edges, cross, cam_observed, pt_observed, lam):
    """Node features and normalized covisibility of one scaled Schur system.
    cam_gram (C,cw,cw), pt_gram (P,pw,pw) full symmetric Gram blocks of the
    column-scaled Jacobian; edges (E,2) = (camera, point); cross (E,cw,pw);
    returns (X0, A, Lc)."""
    C, cw = cam_gram.shape[0], cam_gram.shape[1]
    pw = pt_gram.shape[1] if len(pt_gram.shape) == 3 else 0
    Lc = np.zeros((C, cw, cw))
    for i in range(C):
        Lc[i] = np.linalg.cholesky(cam_gram[i] + lam * np.eye(cw)) if cam_observed[i] else np.sqrt(lam) * np.eye(cw)
    Lp = np.zeros((pt_gram.shape[0], pw, pw))
    for p in range(pt_gram.shape[0]):
        Lp[p] = np.linalg.cholesky(pt_gram[p] + lam * np.eye(pw)) if pt_observed[p] else np.sqrt(lam) * np.eye(pw)
    U = np.zeros((C, cw, cw))
    Kmat = np.zeros((len(edges), pw, pw))
    for e, (c, p) in enumerate(edges):
        E = cross[e]
        Cinv = np.linalg.inv(Lp[p] @ Lp[p].T)
        U[c] += E @ Cinv @ E.T
        Eb = np.linalg.solve(Lc[c], E)
        Lpi = np.linalg.inv(Lp[p])
        Kmat[e] = Lpi @ (Eb.T @ Eb) @ Lpi.T
    W = np.zeros((C, C))
    by_point = {}
    for e, (c, p) in enumerate(edges):
        by_point.setdefault(int(p), []).append(e)
    for es in by_point.values():
        for a in range(len(es)):
            for b in range(a + 1, len(es)):
                ci, cj = edges[es[a]][0], edges[es[b]][0]
                if ci == cj or not cam_observed[ci] or not cam_observed[cj]:
                    continue
                w = float(np.sum(Kmat[es[a]] * Kmat[es[b]]))
                W[ci, cj] += w
                W[cj, ci] += w
    S = np.sqrt(np.maximum(W, 0.0))
    rows = S.sum(1)
    A = np.where(rows[:, None] > 0, S / np.where(rows > 0, rows, 1.0)[:, None], 0.0)
    X0 = np.zeros((C, FEATURES))
    for i in range(C):
        if not cam_observed[i]:
            X0[i, 49] = 1.0
            continue
        Li = np.linalg.inv(Lc[i])
        P = Li @ U[i] @ Li.T
        for k, (rr, c) in enumerate(_lower_index(cw)):
            X0[i, k] = P[rr, c]
        X0[i, 45] = np.log1p(np.count_nonzero(S[i] > 0)) / 4.0
        X0[i, 46] = np.log1p(rows[i])
        X0[i, 47] = np.log10(max(lam, 1e-12)) / 12.0
        X0[i, 48] = np.trace(P) / cw
        X0[i, 49] = 1.0
    return X0, A, Lc
