"""ORACLE — test infrastructure only.

ctypes face of oracle/liboracle.so, the sequential f64 CPU restatement of
fagra's hot path (see oracle.cpp for the per-function citations). Only the
test suite, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
size_t = C.c_size_t
ptrdiff_t = C.c_ssize_t
dptr = C.POINTER(C.c_double)


def _load():
    if not LIB.exists():
        from .build import build
        build()
    return C.CDLL(str(LIB))


lib = _load()


class Diag(C.Structure):
    _fields_ = [("termination", C.c_int), ("iterations", size_t), ("damping", C.c_double),
                ("estimated", C.c_double), ("reduced", C.c_double), ("scaled", C.c_double),
                ("original", C.c_double), ("has_estimated", C.c_int), ("has_reduced", C.c_int),
                ("has_scaled", C.c_int), ("has_original", C.c_int)]


class OptOpts(C.Structure):
    _fields_ = [("max_iterations", size_t), ("gradient_tolerance", C.c_double), ("step_tolerance", C.c_double),
                ("cost_tolerance", C.c_double)]


class LmOpts(C.Structure):
    _fields_ = [("initial_damping", C.c_double), ("min_damping", C.c_double), ("max_damping", C.c_double),
                ("min_column_norm", C.c_double), ("acceptance_threshold", C.c_double), ("max_trials", size_t)]


class Report(C.Structure):
    _fields_ = [("iterations", size_t), ("initial_cost", C.c_double), ("final_cost", C.c_double),
                ("termination", C.c_int)]


class LmStats(C.Structure):
    _fields_ = [("linearizations", size_t), ("attempts", size_t), ("rejected_steps", size_t),
                ("accepted_steps", size_t), ("cost_evaluations", size_t), ("damping", C.c_double),
                ("cost", C.c_double), ("gradient_norm", C.c_double), ("step_norm", C.c_double),
                ("has_cost", C.c_int), ("has_gradient_norm", C.c_int), ("has_step_norm", C.c_int),
                ("last_rejection", C.c_int), ("linear_solves", size_t), ("linear_iterations", size_t)]


class LsmrDiag(C.Structure):
    _fields_ = [("termination", C.c_int), ("iterations", size_t), ("finite_step", C.c_int),
                ("estimated_absolute", C.c_double), ("estimated_relative", C.c_double),
                ("original_absolute", C.c_double), ("original_relative", C.c_double),
                ("scaled_absolute", C.c_double), ("scaled_relative", C.c_double),
                ("min_scale", C.c_double), ("max_scale", C.c_double), ("damping", C.c_double),
                ("block_fallbacks", size_t), ("has_estimated", C.c_int), ("has_original", C.c_int),
                ("has_scaled", C.c_int), ("has_scales", C.c_int), ("has_damping", C.c_int)]


ACCEPT = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(LmStats))
COST = C.CFUNCTYPE(C.c_int, C.c_void_p, dptr, dptr)
LIN = C.CFUNCTYPE(C.c_int, C.c_void_p, dptr, C.c_void_p)

_sig = {
    "or_bal_project": (C.c_int, [dptr, dptr, dptr]),
    "or_bal_jacobians": (None, [dptr, dptr, dptr, dptr]),
    "or_rotation": (None, [dptr, dptr]),
    "or_schur_create": (C.c_void_p, [size_t, size_t, size_t]),
    "or_schur_destroy": (None, [C.c_void_p]),
    "or_schur_set_limits": (None, [C.c_void_p, size_t, C.c_double]),
    "or_schur_prepare": (C.c_int, [C.c_void_p, size_t]),
    "or_schur_clear": (None, [C.c_void_p]),
    "or_schur_accumulate": (C.c_int, [C.c_void_p, size_t, dptr, size_t, C.POINTER(size_t), C.POINTER(size_t),
                                      C.POINTER(dptr), C.POINTER(ptrdiff_t), C.POINTER(ptrdiff_t)]),
    "or_schur_gradient_norm": (C.c_int, [C.c_void_p, dptr]),
    "or_schur_prepare_damping": (C.c_int, [C.c_void_p, C.c_double]),
    "or_schur_solve_damped": (C.c_int, [C.c_void_p, C.c_double, dptr, dptr]),
    "or_schur_solve": (C.c_int, [C.c_void_p, dptr]),
    "or_schur_work": (None, [C.c_void_p, C.POINTER(size_t), C.POINTER(size_t)]),
    "or_schur_diagnostics": (None, [C.c_void_p, C.POINTER(Diag)]),
    "or_schur_sizes": (None, [C.c_void_p] + [C.POINTER(size_t)] * 7),
    "or_schur_export": (None, [C.c_void_p] + [C.POINTER(size_t)] * 4 + [dptr] * 6),
    "or_schur_reduced_apply": (None, [C.c_void_p, C.c_double, dptr, dptr]),
    "or_schur_reduced_rhs": (None, [C.c_void_p, dptr]),
    "or_model_create": (C.c_void_p, [size_t]),
    "or_model_destroy": (None, [C.c_void_p]),
    "or_model_accumulate": (C.c_int, [C.c_void_p, size_t, dptr, size_t, C.POINTER(size_t), C.POINTER(size_t),
                                      C.POINTER(dptr), C.POINTER(ptrdiff_t), C.POINTER(ptrdiff_t)]),
    "or_model_prepare_scales": (C.c_int, [C.c_void_p, C.c_double]),
    "or_model_verify": (None, [C.c_void_p, dptr, C.c_double, dptr, dptr, dptr]),
    "or_model_state": (None, [C.c_void_p, dptr, dptr]),
    "or_blockfactors_run": (C.c_int, [size_t, size_t, size_t, C.POINTER(size_t), dptr, size_t, dptr, dptr, size_t,
                                      C.POINTER(size_t)]),
    "or_bal_create": (C.c_void_p, [size_t, size_t, size_t, dptr, dptr, C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_uint32), dptr]),
    "or_bal_destroy": (None, [C.c_void_p]),
    "or_bal_cost": (C.c_int, [C.c_void_p, dptr]),
    "or_bal_get": (None, [C.c_void_p, dptr, dptr]),
    "or_bal_order": (None, [C.c_void_p, C.POINTER(size_t)]),
    "or_bal_linearize": (C.c_int, [C.c_void_p, C.c_void_p]),
    "or_lm_bal": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(OptOpts), C.POINTER(LmOpts), C.POINTER(Report),
                            C.POINTER(LmStats), ACCEPT, C.c_void_p]),
    "or_lm_bal_to_cost": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(OptOpts), C.POINTER(LmOpts), C.c_double,
                                    C.POINTER(Report), C.POINTER(LmStats)]),
    "or_gn_bal": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(OptOpts), C.POINTER(Report)]),
    "or_cbproblem_create": (C.c_void_p, [size_t, dptr, COST, LIN, C.c_void_p]),
    "or_cbproblem_destroy": (None, [C.c_void_p]),
    "or_cbproblem_get": (None, [C.c_void_p, dptr]),
    "or_cbproblem_emit": (C.c_int, [C.c_void_p, size_t, dptr, size_t, C.POINTER(size_t), C.POINTER(size_t),
                                    C.POINTER(dptr), C.POINTER(ptrdiff_t), C.POINTER(ptrdiff_t)]),
    "or_lm_cb": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(OptOpts), C.POINTER(LmOpts), C.POINTER(Report),
                           C.POINTER(LmStats)]),
    "or_gn_cb": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(OptOpts), C.POINTER(Report)]),
    "or_lsmr_create": (C.c_void_p, []),
    "or_lsmr_set": (None, [C.c_void_p, size_t, C.c_double, C.c_int, C.c_int]),
    "or_lsmr_diagnostics": (None, [C.c_void_p, C.POINTER(LsmrDiag)]),
    "or_lsmr_damped_products": (None, [C.c_void_p, C.c_double, C.c_int, dptr, dptr, dptr, dptr]),
    "or_lsmr_precond": (None, [C.c_void_p, dptr, dptr, dptr, dptr]),
    "or_lsmr_scales": (None, [C.c_void_p, dptr]),
    "or_dense_normal_create": (C.c_void_p, []),
    "or_dense_schur_create": (C.c_void_p, [size_t, C.POINTER(size_t), size_t]),
    "or_dense_qr_create": (C.c_void_p, [C.c_double]),
    "or_dense_qr_set_tolerance": (None, [C.c_void_p, C.c_double]),
    "or_dense_normal_state": (None, [C.c_void_p, dptr, dptr]),
    "or_dense_normal_information": (C.c_int, [C.c_void_p, C.c_double]),
    "or_backend_covariance": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(size_t), size_t, C.c_double, dptr]),
    "or_eliminate": (C.c_int, [size_t, size_t, dptr, size_t, C.c_double, dptr, dptr, dptr, C.POINTER(size_t),
                               C.POINTER(size_t)]),
    "or_pose_exp": (None, [dptr, dptr]),
    "or_pose_log": (None, [dptr, dptr]),
    "or_pose_compose": (None, [dptr, dptr, dptr]),
    "or_pose_inverse": (None, [dptr, dptr]),
    "or_pose_adjoint": (None, [dptr, dptr]),
    "or_pose_right_jacobian": (None, [dptr, dptr]),
    "or_pose_log_jacobian": (C.c_int, [dptr, dptr]),
    "or_window_solve": (C.c_int, [size_t, dptr, dptr, size_t, C.POINTER(C.c_uint32), dptr, C.POINTER(OptOpts),
                                  C.POINTER(LmOpts), size_t, C.POINTER(Report), C.POINTER(LmStats), dptr, dptr, dptr,
                                  C.POINTER(size_t), C.POINTER(C.c_uint32), C.POINTER(size_t), C.POINTER(size_t)]),
    "or_window_cost": (C.c_int, [size_t, dptr, dptr, size_t, C.POINTER(C.c_uint32), dptr, dptr]),
    "or_window_solve_prior": (C.c_int, [size_t, dptr, size_t, size_t, dptr, dptr, dptr, size_t,
                                        C.POINTER(C.c_uint32), dptr, C.POINTER(OptOpts), C.POINTER(LmOpts), size_t,
                                        C.POINTER(Report), C.POINTER(LmStats), dptr, dptr, dptr, C.POINTER(size_t),
                                        C.POINTER(C.c_uint32), C.POINTER(size_t), C.POINTER(size_t)]),
    "or_window_cost_prior": (C.c_int, [size_t, dptr, size_t, size_t, dptr, dptr, dptr, size_t,
                                       C.POINTER(C.c_uint32), dptr, dptr]),
}
for _n, (_r, _a) in _sig.items():
    _f = getattr(lib, _n)
    _f.restype = _r
    _f.argtypes = _a

TERM = {0: None, 1: "Converged", 2: "IterationLimit", 3: "NotPositiveDefinite", 4: "NonFinite"}


def _dp(a):
    return a.ctypes.data_as(dptr)


def pack_blocks(residual, jacobians):
    r = np.ascontiguousarray(np.asarray(residual, np.float64).reshape(-1))
    blocks = [(int(c), np.asarray(j, np.float64)) for c, j in jacobians]
    nb = len(blocks)
    cols = (size_t * max(nb, 1))(*[c for c, _ in blocks])
    widths = (size_t * max(nb, 1))()
    ptrs = (dptr * max(nb, 1))()
    rs = (ptrdiff_t * max(nb, 1))()
    cs = (ptrdiff_t * max(nb, 1))()
    keep = [r]
    for k, (_, j) in enumerate(blocks):
        j2 = j.reshape(len(r), -1) if j.ndim != 2 else j
        keep.append(j2)
        widths[k] = j2.shape[1]
        ptrs[k] = j2.ctypes.data_as(dptr)
        rs[k] = j2.strides[0] // 8
        cs[k] = j2.strides[1] // 8
    return (len(r), _dp(r), nb, cols, widths, ptrs, rs, cs), keep


def project(cam, X):
    cam = np.ascontiguousarray(cam, np.float64)
    X = np.ascontiguousarray(X, np.float64)
    pix = np.zeros(2)
    st = lib.or_bal_project(_dp(cam), _dp(X), _dp(pix))
    return pix, st


def jacobians(cam, X):
    cam = np.ascontiguousarray(cam, np.float64)
    X = np.ascontiguousarray(X, np.float64)
    jc = np.zeros(18)
    jp = np.zeros(6)
    lib.or_bal_jacobians(_dp(cam), _dp(X), _dp(jc), _dp(jp))
    return jc.reshape(9, 2).T.copy(), jp.reshape(3, 2).T.copy()


class Schur:
    """Oracle Schur backend (src/schur.rs restated)."""

    def __init__(self, retained, cw, pw):
        self.h = lib.or_schur_create(retained, cw, pw)
        self.retained, self.cw, self.pw = retained, cw, pw
        self.max_iterations = 1000
        self.relative_tolerance = max(1e-10, 128 * np.finfo(float).eps)
        self.dim = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_schur_destroy(self.h)
            self.h = None

    def _limits(self):
        lib.or_schur_set_limits(self.h, self.max_iterations, self.relative_tolerance)

    def covariance(self, columns, tol=64 * np.finfo(float).eps):
        """LinearizedModel::covariance of the cached model (src/linear_model.rs:122-167)."""
        cols = np.ascontiguousarray(np.asarray(columns, np.uint64))
        k = len(cols)
        out = np.zeros(max(k * k, 1))
        st = lib.or_backend_covariance(self.h, 0, cols.ctypes.data_as(C.POINTER(size_t)), k, tol, _dp(out))
        return st, out[:k * k].reshape(k, k).T.copy()

    def prepare(self, dim):
        self._limits()
        self.dim = dim
        return lib.or_schur_prepare(self.h, dim)

    def clear(self):
        lib.or_schur_clear(self.h)

    def accumulate(self, residual, jacobians):
        args, keep = pack_blocks(residual, jacobians)
        return lib.or_schur_accumulate(self.h, *args)

    def gradient_norm(self):
        out = C.c_double()
        st = lib.or_schur_gradient_norm(self.h, C.byref(out))
        return st, out.value

    def prepare_damping(self, floor):
        return lib.or_schur_prepare_damping(self.h, floor)

    def solve_damped(self, lam):
        self._limits()
        d = np.zeros(self.dim)
        p = C.c_double()
        st = lib.or_schur_solve_damped(self.h, lam, _dp(d), C.byref(p))
        return st, d, p.value

    def solve(self):
        self._limits()
        d = np.zeros(self.dim)
        st = lib.or_schur_solve(self.h, _dp(d))
        return st, d

    def work(self):
        s, i = size_t(), size_t()
        lib.or_schur_work(self.h, C.byref(s), C.byref(i))
        return s.value, i.value

    def diagnostics(self):
        d = Diag()
        lib.or_schur_diagnostics(self.h, C.byref(d))
        o = lambda f, v: v if f else None  # noqa: E731
        return dict(termination=TERM[d.termination], iterations=d.iterations, damping=d.damping,
                    estimated=o(d.has_estimated, d.estimated), reduced=o(d.has_reduced, d.reduced),
                    scaled=o(d.has_scaled, d.scaled), original=o(d.has_original, d.original))

    def export(self):
        sz = [size_t() for _ in range(7)]
        lib.or_schur_sizes(self.h, *[C.byref(s) for s in sz])
        nb, ne, nv, nvar, ngram, rows, cols = (s.value for s in sz)
        b5 = np.zeros((max(nb, 1), 5), np.uint64)
        e4 = np.zeros((max(ne, 1), 4), np.uint64)
        own = np.zeros(max(cols, 1), np.uint64)
        v3 = np.zeros((max(nvar, 1), 3), np.uint64)
        vals, neg, g, sc = np.zeros(max(nv, 1)), np.zeros(max(rows, 1)), np.zeros(max(cols, 1)), np.zeros(max(cols, 1))
        gram = np.zeros(max(ngram, 1))
        cross = np.zeros(max(ne * self.cw * self.pw, 1))
        sp = C.POINTER(size_t)
        lib.or_schur_export(self.h, b5.ctypes.data_as(sp), e4.ctypes.data_as(sp), own.ctypes.data_as(sp),
                            v3.ctypes.data_as(sp), _dp(vals), _dp(neg), _dp(g), _dp(sc), _dp(gram), _dp(cross))
        return dict(blocks=b5[:nb], edges=e4[:ne], owners=own[:cols], variables=v3[:nvar], values=vals[:nv],
                    negative_residual=neg[:rows], gradient=g[:cols], scales=sc[:cols], gram=gram[:ngram],
                    cross=cross[:ne * self.cw * self.pw], rows=rows, cols=cols)

    def reduced_apply(self, lam, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        lib.or_schur_reduced_apply(self.h, lam, _dp(x), _dp(y))
        return y


class Lsmr(Schur):
    """Oracle LSMR backend (src/lsmr.rs restated; faer's LSMR per Fong & Saunders).

    Shares the generic backend entry points with Schur; the options mirror the
    reference's public fields."""

    def __init__(self):  # noqa: D107 - Schur.__init__ is not called on purpose
        self.h = lib.or_lsmr_create()
        self.max_iterations = 1000
        self.relative_tolerance = max(1e-10, 128 * np.finfo(float).eps)
        self.diagonal_preconditioning = True
        self.block_preconditioning = False
        self.dim = 0
        self.rows = 0

    def _limits(self):
        lib.or_lsmr_set(self.h, self.max_iterations, self.relative_tolerance, int(self.diagonal_preconditioning),
                        int(self.block_preconditioning))

    def prepare(self, dim):
        self.rows = 0
        return super().prepare(dim)

    def clear(self):
        self.rows = 0
        super().clear()

    def accumulate(self, residual, jacobians):
        args, keep = pack_blocks(residual, jacobians)
        st = lib.or_schur_accumulate(self.h, *args)
        if st == 0:
            self.rows += args[0]
        return st

    def prepare_damping(self, floor):
        self._limits()
        return super().prepare_damping(floor)

    def diagnostics(self):
        d = LsmrDiag()
        lib.or_lsmr_diagnostics(self.h, C.byref(d))
        o = lambda f, v: v if f else None  # noqa: E731
        return dict(termination=TERM[d.termination], iterations=d.iterations, finite_step=bool(d.finite_step),
                    estimated_absolute=o(d.has_estimated, d.estimated_absolute),
                    estimated_relative=o(d.has_estimated, d.estimated_relative),
                    original_absolute=o(d.has_original, d.original_absolute),
                    original_relative=o(d.has_original, d.original_relative),
                    scaled_absolute=o(d.has_scaled, d.scaled_absolute),
                    scaled_relative=o(d.has_scaled, d.scaled_relative),
                    min_scale=o(d.has_scales, d.min_scale), max_scale=o(d.has_scales, d.max_scale),
                    damping=o(d.has_damping, d.damping), block_fallbacks=d.block_fallbacks)

    def scales(self):
        out = np.zeros(max(self.dim, 1))
        lib.or_lsmr_scales(self.h, _dp(out))
        return out[:self.dim]

    def damped_products(self, lam, scaled, x, y):
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        fwd = np.zeros(self.rows + self.dim)
        tr = np.zeros(self.dim)
        lib.or_lsmr_damped_products(self.h, lam, int(scaled), _dp(x), _dp(fwd), _dp(y), _dp(tr))
        return fwd, tr

    def precond(self, x, y):
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        px, pty = np.zeros(self.dim), np.zeros(self.dim)
        lib.or_lsmr_precond(self.h, _dp(x), _dp(px), _dp(y), _dp(pty))
        return px, pty


class _Generic(Schur):
    """Shared generic-backend calls (prepare/accumulate/damping/solve/work)."""

    def __init__(self, handle, dim_hint=0):  # noqa: D107 - Schur.__init__ is not called on purpose
        self.h = handle
        self.dim = dim_hint
        self.max_iterations = 1000
        self.relative_tolerance = max(1e-10, 128 * np.finfo(float).eps)

    def _limits(self):
        pass

    def covariance(self, columns, tol=64 * np.finfo(float).eps):
        cols = np.ascontiguousarray(np.asarray(columns, np.uint64))
        k = len(cols)
        out = np.zeros(max(k * k, 1))
        st = lib.or_backend_covariance(self.h, self._kind, cols.ctypes.data_as(C.POINTER(size_t)), k, tol, _dp(out))
        return st, out[:k * k].reshape(k, k).T.copy()


class DenseNormal(_Generic):
    """DenseNormalCholesky (src/normal.rs)."""
    _kind = 1

    def __init__(self):
        super().__init__(lib.or_dense_normal_create())

    def state(self):
        normal = np.zeros(max(self.dim * self.dim, 1))
        rhs = np.zeros(max(self.dim, 1))
        lib.or_dense_normal_state(self.h, _dp(normal), _dp(rhs))
        return normal[:self.dim * self.dim].reshape(self.dim, self.dim).T.copy(), rhs[:self.dim]

    def information(self, tol):
        return lib.or_dense_normal_information(self.h, tol)


class DenseSchur(_Generic):
    """DenseSchur (src/dense_schur.rs): retained prefix + landmark widths."""
    _kind = 2

    def __init__(self, retained, widths=()):
        w = (size_t * max(len(widths), 1))(*widths)
        super().__init__(lib.or_dense_schur_create(retained, w, len(widths)))


class DenseQr(_Generic):
    """DenseQr (src/qr.rs)."""
    _kind = 0

    def __init__(self, relative_rank_tolerance=64 * np.finfo(float).eps):
        super().__init__(lib.or_dense_qr_create(relative_rank_tolerance))

    def set_tolerance(self, tol):
        lib.or_dense_qr_set_tolerance(self.h, tol)


def eliminate(rows, removed, tol=-1.0):
    """Elimination::reduce (src/marginalization.rs:458-513) on row-major [J | r]."""
    rows = np.ascontiguousarray(np.asarray(rows, np.float64))
    m, width = rows.shape
    n = width - 1
    a = np.zeros(max(m * n, 1))
    b = np.zeros(max(m, 1))
    const = C.c_double()
    rank, nrows = size_t(), size_t()
    st = lib.or_eliminate(m, n, _dp(rows), removed, tol, _dp(a), _dp(b), C.byref(const), C.byref(rank),
                          C.byref(nrows))
    k, sep = nrows.value, n - removed
    return st, a[:k * sep].reshape(sep, k).T.copy(), b[:k].copy(), const.value, rank.value


def pose_exp(d):
    d = np.ascontiguousarray(d, np.float64)
    out = np.zeros(7)
    lib.or_pose_exp(_dp(d), _dp(out))
    return out


def pose_log(p):
    p = np.ascontiguousarray(p, np.float64)
    out = np.zeros(6)
    lib.or_pose_log(_dp(p), _dp(out))
    return out


def pose_compose(a, b):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    out = np.zeros(7)
    lib.or_pose_compose(_dp(a), _dp(b), _dp(out))
    return out


def pose_inverse(a):
    a = np.ascontiguousarray(a, np.float64)
    out = np.zeros(7)
    lib.or_pose_inverse(_dp(a), _dp(out))
    return out


def pose_adjoint(p):
    p = np.ascontiguousarray(p, np.float64)
    out = np.zeros(36)
    lib.or_pose_adjoint(_dp(p), _dp(out))
    return out.reshape(6, 6)


def pose_right_jacobian(d):
    d = np.ascontiguousarray(d, np.float64)
    out = np.zeros(36)
    lib.or_pose_right_jacobian(_dp(d), _dp(out))
    return out.reshape(6, 6)


def pose_log_jacobian(d):
    d = np.ascontiguousarray(d, np.float64)
    out = np.zeros(36)
    st = lib.or_pose_log_jacobian(_dp(d), _dp(out))
    return st, out.reshape(6, 6)


def _marginal(marginal):
    """(A m x 6s, b m, refs s x 7) -> column-major A, b, refs, m, s."""
    A, b, refs = marginal
    A = np.asarray(A, np.float64)
    refs = np.ascontiguousarray(np.asarray(refs, np.float64).reshape(-1, 7))
    return (np.ascontiguousarray(A.T).reshape(-1), np.ascontiguousarray(np.asarray(b, np.float64).reshape(-1)), refs,
            A.shape[0], len(refs))


def window_solve(poses, prior, rel_ij, rel_z, removed=10, max_iterations=20, gradient_tolerance=1e-8,
                 step_tolerance=1e-10, cost_tolerance=1e-12, lm_options=None, marginal=None):
    """LM over DenseSchur(6n, []) for one pose-graph window, then square-root
    marginalization of its oldest `removed` poses. marginal = (A, b, refs):
    a prior on the first len(refs) poses in place of the anchor prior."""
    poses = np.ascontiguousarray(np.array(poses, np.float64).reshape(-1, 7))
    n = len(poses)
    prior = np.ascontiguousarray(prior, np.float64)
    ij = np.ascontiguousarray(np.asarray(rel_ij, np.uint32).reshape(-1, 2))
    z = np.ascontiguousarray(np.asarray(rel_z, np.float64).reshape(-1, 7))
    o = OptOpts(max_iterations, gradient_tolerance, step_tolerance, cost_tolerance)
    lo = LmOpts(*(lm_options or (1e-3, 1e-12, 1e12, 1e-6, 1e-4, 16)))
    rep, st = Report(), LmStats()
    cap = 6 * n + 6
    a = np.zeros(cap * cap)
    b = np.zeros(cap)
    const = C.c_double()
    rows, nsep, rank = size_t(), size_t(), size_t()
    sep = np.zeros(max(n, 1), np.uint32)
    u32 = C.POINTER(C.c_uint32)
    if marginal is None:
        code = lib.or_window_solve(n, _dp(poses), _dp(prior), len(ij), ij.ctypes.data_as(u32), _dp(z), C.byref(o),
                                   C.byref(lo), removed, C.byref(rep), C.byref(st), _dp(a), _dp(b), C.byref(const),
                                   C.byref(rows), sep.ctypes.data_as(u32), C.byref(nsep), C.byref(rank))
    else:
        A, bb, refs, m, ns = _marginal(marginal)
        code = lib.or_window_solve_prior(n, _dp(poses), ns, m, _dp(A), _dp(bb), _dp(refs), len(ij),
                                         ij.ctypes.data_as(u32), _dp(z), C.byref(o), C.byref(lo), removed,
                                         C.byref(rep), C.byref(st), _dp(a), _dp(b), C.byref(const), C.byref(rows),
                                         sep.ctypes.data_as(u32), C.byref(nsep), C.byref(rank))
    k, s = rows.value, 6 * nsep.value
    return dict(code=code, poses=poses, report=rep, stats=st, prior_a=a[:k * s].reshape(s, k).T.copy(),
                prior_b=b[:k].copy(), prior_constant=const.value, separator=sep[:nsep.value].copy(),
                rank=rank.value)


def window_cost(poses, prior, rel_ij, rel_z, marginal=None):
    poses = np.ascontiguousarray(np.array(poses, np.float64).reshape(-1, 7))
    prior = np.ascontiguousarray(prior, np.float64)
    ij = np.ascontiguousarray(np.asarray(rel_ij, np.uint32).reshape(-1, 2))
    z = np.ascontiguousarray(np.asarray(rel_z, np.float64).reshape(-1, 7))
    out = C.c_double()
    u32 = C.POINTER(C.c_uint32)
    if marginal is None:
        st = lib.or_window_cost(len(poses), _dp(poses), _dp(prior), len(ij), ij.ctypes.data_as(u32), _dp(z),
                                C.byref(out))
    else:
        A, bb, refs, m, ns = _marginal(marginal)
        st = lib.or_window_cost_prior(len(poses), _dp(poses), ns, m, _dp(A), _dp(bb), _dp(refs), len(ij),
                                      ij.ctypes.data_as(u32), _dp(z), C.byref(out))
    return st, out.value


class Bal:
    """Oracle BAL problem (examples/bal/model.rs Frame batches)."""

    def __init__(self, cams, pts, oc, op, px):
        self.cams = np.ascontiguousarray(np.asarray(cams, np.float64).reshape(-1, 9))
        self.pts = np.ascontiguousarray(np.asarray(pts, np.float64).reshape(-1, 3))
        self.oc = np.ascontiguousarray(np.asarray(oc, np.uint32))
        self.op = np.ascontiguousarray(np.asarray(op, np.uint32))
        self.px = np.ascontiguousarray(np.asarray(px, np.float64).reshape(-1, 2))
        u32 = C.POINTER(C.c_uint32)
        self.h = lib.or_bal_create(len(self.cams), len(self.pts), len(self.oc), _dp(self.cams), _dp(self.pts),
                                   self.oc.ctypes.data_as(u32), self.op.ctypes.data_as(u32), _dp(self.px))

    @classmethod
    def from_data(cls, d):
        return cls(d.cameras, d.points, d.obs_camera, d.obs_point, d.obs_pixel)

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_bal_destroy(self.h)
            self.h = None

    def dimension(self):
        return 9 * len(self.cams) + 3 * len(self.pts)

    def cost(self):
        out = C.c_double()
        st = lib.or_bal_cost(self.h, C.byref(out))
        return st, out.value

    def parameters(self):
        c = np.zeros_like(self.cams)
        p = np.zeros_like(self.pts)
        lib.or_bal_get(self.h, _dp(c), _dp(p))
        return c, p

    def linearize(self, schur: Schur):
        return lib.or_bal_linearize(self.h, schur.h)

    def lm(self, schur: Schur, max_iterations=20, gradient_tolerance=1e-8, step_tolerance=0.0, cost_tolerance=0.0,
           lm_options=None, on_accept=None):
        schur._limits()
        o = OptOpts(max_iterations, gradient_tolerance, step_tolerance, cost_tolerance)
        lo = LmOpts(*(lm_options or (1e-3, 1e-12, 1e12, 1e-6, 1e-4, 16)))
        rep, st = Report(), LmStats()
        cb = ACCEPT(lambda _u, s: on_accept(s.contents)) if on_accept else ACCEPT()
        code = lib.or_lm_bal(schur.h, self.h, C.byref(o), C.byref(lo), C.byref(rep), C.byref(st), cb, None)
        return code, rep, st

    def lm_to_cost(self, schur: Schur, target_cost: float, max_iterations=50, gradient_tolerance=1e-8,
                   lm_options=None):
        """LM from the current estimates until an accepted cost is at or below
        target_cost (termination 5), or the usual LM stopping rules."""
        schur._limits()
        o = OptOpts(max_iterations, gradient_tolerance, 0.0, 0.0)
        lo = LmOpts(*(lm_options or (1e-3, 1e-12, 1e12, 1e-6, 1e-4, 16)))
        rep, st = Report(), LmStats()
        code = lib.or_lm_bal_to_cost(schur.h, self.h, C.byref(o), C.byref(lo), target_cost, C.byref(rep),
                                     C.byref(st))
        return code, rep, st

    def gn(self, schur: Schur, max_iterations=20, gradient_tolerance=1e-8, step_tolerance=0.0, cost_tolerance=0.0):
        schur._limits()
        o = OptOpts(max_iterations, gradient_tolerance, step_tolerance, cost_tolerance)
        rep = Report()
        code = lib.or_gn_bal(schur.h, self.h, C.byref(o), C.byref(rep))
        return code, rep


class CallbackProblem:
    """Host-evaluated problem for the oracle LM/GN (additive coordinates)."""

    def __init__(self, x0, cost, linearize):
        self.x0 = np.ascontiguousarray(np.asarray(x0, np.float64))
        n = len(self.x0)

        def cost_cb(_u, xp, out):
            try:
                out[0] = float(cost(np.ctypeslib.as_array(xp, shape=(n,)).copy() if n else np.zeros(0)))
                return 0
            except Exception as e:
                return getattr(e, "code", 20)

        def lin_cb(_u, xp, sink):
            def emit(r, blocks):
                args, keep = pack_blocks(r, blocks)
                code = lib.or_cbproblem_emit(sink, *args)
                if code:
                    raise RuntimeError(code)
            try:
                linearize(np.ctypeslib.as_array(xp, shape=(n,)).copy() if n else np.zeros(0), emit)
                return 0
            except RuntimeError as e:
                return int(e.args[0]) if e.args and isinstance(e.args[0], int) else 20
            except Exception as e:
                return getattr(e, "code", 20)

        self._c = COST(cost_cb)
        self._l = LIN(lin_cb)
        self.h = lib.or_cbproblem_create(n, _dp(self.x0), self._c, self._l, None)
        self.n = n

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_cbproblem_destroy(self.h)
            self.h = None

    @property
    def x(self):
        out = np.zeros(self.n)
        lib.or_cbproblem_get(self.h, _dp(out))
        return out

    def lm(self, schur, max_iterations=50, gradient_tolerance=1e-8, step_tolerance=1e-10, cost_tolerance=1e-12,
           lm_options=None):
        schur._limits()
        o = OptOpts(max_iterations, gradient_tolerance, step_tolerance, cost_tolerance)
        lo = LmOpts(*(lm_options or (1e-3, 1e-12, 1e12, 1e-6, 1e-4, 16)))
        rep, st = Report(), LmStats()
        code = lib.or_lm_cb(schur.h, self.h, C.byref(o), C.byref(lo), C.byref(rep), C.byref(st))
        return code, rep, st

    def gn(self, schur, max_iterations=50, gradient_tolerance=1e-8, step_tolerance=1e-10, cost_tolerance=1e-12):
        schur._limits()
        o = OptOpts(max_iterations, gradient_tolerance, step_tolerance, cost_tolerance)
        rep = Report()
        code = lib.or_gn_cb(schur.h, self.h, C.byref(o), C.byref(rep))
        return code, rep


class Model:
    """LinearizedModel alone (src/linear_model.rs) for its known-answer test."""

    def __init__(self, dim):
        self.h = lib.or_model_create(dim)
        self.dim = dim
        self.rows = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib.or_model_destroy(self.h)
            self.h = None

    def accumulate(self, residual, jacobians):
        args, keep = pack_blocks(residual, jacobians)
        self.rows += args[0]
        return lib.or_model_accumulate(self.h, *args)

    def prepare_scales(self, floor):
        return lib.or_model_prepare_scales(self.h, floor)

    def verify(self, step, lam):
        step = np.ascontiguousarray(step, np.float64)
        out = np.zeros(4)
        nr = np.zeros(self.dim)
        ref = np.zeros(self.dim)
        lib.or_model_verify(self.h, _dp(step), lam, _dp(out), _dp(nr), _dp(ref))
        return dict(predicted=out[0], finite_step=bool(out[1]), residual_norm=out[2], reference_norm=out[3],
                    normal_residual=nr, reference=ref)

    def state(self):
        g = np.zeros(self.dim)
        neg = np.zeros(max(self.rows, 1))
        lib.or_model_state(self.h, _dp(g), _dp(neg))
        return g, neg[:self.rows]


def block_factors_fallbacks(rows, cols, blocks5, values, scales, lambdas):
    b5 = np.ascontiguousarray(np.asarray(blocks5, np.uint64).reshape(-1, 5)).astype(np.uint64)
    vals = np.ascontiguousarray(np.asarray(values, np.float64))
    sc = np.ascontiguousarray(np.asarray(scales, np.float64))
    lam = np.ascontiguousarray(np.asarray(lambdas, np.float64))
    out = np.zeros(len(lam), np.uint64)
    sp = C.POINTER(size_t)
    st = lib.or_blockfactors_run(rows, cols, len(b5), b5.ctypes.data_as(sp), _dp(vals), len(vals), _dp(sc),
                                 _dp(lam), len(lam), out.ctypes.data_as(sp))
    return st, [int(x) for x in out]
