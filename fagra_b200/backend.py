"""Python face of the device backend, shaped like fagra's Rust API.

`Schur` mirrors `fagra::Schur` (src/schur.rs): public fields `max_iterations`,
`relative_tolerance`, `collect_timings`; the LeastSquaresBackend methods
(src/optimization.rs:131-169); `statistics()`, `diagnostics()`, `timings()`.
Every numerical step runs in libfagra_b200.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Iterable, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import lib, size_t, ptrdiff_t, dptr
from .errors import raise_for_status

TERMINATIONS = {0: None, 1: "Converged", 2: "IterationLimit", 3: "NotPositiveDefinite", 4: "NonFinite"}
PRECISIONS = {"f64": 0, "f32": 1}
PRECONDITIONERS = {"retained_blocks": 0, "schur_diagonal": 1, "learned": 2}


@dataclass
class DampedStep:
    """src/optimization.rs:171-177 (delta copied out of the pinned mirror)."""
    delta: np.ndarray
    predicted_reduction: float


@dataclass
class LinearSolveWork:
    solves: int
    iterations: int


@dataclass
class SchurDiagnostics:
    termination: Optional[str]
    iterations: int
    damping: float
    estimated_relative_residual: Optional[float]
    reduced_relative_residual: Optional[float]
    scaled_relative_residual: Optional[float]
    original_relative_residual: Optional[float]
    refinements: int
    # learned preconditioner only: the preconditioner whose step was kept, the
    # fallback taken (None, "failed", "more_iterations") and both solves' counts
    preconditioner_used: str = "retained_blocks"
    learned_fallback: Optional[str] = None
    learned_iterations: int = 0
    block_jacobi_iterations: int = 0
    coarse_vectors: int = 0
    learned_seconds: float = 0.0
    block_jacobi_seconds: float = 0.0


@dataclass
class SchurTimings:
    preparation: float
    factorization: float
    linear_solve: float
    products: float
    preconditioner: float
    verification: float


def _dp(a: np.ndarray):
    return a.ctypes.data_as(dptr)


def _covariance(handle, columns, tol: float) -> np.ndarray:
    """CovarianceBackend::covariance + SelectedCovariance (src/covariance.rs:225-270):
    the selected block of the undamped inverse information, selection order."""
    cols = (size_t * max(len(columns), 1))(*[int(c) for c in columns])
    k = len(columns)
    out = np.zeros(max(k * k, 1))
    raise_for_status(lib.fg_backend_covariance(handle, cols, k, tol, _dp(out)))
    return out[:k * k].reshape(k, k).T.copy()


class Schur:
    """Device Schur-PCG backend: `Schur::new(retained, retained_width, eliminated_width)`."""

    def __init__(self, retained_dimension: int, retained_block_width: int, eliminated_block_width: int, *,
                 precision: str = "f64", preconditioner: str = "retained_blocks", coarse_correction: bool = False,
                 device: int = 0):
        o = _lib.SchurOptions()
        lib.fg_schur_default_options(C.byref(o))
        o.precision = PRECISIONS[precision]
        o.preconditioner = PRECONDITIONERS[preconditioner]
        o.coarse_correction = int(bool(coarse_correction))
        o.device = device
        self._opts = o
        h = C.c_void_p()
        raise_for_status(lib.fg_schur_create(retained_dimension, retained_block_width, eliminated_block_width,
                                             C.byref(o), C.byref(h)))
        self._h = h
        self.retained = retained_dimension
        self.widths = (retained_block_width, eliminated_block_width)
        self.precision = precision
        self.device = device

    # ---- public fields
    def _get(self, name):
        return getattr(self._opts, name)

    def _set(self, name, value):
        setattr(self._opts, name, value)
        raise_for_status(lib.fg_schur_set_options(self._h, C.byref(self._opts)))

    max_iterations = property(lambda s: s._get("max_iterations"), lambda s, v: s._set("max_iterations", v))
    relative_tolerance = property(lambda s: s._get("relative_tolerance"),
                                  lambda s, v: s._set("relative_tolerance", v))
    collect_timings = property(lambda s: bool(s._get("collect_timings")),
                               lambda s, v: s._set("collect_timings", int(bool(v))))
    preconditioner = property(lambda s: {v: k for k, v in PRECONDITIONERS.items()}[s._get("preconditioner")],
                              lambda s, v: s._set("preconditioner", PRECONDITIONERS[v]))
    residual_replacement = property(lambda s: s._get("residual_replacement"),
                                    lambda s, v: s._set("residual_replacement", v))
    operator_variant = property(lambda s: s._get("operator_variant"), lambda s, v: s._set("operator_variant", v))
    coarse_correction = property(lambda s: bool(s._get("coarse_correction")),
                                 lambda s, v: s._set("coarse_correction", int(bool(v))))
    # learned preconditioner: "compare" (default; one block-Jacobi comparison,
    # the network is dropped when it loses) or "always"
    learned_policy = property(lambda s: ("compare", "always")[s._get("learned_policy")],
                              lambda s, v: s._set("learned_policy", {"compare": 0, "always": 1}[v]))

    def accumulate_pairs_device(self, count: int, rows: int, retained_variable: int, eliminated_variable: int,
                                residual: int, retained_jacobian: int, eliminated_jacobian: int) -> None:
        """A device batch of `count` bipartite emissions (device pointers,
        SoA layout of fg_schur_accumulate_pairs_device)."""
        raise_for_status(lib.fg_schur_accumulate_pairs_device(
            self._h, count, rows, C.c_void_p(retained_variable), C.c_void_p(eliminated_variable),
            C.c_void_p(residual), C.c_void_p(retained_jacobian), C.c_void_p(eliminated_jacobian)))

    def set_poll_limit(self, polls: int) -> None:
        """Test hook: polls after which the ring operator's slot wait gives up
        (the solve then raises DeviceTimeout); 0 restores the default."""
        raise_for_status(lib.fg_schur_set_poll_limit(self._h, polls))

    def operator_info(self):
        """(variant in use, measured seconds per application of variants 1..4)."""
        var, sec = C.c_int(), (C.c_double * 4)()
        raise_for_status(lib.fg_schur_operator_info(self._h, C.byref(var), sec))
        return var.value, list(sec)

    @property
    def handle(self):
        return self._h

    def attach_learned(self, network) -> None:
        """Attach (None: detach) the network used by preconditioner="learned".
        Re-arms the one-time block-Jacobi comparison."""
        raise_for_status(lib.fg_schur_attach_learned(self._h, network.handle if network is not None else None))
        self._learned = network  # the backend holds a pointer: keep the network alive

    def close(self):
        if getattr(self, "_h", None):
            lib.fg_backend_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- LeastSquaresBackend
    def prepare(self, dimension: int) -> None:
        raise_for_status(lib.fg_backend_prepare(self._h, dimension))
        self._dim = dimension

    def clear(self) -> None:
        raise_for_status(lib.fg_backend_clear(self._h))

    def accumulate(self, residual: Sequence[float], jacobians: Iterable[Tuple[int, np.ndarray]]) -> None:
        accumulate_into(self._h, residual, jacobians)

    def gradient_norm(self) -> float:
        out = C.c_double()
        raise_for_status(lib.fg_backend_gradient_norm(self._h, C.byref(out)))
        return out.value

    def solve(self) -> np.ndarray:
        p = dptr()
        n = size_t()
        raise_for_status(lib.fg_backend_solve(self._h, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0)

    def prepare_damping(self, min_column_norm: float) -> None:
        raise_for_status(lib.fg_backend_prepare_damping(self._h, min_column_norm))

    def solve_damped(self, damping: float) -> DampedStep:
        p = dptr()
        n = size_t()
        pred = C.c_double()
        raise_for_status(lib.fg_backend_solve_damped(self._h, damping, C.byref(p), C.byref(n), C.byref(pred)))
        delta = np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0)
        return DampedStep(delta, pred.value)

    def linear_solve_work(self) -> LinearSolveWork:
        s, i, a = size_t(), size_t(), C.c_int()
        raise_for_status(lib.fg_backend_linear_solve_work(self._h, C.byref(s), C.byref(i), C.byref(a)))
        return LinearSolveWork(s.value, i.value)

    statistics = linear_solve_work

    def diagnostics(self) -> SchurDiagnostics:
        d = _lib.SchurDiagnosticsC()
        raise_for_status(lib.fg_schur_get_diagnostics(self._h, C.byref(d)))
        opt = lambda flag, v: v if flag else None  # noqa: E731
        return SchurDiagnostics(TERMINATIONS[d.termination], d.iterations, d.damping,
                                opt(d.has_estimated, d.estimated_relative_residual),
                                opt(d.has_reduced, d.reduced_relative_residual),
                                opt(d.has_scaled, d.scaled_relative_residual),
                                opt(d.has_original, d.original_relative_residual), d.refinements,
                                {v: k for k, v in PRECONDITIONERS.items()}[d.preconditioner_used],
                                (None, "failed", "more_iterations")[d.learned_fallback], d.learned_iterations,
                                d.block_jacobi_iterations, d.coarse_vectors, d.learned_seconds,
                                d.block_jacobi_seconds)

    def timings(self) -> SchurTimings:
        t = _lib.SchurTimingsC()
        raise_for_status(lib.fg_schur_get_timings(self._h, C.byref(t)))
        return SchurTimings(t.preparation, t.factorization, t.linear_solve, t.products, t.preconditioner,
                            t.verification)

    # ---- structure / model export (index maps in the reference layouts)
    def structure(self) -> dict:
        sizes = [size_t() for _ in range(6)]
        raise_for_status(lib.fg_schur_structure_sizes(self._h, *[C.byref(s) for s in sizes]))
        nb, ne, nv, nvar, rows, cols = (s.value for s in sizes)
        b5 = np.zeros((max(nb, 1), 5), np.uint64)
        e4 = np.zeros((max(ne, 1), 4), np.uint64)
        own = np.zeros(max(cols, 1), np.uint64)
        v3 = np.zeros((max(nvar, 1), 3), np.uint64)
        u64 = C.POINTER(C.c_uint64)
        raise_for_status(lib.fg_schur_export_structure(
            self._h, b5.ctypes.data_as(u64), e4.ctypes.data_as(u64), own.ctypes.data_as(u64),
            v3.ctypes.data_as(u64)))
        return dict(blocks=b5[:nb], edges=e4[:ne], owners=own[:cols], variables=v3[:nvar], rows=rows, cols=cols,
                    nvalues=nv)

    def model(self, damping_ready: bool = True) -> dict:
        s = self.structure()
        nv, rows, cols = s["nvalues"], s["rows"], s["cols"]
        var = s["variables"]
        ngram = int(sum(int(w) * int(w) for w in var[:, 1])) if len(var) else 0
        cw, pw = self.widths
        out = dict(values=np.zeros(max(nv, 1)), negative_residual=np.zeros(max(rows, 1)),
                   gradient=np.zeros(max(cols, 1)), scales=np.zeros(max(cols, 1)), gram=np.zeros(max(ngram, 1)),
                   cross=np.zeros(max(len(s["edges"]) * cw * pw, 1)))
        raise_for_status(lib.fg_schur_export_model(self._h, *[_dp(out[k]) for k in
                                                              ("values", "negative_residual", "gradient", "scales",
                                                               "gram", "cross")]))
        out["values"] = out["values"][:nv]
        out["negative_residual"] = out["negative_residual"][:rows]
        out["gradient"] = out["gradient"][:cols]
        out["scales"] = out["scales"][:cols]
        out["gram"] = out["gram"][:ngram]
        out["cross"] = out["cross"][:len(s["edges"]) * cw * pw]
        return out

    def covariance(self, columns, relative_pivot_tolerance: float = 64 * np.finfo(float).eps) -> np.ndarray:
        """Schur delegates to LinearizedModel::covariance (src/schur.rs:548-556): a
        dense normal matrix of the cached Jacobian, then the selected inverse."""
        return _covariance(self._h, columns, relative_pivot_tolerance)

    def reduced_apply(self, damping: float, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        raise_for_status(lib.fg_schur_reduced_apply(self._h, damping, _dp(x), _dp(y)))
        return y


@dataclass
class LsmrDiagnostics:
    """src/lsmr.rs:68-104 (None where the reference has None)."""
    termination: Optional[str]
    iterations: int
    finite_step: bool
    estimated_absolute_residual: Optional[float]
    estimated_relative_residual: Optional[float]
    original_absolute_residual: Optional[float]
    original_relative_residual: Optional[float]
    scaled_absolute_residual: Optional[float]
    scaled_relative_residual: Optional[float]
    min_scale: Optional[float]
    max_scale: Optional[float]
    damping: Optional[float]
    block_fallbacks: int


@dataclass
class LsmrTimings:
    preparation: float
    factorization: float
    linear_solve: float
    forward: float
    transpose: float
    preconditioner: float
    residual_checks: float


class Lsmr:
    """Device LSMR backend: `Lsmr::default()` (src/lsmr.rs:339-362) with the public
    fields `max_iterations`, `relative_tolerance`, `diagonal_preconditioning`,
    `block_preconditioning` and `collect_timings`."""

    def __init__(self, *, precision: str = "f64", device: int = 0):
        o = _lib.LsmrOptions()
        lib.fg_lsmr_default_options(C.byref(o))
        o.precision = PRECISIONS[precision]
        if precision == "f32":  # Lsmr::<f32>::default(): max(1e-10, 128 eps_f32)
            o.relative_tolerance = max(1e-10, 128 * float(np.finfo(np.float32).eps))
        o.device = device
        self._opts = o
        h = C.c_void_p()
        raise_for_status(lib.fg_lsmr_create(C.byref(o), C.byref(h)))
        self._h = h
        self.precision = precision
        self.device = device
        self._dim = 0
        self._rows = 0

    def _get(self, name):
        return getattr(self._opts, name)

    def _set(self, name, value):
        setattr(self._opts, name, value)
        raise_for_status(lib.fg_lsmr_set_options(self._h, C.byref(self._opts)))

    max_iterations = property(lambda s: s._get("max_iterations"), lambda s, v: s._set("max_iterations", v))
    relative_tolerance = property(lambda s: s._get("relative_tolerance"),
                                  lambda s, v: s._set("relative_tolerance", v))
    diagonal_preconditioning = property(lambda s: bool(s._get("diagonal_preconditioning")),
                                        lambda s, v: s._set("diagonal_preconditioning", int(bool(v))))
    block_preconditioning = property(lambda s: bool(s._get("block_preconditioning")),
                                     lambda s, v: s._set("block_preconditioning", int(bool(v))))
    collect_timings = property(lambda s: bool(s._get("collect_timings")),
                               lambda s, v: s._set("collect_timings", int(bool(v))))

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib.fg_backend_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- LeastSquaresBackend
    def covariance(self, columns, relative_pivot_tolerance: float = 64 * np.finfo(float).eps) -> np.ndarray:
        """Lsmr delegates to LinearizedModel::covariance (src/lsmr.rs:598-604)."""
        return _covariance(self._h, columns, relative_pivot_tolerance)

    def prepare(self, dimension: int) -> None:
        raise_for_status(lib.fg_backend_prepare(self._h, dimension))
        self._dim = dimension
        self._rows = 0

    def clear(self) -> None:
        raise_for_status(lib.fg_backend_clear(self._h))
        self._rows = 0

    def accumulate(self, residual: Sequence[float], jacobians: Iterable[Tuple[int, np.ndarray]]) -> None:
        accumulate_into(self._h, residual, jacobians)
        self._rows += int(np.asarray(residual).size)

    def gradient_norm(self) -> float:
        out = C.c_double()
        raise_for_status(lib.fg_backend_gradient_norm(self._h, C.byref(out)))
        return out.value

    def solve(self) -> np.ndarray:
        p = dptr()
        n = size_t()
        raise_for_status(lib.fg_backend_solve(self._h, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0)

    def prepare_damping(self, min_column_norm: float) -> None:
        raise_for_status(lib.fg_backend_prepare_damping(self._h, min_column_norm))

    def solve_damped(self, damping: float) -> DampedStep:
        p = dptr()
        n = size_t()
        pred = C.c_double()
        raise_for_status(lib.fg_backend_solve_damped(self._h, damping, C.byref(p), C.byref(n), C.byref(pred)))
        delta = np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0)
        return DampedStep(delta, pred.value)

    def linear_solve_work(self) -> LinearSolveWork:
        s, i, a = size_t(), size_t(), C.c_int()
        raise_for_status(lib.fg_backend_linear_solve_work(self._h, C.byref(s), C.byref(i), C.byref(a)))
        return LinearSolveWork(s.value, i.value)

    statistics = linear_solve_work

    def diagnostics(self) -> LsmrDiagnostics:
        d = _lib.LsmrDiagnosticsC()
        raise_for_status(lib.fg_lsmr_get_diagnostics(self._h, C.byref(d)))
        o = lambda flag, v: v if flag else None  # noqa: E731
        return LsmrDiagnostics(TERMINATIONS[d.termination], d.iterations, bool(d.finite_step),
                               o(d.has_estimated, d.estimated_absolute_residual),
                               o(d.has_estimated, d.estimated_relative_residual),
                               o(d.has_original, d.original_absolute_residual),
                               o(d.has_original, d.original_relative_residual),
                               o(d.has_scaled, d.scaled_absolute_residual),
                               o(d.has_scaled, d.scaled_relative_residual),
                               o(d.has_scales, d.min_scale), o(d.has_scales, d.max_scale),
                               o(d.has_damping, d.damping), d.block_fallbacks)

    def timings(self) -> LsmrTimings:
        t = _lib.LsmrTimingsC()
        raise_for_status(lib.fg_lsmr_get_timings(self._h, C.byref(t)))
        return LsmrTimings(t.preparation, t.factorization, t.linear_solve, t.forward, t.transpose,
                           t.preconditioner, t.residual_checks)

    def damped_products(self, damping: float, scaled: bool, x: np.ndarray, y: np.ndarray):
        """Damped operator products on the device: (A x, A^T y)."""
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        fwd = np.zeros(self._rows + self._dim)
        tr = np.zeros(self._dim)
        raise_for_status(lib.fg_lsmr_damped_products(self._h, damping, int(bool(scaled)), _dp(x), _dp(fwd), _dp(y),
                                                     _dp(tr)))
        return fwd, tr

    def time_iteration(self, damping: float, repetitions: int = 64):
        sec, by = C.c_double(), C.c_double()
        raise_for_status(lib.fg_lsmr_time_iteration(self._h, damping, repetitions, C.byref(sec), C.byref(by)))
        return sec.value, by.value


def accumulate_into(handle, residual, jacobians) -> None:
    """Emit one residual with its (column offset, Jacobian) blocks through the C ABI."""
    r = np.ascontiguousarray(np.asarray(residual, dtype=np.float64).reshape(-1))
    blocks = [(int(c), np.asarray(j, dtype=np.float64)) for c, j in jacobians]
    nb = len(blocks)
    cols = (size_t * max(nb, 1))(*[c for c, _ in blocks])
    widths = (size_t * max(nb, 1))()
    ptrs = (dptr * max(nb, 1))()
    rs = (ptrdiff_t * max(nb, 1))()
    cs = (ptrdiff_t * max(nb, 1))()
    keep = []
    for k, (_, j) in enumerate(blocks):
        j2 = j.reshape(len(r), -1) if j.ndim != 2 else j
        keep.append(j2)
        widths[k] = j2.shape[1]
        ptrs[k] = j2.ctypes.data_as(dptr)
        rs[k] = j2.strides[0] // 8
        cs[k] = j2.strides[1] // 8
    raise_for_status(lib.fg_backend_accumulate(handle, len(r), _dp(r), nb, cols, widths, ptrs, rs, cs))


class _DenseBackend:
    """Shared LeastSquaresBackend calls of the dense device backends."""

    _h = None

    def close(self):
        if getattr(self, "_h", None):
            lib.fg_backend_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def prepare(self, dimension: int) -> None:
        raise_for_status(lib.fg_backend_prepare(self._h, dimension))
        self._dim = dimension

    def clear(self) -> None:
        raise_for_status(lib.fg_backend_clear(self._h))

    def accumulate(self, residual, jacobians) -> None:
        accumulate_into(self._h, residual, jacobians)

    def gradient_norm(self) -> float:
        out = C.c_double()
        raise_for_status(lib.fg_backend_gradient_norm(self._h, C.byref(out)))
        return out.value

    def solve(self) -> np.ndarray:
        p, n = dptr(), size_t()
        raise_for_status(lib.fg_backend_solve(self._h, C.byref(p), C.byref(n)))
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0)

    def prepare_damping(self, min_column_norm: float) -> None:
        raise_for_status(lib.fg_backend_prepare_damping(self._h, min_column_norm))

    def solve_damped(self, damping: float) -> DampedStep:
        p, n, pred = dptr(), size_t(), C.c_double()
        raise_for_status(lib.fg_backend_solve_damped(self._h, damping, C.byref(p), C.byref(n), C.byref(pred)))
        delta = np.ctypeslib.as_array(p, shape=(n.value,)).copy() if n.value else np.zeros(0)
        return DampedStep(delta, pred.value)

    def covariance(self, columns, relative_pivot_tolerance: float = 64 * np.finfo(float).eps) -> np.ndarray:
        return _covariance(self._h, columns, relative_pivot_tolerance)


class DenseNormalCholesky(_DenseBackend):
    """Device DenseNormalCholesky (src/normal.rs)."""

    def __init__(self, *, device: int = 0):
        h = C.c_void_p()
        raise_for_status(lib.fg_dense_normal_create(device, C.byref(h)))
        self._h = h


class DenseSchur(_DenseBackend):
    """Device DenseSchur (src/dense_schur.rs): retained prefix + landmark widths."""

    def __init__(self, retained_dimension: int, eliminated_widths=(), *, device: int = 0):
        w = (size_t * max(len(eliminated_widths), 1))(*[int(x) for x in eliminated_widths])
        h = C.c_void_p()
        raise_for_status(lib.fg_dense_schur_create(retained_dimension, w, len(eliminated_widths), device,
                                                   C.byref(h)))
        self._h = h


class DenseQr(_DenseBackend):
    """Device DenseQr (src/qr.rs)."""

    def __init__(self, relative_rank_tolerance: float = 64 * np.finfo(float).eps, *, device: int = 0):
        h = C.c_void_p()
        raise_for_status(lib.fg_dense_qr_create(relative_rank_tolerance, device, C.byref(h)))
        self._h = h
        self._tol = relative_rank_tolerance

    @property
    def relative_rank_tolerance(self):
        return self._tol

    @relative_rank_tolerance.setter
    def relative_rank_tolerance(self, v):
        raise_for_status(lib.fg_dense_qr_set_tolerance(self._h, v))
        self._tol = v
