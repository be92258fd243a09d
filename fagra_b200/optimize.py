"""Nonlinear optimizers over the device backend, shaped like fagra's
`LevenbergMarquardt` / `GaussNewton` (src/optimization/*.rs).

The loops themselves run in the library's C++ driver (fg_lm_solve_bal,
fg_lm_optimize, ...); this module holds the option structs and the
`solve_batch*` entry points.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import _lib
from ._lib import lib, dptr
from .backend import Schur, accumulate_into
from .errors import FagraError, error_for, raise_for_status

TERMINATION = {1: "NoVariables", 2: "GradientTolerance", 3: "StepTolerance", 4: "CostTolerance"}
REJECTION = {0: None, 1: "LinearSolve", 2: "Prediction", 3: "InvalidEvaluation", 4: "PoorAgreement"}


@dataclass
class OptimizeOptions:
    """src/optimization.rs:40-67 (defaults for f64)."""
    max_iterations: int = 50
    gradient_tolerance: float = 1e-8
    step_tolerance: float = 1e-10
    cost_tolerance: float = 1e-12

    def c(self):
        return _lib.OptimizeOptionsC(self.max_iterations, self.gradient_tolerance, self.step_tolerance,
                                     self.cost_tolerance)


@dataclass
class LmOptions:
    """src/optimization/levenberg_marquardt.rs:17-46."""
    initial_damping: float = 1e-3
    min_damping: float = 1e-12
    max_damping: float = 1e12
    min_column_norm: float = 1e-6
    acceptance_threshold: float = 1e-4
    max_trials: int = 16

    def c(self):
        return _lib.LmOptionsC(self.initial_damping, self.min_damping, self.max_damping, self.min_column_norm,
                               self.acceptance_threshold, self.max_trials)


@dataclass
class OptimizeReport:
    iterations: int
    initial_cost: float
    final_cost: float
    termination: str


@dataclass
class LinearSolveWork:
    solves: int
    iterations: int


@dataclass
class LmStatistics:
    linearizations: int = 0
    attempts: int = 0
    rejected_steps: int = 0
    accepted_steps: int = 0
    cost_evaluations: int = 0
    damping: float = 0.0
    cost: Optional[float] = None
    gradient_norm: Optional[float] = None
    step_norm: Optional[float] = None
    last_rejection: Optional[str] = None
    linear_solve: Optional[LinearSolveWork] = None

    @staticmethod
    def from_c(s: "_lib.LmStatisticsC") -> "LmStatistics":
        return LmStatistics(s.linearizations, s.attempts, s.rejected_steps, s.accepted_steps, s.cost_evaluations,
                            s.damping, s.cost if s.has_cost else None,
                            s.gradient_norm if s.has_gradient_norm else None,
                            s.step_norm if s.has_step_norm else None, REJECTION[s.last_rejection],
                            LinearSolveWork(s.linear_solves, s.linear_iterations) if s.linear_work_available
                            else None)


@dataclass
class LmWork:
    """levenberg_marquardt.rs:124-141."""
    linearizations: int = 0
    attempts: int = 0
    rejected_steps: int = 0
    accepted_steps: int = 0
    cost_evaluations: int = 0
    linear_solve: Optional[LinearSolveWork] = field(default_factory=lambda: LinearSolveWork(0, 0))


@dataclass
class LmOutcome:
    """levenberg_marquardt.rs:175-184: result is a report or the raised error."""
    result: object
    statistics: LmStatistics
    work: LmWork


class LevenbergMarquardt:
    """`LevenbergMarquardt::new(backend)` with `options` and `on_accept`."""

    def __init__(self, backend: Schur):
        self._backend = backend
        self.options = LmOptions()
        self.on_accept: Optional[Callable[[LmStatistics], None]] = None
        self._stats = LmStatistics(damping=0.0)

    def backend(self) -> Schur:
        return self._backend

    def statistics(self) -> LmStatistics:
        return self._stats

    def _run(self, problem, options: OptimizeOptions):
        rep = _lib.ReportC()
        st = _lib.LmStatisticsC()
        if hasattr(problem, "_bal_handle"):
            obs = self.on_accept
            cb = _lib.ACCEPT_CB(lambda _u, p: obs(LmStatistics.from_c(p.contents))) if obs else _lib.ACCEPT_CB()
            code = lib.fg_lm_solve_bal(self._backend.handle, problem._bal_handle, C.byref(options.c()),
                                       C.byref(self.options.c()), C.byref(rep), C.byref(st), cb, None)
        else:
            code = problem._lm(self._backend, options, self.options, rep, st)
        self._stats = LmStatistics.from_c(st)
        return code, rep

    def solve_batch(self, problem, options: Optional[OptimizeOptions] = None) -> OptimizeReport:
        code, rep = self._run(problem, options or OptimizeOptions())
        raise_for_status(code)
        return OptimizeReport(rep.iterations, rep.initial_cost, rep.final_cost, TERMINATION[rep.termination])

    optimize_with = solve_batch

    def solve_batch_with_covariance(self, problem, options: Optional[OptimizeOptions] = None, columns=(),
                                    relative_pivot_tolerance: float = 64 * np.finfo(float).eps):
        """levenberg_marquardt.rs:218-231: solve, then the selected covariance of
        the undamped model linearized at the final estimates."""
        report = self.solve_batch(problem, options)
        return report, _final_covariance(self._backend, problem, columns, relative_pivot_tolerance)

    def solve_batch_with_outcome(self, problem, options: Optional[OptimizeOptions] = None) -> LmOutcome:
        code, rep = self._run(problem, options or OptimizeOptions())
        s = self._stats
        result = (OptimizeReport(rep.iterations, rep.initial_cost, rep.final_cost, TERMINATION[rep.termination])
                  if code == 0 else error_for(code))
        ls = LinearSolveWork(0, 0) if s.attempts == 0 else s.linear_solve
        return LmOutcome(result, s, LmWork(s.linearizations, s.attempts, s.rejected_steps, s.accepted_steps,
                                           s.cost_evaluations, ls))


class GaussNewton:
    """`GaussNewton::new(backend)`."""

    def __init__(self, backend: Schur):
        self._backend = backend

    def backend(self) -> Schur:
        return self._backend

    def solve_batch(self, problem, options: Optional[OptimizeOptions] = None) -> OptimizeReport:
        options = options or OptimizeOptions()
        rep = _lib.ReportC()
        if hasattr(problem, "_bal_handle"):
            code = lib.fg_gn_solve_bal(self._backend.handle, problem._bal_handle, C.byref(options.c()), C.byref(rep))
        else:
            code = problem._gn(self._backend, options, rep)
        raise_for_status(code)
        return OptimizeReport(rep.iterations, rep.initial_cost, rep.final_cost, TERMINATION[rep.termination])

    optimize_with = solve_batch

    def solve_batch_with_covariance(self, problem, options: Optional[OptimizeOptions] = None, columns=(),
                                    relative_pivot_tolerance: float = 64 * np.finfo(float).eps):
        """gauss_newton.rs solve_batch_with_covariance: solve, then the selected
        covariance of the model at the final estimates."""
        report = self.solve_batch(problem, options)
        return report, _final_covariance(self._backend, problem, columns, relative_pivot_tolerance)


def _final_covariance(backend, problem, columns, tol):
    """Workspace::covariance (src/optimization.rs:268-284): linearize at the final
    estimates, then CovarianceBackend::covariance on that model."""
    backend.prepare(problem.dimension() if hasattr(problem, "_bal_handle") else len(problem.x))
    if hasattr(problem, "_bal_handle"):
        problem.linearize(backend)
    else:
        backend.clear()
        problem._linearize(problem.x.copy(), lambda r, blocks: backend.accumulate(r, blocks))
    return backend.covariance(columns, tol)


class CallbackProblem:
    """A host-evaluated problem over additive real coordinates.

    `cost(x) -> float` evaluates the objective; `linearize(x, emit)` calls
    `emit(residual, [(col, J), ...])` once per residual, in factor order.
    Raise `fagra_b200.errors.InvalidEvaluation` for invalid trial states.
    """

    def __init__(self, x0, cost: Callable, linearize: Callable):
        self.x = np.ascontiguousarray(np.asarray(x0, dtype=np.float64).copy())
        self._cost = cost
        self._linearize = linearize

    def _callbacks(self):
        n = len(self.x)

        def cost_cb(_u, xp, out):
            try:
                x = np.ctypeslib.as_array(xp, shape=(n,)) if n else np.zeros(0)
                out[0] = float(self._cost(x.copy()))
                return 0
            except FagraError as e:
                return e.code
            except Exception:
                return 20

        def lin_cb(_u, xp, handle):
            try:
                x = np.ctypeslib.as_array(xp, shape=(n,)) if n else np.zeros(0)
                self._linearize(x.copy(), lambda r, blocks: accumulate_into(handle, r, blocks))
                return 0
            except FagraError as e:
                return e.code
            except Exception:
                return 20

        cbs = _lib.ProblemCallbacksC(n, _lib.COST_CB(cost_cb), _lib.LIN_CB(lin_cb))
        return cbs

    def _lm(self, backend, options, lm_options, rep, st):
        cbs = self._callbacks()
        return lib.fg_lm_optimize(backend.handle, C.byref(cbs), None, self.x.ctypes.data_as(dptr),
                                  C.byref(options.c()), C.byref(lm_options.c()), C.byref(rep), C.byref(st))

    def _gn(self, backend, options, rep):
        cbs = self._callbacks()
        return lib.fg_gn_optimize(backend.handle, C.byref(cbs), None, self.x.ctypes.data_as(dptr),
                                  C.byref(options.c()), C.byref(rep))
