"""fagra_b200 — a B200 (sm_100a) linear-solve and linearization backend for the
fagra factor-graph library.

The numerical work lives in libfagra_b200.so (hand-written CUDA); this
package is its Python face, shaped like fagra's Rust API:

    from fagra_b200 import Schur, LevenbergMarquardt, BalProblem
    backend = Schur(9 * cameras, 9, 3)
    lm = LevenbergMarquardt(backend)
    report = lm.solve_batch(BalProblem.from_data(data))
"""
from ._lib import device_count, kernel_launches, last_error, device_stream, LIB_PATH  # noqa: F401
from .errors import *  # noqa: F401,F403
from .backend import (Schur, Lsmr, DampedStep, SchurDiagnostics, SchurTimings, LsmrDiagnostics,  # noqa: F401
                      LsmrTimings, DenseNormalCholesky, DenseSchur, DenseQr)
from .optimize import (LevenbergMarquardt, GaussNewton, OptimizeOptions, LmOptions, LmStatistics,  # noqa: F401
                       LmOutcome, LmWork, CallbackProblem, OptimizeReport)
from .bal import BalProblem  # noqa: F401
from .learned import LearnedPreconditioner  # noqa: F401

__version__ = "0.1.0"
