"""Error types mirroring fagra's src/error.rs, mapped from fg_status codes."""
from __future__ import annotations


class FagraError(Exception):
    """Base class for every error raised through the C ABI."""

    code = -1

    def __init__(self, message: str = ""):
        super().__init__(message or type(self).__name__)


class SolverError(FagraError):
    """src/error.rs:39-76 SolverError."""


class EvaluationError(SolverError):
    """src/error.rs:19-37 EvaluationError (wrapped by SolverError::Evaluation)."""


class DuplicateCovarianceBlock(SolverError): code = 1
class SingularInformation(SolverError): code = 2
class InvalidInformation(SolverError): code = 3
class InvalidRankTolerance(SolverError): code = 4
class BatchNotEmpty(SolverError): code = 5
class InvalidOptions(SolverError): code = 6
class KeyError_(SolverError): code = 7
class LinearSolveFailed(SolverError): code = 8
class NoConvergence(SolverError): code = 9
class NoProgress(SolverError): code = 10
class InvalidEvaluation(EvaluationError): code = 20
class DimensionMismatch(EvaluationError): code = 21
class InvalidEmission(EvaluationError): code = 22
class UnsupportedStructure(EvaluationError): code = 23


class DeviceError(FagraError):
    """CUDA-side failures with no counterpart in the CPU reference."""


class CudaError(DeviceError): code = 40
class OutOfMemory(DeviceError): code = 41
class DeviceTimeout(DeviceError): code = 42
class NullArgument(DeviceError): code = 43
class NoDevice(DeviceError): code = 44


BY_CODE = {cls.code: cls for cls in [
    DuplicateCovarianceBlock, SingularInformation, InvalidInformation, InvalidRankTolerance, BatchNotEmpty,
    InvalidOptions, KeyError_, LinearSolveFailed, NoConvergence, NoProgress, InvalidEvaluation,
    DimensionMismatch, InvalidEmission, UnsupportedStructure, CudaError, OutOfMemory, DeviceTimeout,
    NullArgument, NoDevice]}


def error_for(code: int, message: str = "") -> FagraError:
    cls = BY_CODE.get(int(code), FagraError)
    return cls(message)


def raise_for_status(code: int) -> None:
    if code:
        from ._lib import last_error
        raise error_for(code, f"{BY_CODE.get(int(code), FagraError).__name__}: {last_error()}")
