"""The C-ABI library loads, exports every symbol include/fagra_b200.h declares,
and fails loudly (no CPU fallback) when no CUDA device is present."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "fagra_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"FG_API\s+[\w\s\*]+?\b(fg_\w+)\s*\(", text)))


def test_header_declares_the_backend_trait():
    names = declared_functions()
    for required in ["fg_schur_create", "fg_backend_prepare", "fg_backend_clear", "fg_backend_accumulate",
                     "fg_backend_gradient_norm", "fg_backend_solve", "fg_backend_prepare_damping",
                     "fg_backend_solve_damped", "fg_backend_linear_solve_work", "fg_lm_solve_bal",
                     "fg_bal_linearize"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    import fagra_b200
    lib = ctypes.CDLL(str(fagra_b200.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol():
    from fagra_b200 import _lib
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_no_cpu_fallback_without_a_device():
    import fagra_b200
    if fagra_b200.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(fagra_b200.NoDevice):
        fagra_b200.Schur(9, 9, 3)


def test_default_options_match_the_reference():
    # src/schur.rs:155-158, src/optimization.rs:57-67, levenberg_marquardt.rs:35-46
    from fagra_b200 import _lib
    o = _lib.SchurOptions()
    _lib.lib.fg_schur_default_options(ctypes.byref(o))
    assert o.max_iterations == 1000 and o.relative_tolerance == 1e-10
    oo = _lib.OptimizeOptionsC()
    _lib.lib.fg_optimize_default_options(ctypes.byref(oo))
    assert (oo.max_iterations, oo.gradient_tolerance, oo.step_tolerance, oo.cost_tolerance) == (50, 1e-8, 1e-10,
                                                                                                  1e-12)
    lo = _lib.LmOptionsC()
    _lib.lib.fg_lm_default_options(ctypes.byref(lo))
    assert (lo.initial_damping, lo.min_damping, lo.max_damping, lo.min_column_norm, lo.acceptance_threshold,
            lo.max_trials) == (1e-3, 1e-12, 1e12, 1e-6, 1e-4, 16)
