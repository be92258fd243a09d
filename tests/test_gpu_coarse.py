"""Two-level PCG on the reduced camera system: block-Jacobi plus a coarse
correction on the 7 similarity-gauge directions of bundle adjustment, which the
device BAL problem supplies at every linearization. The step must equal the
one-level PCG step (fagra's Schur, src/schur.rs:204-310) and take fewer
iterations."""
import json
from pathlib import Path

import numpy as np
import pytest

import fagra_b200 as fg
from fagra_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = json.loads((Path(__file__).parent / "golden" / "bal16_oracle.json").read_text())


def _backend(d, **kw):
    b = fg.Schur(9 * d.num_cameras, 9, 3, **kw)
    p = fg.BalProblem.from_data(d)
    b.prepare(p.dimension())
    p.linearize(b)
    b.prepare_damping(1e-6)
    return b


# Both solves meet the reduced-residual tolerance; the gauge components of the
# step are resolved only to that tolerance over the gauge eigenvalues (~2 lambda),
# so the steps agree to ~1e-10 / lambda relative, the predicted reductions
# (blind to the gauge) much closer.
@pytest.mark.parametrize("precision,tol", [("f64", 2e-6), ("f32", 2e-5)])
@pytest.mark.parametrize("name,kw", [("bal16", {}), ("bal1k", dict(cameras=100, points=15000, seed=9))])
def test_coarse_correction_keeps_the_step_and_cuts_iterations(precision, tol, name, kw):
    d = synthetic.generate(name, **kw)
    one = _backend(d, precision=precision)
    two = _backend(d, precision=precision, coarse_correction=True)
    for lam in (1e-4, 1e-2, 1.0):
        a = one.solve_damped(lam)
        da = one.diagnostics()
        b = two.solve_damped(lam)
        db = two.diagnostics()
        assert da.coarse_vectors == 0 and db.coarse_vectors == (7 if lam <= 0.1 else 0)
        assert db.termination == "Converged" and db.reduced_relative_residual < 1e-8
        assert np.linalg.norm(b.delta - a.delta) <= tol * np.linalg.norm(a.delta), lam
        assert abs(b.predicted_reduction - a.predicted_reduction) <= 1e-3 * tol * abs(a.predicted_reduction)
        print(f"{name} {precision} lambda {lam}: iterations {da.iterations} -> {db.iterations}")
        if lam <= 1e-2:
            assert db.iterations < da.iterations


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_lm_with_coarse_correction_reaches_the_oracle_cost(precision):
    d = synthetic.generate("bal16")
    b = fg.Schur(9 * d.num_cameras, 9, 3, precision=precision, coarse_correction=True)
    out = fg.LevenbergMarquardt(b).solve_batch_with_outcome(fg.BalProblem.from_data(d),
                                                            fg.OptimizeOptions(50, 1e-8, 0.0, 0.0))
    assert abs(out.statistics.cost - GOLD["final_cost"]) <= 1e-6 * GOLD["final_cost"]


def test_coarse_correction_without_a_basis_is_one_level():
    from tests import cases
    emissions, J, r = cases.twelve_column_schur_emissions()
    b = fg.Schur(6, 2, 2, coarse_correction=True)
    b.prepare(12)
    b.clear()
    for res, blocks in emissions:
        b.accumulate(res, blocks)
    b.prepare_damping(0.1)
    b.solve_damped(0.01)
    assert b.diagnostics().coarse_vectors == 0


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_single_launch_and_polled_pcg_take_the_same_steps(precision, monkeypatch):
    """A damped solve runs its CG loop as one conditional-graph launch (the
    device decides when to stop); FAGRA_B200_POLLED_GRAPHS at backend creation
    selects the fallback, graphs of 8 iterations polled from the host. Both
    run the same kernels in the same order: the same iterations and the same
    step (FP64 atomic sums may reorder the last bits, which the FP32
    recurrences carry further: 1e-9 / 1e-7 relative, far inside the CG
    tolerance), with different launch counts showing that the two paths ran."""
    d = synthetic.generate("bal1k", cameras=100, points=15000, seed=9)
    one = _backend(d, precision=precision, coarse_correction=True)
    monkeypatch.setenv("FAGRA_B200_POLLED_GRAPHS", "1")
    two = _backend(d, precision=precision, coarse_correction=True)
    monkeypatch.delenv("FAGRA_B200_POLLED_GRAPHS")
    for lam in (1e-4, 1e-2, 1.0):
        l0 = fg.kernel_launches()
        a = one.solve_damped(lam)
        l1 = fg.kernel_launches()
        b = two.solve_damped(lam)
        l2 = fg.kernel_launches()
        da, db = one.diagnostics(), two.diagnostics()
        assert da.termination == db.termination == "Converged"
        assert abs(da.iterations - db.iterations) <= 1, lam
        tol = 1e-9 if precision == "f64" else 1e-7
        assert np.linalg.norm(b.delta - a.delta) <= tol * np.linalg.norm(a.delta), lam
        assert l1 - l0 != l2 - l1, lam
