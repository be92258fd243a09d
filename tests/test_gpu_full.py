"""Full-size parity on the bal1k workload (1,000 cameras, 200,000 points,
1,099,832 observations): LM with the device Schur backend reaches the f64
oracle's final cost (tests/golden/bal1k_oracle.json, the oracle's 20-step
LM run) within 1e-6 relative, and every accepted step's PCG solve meets the
1e-8 reduced-residual bar, for the FP32 two-level form and for the f64
form."""
import json
from pathlib import Path

import pytest

import fagra_b200 as fg
from fagra_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = json.loads((Path(__file__).parent / "golden" / "bal1k_oracle.json").read_text())


@pytest.fixture(scope="module")
def bal1k():
    return synthetic.generate("bal1k")


@pytest.mark.parametrize("form", [dict(precision="f32", coarse_correction=True, tol=1e-8),
                                  dict(precision="f64", coarse_correction=False, tol=1e-10)])
def test_bal1k_lm_reaches_the_oracle_cost_with_every_step_converged(bal1k, form):
    d = bal1k
    assert (d.num_cameras, d.num_points, d.num_observations) == (GOLD["cameras"], GOLD["points"],
                                                                  GOLD["observations"])
    kw = dict(form)
    tol = kw.pop("tol")
    b = fg.Schur(9 * d.num_cameras, 9, 3, **kw)
    b.relative_tolerance = tol
    lm = fg.LevenbergMarquardt(b)
    residuals, costs = [], []

    def seen(s):
        costs.append(s.cost)
        residuals.append(b.diagnostics().reduced_relative_residual)

    lm.on_accept = seen
    out = lm.solve_batch_with_outcome(fg.BalProblem.from_data(d), fg.OptimizeOptions(20, 1e-8, 0.0, 0.0))
    target = GOLD["final_cost"]
    assert abs(out.statistics.cost - target) <= 1e-6 * target, (out.statistics.cost, target)
    assert residuals and max(residuals) < 1e-8, residuals
    # the first accepted costs follow the oracle's trace
    for got, ref in list(zip(costs, GOLD["accepted_costs"]))[:3]:
        assert abs(got - ref) <= 1e-6 * ref, (got, ref)
