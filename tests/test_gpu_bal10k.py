"""Full-size parity on the bal10k workload (10,000 cameras, 2,000,000 points,
7,998,238 observations; track length 2 + geometric with mean 4, so a few
points have more than 32 observations): the FP32 two-level form, whose
operator keeps its camera sums in the global accumulator at this camera
count, reaches the f64 oracle's final cost (tests/golden/bal10k_oracle.json,
the oracle's 20-step LM run) within 1e-6 relative with every accepted step's
reduced residual below 1e-8; and its reduced operator is symmetric and agrees
with the f64-record operator."""
import json
from pathlib import Path

import numpy as np
import pytest

import fagra_b200 as fg
from fagra_b200 import synthetic

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
GOLD_PATH = Path(__file__).parent / "golden" / "bal10k_oracle.json"


@pytest.fixture(scope="module")
def bal10k():
    d = synthetic.generate("bal10k")
    assert (d.num_cameras, d.num_points, d.num_observations) == (10_000, 2_000_000, 7_998_238)
    return d


def test_bal10k_fp32_lm_reaches_the_oracle_cost(bal10k):
    if not GOLD_PATH.exists():
        pytest.skip("tests/golden/bal10k_oracle.json not generated (tests/golden/make_bal1k.py bal10k)")
    GOLD = json.loads(GOLD_PATH.read_text())
    d = bal10k
    b = fg.Schur(9 * d.num_cameras, 9, 3, precision="f32", coarse_correction=True)
    b.relative_tolerance = 1e-8
    lm = fg.LevenbergMarquardt(b)
    residuals, costs = [], []

    def seen(s):
        costs.append(s.cost)
        residuals.append(b.diagnostics().reduced_relative_residual)

    lm.on_accept = seen
    lm.solve_batch_with_outcome(fg.BalProblem.from_data(d), fg.OptimizeOptions(50, 1e-8, 0.0, 0.0))
    target = GOLD["final_cost"]
    assert min(costs) <= target * (1 + 1e-6), (min(costs), target)
    assert residuals and max(residuals) < 1e-8, max(residuals)
    for got, ref in list(zip(costs, GOLD["accepted_costs"]))[:2]:
        assert abs(got - ref) <= 1e-6 * ref, (got, ref)


def test_bal10k_operator_symmetric_and_matches_f64_records(bal10k):
    d = bal10k
    p = fg.BalProblem.from_data(d)
    ops = {}
    for prec in ("f32", "f64"):
        b = fg.Schur(9 * d.num_cameras, 9, 3, precision=prec)
        b.prepare(p.dimension())
        p.linearize(b)
        b.prepare_damping(1e-6)
        ops[prec] = b
    rng = np.random.default_rng(17)
    x, y = rng.normal(size=9 * d.num_cameras), rng.normal(size=9 * d.num_cameras)
    sx, sy = ops["f32"].reduced_apply(1e-3, x), ops["f32"].reduced_apply(1e-3, y)
    assert abs(x @ sy - y @ sx) <= 1e-5 * abs(x @ sy)
    ref = ops["f64"].reduced_apply(1e-3, x)
    assert np.linalg.norm(sx - ref) <= 2e-5 * np.linalg.norm(ref)
