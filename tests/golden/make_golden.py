"""Regenerates tests/golden/bal16_oracle.json: the CPU oracle's 20-step LM run
on the bal16 workload (16 cameras, 1,000 points, 4,000 observations) with the
Schur backend at its default controls (CG relative tolerance 1e-10, 1,000
iterations; LM gradient tolerance 1e-8, step and cost tolerances 0).

Run from the repository root: python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from fagra_b200 import synthetic  # noqa: E402


def main():
    d = synthetic.generate("bal16")
    bal = oracle.Bal.from_data(d)
    costs, cgs = [], []

    def seen(s):
        costs.append(s.cost)
        cgs.append(s.linear_iterations)

    code, rep, st = bal.lm(oracle.Schur(9 * d.num_cameras, 9, 3), max_iterations=20, on_accept=seen)
    out = dict(workload="bal16", cameras=d.num_cameras, points=d.num_points, observations=d.num_observations,
               status=code, initial_cost=rep.initial_cost, final_cost=st.cost, accepted_costs=costs, accepted_cg=cgs,
               accepted=st.accepted_steps, rejected=st.rejected_steps, linearizations=st.linearizations,
               cg_iterations=st.linear_iterations, solves=st.linear_solves)
    path = Path(__file__).parent / "bal16_oracle.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps({k: v for k, v in out.items() if not k.startswith("accepted_")}))


if __name__ == "__main__":
    main()
