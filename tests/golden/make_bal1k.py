"""Regenerates tests/golden/bal1k_oracle.json: the CPU oracle's f64 LM run on
the bal1k workload (1,000 cameras, 200,000 points, track length U{3..8}),
Schur backend at default controls (CG tolerance 1e-10, 1,000 iterations),
LM 20 steps, gradient tolerance 1e-8, step/cost tolerances 0. The final cost
is the target of the time-to-1e-6-relative-cost benchmark. Takes tens of
minutes on one core. Run from the repository root."""
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from fagra_b200 import synthetic  # noqa: E402


def main(name="bal1k"):
    d = synthetic.generate(name)
    bal = oracle.Bal.from_data(d)
    trace = []
    t0 = time.time()

    def seen(s):
        trace.append(dict(cost=s.cost, t=time.time() - t0, cg=s.linear_iterations, accepted=s.accepted_steps))
        print(trace[-1], flush=True)

    code, rep, st = bal.lm(oracle.Schur(9 * d.num_cameras, 9, 3), max_iterations=20, on_accept=seen)
    out = dict(workload=name, cameras=d.num_cameras, points=d.num_points, observations=d.num_observations,
               status=code, initial_cost=rep.initial_cost, final_cost=st.cost,
               accepted_costs=[t["cost"] for t in trace], accepted_seconds=[t["t"] for t in trace],
               accepted_cg=[t["cg"] for t in trace],
               accepted=st.accepted_steps, rejected=st.rejected_steps, linearizations=st.linearizations,
               cg_iterations=st.linear_iterations, solves=st.linear_solves, seconds=time.time() - t0, cores=1)
    path = Path(__file__).parent / f"{name}_oracle.json"
    path.write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps({k: v for k, v in out.items() if not k.startswith("accepted_")}))


if __name__ == "__main__":
    main(*sys.argv[1:])
