"""The reference arm of bench.py on CPU: its JSON line keeps the bench
contract (one line, the metric and config of the GPU arm, a timed full oracle
solve as value, cpu_baseline and a zero-copy e2e), loads no product library,
and a non-zero torchrun rank exits 0 without work. The bal16 workload keeps
it to a fraction of a second of oracle time."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(extra_env=None, *args):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "bal16",
                           *args], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_contract_line():
    res = _run(None, "--steps", "2", "--warmup", "1")
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "BA time to 1e-6 relative cost (bal16)"
    assert d["unit"] == "s" and d["higher_is_better"] is False and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] == d["value"] * 1e3
    assert d["config"]["workload"].startswith("bal16: 16 cameras, 1000 points, 4000 observations")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] == 1 and cb["value"] == d["value"]
    assert "one full oracle LM solve to the target" in cb["sample"]
    assert d["e2e"] == dict(value=d["value"], unit="s", h2d_bytes_per_step=0, d2h_bytes_per_step=0)
    assert d["libraries_loaded"] == ["oracle/liboracle.so"]


def test_reference_arm_other_ranks_exit_without_work():
    res = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--steps", "1", "--warmup", "0", "--gpus", "2")
    assert res.returncode == 0, res.stderr[-2000:]
    assert not [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
