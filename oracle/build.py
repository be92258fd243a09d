"""Build the CPU oracle (test infrastructure): oracle/liboracle.so from oracle.cpp.

The oracle is a plain f64 restatement of fagra's hot path used only as the
checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle.cpp"
OUT = HERE / "liboracle.so"


def build(force: bool = False) -> Path:
    sources = [SRC, *HERE.glob("*.hpp")]
    if not force and OUT.exists() and OUT.stat().st_mtime >= max(p.stat().st_mtime for p in sources):
        return OUT
    # -ffp-contract=off keeps the sequential f64 arithmetic free of fused
    # multiply-adds, like the Rust reference.
    # written next to the target and renamed, so a process that has the old
    # library mapped keeps a consistent file
    tmp = OUT.with_suffix(f".so.{os.getpid()}")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
           str(SRC), "-o", str(tmp)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
