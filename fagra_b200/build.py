"""Build the sm_100a shared library in-tree: fagra_b200/libfagra_b200.so.

Usage: python -m fagra_b200.build [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OUT = HERE / "libfagra_b200.so"
OBJ = HERE / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr", "-I", str(INCLUDE),
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _compile(src: Path, extra: list[str]) -> Path:
    obj = OBJ / (src.stem + ".o")
    deps = [src, *CSRC.glob("*.cuh"), INCLUDE / "fagra_b200.h"]
    if obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(jobs: int | None = None, verbose: bool = False, extra: list[str] | None = None) -> Path:
    OBJ.mkdir(exist_ok=True)
    extra = extra or []
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), srcs))
    if OUT.exists() and all(OUT.stat().st_mtime >= o.stat().st_mtime for o in objs):
        return OUT
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(OUT)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(f"built {OUT}")
    return OUT


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_verbose else []
    build(a.jobs, verbose=True, extra=extra)
    return 0


if __name__ == "__main__":
    sys.exit(main())
