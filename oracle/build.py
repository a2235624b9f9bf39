"""Build recipe of the CPU oracle (test infrastructure): oracle/libpd_oracle.so.

The reference (ParticleDynamics.jl) is Julia + CUDA.jl with no C/C++ sources,
so there is no reference library to compile into oracle/_ref; the oracle is the
C restatement in pd_oracle.c, compiled here with OpenMP and without
floating-point contraction (the cluster-list restatement is compared bit for bit).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "pd_oracle.c"
LIB = HERE / "libpd_oracle.so"


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-std=gnu11",
           "-o", str(tmp), str(SRC), "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
