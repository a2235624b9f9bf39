"""Build libpdb200.so (CUDA, sm_100a) next to this file.

The library is compiled directly with nvcc for ``sm_100a`` only; the result is
an in-tree shared object that the Python host side loads with ctypes (and that
Julia host code would ``ccall``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libpdb200.so"
ROOT = HERE.parent

SOURCES = ["cluster_list.cu", "cluster_pairs.cu", "mesh.cu", "md.cu", "noalloc.cu", "ell.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libpdb200")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp"))
    deps.append(ROOT / "include" / "pdb200.h")
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if a source is newer than the shared object."""
    if not force and not _stale():
        return LIB
    cuda_lib = Path(nvcc()).resolve().parent.parent / "lib64"
    cmd = [
        nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
        "-Xcompiler", "-O2", "-o", str(LIB), *[str(CSRC / s) for s in SOURCES],
        f"-L{cuda_lib}", "-lcufft", "-Xlinker", f"-rpath,{cuda_lib}",
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    tmp = LIB.with_suffix(".so.tmp")
    cmd[cmd.index(str(LIB))] = str(tmp)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stdout + res.stderr, file=sys.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
