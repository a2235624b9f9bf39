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

# the mesh's gather and spread variants are spread over several units so that they compile in parallel
SOURCES = ["mesh_gather_ad.cu", "mesh_gather_ik.cu", "mesh_gather_esp.cu", "mesh_gather_ad_join.cu",
           "mesh_gather_ik_join.cu", "mesh_gather_esp_join.cu", "mesh_spread.cu", "cluster_pairs.cu", "cluster_pairs_excl.cu", "ell.cu",
           "batch.cu", "batch_mesh.cu", "mesh.cu", "cluster_list.cu", "md.cu", "noalloc.cu", "mlp.cu", "learned.cu", "ewald.cu",
           "gsd.cpp", "snapshot.cu"]
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


def _compile(src: Path, obj: Path, verbose: bool) -> str:
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
           "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n" + res.stdout + res.stderr)
    return res.stdout + res.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if a source is newer than the shared object.

    Each translation unit is compiled to an object under ``_build/`` in parallel (a unit is
    recompiled when it, a shared header or this script is newer than its object), then the
    objects are linked into the shared library."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + [ROOT / "include" / "pdb200.h", Path(__file__)]
    newest_header = max(p.stat().st_mtime for p in headers if p.exists())
    jobs = []
    for s in SOURCES:
        src, obj = CSRC / s, objdir / (Path(s).stem + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header):
            jobs.append((src, obj))
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for out in ex.map(lambda j: _compile(j[0], j[1], verbose), jobs):
            if verbose and out:
                print(out, file=sys.stderr)
    cuda_lib = Path(nvcc()).resolve().parent.parent / "lib64"
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *[str(objdir / (Path(s).stem + ".o")) for s in SOURCES],
           f"-L{cuda_lib}", "-lcufft", "-Xlinker", f"-rpath,{cuda_lib}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
