"""Ahead-of-time build of libxac.so for sm_100a (in-tree, so the library travels with the sources).

The lattice-Boltzmann kernels are compiled with ``--fmad=false``: every multiply and add is rounded
separately, in the operand order of the reference's kernels, so the FP32 path is reproducible bit for
bit against a CPU restatement compiled the same way.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libxac.so"
BUILD = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"] + ARCH

# (source, extra flags)
UNITS = [
    ("ops_reference_layout.cu", ["--fmad=false"]),
    ("lattice.cu", ["--fmad=false"]),
    ("step_f32.cu", ["--fmad=false"]),
    ("step_f16.cu", ["--fmad=false"]),
    ("step_bf16.cu", ["--fmad=false"]),
    ("step_f32t16.cu", ["--fmad=false"]),
    ("stats_noalloc.cu", ["--fmad=false"]),
    ("conv3d.cu", []),
    ("designs.cu", ["--fmad=false"]),
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libxac.so")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "xac.h"]
    objs, jobs = [], []
    for src, extra in UNITS:
        obj = BUILD / (Path(src).stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [CSRC / src] + headers):
            jobs.append([nvcc, *COMMON, *extra, "-c", str(CSRC / src), "-o", str(obj)])
    # units compile independently: run them side by side
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd), flush=True)
        for f in [ex.submit(subprocess.run, cmd, check=True) for cmd in jobs]:
            f.result()
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
