"""Builds libwindfvm.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python -m unitywindsimulation_b200.build
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
SOURCES = ["wf_api.cu", "wf_kernels.cu", "wf_sweeps.cu", "wf_batch.cu", "wf_noalloc.cu", "wf_adjoint.cu", "wf_nested.cu", "wf_export.cu", "wf_raster.cu", "wf_nonuniform.cu", "wf_pres_tma.cu", "wf_vel_tma.cu"]
HEADERS = ["wf_common.cuh", "wf_kernels.cuh", "wf_solver.cuh", "wf_sweeps.cuh", "wf_tma.cuh", "wf_gridbar.cuh"]
OUT = os.path.join(HERE, "libwindfvm.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "windfvm.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    cmd = [nvcc_path(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", OUT, *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
