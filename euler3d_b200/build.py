"""Build recipe of the euler3d_b200 shared library (sm_100a) with nvcc, in-tree.

``python -m euler3d_b200.build`` (or ``build()``) compiles ``csrc/*`` into
``euler3d_b200/libeuler3d_b200.so``.  The CUDA translation units are compiled
with ``-fmad=false`` so that no multiply-add is contracted behind the source's back: the exact
mode rounds as the reference's source order does, and the FP64 mode fuses only where its source
says ``fma()``, so every kernel variant computes the same bits whatever its register budget.  Host
code is compiled with ``-ffp-contract=off`` for the same reason.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD_DIR = os.path.join(HERE, "_build")
LIB_NAME = "libeuler3d_b200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", f"-I{INCLUDE}", f"-I{CSRC}",
          "--expt-relaxed-constexpr"]
# (source, extra flags)
SOURCES = [
    ("stage_exact.cu", ["-fmad=false"]),
    ("stage_fast.cu", ["-fmad=false"]),
    ("stage_f32.cu", ["-fmad=false"]),
    ("solver.cu", ["-fmad=false"]),
    ("batch.cu", ["-fmad=false"]),
    ("outputs.cu", ["-fmad=false"]),
    ("capi.cpp", []),
    ("mesh_prep.cpp", []),
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _needs(obj: str, deps: List[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "euler3d_b200.h"))
    objs = []
    for src, extra in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src + ".o")
        objs.append(obj)
        if not _needs(obj, [path, __file__] + headers) and not ptxas_info:
            continue
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", path, "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if ptxas_info and r.stderr:
            print(r.stderr, file=sys.stderr)
    if _needs(LIB_PATH, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB_PATH, *objs, "-Xcompiler", "-pthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
