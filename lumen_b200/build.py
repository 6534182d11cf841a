"""Build liblumen.so (the CUDA kernels and the C interface) in-tree for sm_100a.

``python -m lumen_b200.build`` or ``lumen_b200.build.build()``. Objects go to
lumen_b200/_build/, the library to lumen_b200/liblumen.so. The forward
kernels are compiled with --fmad=false (no fused multiply-add contraction)
so the projection, keys, alpha decisions and transmittance round exactly as
the reference's operation order prescribes. The backward (gradients, held
to a tolerance rather than to bits) is compiled with contraction; the
forward decisions it repeats are written there with explicitly rounded
operations.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblumen.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

SOURCES = ["project.cu", "sort.cu", "composite.cu", "backward.cu", "forward.cu", "capi.cu", "noalloc.cu", "serve.cu", "ply.cu", "train.cu", "depth.cu", "spatial.cu"]

# sources compiled with fused multiply-add contraction
CONTRACTED = {"backward.cu"}

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-I" + os.path.join(ROOT, "include"),
]


def _deps_mtime() -> float:
    m = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    fmad = "--fmad=true" if src in CONTRACTED else "--fmad=false"
    cmd = [NVCC, *NVCC_FLAGS, fmad, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every .cu for sm_100a and link liblumen.so (cudart static)."""
    os.makedirs(BUILD, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps_mtime():
        return LIB
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "static",
           "-o", LIB, *objs, "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
