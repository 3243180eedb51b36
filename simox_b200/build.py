"""Build libsimox_b200.so in-tree with nvcc for sm_100a.

    python -m simox_b200.build          # compile (parallel per translation unit)

The library links cuFFT and the CUDA runtime dynamically (rpath to the CUDA
toolkit), so it loads on any host with the same CUDA 12 toolkit layout.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "libsimox_b200.so")
OBJDIR = os.path.join(ROOT, "_build", "obj")
SOURCES = ["api.cu", "cells.cu", "pair.cu", "pair_half.cu", "pme.cu", "ctip.cu", "integrate.cu", "noalloc.cu", "batch.cu", "adjoint.cu", "oxidation.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def cuda_home() -> str:
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nv = shutil.which("nvcc")
    if nv:
        return os.path.dirname(os.path.dirname(nv))
    raise RuntimeError("nvcc not found")


def _flags(extra=()):
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE,
                   "-I" + CSRC] + list(extra)


def _up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "simox_gpu.h")]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    if not force and _up_to_date():
        return OUT
    ch = cuda_home()
    nvcc = os.path.join(ch, "bin", "nvcc")
    os.makedirs(OBJDIR, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_v else []

    def compile_one(src):
        obj = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        cmd = [nvcc] + _flags(extra) + ["-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return obj, (r.stdout + r.stderr)

    with cf.ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    if verbose or ptxas_v:
        for _, log in results:
            if log.strip():
                print(log)
    objs = [o for o, _ in results]
    lib64 = os.path.join(ch, "lib64")
    tmp = OUT + ".tmp"
    cmd = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs + [
        "-L" + lib64, "-lcufft", "-Xlinker", "-rpath=" + lib64]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="-v" in sys.argv)
    print(OUT)
