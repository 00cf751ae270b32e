"""Builds libeafcg.so in-tree for sm_100a with nvcc (no JIT cache).

    python hornofusion-full3d_b200/build.py [--verbose-ptxas] [--force]

Every translation unit under csrc/ is compiled with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the FP64 solver
unit additionally gets ``-fmad=false`` so that its arithmetic is rounded the
way the reference's default (non-FMA) gfortran build rounds it. The CUDA
runtime is linked statically, so the library does not depend on the
runtime version another module of the process (e.g. PyTorch) carries.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libeafcg.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
          "-I", INCLUDE, "-I", CSRC, "--expt-relaxed-constexpr"]
# Per-unit extra flags.
UNITS = {
    "api.cu": [],
    "api_pressure.cu": [],
    "cg_f64.cu": ["-fmad=false"],
    "cg_dsm.cu": ["-fmad=false"],
    "cg_mixed.cu": [],
    "batch.cu": [],
    "noalloc.cu": ["-fmad=false"],
    "serve.cu": [],
    "diag.cu": [],
    "tdma.cu": ["-fmad=false"],
    "pcorr.cu": ["-fmad=false"],
    "multirank.cu": [],
    "assemble.cu": ["-fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc",
                 shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas: bool = False, force: bool = False, quiet: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
               if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "eafcg.h"))
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD_DIR, unit.replace(".cu", ".o"))
        objs.append(obj)
        if not force and not _stale(obj, [src] + headers):
            continue
        cmd = [nvcc()] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        if not quiet:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if not quiet:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    build(args.verbose_ptxas, args.force)
    return 0


if __name__ == "__main__":
    sys.exit(main())
