"""Builds libadi_b200.so in-tree (next to the Python binding) for sm_100a.

    python cmc-fluid-solver_b200/build_adi.py [--force]

Each .cu is compiled to an object with nvcc (-gencode arch=compute_100a,code=sm_100a),
then linked into one shared library with the CUDA runtime.  Files whose arithmetic
must reproduce the reference's float results bit for bit are compiled with
--fmad=false; host code of every file is compiled with -ffp-contract=off.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "adi_b200", "libadi_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
          f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}", "--expt-relaxed-constexpr"]

# (source, extra flags)
SOURCES = [
    ("adi_api.cu", ["--fmad=false"]),
    ("segments.cu", []),
    ("layer_ops.cu", ["--fmad=false"]),
    ("sweep_exact.cu", ["--fmad=false"]),
    ("sweep_fast.cu", []),
    ("sweep_zwarp.cu", []),
    ("sweep_xytma.cu", []),
    ("sweep_xypair.cu", []),
    ("adjoint.cu", []),
    ("adjoint_fast.cu", []),
    ("adi2d.cu", ["--fmad=false"]),
    ("masks.cu", ["--fmad=false"]),
    ("netcdf_out.cu", []),
]


def _stale(src: str, obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "adi_b200.h"))
    objs = []
    changed = force
    for src, extra in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(s, o, headers):
            cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            changed = True
    if changed or not os.path.exists(OUT):
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True, ptxas_info=a.ptxas_info))
    sys.exit(0)
