"""Compile the CUDA library in-tree: csrc/*.cu, csrc/*.cpp -> libnuppn_b200.so (sm_100a only).

solver.cu is compiled twice: once with the thread group = the whole CTA (one zone per CTA, namespace
nuppn::cta) and once with the group = one warp (one zone per warp, namespace nuppn::warp). The
objects are compiled in parallel into _build/ and linked with capi.cu and net_host.cpp.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnuppn_b200.so")
# (source, extra defines, object)
UNITS = [("solver.cu", ["-DNUPPN_GROUP_WARP=0"], "solver_cta.o"),
         ("solver.cu", ["-DNUPPN_GROUP_WARP=1"], "solver_warp.o"),
         ("capi.cu", [], "capi.o"),
         ("net_host.cpp", [], "net_host.o"),
         ("netsetup.cpp", [], "netsetup.o"),
         ("output.cpp", [], "output.o"),
         ("tppnp_io.cpp", [], "tppnp_io.o"),
         ("mixing.cu", [], "mixing.o")]
# --fmad=false: products are rounded before they are added, as in the reference's CPU build (x86-64
# without FMA). The Bader-Deuflhard error test of some cooling intervals rests on a cancellation of
# two rounded products of the same factors (a dX/dt term against U(r, c) x(c) in the back
# substitution), which is exact without contraction and leaves a residue of ~1e-16 of the terms
# (far above the abundances involved) with it. Explicit fma() calls are unaffected.
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--fmad=false", "-gencode", "arch=compute_100a,code=sm_100a",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = sorted({os.path.join(CSRC, u[0]) for u in UNITS})
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(HERE, "..", "include", "nuppn.h"))
    deps.append(os.path.abspath(__file__))  # flags
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    os.makedirs(OBJ, exist_ok=True)
    procs = []
    for src, defs, obj in UNITS:
        cmd = [nvcc(), *NVCC_FLAGS, *defs, "-c", "-o", os.path.join(OBJ, obj), src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((cmd, subprocess.Popen(cmd, cwd=CSRC)))
    for cmd, p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", "-o", LIB, *[os.path.join(OBJ, u[2]) for u in UNITS]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
