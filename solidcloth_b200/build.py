"""Build libsolidcloth_b200.so (sm_100a) in-tree with nvcc.

    python -m solidcloth_b200.build

The kernels are compiled with -fmad=false and IEEE division/square root
(nvcc's defaults without --use_fast_math) so their arithmetic follows the
reference's operation order; host code with -ffp-contract=off for the same
reason. solver_fast.cu, the fast build of the solver (csrc/solver.cuh), is the
one exception: FMA contraction and approximate division / square root.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libsolidcloth_b200.so"
SOURCES = ["step_kernels.cu", "solver_fast.cu", "cloth.cu", "capi.cu", "noalloc.cu", "render.cu"]
# per-source replacements of the default numerics flags
FAST = {"solver_fast.cu": ["-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--extended-lambda",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden", "-ccbin", "g++"]


def nvcc() -> str:
    cand = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def build(verbose: bool = False, ptxas_v: bool = False) -> Path:
    LIBDIR.mkdir(exist_ok=True)
    objs = []
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [PKG.parent / "include" / "solidcloth_b200.h"]
    hdr_time = max(h.stat().st_mtime for h in headers)
    for src in SOURCES:
        s = CSRC / src
        o = LIBDIR / (s.stem + ".o")
        if not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hdr_time):
            flags = [f for f in FLAGS if not (src in FAST and f == "-fmad=false")] + FAST.get(src, [])
            cmd = [nvcc(), *ARCH, *flags, "-c", str(s), "-o", str(o)]
            if ptxas_v:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        objs.append(str(o))
    if not LIB.exists() or LIB.stat().st_mtime < max(Path(o).stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_v="-v" in sys.argv)
    print(LIB)
