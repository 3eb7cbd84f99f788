"""Build recipe of the CUDA library libbv_b200.so (sm_100a).

    python -m blade_volume_b200.build        # or __graft_entry__.build()

Every .cu file under csrc/ is compiled by nvcc for sm_100a and linked into
blade_volume_b200/libbv_b200.so, in-tree next to this file.  The walk kernels
are compiled with -fmad=false: each FP32/FP64 expression is then the exact
sequence of rounded operations it is written as, which is what makes cell
sequences, t values and colours bit-identical to the CPU restatement.  Host
code is built with -ffp-contract=off for the same reason: the PowerFoam splat
tracer forms its Cech clip planes on the host in the kernel's FP32 order.
"""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libbv_b200.so")
BUILD_DIR = os.path.join(ROOT, "_build", "bv_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
              "-ffp-contract=off", "-fmad=false",
              "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(INCLUDE, "*.h")))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in sources() + headers() + [__file__])


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False,
          out: str = LIB, defines=()) -> str:
    """Compile every csrc/*.cu for sm_100a and link ``out``.  ``defines``
    (e.g. ``["BV_FACE_UNROLL=2"]``) override the kernels' tuning knobs."""
    if out == LIB and not defines and not force and not stale():
        return LIB
    bdir = BUILD_DIR if not defines else BUILD_DIR + "_" + "_".join(
        d.replace("=", "") for d in defines)
    os.makedirs(bdir, exist_ok=True)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    extra += ["-D" + d for d in defines]
    for src in sources():
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-dc" if False else "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = out + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs, "-lcudart_static",
           "-lrt", "-ldl", "-lpthread"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build(force=True, verbose=True, ptxas_info="--ptxas" in sys.argv))
