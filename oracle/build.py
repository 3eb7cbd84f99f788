"""Build recipe for the CPU oracle (test infrastructure).

Compiles oracle/bv_oracle.c with gcc into oracle/_build/libbv_oracle.so.
FP contraction is disabled so that every FP32 expression is evaluated in the
reference's written order; OpenMP parallelises the image loops.

The reference itself (Rust + WGSL, git dependencies not vendored) cannot be
compiled on this machine, so there is no oracle/_ref build.
"""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libbv_oracle.so")
SOURCES = [os.path.join(HERE, "bv_oracle.c")]
CFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
          "-std=c11", "-Wall", "-Wextra"]


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = SOURCES + [os.path.join(HERE, "bv_oracle.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False) -> str:
    if force or stale():
        os.makedirs(OUT_DIR, exist_ok=True)
        tmp = LIB + ".tmp"
        subprocess.check_call(["gcc", *CFLAGS, "-o", tmp, *SOURCES, "-lm"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
