"""Build recipe for the oracle's C core (test infrastructure only).

Compiles oracle/cimx_oracle.c into oracle/_lib/libcimx_oracle.so with gcc,
-ffp-contract=off (only the explicit fmaf()/fma() calls fuse) and OpenMP.
The cuCIM reference itself cannot be compiled into a CPU library: its
kernels are CUDA C strings generated at run time by CuPy, so there is no
oracle/_ref build.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cimx_oracle.c")
OUT_DIR = os.path.join(HERE, "_lib")
OUT = os.path.join(OUT_DIR, "libcimx_oracle.so")


def build(force=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    if (
        not force
        and os.path.exists(OUT)
        and os.path.getmtime(OUT) >= os.path.getmtime(SRC)
    ):
        return OUT
    cmd = [
        "gcc",
        "-O3",
        "-fPIC",
        "-shared",
        "-ffp-contract=off",
        "-fno-fast-math",
        "-fopenmp",
        "-o",
        OUT,
        SRC,
        "-lm",
    ]
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
