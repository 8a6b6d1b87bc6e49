"""Builds the CPU oracle (test infrastructure) into oracle/libodevec_oracle.so.

gcc -O2 -ffp-contract=off: no floating-point contraction, so every product and
sum is a separately rounded IEEE operation, as in the CUDA kernels built with
--fmad=false.  OpenMP parallelises over groups of cells.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "odevec_oracle.c")
LIB = os.path.join(HERE, "libodevec_oracle.so")


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [SRC, os.path.join(HERE, "..", "include", "odevec_b200.h")]
    gen = os.path.join(HERE, "..", "odevec_b200", "csrc")
    for root, _, files in os.walk(gen):
        deps += [os.path.join(root, f) for f in files if f.endswith((".h", ".inc"))]
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps)):
        return LIB
    cmd = ["gcc", "-std=gnu11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-fopenmp", "-Wall", "-Wno-unused-function", "-Wno-unused-variable", "-o", LIB + ".tmp",
           SRC, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
