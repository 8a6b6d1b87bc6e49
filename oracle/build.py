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
LIB_LIBM = os.path.join(HERE, "libodevec_oracle_libm.so")


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _cpu_tag() -> str:
    """identifies the host CPU (model and instruction-set flags) so that a
    -march=native build is never loaded on another kind of CPU"""
    import hashlib
    flags = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                flags = line
                break
    except OSError:
        pass
    return hashlib.sha1((cpu_model() + flags).encode()).hexdigest()[:10]


def fast_lib_path() -> str:
    return os.path.join(HERE, "libodevec_oracle_fast_%s.so" % _cpu_tag())


def build(force: bool = False, verbose: bool = False, libm: bool = False, fast: bool = False) -> str:
    """libm: the variant whose exp/log/log10/pow are the C library's (-DOV_LIBM),
    compared bit for bit with runs of the reference's own solver module.
    fast: the CPU baseline's build, -O3 -march=native with floating-point
    contraction allowed (not bit-identical to the GPU kernels); built on the
    host that loads it."""
    lib = LIB_LIBM if libm else (fast_lib_path() if fast else LIB)
    deps = [SRC, os.path.join(HERE, "..", "include", "odevec_b200.h")]
    gen = os.path.join(HERE, "..", "odevec_b200", "csrc")
    for root, _, files in os.walk(gen):
        deps += [os.path.join(root, f) for f in files if f.endswith((".h", ".inc"))]
    if (not force and os.path.exists(lib)
            and os.path.getmtime(lib) >= max(os.path.getmtime(d) for d in deps)):
        return lib
    opt = ["-O3", "-march=native", "-ffp-contract=fast"] if fast else ["-O2", "-ffp-contract=off"]
    cmd = ["gcc", "-std=gnu11"] + opt + ["-fno-fast-math", "-fPIC", "-shared",
           "-fopenmp", "-Wall", "-Wno-unused-function", "-Wno-unused-variable", "-o", lib + ".tmp",
           SRC, "-lm"] + (["-DOV_LIBM"] if libm else [])
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    print(build(force="--force" in sys.argv, verbose=True, libm=True))
