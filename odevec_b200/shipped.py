"""The network variants compiled into the library by default.

Each entry is a preprocessor command line (the reference's flags).  The
defaults follow the reference drivers: ROBER with nvector=32 lockstep and
dt_min=1e-20 (``tests/rober.f90:44``), OREGO per cell with the default
dt_min, PRIMORDIAL per cell with dt_min=1e-20 (``tests/primordial.f90:45``)
in dense, FF- and CMK-ordered CSC packaging, the symbolic-LU and
difference-quotient Jacobian methods on dense variants, the synthetic
64-species network read from a KROME-format dump, and a toy KROME-layout
network with the heating/cooling temperature equation (--heatcool=1).
"""
import os

from . import pre_odevec

HERE = os.path.dirname(os.path.abspath(__file__))
SYN64_DUMP = os.path.join(HERE, "data", "syn64_krome.py")
HCTOY_DUMP = os.path.join(HERE, "data", "hctoy_krome.py")

SHIPPED = [
    ["--example=ROBER", "--packaging=DENSE", "--nvector=32", "--dt_min=1e-20"],
    ["--example=ROBER", "--packaging=CSC", "--nvector=32", "--dt_min=1e-20"],
    ["--example=OREGO", "--packaging=CSC", "--ordering=CMK", "--nvector=1"],
    ["--example=OREGO", "--packaging=DENSE", "--nvector=1"],
    ["--example=PRIMORDIAL", "--packaging=DENSE", "--nvector=1", "--dt_min=1e-20"],
    ["--example=PRIMORDIAL", "--packaging=CSC", "--ordering=FF", "--nvector=1", "--dt_min=1e-20"],
    ["--example=PRIMORDIAL", "--packaging=CSC", "--ordering=CMK", "--nvector=1", "--dt_min=1e-20"],
    # the reference's other two Jacobian methods: the symbolic LU (LUmethod 2,
    # tractable for the small networks) and difference quotients (LUmethod 3)
    ["--example=ROBER", "--packaging=DENSE", "--nvector=32", "--dt_min=1e-20", "--LUmethod=2"],
    ["--example=OREGO", "--packaging=DENSE", "--nvector=1", "--LUmethod=2"],
    ["--example=ROBER", "--packaging=DENSE", "--nvector=32", "--dt_min=1e-20", "--LUmethod=3"],
    ["--example=PRIMORDIAL", "--packaging=DENSE", "--nvector=1", "--dt_min=1e-20", "--LUmethod=3"],
]


def emit_all(outdir: str = pre_odevec.GEN_DIR, quiet: bool = True):
    import contextlib
    import io
    os.makedirs(outdir, exist_ok=True)
    systems = []
    krome = [["--krome_setupfile=" + SYN64_DUMP, "--name=SYN64", "--packaging=CSC",
              "--ordering=CMK", "--nvector=1", "--dt_min=1e-20"],
             # the heating/cooling temperature equation (--heatcool=1) on a
             # toy network with toy heating and cooling laws
             ["--krome_setupfile=" + HCTOY_DUMP, "--name=HCTOY", "--packaging=DENSE", "--nvector=1",
              "--dt_min=1e-20", "--heatcool=1", "--heatcool_header=heatcool_hctoy.h"]]
    for argv in SHIPPED + krome:
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf) if quiet else contextlib.nullcontext():
            systems.append(pre_odevec.main(argv + ["--outdir=" + outdir]))
    return systems


if __name__ == "__main__":
    for s in emit_all(quiet=False):
        print(s.tag, "nnz", s.nnz)
