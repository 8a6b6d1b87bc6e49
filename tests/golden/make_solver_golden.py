#!/usr/bin/env python
"""Generates tests/golden/ref_solver.json: outputs of the reference's own
solver module on seeded inputs.

Run in a container where the reference sources are mounted (read-only) at
``REF`` (default /root/reference); the GPU machines never run this script,
they only read the JSON it writes.

For every case:

1. the reference's ``pre_odevec.py`` (in a shimmed temporary copy, see
   make_golden.py) writes ``build/odevec.f90`` and ``build/odevec_commons.f90``
   for the case's example, packaging, ordering, LU method and ``--nvector``;
2. ``f90py`` translates those two generated modules, statement by statement,
   into Python/NumPy with gfortran -O2 semantics (the C library's
   exp/log/pow, IEEE binary64/binary32 arithmetic, no contraction), with
   ``HAVE_COEFFICIENTS`` defined for networks with rate coefficients, as the
   reference's CI builds them (``.gitlab-ci.yml:15``);
3. a driver calls the translated ``InitOdevec`` and ``SolveODE`` the way the
   reference's test programs do (``tests/rober.f90:41-62``,
   ``tests/orego.f90:42-58``, ``tests/primordial.f90:43-92``: a ladder of
   ``t_stop`` values on one solver object, time carried, ``dt`` reset or
   carried, mass fractions converted around each call), on seeded cells
   instead of the programs' one fixed state, with the drivers' Fortran
   literal kinds (``1e11``, ``0.01``, ``1e-10``, ``2.2954626201190183E-026``
   are single precision);
4. after every call the state ``y``, ``time``, ``dt`` and eight counters are
   recorded: accepted steps (calls of SolveLinearSystem), predictor attempts
   (calls of PredictSolution), error-test failures and Newton failures (the
   statements that increment FailedErrorTests / FailedCorrections), Newton
   iterations (calls of CalcResiduum), Jacobian evaluations (the statement
   ``this%UpdateJac = .false.``), the final order, and the Nordsieck passes
   of PredictSolution and ResetSystem (order*(order+1)/2 per call).

Only numbers are written (hex floats), never the generated or translated
source.  Usage: ``python tests/golden/make_solver_golden.py [REF] [case ...]``.
"""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import f90py as F  # noqa: E402
import make_golden as MG  # noqa: E402

REF = "/root/reference"
OUT = os.path.join(HERE, "ref_solver.json")


def f32(x):
    """a Fortran default-real literal, widened to double"""
    return np.float64(F._f32_literal(x if isinstance(x, str) else repr(float(x))))


PROBES = {"lte": ("solvelinearsystem", "this%FailedErrorTests = this%FailedErrorTests + 1"),
          "conv": ("solvelinearsystem", "this%FailedCorrections = this%FailedCorrections + 1"),
          "jac": ("solvelinearsystem", "this%UpdateJac = .false.")}


# --------------------------------------------------------------------- inputs
def rober_ladder():
    """tests/rober.f90:47-62: t_stop = 1e-10, *10 while below the real
    literal 1e11; dt = 1d-10 before each call; rtol = 10**(-2-24/4)."""
    ts, t = [], np.float64(1e-10)
    while t < f32("1e11"):
        ts.append(t)
        t = t * np.float64(10.0)
    rtol = np.float64(F._libm_pow(10.0, float(np.float64(-2.0) - np.float64(24) * np.float64(0.25))))
    return ts, rtol, np.float64(1e-6) * rtol


def rober_cells(n, seed):
    """seeded ROBER states: y1 ~ U(0.9, 1), y2 = 0, y3 = 1 - y1"""
    rng = np.random.default_rng(seed)
    y1 = rng.uniform(0.9, 1.0, n)
    y = np.zeros((3, n))
    y[0] = y1
    y[2] = 1.0 - y1
    return y


def orego_ladder(ncalls):
    """tests/orego.f90:44-58: t_stop = 1.0, + the real literal 0.01 while not
    above 360.0 (the first ncalls of them); dt = 1d-10 before each call;
    rtol = 10**(-2-32/4)."""
    ts, t = [], np.float64(1.0)
    while t <= f32("360.0") and len(ts) < ncalls:
        ts.append(t)
        t = t + f32("0.01")
    rtol = np.float64(F._libm_pow(10.0, float(np.float64(-2.0) - np.float64(32) * np.float64(0.25))))
    return ts, rtol, np.float64(1e-6) * rtol


def orego_cells(n, seed):
    """(1, 2, 3), each component scaled by 10^U(log10 0.9, log10 1.1)"""
    rng = np.random.default_rng(seed)
    base = np.array([1.0, 2.0, 3.0])[:, None]
    return base * 10.0 ** rng.uniform(np.log10(0.9), np.log10(1.1), (3, n))


# PRIMORDIAL: the reference driver's inverse masses and masses of the 12
# chemical species (tests/primordial.f90:145-210)
PRIM_IMASS = [1.09776932527e+27, 5.9721335838e+23, 5.97538433901e+23, 1.49430705554e+23,
              2.9876921695e+23, 2.98861411108e+23, 1.99220448934e+23, 5.97863863505e+23,
              1.4945104915e+23, 2.98850552203e+23, 2.98942796572e+23, 1.49471398286e+23]
PRIM_MASS = [9.10938188e-28, 1.67444345638e-24, 1.67353251819e-24, 6.69206503638e-24,
             3.34706503638e-24, 3.34603251819e-24, 5.01956503638e-24, 1.67262158e-24,
             6.69115409819e-24, 3.34615409819e-24, 3.34512158e-24, 6.69024316e-24]


def primordial_x0():
    """tests/primordial.f90:48-68: single-precision literals, normalised by
    the (sequential) sum of the 12 mass fractions."""
    x = np.full(12, f32("1e-20"))
    vals = {3: "0.75615", 1: "4.46406e-8", 8: "8.1967e-5", 6: "1.0e-40", 11: "1.0e-40", 4: "0.24375",
            9: "1.0e-40", 10: "1.0e-40", 5: "1.5123e-6", 7: "1.0e-40", 2: "1.0e-40", 12: "1.0e-40"}
    for i, v in vals.items():
        x[i - 1] = f32(v)
    return x / F._sum(x)


def x2n(x, rho):
    """krome_x2n (tests/primordial.f90:128-138): rhogas * x(:) * imass"""
    return rho * x * np.array(PRIM_IMASS)


def n2x(n, rho):
    """krome_n2x (tests/primordial.f90:113-122): n(:) * mass / rhogas"""
    return n[:12] * np.array(PRIM_MASS) / rho


def primordial_bench_cells(n, seed):
    """cells of the PRIMORDIAL bench workload's distributions, with Tgas at
    the reference's fixed 1000 K"""
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from odevec_b200 import workloads as W
    wl = W.primordial(ncells=n, seed=seed)
    y = wl.y.copy()
    y[14] = 1000.0
    return y, wl.t_stop, wl.dt0, wl.rtol, wl.atol, wl.dt_min


# --------------------------------------------------------------------- driver
class Case:
    def __init__(self, name, tag, ex, pack, order, lum, nvector, runs, defines=(), check_neg=False,
                 krome=None):
        self.name, self.tag, self.ex, self.pack, self.order = name, tag, ex, pack, order
        self.lum, self.nvector, self.runs, self.defines = lum, nvector, runs, defines
        self.check_neg = check_neg
        self.krome = krome      # KROME dump for --heatcool=1 cases


# heating and cooling of the HCTOY test network as Fortran functions with
# KROME's interfaces (heating(n, Tgas, k, nH2dust), cooling(n, Tgas)); the
# same laws, in the same operation order, as odevec_b200/csrc/heatcool_hctoy.h
HCTOY_FORTRAN = """
module hctoy_heatcool
contains
  function heating(y, Tgas, k, nh2dust)
    implicit none
    double precision, dimension(:,:) :: y, k
    double precision, dimension(:) :: Tgas, nh2dust
    double precision, dimension(size(y,1)) :: heating
    heating = 1.0d-25*(y(:,3) + y(:,4) + y(:,5))
  end function heating
  function cooling(y, Tgas)
    implicit none
    double precision, dimension(:,:) :: y
    double precision, dimension(:) :: Tgas
    double precision, dimension(size(y,1)) :: cooling
    cooling = 1.0d-23*y(:,1)*y(:,2)*sqrt(Tgas) + 2.0d-24*y(:,4)*Tgas
  end function cooling
end module hctoy_heatcool
"""


def krome_shim(commons, neq):
    """The reference's --heatcool=1 output is a fragment for KROME's build
    (pre_odevec.py:148-190, 556-561): it calls KROME's heating/cooling and
    uses krome_gamma, boltzmann_erg, nmols, Tgas, nH2dust, yy, dyy, dy, dy0,
    dy1 without declaring them, leaves #KROME_ placeholders for KROME's
    preprocessor, and its template has no #ODEVEC_DY0 line to compute dy0.
    This supplies that context the way KROME does and changes nothing the
    reference wrote: the placeholders are dropped (no quench, no floor);
    krome_gamma -> 5/3, boltzmann_erg -> 1.380648d-16, nmols -> neq-4;
    Tgas = y(:,neq-1) and nH2dust = 0 at the entry of GetRHS and GetJac; the
    scratch arrays are declared in GetJac, and dy0 = the heating/cooling term
    of y (the reference's own Tgas right-hand side) before the Jacobian."""
    c = commons.replace("#KROME_coolingQuench #KROME_coolfloor", "")
    c = c.replace("krome_gamma(:)", "(5d0/3d0)").replace("boltzmann_erg", "1.380648d-16")
    c = c.replace("y(:,1:nmols)", "y(:,1:%d)" % (neq - 4))
    # the generated Tgas right-hand side, joined, as the dy0 statement
    joined = re.sub(r"&\s*\n\s*", "", c)
    m = re.search(r"rhs\(:,%d\) = (.*)\n" % (neq - 1), joined)
    dy0 = "      dy0(:) = " + m.group(1).strip() + "\n"
    out = []
    sub = None
    for line in c.split("\n"):
        ms = re.match(r"\s*subroutine\s+(\w+)", line, re.I)
        if ms:
            sub = ms.group(1).lower()
        st = line.strip().lower()
        if sub in ("getrhs", "getjac") and st == "#ifdef have_coefficients":
            out.append("    double precision, dimension(this%nvector) :: Tgas, nH2dust")
            if sub == "getjac":
                out.append("    double precision, dimension(this%nvector) :: dyy, dy0, dy1")
                out.append("    double precision, dimension(this%nvector,this%neq) :: yy, dy")
        out.append(line)
        if sub in ("getrhs", "getjac") and st == "#endif":
            out.append("      Tgas(:) = y(:,%d)" % (neq - 1))
            out.append("      nH2dust(:) = 0d0")
            if sub == "getjac":
                out.append(dy0.rstrip("\n"))
            sub = None
    return "\n".join(out)


def translate_case(work, case):
    if case.krome:
        cmd = [sys.executable, "pre_odevec.py", "--nvector=%d" % case.nvector,
               "--krome_setupfile=%s" % case.krome, "--heatcool=1",
               "--packaging=%s" % case.pack, "--ordering=%s" % case.order, "--LUmethod=%d" % case.lum]
    else:
        cmd = [sys.executable, "pre_odevec.py", "--nvector=%d" % case.nvector, "--example=%s" % case.ex,
               "--packaging=%s" % case.pack, "--ordering=%s" % case.order, "--LUmethod=%d" % case.lum]
    subprocess.run(cmd, cwd=work, capture_output=True, text=True, check=True)
    b = os.path.join(work, "build")
    srcs = [open(os.path.join(b, "odevec.f90")).read(), open(os.path.join(b, "odevec_commons.f90")).read()]
    if case.krome:
        neq = int(re.search(r"integer :: neq=(\d+)", srcs[0]).group(1))
        srcs = [srcs[0], HCTOY_FORTRAN, krome_shim(srcs[1], neq)]
    _, ns = F.translate(srcs, defines=case.defines, probes=PROBES)
    return ns


def hexs(a):
    return [float(v).hex() for v in np.asarray(a, dtype=np.float64).ravel()]


def run_ladder(ns, case, run):
    """One solver object of nvector cells through a ladder of SolveODE calls.
    run: dict(y0 (neq, nvector), t0, dt0, t_stops, dt_reset|None, rtol, atol,
    dt_min|None, rho|None (then y0 holds mass fractions), masks|None)"""
    ode = ns["T_odevec"]()
    ns["p_initodevec"](ode)
    ode.relativetolerance = np.float64(run["rtol"])
    ode.absolutetolerance = np.float64(run["atol"])
    if run.get("dt_min") is not None:
        ode.minimaltimestep = np.float64(run["dt_min"])
    dt_min = ode.minimaltimestep
    ode.checknegatives = bool(case.check_neg)
    neq = ode.neq
    rho = run.get("rho")
    x = None
    if rho is not None:
        x = np.array(run["y0"], dtype=np.float64)
        ode.y.a[:, :] = 0.0
        ode.y.a[:, 14] = 1000.0      # Tgas row: passive, the reference's coe() fixes 1000 K
    else:
        ode.y.a[:, :] = np.asarray(run["y0"], dtype=np.float64).T
    t = F.Ref(np.float64(run["t0"]))
    dt = F.Ref(np.float64(run["dt0"]))
    pp = {"n": 0}

    def hook(fr):
        pp["n"] += fr["v_this"].order * (fr["v_this"].order + 1) // 2
    F.HOOKS["predictsolution"] = hook
    F.HOOKS["resetsystem"] = hook
    calls = []
    for k, ts in enumerate(run["t_stops"]):
        if run.get("dt_reset") is not None:
            dt.v = np.float64(run["dt_reset"])
        if rho is not None:
            for i in range(case.nvector):
                ode.y.a[i, :12] = x2n(x[:12, i], rho[i])
        y_in = ode.y.a.T.copy()
        dt_in, t_in = dt.v, t.v
        mask = None
        if run.get("masks") is not None and run["masks"][k] is not None:
            mask = F.FArray(np.asarray(run["masks"][k], dtype=bool))
        F.reset_counters()
        pp["n"] = 0
        try:
            ns["p_solveode"](ode, t, dt, F.Ref(np.float64(ts)), ode.y, ns["p_getrhs"], ns["p_getjac"],
                             ns["p_getlu"], mask)
            stopped = ""
        except F.FortranStop:
            stopped = F.PRINTED[-1] if F.PRINTED else "stop"
        rec = {"t_stop": float(ts).hex(), "t_in": float(t_in).hex(), "dt_in": float(dt_in).hex(),
               "y_in": hexs(y_in), "y": hexs(ode.y.a.T), "t": float(t.v).hex(), "dt": float(dt.v).hex(),
               "stats": [F.CALLS.get("solvelinearsystem", 0), F.CALLS.get("predictsolution", 0),
                         F.HITS.get("lte", 0), F.HITS.get("conv", 0), F.CALLS.get("calcresiduum", 0),
                         F.HITS.get("jac", 0), int(ode.order), pp["n"]]}
        if mask is not None:
            rec["mask"] = [int(v) for v in mask.a]
        if stopped:
            rec["stopped"] = stopped
        calls.append(rec)
        if stopped:
            break
        if rho is not None:
            for i in range(case.nvector):
                x[:12, i] = n2x(ode.y.a[i, :], rho[i])
    return {"neq": int(neq), "nvector": case.nvector, "rtol": float(run["rtol"]).hex(),
            "atol": float(run["atol"]).hex(), "dt_min": float(dt_min).hex(),
            "dt_reset": None if run.get("dt_reset") is None else float(run["dt_reset"]).hex(),
            "rho": None if rho is None else hexs(rho), "calls": calls}


def cases():
    rts, rrtol, ratol = rober_ladder()
    C = []
    rober_run = {"y0": rober_cells(32, 5), "t0": 0.0, "dt0": 1e-5, "t_stops": rts, "dt_reset": 1e-10,
                 "rtol": rrtol, "atol": ratol, "dt_min": 1e-20}
    # masked calls: the first three calls leave cells 3, 17 and 30 out
    masks = [None] * len(rts)
    m = np.ones(32, bool)
    m[[3, 17, 30]] = False
    for k in range(3):
        masks[k] = m
    C.append(Case("rober_dense", "ROBER_DENSE_NONE", "ROBER", "DENSE", "None", 1, 32, [rober_run]))
    C.append(Case("rober_dense_masked", "ROBER_DENSE_NONE", "ROBER", "DENSE", "None", 1, 32,
                  [dict(rober_run, masks=masks, t_stops=rts[:8])]))
    C.append(Case("rober_csc", "ROBER_CSC_NONE", "ROBER", "CSC", "None", 1, 32, [rober_run]))
    C.append(Case("rober_lu2", "ROBER_DENSE_NONE_LU2", "ROBER", "DENSE", "None", 2, 32, [rober_run]))
    C.append(Case("rober_lu3", "ROBER_DENSE_NONE_LU3", "ROBER", "DENSE", "None", 3, 32, [rober_run]))
    # CheckNegatives at a loose tolerance, where predictions go negative
    loose = {"y0": rober_cells(32, 6), "t0": 0.0, "dt0": 1e-5, "t_stops": rts, "dt_reset": 1e-10,
             "rtol": 1e-3, "atol": 1e-9, "dt_min": 1e-20}
    C.append(Case("rober_checkneg", "ROBER_DENSE_NONE", "ROBER", "DENSE", "None", 1, 32, [loose],
                  check_neg=True))
    ots, ortol, oatol = orego_ladder(120)
    y = orego_cells(2, 7)
    orego_runs = [{"y0": y[:, i:i + 1], "t0": 0.0, "dt0": 1e-10, "t_stops": ots, "dt_reset": 1e-10,
                   "rtol": ortol, "atol": oatol} for i in range(2)]
    C.append(Case("orego_dense_ladder", "OREGO_DENSE_NONE", "OREGO", "DENSE", "None", 1, 1, orego_runs))
    # the OREGO workload: single solves to t_end ~ U(30, 360), rtol 1e-6, atol 1e-10
    rng = np.random.default_rng(8)
    y = orego_cells(6, 9)
    tends = rng.uniform(30.0, 360.0, 6)
    single = [{"y0": y[:, i:i + 1], "t0": 0.0, "dt0": 1e-10, "t_stops": [tends[i]], "dt_reset": None,
               "rtol": 1e-6, "atol": 1e-10} for i in range(6)]
    C.append(Case("orego_csc_cmk", "OREGO_CSC_CMK", "OREGO", "CSC", "CMK", 1, 1, single))
    C.append(Case("orego_lu2", "OREGO_DENSE_NONE_LU2", "OREGO", "DENSE", "None", 2, 1, single[:3]))
    # PRIMORDIAL: the driver's ladder (mass fractions, 1e8 s steps to 1e10)
    pts, t = [], np.float64(0.0)
    while True:
        t = t + np.float64(1e8)
        pts.append(t)
        if not t < f32("1e10"):
            break
    x0 = np.zeros((16, 1))
    x0[:12, 0] = primordial_x0()
    prim_ladder = {"y0": x0, "t0": 0.0, "dt0": f32("2.2954626201190183E-026"), "t_stops": pts,
                   "dt_reset": None, "rtol": 1e-4, "atol": 1e-20, "dt_min": 1e-20,
                   "rho": np.array([f32("1e-10")])}
    C.append(Case("primordial_csc_ff_ladder", "PRIMORDIAL_CSC_FF", "PRIMORDIAL", "CSC", "FF", 1, 1,
                  [prim_ladder], defines=("HAVE_COEFFICIENTS",)))
    # the PRIMORDIAL workload's cells (Tgas 1000 K), single solves at rtol 1e-6
    yb, tsb, dtb, rt, at, dm = primordial_bench_cells(6, 31)
    bench = [{"y0": yb[:, i:i + 1], "t0": 0.0, "dt0": dtb[i], "t_stops": [tsb[i]], "dt_reset": None,
              "rtol": rt, "atol": at, "dt_min": dm} for i in range(6)]
    C.append(Case("primordial_csc_ff", "PRIMORDIAL_CSC_FF", "PRIMORDIAL", "CSC", "FF", 1, 1, bench,
                  defines=("HAVE_COEFFICIENTS",)))
    C.append(Case("primordial_csc_cmk", "PRIMORDIAL_CSC_CMK", "PRIMORDIAL", "CSC", "CMK", 1, 1, bench[:2],
                  defines=("HAVE_COEFFICIENTS",)))
    C.append(Case("primordial_dense", "PRIMORDIAL_DENSE_NONE", "PRIMORDIAL", "DENSE", "None", 1, 1,
                  bench[2:4], defines=("HAVE_COEFFICIENTS",)))
    C.append(Case("primordial_lu3", "PRIMORDIAL_DENSE_NONE_LU3", "PRIMORDIAL", "DENSE", "None", 3, 1,
                  bench[4:6], defines=("HAVE_COEFFICIENTS",)))
    # --heatcool=1: the heating/cooling test network's cells, single solves
    # and a ladder of hydro steps with dt carried
    from odevec_b200 import workloads as W
    wl = W.hctoy(ncells=6, seed=41)
    hc = [{"y0": wl.y[:, i:i + 1], "t0": 0.0, "dt0": wl.dt0[i], "t_stops": [wl.t_stop[i]], "dt_reset": None,
           "rtol": wl.rtol, "atol": wl.atol, "dt_min": wl.dt_min} for i in range(4)]
    hc.append({"y0": wl.y[:, 4:5], "t0": 0.0, "dt0": 1e-10, "t_stops": [np.float64(1e9) * (k + 1) for k in range(20)],
               "dt_reset": None, "rtol": wl.rtol, "atol": wl.atol, "dt_min": wl.dt_min})
    dump = os.path.join(os.path.dirname(os.path.dirname(HERE)), "odevec_b200", "data", "hctoy_krome.py")
    C.append(Case("hctoy_heatcool", "HCTOY_DENSE_NONE", "KROME", "DENSE", "None", 1, 1, hc, krome=dump))
    return C


def main(argv):
    global REF
    args = [a for a in argv if not a.startswith("-")]
    if args and os.path.isdir(args[0]):
        REF = args.pop(0)
    MG.REF = REF
    wanted = set(args)
    out = json.load(open(OUT)) if os.path.exists(OUT) and wanted else {}
    work = tempfile.mkdtemp(prefix="odevec_ref_")
    try:
        ref = os.path.join(work, "ref")
        MG.shim_copy(ref)
        os.makedirs(os.path.join(ref, "build"), exist_ok=True)
        for case in cases():
            if wanted and case.name not in wanted:
                continue
            t0 = time.time()
            ns = translate_case(ref, case)
            runs = [run_ladder(ns, case, r) for r in case.runs]
            out[case.name] = {"tag": case.tag, "check_negatives": int(case.check_neg), "runs": runs,
                              "reference": {"example": case.ex, "packaging": case.pack,
                                            "ordering": case.order, "LUmethod": case.lum,
                                            "nvector": case.nvector}}
            ncalls = sum(len(r["calls"]) for r in runs)
            print("%-26s %3d runs %5d calls %6.1f s" % (case.name, len(runs), ncalls, time.time() - t0))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    with open(OUT, "w") as fh:
        json.dump({k: out[k] for k in sorted(out)}, fh, separators=(",", ":"))
    print("wrote", OUT)


if __name__ == "__main__":
    main(sys.argv[1:])
