"""GPU runs of the reference's own driver ladders against the oracle.

Every case of tests/golden/ref_solver.json (outputs of the reference's
generated solver module on seeded inputs, see tests/test_reference_pin.py)
is replayed on the GPU through the C ABI in the FP64 form without fused
multiply-add: the same ladder of SolveODE calls, the time carried, dt reset
or carried, mass fractions converted on the device (odevec_convert), and the
previous call's last Newton correction carried in the resident workspace
(odevec_solve_resident with resume = 2 after the first call), as the
reference's solver object keeps this%en_old.  Each call must equal the
oracle's same ladder bit for bit: states, times, steps, status and all
counters.  The oracle in its libm form equals the reference bit for bit on
these ladders (tests/test_reference_pin.py), so this measures the kernel
against the reference's own outputs up to the elementary functions.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_solver.json")
CASES = json.load(open(FIX)) if os.path.exists(FIX) else {}


def _h(v):
    return np.array([float.fromhex(x) for x in v])


def gpu_ladder(S, case, run):
    import torch
    from odevec_b200 import driver as D
    nv, neq = run["nvector"], run["neq"]
    tag = case["tag"]
    ode = S.Odevec(tag, RelativeTolerance=float.fromhex(run["rtol"]),
                   AbsoluteTolerance=float.fromhex(run["atol"]), MinimalTimestep=float.fromhex(run["dt_min"]),
                   CheckNegatives=bool(case["check_negatives"]), nvector=nv, precision="fp64",
                   raise_on_failure=False)
    S.InitOdevec(ode)
    try:
        ws = S.Workspace(ode, nv)
        rho = None if run["rho"] is None else torch.tensor(_h(run["rho"]), device="cuda")
        first = run["calls"][0]
        y = torch.tensor(_h(first["y_in"]).reshape(neq, nv), device="cuda")
        t = torch.full((nv,), float.fromhex(first["t_in"]), dtype=torch.float64, device="cuda")
        dt = torch.full((nv,), float.fromhex(first["dt_in"]), dtype=torch.float64, device="cuda")
        for k, call in enumerate(run["calls"]):
            if k:
                if rho is not None:
                    x = D.convert(tag, y, rho, D.OV_N2X)
                    y = D.convert(tag, x, rho, D.OV_X2N)
                if run["dt_reset"] is not None:
                    dt.fill_(float.fromhex(run["dt_reset"]))
            mask = None
            if "mask" in call:
                mask = torch.tensor(call["mask"], dtype=torch.uint8, device="cuda")
            ts = torch.full((nv,), float.fromhex(call["t_stop"]), dtype=torch.float64, device="cuda")
            t, dt = S.SolveODE(ode, t, dt, ts, y, Mask=mask, workspace=ws, resume="en_old" if k else False)
            torch.cuda.synchronize()
            yield (y.cpu().numpy().copy(), t.cpu().numpy().copy(), dt.cpu().numpy().copy(),
                   ode.status.cpu().numpy().copy(), ode.stats.cpu().numpy().copy())
    finally:
        S.CloseOdevec(ode)


def _runs():
    for name in sorted(CASES):
        for i in range(len(CASES[name]["runs"])):
            yield pytest.param(name, i, id="%s-%d" % (name, i))


@pytest.mark.skipif(not CASES, reason="no reference fixtures")
@pytest.mark.parametrize("name,irun", list(_runs()))
def test_gpu_reference_ladder_equals_oracle(gpu_lib, name, irun):
    from test_reference_pin import replay
    case = CASES[name]
    run = case["runs"][irun]
    for k, (g, (call, _, o)) in enumerate(zip(gpu_ladder(gpu_lib, case, run), replay(case, run, libm=False))):
        for what, a, b in zip(["y", "t", "dt", "status", "stats"], g, o):
            assert np.array_equal(a, b), "%s run %d call %d: %s differs" % (name, irun, k, what)
