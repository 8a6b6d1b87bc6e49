"""The oracle against outputs of the reference's own solver module.

tests/golden/ref_solver.json holds what the reference's generated Fortran
(``build/odevec.f90`` + ``build/odevec_commons.f90`` written by its
``pre_odevec.py``) computes on seeded inputs, run through a statement-by-
statement translation with gfortran's arithmetic (tests/golden/f90py.py,
tests/golden/make_solver_golden.py).  Each case replays the reference
drivers' loops: every SolveODE call's state, time, step and counters.

The reference's solver object keeps ``this%en_old`` (the last Newton
correction) from one SolveODE call to the next; the oracle carries it in its
workspace (resume "en_old"), which the library's odevec_solve_resident
offers with resume = 2.

The oracle is built in its libm form here (exp, log, log10 and pow from the
C library, as in the compiled Fortran), so the comparison is bit for bit:
states, times, step sizes and all eight counters of every call.  The
default oracle -- the one the GPU kernels match bit for bit -- differs from
the libm form only in those four functions (at most 2 ulp each,
tests/test_math.py); test_default_oracle_tracks_reference shows what that
does on the PRIMORDIAL workload's cells.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_solver.json")
STAT_NAMES = ["steps", "attempts", "error-test failures", "Newton failures", "Newton iterations",
              "Jacobians", "order", "Nordsieck passes"]
CASES = json.load(open(FIX)) if os.path.exists(FIX) else {}


def _h(v):
    return np.array([float.fromhex(x) for x in v])


def replay(case, run, libm=True):
    """Runs the oracle through the run's ladder, each call on the state the
    oracle itself produced (time carried, dt reset or carried, mass fractions
    converted as the reference driver does, en_old carried).  Yields
    (call record, inputs, outputs) per call."""
    nv, neq = run["nvector"], run["neq"]
    tag = case["tag"]
    rtol, atol, dt_min = (float.fromhex(run[k]) for k in ("rtol", "atol", "dt_min"))
    rho = None if run["rho"] is None else _h(run["rho"])
    ws = O.workspace(tag, nv, nv)
    y = t = dt = None
    for k, call in enumerate(run["calls"]):
        if k == 0:
            y = _h(call["y_in"]).reshape(neq, nv)
            t = np.full(nv, float.fromhex(call["t_in"]))
            dt = np.full(nv, float.fromhex(call["dt_in"]))
        else:
            if rho is not None:    # number densities -> mass fractions -> number densities
                y = O.convert(tag, O.convert(tag, y, rho, 1), rho, 0)
            if run["dt_reset"] is not None:
                dt = np.full(nv, float.fromhex(run["dt_reset"]))
        mask = np.array(call["mask"], np.uint8) if "mask" in call else None
        inputs = (y.copy(), t.copy(), dt.copy())
        out = O.solve(tag, y, t, dt, np.full(nv, float.fromhex(call["t_stop"])), rtol, atol, dt_min,
                      group=nv, check_negatives=bool(case["check_negatives"]), mask=mask, libm=libm,
                      ws=ws, resume="en_old" if k else False)
        yield call, inputs, out
        y, t, dt = out[0], out[1], out[2]


def _runs():
    for name in sorted(CASES):
        for i in range(len(CASES[name]["runs"])):
            yield pytest.param(name, i, id="%s-%d" % (name, i))


@pytest.mark.skipif(not CASES, reason="no reference fixtures")
@pytest.mark.parametrize("name,irun", list(_runs()))
def test_oracle_equals_reference(name, irun):
    case = CASES[name]
    run = case["runs"][irun]
    nv, neq = run["nvector"], run["neq"]
    for k, (call, (yi, ti, dti), (yo, to, dto, st, stats)) in enumerate(replay(case, run)):
        where = "%s run %d call %d (t_stop %s)" % (name, irun, k, float.fromhex(call["t_stop"]))
        assert np.array_equal(yi, _h(call["y_in"]).reshape(neq, nv)), where + ": input state"
        assert np.all(ti == float.fromhex(call["t_in"])) and np.all(dti == float.fromhex(call["dt_in"])), \
            where + ": input time or step"
        assert "stopped" not in call, where
        assert np.all(st == 0), where
        ref_y = _h(call["y"]).reshape(neq, nv)
        assert np.array_equal(yo, ref_y), "%s: y differs, max rel %.3g" % (
            where, np.max(np.abs(yo - ref_y) / np.maximum(np.abs(ref_y), 1e-300)))
        assert np.all(to == float.fromhex(call["t"])), where + ": time"
        assert np.all(dto == float.fromhex(call["dt"])), where + ": dt"
        for j, nm in enumerate(STAT_NAMES):
            assert np.all(stats[:, j] == call["stats"][j]), "%s: %s %s != %d" % (
                where, nm, stats[:, j], call["stats"][j])


@pytest.mark.skipif(not CASES, reason="no reference fixtures")
@pytest.mark.parametrize("name", ["primordial_csc_ff", "primordial_csc_cmk", "primordial_dense",
                                  "primordial_lu3", "rober_dense_masked", "rober_checkneg"])
def test_default_oracle_tracks_reference(name):
    """The oracle the GPU kernels equal bit for bit (its own exp/log/pow, at
    most 2 ulp from the C library's) on the PRIMORDIAL workload's cells and
    two ROBER ladders: the same counters on every call and states within
    1e-4 rtol (species above atol/rtol).  On long oscillatory or restart-
    prone runs (the OREGO solves to t ~ 360, the 100-call PRIMORDIAL ladder)
    a last-bit difference in a step-size power moves a step decision and the
    trajectories separate by the algorithm's own global error, so there the
    bit-for-bit comparison of the libm form above is the evidence."""
    case = CASES[name]
    for run in case["runs"]:
        nv, neq = run["nvector"], run["neq"]
        atol, rtol = float.fromhex(run["atol"]), float.fromhex(run["rtol"])
        for call, _, (yo, to, dto, st, stats) in replay(case, run, libm=False):
            ref_y = _h(call["y"]).reshape(neq, nv)
            big = np.abs(ref_y) > atol / rtol
            rel = np.abs(yo - ref_y)[big] / np.abs(ref_y[big])
            assert np.all(st == 0)
            assert np.all(to == float.fromhex(call["t"]))
            assert np.all(stats == np.array(call["stats"])[None, :]), (name, stats[0], call["stats"])
            assert rel.size == 0 or rel.max() < 1e-4 * rtol, (name, float(rel.max()), rtol)


@pytest.mark.skipif(not CASES, reason="no reference fixtures")
def test_fixture_coverage():
    """The fixtures exercise what the parity claims rest on."""
    tags = {c["tag"] for c in CASES.values()}
    for tag in ("ROBER_DENSE_NONE", "ROBER_CSC_NONE", "ROBER_DENSE_NONE_LU2", "ROBER_DENSE_NONE_LU3",
                "OREGO_DENSE_NONE", "OREGO_CSC_CMK", "OREGO_DENSE_NONE_LU2", "PRIMORDIAL_CSC_FF",
                "PRIMORDIAL_CSC_CMK", "PRIMORDIAL_DENSE_NONE", "PRIMORDIAL_DENSE_NONE_LU3", "HCTOY_DENSE_NONE"):
        assert tag in tags, tag
    assert any(c["check_negatives"] for c in CASES.values())
    assert any("mask" in call for c in CASES.values() for r in c["runs"] for call in r["calls"])
    tot = np.zeros(8, np.int64)
    for c in CASES.values():
        for r in c["runs"]:
            for call in r["calls"]:
                tot += np.array(call["stats"])
    # error-test failures, Newton failures and thousands of steps were exercised
    assert tot[2] > 0 and tot[3] > 0 and tot[0] > 1000, tot


@pytest.mark.skipif(not CASES, reason="no reference fixtures")
def test_driver_schedules_are_the_reference_drivers():
    """odevec_b200.driver's rober/orego/primordial schedules give the ladders,
    tolerances and first inputs of the reference drivers' runs above."""
    from odevec_b200 import driver as D
    r = CASES["rober_dense"]["runs"][0]
    s = D.rober_schedule(ncells=32)
    assert [float(v).hex() for v in s.t_stops] == [c["t_stop"] for c in r["calls"]]
    assert float(s.rtol).hex() == r["rtol"] and float(s.atol).hex() == r["atol"]
    assert float(s.dt_reset).hex() == r["dt_reset"]
    o = CASES["orego_dense_ladder"]["runs"][0]
    s = D.orego_schedule(ncells=1, network="OREGO_DENSE_NONE")
    assert [float(v).hex() for v in s.t_stops[:len(o["calls"])]] == [c["t_stop"] for c in o["calls"]]
    assert float(s.rtol).hex() == o["rtol"] and float(s.atol).hex() == o["atol"]
    p = CASES["primordial_csc_ff_ladder"]["runs"][0]
    s = D.primordial_schedule(ncells=1)
    assert [float(v).hex() for v in s.t_stops] == [c["t_stop"] for c in p["calls"]]
    assert float(s.dt).hex() == p["calls"][0]["dt_in"]
    assert [float(v).hex() for v in s.rho] == p["rho"]
    n0 = O.convert("PRIMORDIAL_CSC_FF", s.y0, s.rho, 0)
    assert np.array_equal(n0, _h(p["calls"][0]["y_in"]).reshape(16, 1))
