"""Serving scheduler: continuous batching with admission by memory budget.

CPU tests drive the scheduler with the oracle backend; the GPU test checks
that a request's results are bit-identical alone and in a mix."""
import numpy as np
import pytest

from odevec_b200 import serving as SV
from oracle_backend import OracleBackend


def small_stream(n=6, steps=3, seed=9):
    return SV.make_stream(seed=seed, rate=2000.0, duration=1.0,
                          networks=("ROBER_DENSE_NONE", "PRIMORDIAL_CSC_FF", "SYN64_CSC_CMK"),
                          cells=(32, 96), dt_hydro=(1e2, 1e8), steps=steps, max_requests=n)


class BudgetProbe(OracleBackend):
    def __init__(self):
        super().__init__()
        self.live = 0.0
        self.peak = 0.0

    def admit(self, r):
        self.live += self.bytes_needed(r)
        self.peak = max(self.peak, self.live)
        return super().admit(r)

    def release(self, h):
        self.live -= self.bytes_needed(h["r"])
        return super().release(h)


def test_scheduler_completes_all_steps_within_budget(oracle):
    reqs = small_stream()
    be = BudgetProbe()
    budget = 2.5 * max(be.bytes_needed(r) for r in reqs)
    recs, res = SV.Scheduler(be, budget, slots=3).run(reqs, realtime=False)
    assert len(recs) == sum(r.steps for r in reqs)
    assert sorted(res) == [r.rid for r in reqs]
    assert be.peak <= budget
    for r in reqs:
        steps = sorted(x.step for x in recs if x.rid == r.rid)
        assert steps == list(range(r.steps))
    s = SV.summarize(recs)
    assert s["cells"] == sum(r.ncells * r.steps for r in reqs) and s["p99_ms"] >= s["p50_ms"]


def test_results_same_alone_and_in_mix(oracle):
    reqs = small_stream()
    _, mixed = SV.Scheduler(OracleBackend(), 1e12, slots=4).run(reqs, realtime=False)
    for r in reqs:
        _, alone = SV.Scheduler(OracleBackend(), 1e12, slots=1).run([r], realtime=False)
        assert np.array_equal(alone[r.rid].y, mixed[r.rid].y)
        assert np.array_equal(alone[r.rid].status, mixed[r.rid].status)


def failing_request(steps=3):
    """Four valid ROBER cells; the third, y = (0.9045, 0, 0.0955), fails
    with DT_MIN_CONV in the first hydro step of 1.83e9 s under the
    reference's restart after three failed error tests (and passes with
    that restart corrected)."""
    y0 = np.array([[0.904506772, 0.904506772, 0.90450677, 0.5],
                   [0.0, 1e-6, 0.0, 1e-7],
                   [0.095493228, 0.095493227, 0.09549323, 0.4999999]])
    from odevec_b200 import workloads as W
    wl = W.BUILDERS["ROBER"](ncells=260944, seed=1002, network="ROBER_DENSE_NONE")
    y0[:, 2] = wl.y[:, 26542]
    return SV.Request(0, "ROBER_DENSE_NONE", y0, 1827450230.062853, steps, 0.0, 1e-4, 1e-10, 1e-20, 1e-10)


def test_failed_cell_is_reported_and_masked_out(oracle):
    r = failing_request()
    _, res = SV.Scheduler(OracleBackend(), 1e12, slots=1).run([r], realtime=False)
    assert list(res[0].status) == [0, 0, 3, 0] and res[0].failed == 1
    # the failed cell stays at its failure state (the diverged iterate, NaN
    # and inf here); the others continue as a request without it
    y1, *_ = oracle.solve(r.network, r.y0, np.zeros(4), np.full(4, r.dt_in), r.dt_hydro, r.rtol, r.atol, r.dt_min)
    assert np.array_equal(res[0].y[:, 2], y1[:, 2], equal_nan=True)
    ok = [0, 1, 3]
    r3 = SV.Request(1, r.network, r.y0[:, ok].copy(), r.dt_hydro, r.steps, 0.0, r.rtol, r.atol, r.dt_min, r.dt_in)
    _, res3 = SV.Scheduler(OracleBackend(), 1e12, slots=1).run([r3], realtime=False)
    assert np.array_equal(res[0].y[:, ok], res3[1].y)
    assert SV.summarize([SV.StepRecord(0, 0, 4, r.network, 0.0, 1.0)], res)["failed_cells"] == 1


def test_resident_steps_equal_oracle_continuation(oracle):
    # the scheduler's per-request result is the oracle's continuation over
    # the request's hydro steps
    r = small_stream(n=1)[0]
    _, res = SV.Scheduler(OracleBackend(), 1e12, slots=1).run([r], realtime=False)
    ws = oracle.workspace(r.network, r.ncells)
    y, t, dt = r.y0, np.zeros(r.ncells), np.full(r.ncells, r.dt_in)
    for k in range(r.steps):
        y, t, dt, st, _ = oracle.solve(r.network, y, t, dt, r.dt_hydro * (k + 1), r.rtol, r.atol, r.dt_min,
                                       ws=ws, resume=k > 0)
    assert np.array_equal(res[r.rid].y, y) and not np.any(res[r.rid].status)


def test_over_budget_request_rejected(oracle):
    reqs = small_stream(n=2)
    with pytest.raises(ValueError, match="budget"):
        SV.Scheduler(OracleBackend(), 16.0, slots=2).run(reqs, realtime=False)


@pytest.mark.gpu
def test_gpu_results_same_alone_and_in_mix(gpu_lib):
    reqs = SV.make_stream(seed=3, rate=500.0, duration=1.0,
                          networks=("ROBER_DENSE_NONE", "PRIMORDIAL_CSC_FF", "SYN64_CSC_CMK"),
                          cells=(1000, 20000), dt_hydro=(1e4, 1e8), steps=4, max_requests=8)
    for precision in ("fp64", "fp32_lu"):
        be = SV.GpuBackend(precision)
        recs, mixed = SV.Scheduler(be, 100e9, slots=8).run(reqs, realtime=False)
        assert len(recs) == sum(r.steps for r in reqs)
        for r in reqs[:4]:
            _, alone = SV.Scheduler(SV.GpuBackend(precision), 100e9, slots=1).run([r], realtime=False)
            assert np.array_equal(alone[r.rid].y, mixed[r.rid].y)
            assert np.array_equal(alone[r.rid].status, mixed[r.rid].status)


@pytest.mark.gpu
def test_gpu_failed_cell_matches_oracle_backend(gpu_lib, oracle):
    r = failing_request()
    _, ref = SV.Scheduler(OracleBackend(), 1e12, slots=1).run([r], realtime=False)
    _, got = SV.Scheduler(SV.GpuBackend("fp64"), 1e12, slots=1).run([r], realtime=False)
    assert np.array_equal(got[0].status, ref[0].status) and got[0].failed == 1
    assert np.array_equal(got[0].y, ref[0].y, equal_nan=True)
    # FP32-LU rounds differently and may take another step sequence (here it
    # passes); a cell that fails there is re-solved in FP64 from its step's
    # inputs, so whatever still fails carries the FP64 status and state
    _, f32 = SV.Scheduler(SV.GpuBackend("fp32_lu"), 1e12, slots=1).run([r], realtime=False)
    for c in np.nonzero(f32[0].status)[0]:
        assert f32[0].status[c] == ref[0].status[c]
        assert np.array_equal(f32[0].y[:, c], ref[0].y[:, c], equal_nan=True)
    ok = f32[0].status == 0
    assert np.all(np.isfinite(f32[0].y[:, ok]))


def test_water_fill_shares():
    """Small requests get the blocks their cells fill; large ones share the
    rest equally; nothing exceeds the capacity."""
    from odevec_b200.serving import water_fill
    assert water_fill({0: 2048, 1: 8, 2: 8}, 444) == {0: 428, 1: 8, 2: 8}
    assert water_fill({0: 2048, 1: 2048}, 444) == {0: 222, 1: 222}
    assert water_fill({0: 100, 1: 2048, 2: 2048}, 444) == {0: 100, 1: 172, 2: 172}
    assert water_fill({5: 3}, 444) == {5: 3}
    s = water_fill({i: 10 * i + 1 for i in range(20)}, 444)
    assert sum(s.values()) <= 444 and all(s[i] <= 10 * i + 1 for i in s)


def test_staging_for_large_networks():
    """Requests run staging 3's shape: with the state vector in shared memory
    above 32 solver species (staging 20), with the history in shared memory
    and soft lockstep up to 12 (staging 21); an explicit staging is kept."""
    import types
    from odevec_b200 import solver
    from odevec_b200.serving import GpuBackend
    be = types.SimpleNamespace(staging=3, S=solver)
    assert GpuBackend.staging_for(be, "SYN64_CSC_CMK") == 20
    assert GpuBackend.staging_for(be, "PRIMORDIAL_CSC_FF") == 21
    assert GpuBackend.staging_for(be, "ROBER_DENSE_NONE") == 21
    be.staging = 8
    assert GpuBackend.staging_for(be, "SYN64_CSC_CMK") == 8
