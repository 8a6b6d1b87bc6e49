"""GPU parity: the CUDA solve path against the CPU oracle.

The FP64 form without fused multiply-add (precision "fp64") must reproduce
the oracle bit for bit: final states, times, last step sizes, status codes
and every per-cell counter.  The fused-multiply-add and FP32-LU forms are
compared within tolerances stated in each test.  All calls go through the
C ABI (odevec_solve / odevec_solve_host).
"""
import numpy as np
import pytest

from odevec_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run_gpu(S, wl, precision="fp64", group=None, host=False, mask=None, check_negatives=False,
            max_attempts=0, dt_min=None, batch=(0, 0, 0), staging=0):
    import torch
    ode = S.Odevec(wl.network, max_cells=wl.ncells if host else 0, RelativeTolerance=wl.rtol,
                   AbsoluteTolerance=wl.atol,
                   MinimalTimestep=wl.dt_min if dt_min is None else dt_min,
                   CheckNegatives=check_negatives, nvector=wl.group if group is None else group,
                   precision=precision, max_attempts=max_attempts, raise_on_failure=False,
                   jac_batch=batch[0], ss_batch=batch[1], max_wait=batch[2], staging=staging)
    S.InitOdevec(ode)
    try:
        if host:
            y = wl.y.copy()
            t, dt = S.SolveODE(ode, wl.t0, wl.dt0, wl.t_stop, y, Mask=mask)
            return y, t, dt, ode.status.copy(), ode.stats.copy()
        y = torch.tensor(wl.y, device="cuda")
        t, dt = S.SolveODE(ode, torch.tensor(wl.t0, device="cuda"), torch.tensor(wl.dt0, device="cuda"),
                           torch.tensor(wl.t_stop, device="cuda"), y, Mask=mask)
        torch.cuda.synchronize()
        return (y.cpu().numpy(), t.cpu().numpy(), dt.cpu().numpy(), ode.status.cpu().numpy(),
                ode.stats.cpu().numpy())
    finally:
        S.CloseOdevec(ode)


def run_oracle(O, wl, group=None, mask=None, check_negatives=False, max_attempts=1000000,
               dt_min=None, rtol=None, atol=None):
    return O.solve(wl.network, wl.y, wl.t0, wl.dt0, wl.t_stop, wl.rtol if rtol is None else rtol,
                   wl.atol if atol is None else atol, wl.dt_min if dt_min is None else dt_min,
                   group=wl.group if group is None else group, check_negatives=check_negatives,
                   mask=mask, max_attempts=max_attempts)


def assert_bitwise(g, o, what=""):
    names = ["y", "t", "dt", "status", "stats"]
    for name, a, b in zip(names, g, o):
        a = np.asarray(a)
        b = np.asarray(b)
        same = (a == b) | (np.isnan(a) & np.isnan(b)) if a.dtype.kind == "f" else (a == b)
        if not np.all(same):
            idx = np.argwhere(~same)[:5]
            raise AssertionError("%s: %s differs at %s: gpu %s oracle %s" % (
                what, name, idx.tolist(), a[tuple(idx[0])], b[tuple(idx[0])]))


CASES = [
    ("ROBER", dict(ncells=256), "ROBER_DENSE_NONE", 32),
    ("ROBER", dict(ncells=256), "ROBER_CSC_NONE", 1),
    ("OREGO", dict(ncells=512), "OREGO_CSC_CMK", 1),
    ("OREGO", dict(ncells=256), "OREGO_DENSE_NONE", 1),
    ("PRIMORDIAL", dict(ncells=512), "PRIMORDIAL_CSC_FF", 1),
    ("PRIMORDIAL", dict(ncells=256), "PRIMORDIAL_CSC_CMK", 1),
    ("PRIMORDIAL", dict(ncells=256), "PRIMORDIAL_DENSE_NONE", 1),
    ("PRIMORDIAL", dict(ncells=256), "PRIMORDIAL_DENSE_NONE", 32),
    ("SYN64", dict(ncells=128), "SYN64_CSC_CMK", 1),
    # LUmethod 2 (symbolic factors) and 3 (difference quotients)
    ("ROBER", dict(ncells=256), "ROBER_DENSE_NONE_LU2", 32),
    ("OREGO", dict(ncells=256), "OREGO_DENSE_NONE_LU2", 1),
    ("ROBER", dict(ncells=256), "ROBER_DENSE_NONE_LU3", 32),
    ("ROBER", dict(ncells=256), "ROBER_DENSE_NONE_LU3", 1),
    ("PRIMORDIAL", dict(ncells=256), "PRIMORDIAL_DENSE_NONE_LU3", 1),
    # --heatcool=1: the heating/cooling temperature row and its difference quotients
    ("HCTOY", dict(ncells=512), "HCTOY_DENSE_NONE", 1),
]


@pytest.mark.parametrize("name,kw,network,group", CASES)
def test_fp64_bit_exact_vs_oracle(gpu_lib, oracle, name, kw, network, group):
    wl = W.BUILDERS[name](network=network, **kw)
    if group == 32 and name == "PRIMORDIAL":
        wl.t_stop[:] = 1e10  # lockstep groups need a common t_stop
    wl.group = group
    g = run_gpu(gpu_lib, wl, "fp64", group=group)
    o = run_oracle(oracle, wl, group=group)
    assert np.all(o[3] == 0), "oracle failures: %s" % np.unique(o[3])
    assert_bitwise(g, o, "%s/%s G=%d" % (name, network, group))


@pytest.mark.parametrize("precision", ["fp64", "fp32_lu"])
def test_scheduling_does_not_change_results(gpu_lib, precision):
    # the Jacobian / step-size batching only reorders work across the lanes
    # of a warp: every cell's result must be bit-identical for any setting
    wl = W.primordial(ncells=2048)
    ref = run_gpu(gpu_lib, wl, precision, batch=(1, 1, -1))
    for batch in [(0, 0, 0), (32, 32, 1000), (5, 20, 2)]:
        g = run_gpu(gpu_lib, wl, precision, batch=batch)
        assert_bitwise(g, ref, "batch %s" % (batch,))
    # every staging (6: staging 3's thread-local kernel in one 384-thread
    # block per SM; 8-12: soft lockstep), with the default batches and with
    # per-cell blocks
    for staging in (1, 2, 3, 4, 6, 8, 9, 10, 12, 17, 21) + ((5, 11) if precision == "fp32_lu" else ()):
        for batch in [(0, 0, 0), (1, 1, -1)]:
            g = run_gpu(gpu_lib, wl, precision, batch=batch, staging=staging)
            assert_bitwise(g, ref, "staging %d batch %s" % (staging, batch))


def test_host_entry_point_matches_device(gpu_lib, oracle):
    wl = W.primordial(ncells=300, network="PRIMORDIAL_CSC_FF")
    g = run_gpu(gpu_lib, wl, "fp64", host=True)
    o = run_oracle(oracle, wl)
    assert_bitwise(g, o, "host path")


def _pinned(a, keep):
    """A copy of NumPy array a in pinned (page-locked, mapped) host memory."""
    import torch
    dt = {np.dtype(np.float64): torch.float64, np.dtype(np.uint8): torch.uint8}[a.dtype]
    buf = torch.empty(a.shape, dtype=dt).pin_memory()
    keep.append(buf)
    x = buf.numpy()
    x[...] = a
    return x


@pytest.mark.parametrize("precision,max_attempts", [("fp64", 0), ("fp32_lu", 0), ("fp32_lu", 5)])
def test_host_entry_point_pinned_arrays_in_place(gpu_lib, oracle, precision, max_attempts):
    """odevec_solve_host with y, time, dt, t_stop and mask in pinned host
    memory: the kernel reads and writes them in place (no copies), with the
    results of the copy path.  With max_attempts 5 every FP32-LU cell fails, is
    restored from the inputs the kernel saved as it loaded them, and is
    solved again in FP64 (the fp64_fma form): the results are that form's."""
    S = gpu_lib
    wl = W.primordial(ncells=300, network="PRIMORDIAL_CSC_FF")
    mask = (np.arange(300) % 7 != 3).astype(np.uint8)
    keep = []

    def solve(prec, pinned):
        ode = S.Odevec(wl.network, max_cells=wl.ncells, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                       MinimalTimestep=wl.dt_min, nvector=1, precision=prec, raise_on_failure=False,
                       max_attempts=max_attempts)
        S.InitOdevec(ode)
        try:
            y = _pinned(wl.y, keep) if pinned else wl.y.copy()
            ts = _pinned(wl.t_stop, keep) if pinned else wl.t_stop.copy()
            m = _pinned(mask, keep) if pinned else mask.copy()
            if pinned:  # time and dt pinned too, updated in place
                t0, d0 = _pinned(wl.t0, keep), _pinned(wl.dt0, keep)
                t, d = S.SolveODE(ode, t0, d0, ts, y, Mask=m, in_place=True)
                assert t is t0 and d is d0
            else:
                t, d = S.SolveODE(ode, wl.t0, wl.dt0, ts, y, Mask=m)
            return y.copy(), t.copy(), d.copy(), ode.status.copy(), ode.stats.copy()
        finally:
            S.CloseOdevec(ode)

    pinned = solve(precision, True)
    assert_bitwise(pinned, solve(precision, False), "pinned vs pageable host arrays")
    if precision == "fp64":
        assert_bitwise(pinned, run_oracle(oracle, wl, mask=mask), "pinned host arrays vs oracle")
    if max_attempts:
        # all but the few cells that finish within 5 attempts end with
        # MAX_STEPS after the FP64 re-solve too, and equal the fp64_fma form
        failed = pinned[3] == 4
        assert failed.sum() >= 250 and not np.any(failed & (mask == 0))
        fma = solve("fp64_fma", True)
        assert np.array_equal(fma[3][failed], pinned[3][failed])
        assert np.array_equal(pinned[0][:, failed], fma[0][:, failed])
        assert np.array_equal(pinned[1][failed], fma[1][failed])
        assert np.array_equal(pinned[2][failed], fma[2][failed])


def _relerr(a, b, floor):
    m = np.abs(b) > floor
    return np.max(np.abs(a[m] - b[m]) / np.abs(b[m])) if np.any(m) else 0.0


@pytest.mark.parametrize("precision", ["fp64_fma", "fp32_lu"])
def test_fast_forms_within_tolerance(gpu_lib, oracle, precision):
    # FMA changes roundings and FP32-LU the Newton iterates, so step
    # sequences differ; both must stay within 10*rtol of the exact FP64 form
    # at the same tolerance (the FP32 factors' share is measured at about
    # 0.1*rtol), for species above 1e-12 of the cell's largest abundance
    wl = W.primordial(ncells=1024)
    g = run_gpu(gpu_lib, wl, precision)
    o = run_oracle(oracle, wl)
    assert np.all(g[3] == 0)
    floor = 1e-12 * np.max(wl.y[:12], axis=0)
    err = np.max([_relerr(g[0][s], o[0][s], floor) for s in range(12)])
    assert err < 10 * wl.rtol, err


def test_mask_semantics(gpu_lib, oracle):
    wl = W.orego(ncells=256)
    mask = (np.arange(256) % 3 != 0).astype(np.uint8)
    g = run_gpu(gpu_lib, wl, "fp64", mask=mask)
    o = run_oracle(oracle, wl, mask=mask)
    assert_bitwise(g, o, "mask")
    off = mask == 0
    assert np.all(g[0][:, off] == wl.y[:, off])       # untouched
    assert np.all(g[1][off] == wl.t_stop[off])        # time = t_stop


def test_lockstep_mask(gpu_lib, oracle):
    wl = W.rober(ncells=128)
    mask = np.ones(128, np.uint8)
    mask[::5] = 0
    mask[64:96] = 0     # one group fully masked
    g = run_gpu(gpu_lib, wl, "fp64", mask=mask)
    o = run_oracle(oracle, wl, mask=mask)
    assert_bitwise(g, o, "lockstep mask")


def test_check_negatives(gpu_lib, oracle):
    wl = W.primordial(ncells=256, network="PRIMORDIAL_CSC_FF")
    g = run_gpu(gpu_lib, wl, "fp64", check_negatives=True)
    o = run_oracle(oracle, wl, check_negatives=True)
    assert_bitwise(g, o, "check negatives")


def test_status_max_attempts(gpu_lib, oracle):
    wl = W.primordial(ncells=64)
    g = run_gpu(gpu_lib, wl, "fp64", max_attempts=7)
    o = run_oracle(oracle, wl, max_attempts=7)
    assert np.all(g[3] == 4)  # OV_ERR_MAX_STEPS
    assert_bitwise(g, o, "max attempts")


def test_status_dt_min(gpu_lib, oracle):
    # OREGO has occasional Newton failures, each dividing dt by 4; with a
    # minimal step of 0.1 most cells end with OV_ERR_DTMIN_CONV
    wl = W.orego(ncells=256)
    g = run_gpu(gpu_lib, wl, "fp64", dt_min=0.1)
    o = run_oracle(oracle, wl, dt_min=0.1)
    assert np.sum(o[3] == 3) > 50
    assert_bitwise(g, o, "dt_min")


@pytest.mark.parametrize("network", ["ROBER_CSC_NONE", "PRIMORDIAL_CSC_FF"])
def test_fix_restart_matches_oracle(gpu_lib, oracle, network):
    # the optional correction of the order-1 restart, at a tight tolerance
    # where the restart happens often
    wl = W.rober(ncells=128, network=network) if network.startswith("ROBER") else \
        W.primordial(ncells=256, network=network)
    wl.group = 1
    wl.rtol = 1e-10
    wl.atol = 1e-16 if network.startswith("ROBER") else 1e-24
    import torch
    ode = gpu_lib.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                         MinimalTimestep=wl.dt_min, nvector=1, precision="fp64", fix_restart=True,
                         raise_on_failure=False)
    gpu_lib.InitOdevec(ode)
    y = torch.tensor(wl.y, device="cuda")
    t, dt = gpu_lib.SolveODE(ode, torch.tensor(wl.t0, device="cuda"), torch.tensor(wl.dt0, device="cuda"),
                             torch.tensor(wl.t_stop, device="cuda"), y)
    g = (y.cpu().numpy(), t.cpu().numpy(), dt.cpu().numpy(), ode.status.cpu().numpy(), ode.stats.cpu().numpy())
    gpu_lib.CloseOdevec(ode)
    o = oracle.solve(wl.network, wl.y, wl.t0, wl.dt0, wl.t_stop, wl.rtol, wl.atol, wl.dt_min, group=1,
                     fix_restart=True)
    assert_bitwise(g, o, "fix_restart")


def test_group_mismatch(gpu_lib, oracle):
    wl = W.rober(ncells=64)
    wl.t_stop[5] = 2e5
    g = run_gpu(gpu_lib, wl, "fp64")
    o = run_oracle(oracle, wl)
    assert np.all(g[3][:32] == 6) and np.all(g[3][32:] == 0)
    assert_bitwise(g, o, "group mismatch")


@pytest.mark.parametrize("precision,tol", [("fp64_fma", 1e-10), ("fp32_lu", 1e-5)])
def test_primordial_conservation_large_sample(gpu_lib, precision, tol):
    # size-independent properties on 65536 cells: hydrogen, helium and
    # deuterium nuclei and charge are linear invariants of the network.  The
    # FP64 Newton corrections preserve them to roundoff; the FP32 LU
    # perturbs each correction at the FP32 level, bounded by 10*rtol.
    wl = W.primordial(ncells=65536)
    g = run_gpu(gpu_lib, wl, precision)
    assert np.all(g[3] == 0)
    a = W.primordial_invariants(wl.y)
    b = W.primordial_invariants(g[0])
    for k in range(3):
        assert np.max(np.abs(b[k] - a[k]) / a[k]) < tol
    assert np.max(np.abs(b[3]) / a[0]) < tol


def test_syn64_mass_conservation(gpu_lib):
    from odevec_b200 import syn64
    wl = W.syn64(ncells=1024)
    g = run_gpu(gpu_lib, wl, "fp32_lu")
    assert np.all(g[3] == 0)
    m = syn64.masses()
    assert np.max(np.abs(m @ g[0] - m @ wl.y) / (m @ wl.y)) < 1e-4


def test_syn64_stagings_bit_exact(gpu_lib, oracle):
    """The 64-species network on every thread-per-cell shape it compiles
    (the soft-lockstep 256- and 512-thread blocks and the shapes with the
    state vector in shared memory exist for networks above 32 solver species
    only), with more cells than one block holds, equals the oracle bit for
    bit."""
    wl = W.syn64(ncells=700)
    o = run_oracle(oracle, wl)
    assert np.all(o[3] == 0)
    for staging in (1, 3, 6, 8, 15, 16, 18, 19, 20):
        assert_bitwise(run_gpu(gpu_lib, wl, "fp64", staging=staging), o, "SYN64 staging %d" % staging)


def _resident_steps(gpu_lib, oracle, wl, precision, nsteps, group, staging=0):
    """Advance the same cells through nsteps successive t_stop values with the
    integrator state kept on the device; compare every step with the oracle's
    continuation."""
    import torch
    ode = gpu_lib.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                         MinimalTimestep=wl.dt_min, nvector=group, precision=precision,
                         raise_on_failure=False, staging=staging)
    gpu_lib.InitOdevec(ode)
    ws_g = gpu_lib.Workspace(ode, wl.ncells)
    ws_o = oracle.workspace(wl.network, wl.ncells, group)
    y_g = torch.tensor(wl.y, device="cuda")
    t_g = torch.tensor(wl.t0, device="cuda")
    d_g = torch.tensor(wl.dt0, device="cuda")
    y_o, t_o, d_o = wl.y.copy(), wl.t0.copy(), wl.dt0.copy()
    try:
        for k in range(nsteps):
            ts = wl.t_stop * (k + 1) / nsteps
            t_g, d_g = gpu_lib.SolveODE(ode, t_g, d_g, torch.tensor(ts, device="cuda"), y_g,
                                        workspace=ws_g, resume=k > 0)
            torch.cuda.synchronize()
            g = (y_g.cpu().numpy(), t_g.cpu().numpy(), d_g.cpu().numpy(), ode.status.cpu().numpy(),
                 ode.stats.cpu().numpy())
            o = oracle.solve(wl.network, y_o, t_o, d_o, ts, wl.rtol, wl.atol, wl.dt_min, group=group,
                             ws=ws_o, resume=k > 0)
            assert np.all(o[3] == 0)
            assert_bitwise(g, o, "resident step %d" % k)
            y_o, t_o, d_o = o[0], o[1], o[2]
    finally:
        gpu_lib.CloseOdevec(ode)
    return k


def test_resident_continuation_matches_oracle(gpu_lib, oracle):
    wl = W.primordial(ncells=512)
    _resident_steps(gpu_lib, oracle, wl, "fp64", 5, 1)
    wl = W.rober(ncells=128)
    _resident_steps(gpu_lib, oracle, wl, "fp64", 4, 32)


def test_resident_fresh_start_equals_solve(gpu_lib):
    # resume = 0 is SolveODE exactly (it only saves the state as well)
    import torch
    wl = W.primordial(ncells=1024)
    a = run_gpu(gpu_lib, wl, "fp32_lu")
    ode = gpu_lib.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                         MinimalTimestep=wl.dt_min, nvector=1, precision="fp32_lu", raise_on_failure=False)
    gpu_lib.InitOdevec(ode)
    y = torch.tensor(wl.y, device="cuda")
    t, dt = gpu_lib.SolveODE(ode, torch.tensor(wl.t0, device="cuda"), torch.tensor(wl.dt0, device="cuda"),
                             torch.tensor(wl.t_stop, device="cuda"), y,
                             workspace=gpu_lib.Workspace(ode, wl.ncells))
    b = (y.cpu().numpy(), t.cpu().numpy(), dt.cpu().numpy(), ode.status.cpu().numpy(), ode.stats.cpu().numpy())
    gpu_lib.CloseOdevec(ode)
    assert_bitwise(b, a, "resident fresh start")


def test_fp32_escalation_rescues_badly_conditioned_cells(gpu_lib):
    # ROBER advanced in hydro steps to ~1e7 s: late-time iteration matrices
    # have condition numbers ~1e14 and an FP32 factorisation can make Newton
    # fail until dt < dt_min.  With escalation every cell finishes, and the
    # rescued cells equal an FP64 solve of the same steps.
    import torch
    wl = W.rober(ncells=51417, seed=1008)
    res = {}
    for prec, esc in (("fp32_lu", False), ("fp32_lu", True), ("fp64_fma", True)):
        ode = gpu_lib.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                             MinimalTimestep=wl.dt_min, nvector=1, precision=prec, raise_on_failure=False,
                             escalation=esc)
        gpu_lib.InitOdevec(ode)
        y = torch.tensor(wl.y, device="cuda")
        t = torch.zeros(wl.ncells, dtype=torch.float64, device="cuda")
        dt = torch.full((wl.ncells,), 1e-10, dtype=torch.float64, device="cuda")
        ws = gpu_lib.Workspace(ode, wl.ncells)
        fails = 0
        for k in range(10):
            ts = torch.full((wl.ncells,), 1013907.692225179 * (k + 1), dtype=torch.float64, device="cuda")
            gpu_lib.SolveODE(ode, t, dt, ts, y, workspace=ws, resume=k > 0)
            fails += int((ode.status != 0).sum().item())
        res[(prec, esc)] = (fails, y.cpu().numpy())
        gpu_lib.CloseOdevec(ode)
    assert res[("fp32_lu", True)][0] == 0
    assert res[("fp64_fma", True)][0] == 0


@pytest.mark.parametrize("ncells", [1, 31, 33, 65, 129])
def test_ragged_sizes_bit_exact(gpu_lib, oracle, ncells):
    # cell counts that leave a warp, a block and the persistent grid partly empty
    wl = W.primordial(ncells=ncells, seed=ncells)
    for staging in (3, 6, 8, 9):
        g = run_gpu(gpu_lib, wl, "fp64", staging=staging)
        assert_bitwise(g, run_oracle(oracle, wl), "ncells %d staging %d" % (ncells, staging))


def test_short_solves_more_cells_than_lanes_bit_exact(gpu_lib, oracle):
    # about 15 trips per cell and two to three cells per lane: lanes go idle
    # often and take new cells on every trip (staging 1) or only on every 16th
    # trip (3, 9), until the work counter runs past the last cell
    wl = W.primordial(ncells=120000, seed=17)
    wl.t_stop[:] = 10.0 ** np.random.default_rng(17).uniform(-4.0, 0.0, wl.ncells)
    o = run_oracle(oracle, wl)
    assert np.all(o[3] == 0)
    for staging in (1, 3, 9):
        assert_bitwise(run_gpu(gpu_lib, wl, "fp64", staging=staging), o, "short solves staging %d" % staging)


def test_empty_and_group_size_errors(gpu_lib):
    import torch
    S = gpu_lib
    wl = W.rober(ncells=64)
    ode = S.Odevec(wl.network, nvector=32, raise_on_failure=False)
    S.InitOdevec(ode)
    try:
        y = torch.empty((3, 0), dtype=torch.float64, device="cuda")
        z = torch.empty(0, dtype=torch.float64, device="cuda")
        S.SolveODE(ode, z, z.clone(), z.clone(), y)  # nothing to do, no launch
        y = torch.tensor(wl.y[:, :33], device="cuda")
        with pytest.raises(S.OdevecError, match="divisible by 32"):
            S.SolveODE(ode, 0.0, 1e-10, 1e5, y)
    finally:
        S.CloseOdevec(ode)


# ------------------------------------ lanes per cell (stagings 7, 13, 14)
# 32, 16 or 8 lanes hold one cell (1, 2 or 4 cells per warp)
WPC_STAGINGS = [7, 13, 14]
WPC_CASES = [
    ("SYN64", dict(ncells=200), "SYN64_CSC_CMK"),
    ("ROBER", dict(ncells=256), "ROBER_CSC_NONE"),
    ("OREGO", dict(ncells=300), "OREGO_CSC_CMK"),
]


@pytest.mark.parametrize("staging", WPC_STAGINGS)
@pytest.mark.parametrize("name,kw,network", WPC_CASES)
def test_warp_per_cell_bit_exact_vs_oracle(gpu_lib, oracle, name, kw, network, staging):
    # K lanes per cell evaluate the network from tables of the emitted code
    # and must reproduce the oracle (and the thread-per-cell kernel) bit for bit
    wl = W.BUILDERS[name](network=network, **kw)
    wl.group = 1
    g = run_gpu(gpu_lib, wl, "fp64", group=1, staging=staging)
    o = run_oracle(oracle, wl, group=1)
    assert np.all(o[3] == 0)
    assert_bitwise(g, o, "%s lanes per cell, staging %d" % (network, staging))
    assert_bitwise(run_gpu(gpu_lib, wl, "fp64", group=1, staging=3), o, "%s thread per cell" % network)


@pytest.mark.parametrize("staging", WPC_STAGINGS)
def test_warp_per_cell_options(gpu_lib, oracle, staging):
    wl = W.syn64(ncells=96)
    mask = (np.arange(96) % 4 != 1).astype(np.uint8)
    assert_bitwise(run_gpu(gpu_lib, wl, "fp64", mask=mask, staging=staging), run_oracle(oracle, wl, mask=mask),
                   "mask")
    assert_bitwise(run_gpu(gpu_lib, wl, "fp64", check_negatives=True, staging=staging),
                   run_oracle(oracle, wl, check_negatives=True), "check negatives")
    g = run_gpu(gpu_lib, wl, "fp64", max_attempts=9, staging=staging)
    assert np.all(g[3] == 4)
    assert_bitwise(g, run_oracle(oracle, wl, max_attempts=9), "max attempts")


@pytest.mark.parametrize("staging", WPC_STAGINGS)
def test_warp_per_cell_resident(gpu_lib, oracle, staging):
    wl = W.syn64(ncells=64)
    _resident_steps(gpu_lib, oracle, wl, "fp64", 3, 1, staging=staging)


def test_warp_per_cell_fast_forms(gpu_lib, oracle):
    from odevec_b200 import syn64
    wl = W.syn64(ncells=256)
    o = run_oracle(oracle, wl)
    m = syn64.masses()
    # FMA and FP32 factors change roundings and with them the step sequence;
    # on this network tiny species then move by far more than rtol, in either
    # kernel.  Errors are taken relative to the species or 1e-6 of the cell's
    # largest one, and the warp kernel must do no worse than the thread kernel.
    floor = 1e-6 * np.max(np.abs(o[0]), axis=0)

    def err(g):
        return np.max(np.abs(g[0] - o[0]) / np.maximum(np.abs(o[0]), floor))

    for precision in ("fp64_fma", "fp32_lu"):
        ref = err(run_gpu(gpu_lib, wl, precision, staging=3))
        for staging in WPC_STAGINGS:
            g = run_gpu(gpu_lib, wl, precision, staging=staging)
            assert np.all(g[3] == 0)
            assert np.max(np.abs(m @ g[0] - m @ wl.y) / (m @ wl.y)) < 1e-4
            assert err(g) <= max(100 * wl.rtol, 2 * ref), (precision, staging, err(g), ref)
    # the automatic staging gives the warp kernel's bits as well
    assert_bitwise(run_gpu(gpu_lib, wl, "fp64"), run_gpu(gpu_lib, wl, "fp64", staging=7), "automatic staging")


@pytest.mark.parametrize("precision", ["fp64", "fp32_lu"])
def test_ranges_equal_whole_solve(gpu_lib, precision):
    """odevec_solve_range: a solve cut into three ranges of cells (row stride
    of the full arrays, resident workspace, two hydro steps) gives the bits of
    the whole solve."""
    import torch
    S = gpu_lib
    wl = W.primordial(ncells=1000, seed=17)

    def run(ranges):
        ode = S.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol, MinimalTimestep=wl.dt_min,
                       nvector=1, precision=precision, raise_on_failure=False)
        S.InitOdevec(ode)
        y = torch.tensor(wl.y, device="cuda")
        t = torch.tensor(wl.t0, device="cuda")
        d = torch.tensor(wl.dt0, device="cuda")
        ws = S.Workspace(ode, wl.ncells)
        status = torch.zeros(wl.ncells, dtype=torch.int32, device="cuda")
        for step in range(2):
            ts = torch.tensor(wl.t_stop * (step + 1), device="cuda")
            for c0, c1 in ranges:
                S.SolveODERange(ode, c0, c1, t, d, ts, y, status, workspace=ws, resume=step > 0)
        torch.cuda.synchronize()
        out = [a.cpu().numpy() for a in (y, t, d, status)]
        S.CloseOdevec(ode)
        return out
    whole = run([(0, wl.ncells)])
    parts = run([(0, 300), (300, 301), (301, wl.ncells)])
    assert np.all(whole[3] == 0)
    for a, b in zip(parts, whole):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name,network,ncells,precision,max_attempts,staging", [
    ("PRIMORDIAL", "PRIMORDIAL_CSC_FF", 100000, "fp64", 0, 0),
    ("PRIMORDIAL", "PRIMORDIAL_CSC_FF", 100000, "fp32_lu", 0, 0),
    ("PRIMORDIAL", "PRIMORDIAL_CSC_FF", 100000, "fp32_lu", 5, 0),   # every cell escalated
    ("PRIMORDIAL", "PRIMORDIAL_CSC_FF", 60000, "fp64", 0, 1),       # refill on every trip
    ("SYN64", "SYN64_CSC_CMK", 5000, "fp64", 0, 7),                 # 32 lanes per cell
    ("ROBER", "ROBER_DENSE_NONE", 65536, "fp64", 0, 0),             # lockstep groups of 32
])
def test_yield_and_continue_equal_one_solve(gpu_lib, name, network, ncells, precision, max_attempts, staging):
    """odevec_set_yield / odevec_solve_continue: with the yield flag set
    before the launch, a launch starts only its first round of cells and
    ends; continuations start the rest.  The results equal one uninterrupted
    solve bit for bit, the FP32-LU escalation included."""
    import torch
    S = gpu_lib
    wl = W.BUILDERS[name](ncells=ncells, network=network)
    if name == "ROBER":
        wl.group = 32

    def run(yielding):
        ode = S.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol, MinimalTimestep=wl.dt_min,
                       nvector=wl.group, precision=precision, max_attempts=max_attempts, raise_on_failure=False,
                       staging=staging)
        S.InitOdevec(ode)
        try:
            y = torch.tensor(wl.y, device="cuda")
            t, d, ts = (torch.tensor(a, device="cuda") for a in (wl.t0, wl.dt0, wl.t_stop))
            st = torch.zeros(ncells, dtype=torch.int32, device="cuda")
            launches = 1
            if yielding:
                flag = torch.ones(1, dtype=torch.int32, device="cuda")
                S.set_yield(ode, flag)
            S.SolveODERange(ode, 0, ncells, t, d, ts, y, st)
            if yielding:
                assert S.cells_started(ode) < ncells  # the first launch yielded
                while S.cells_started(ode) < ncells:
                    S.SolveODERange(ode, 0, ncells, t, d, ts, y, st, cont=True)
                    launches += 1
                    assert launches < 400
                S.set_yield(ode, None)
            torch.cuda.synchronize()
            return [a.cpu().numpy() for a in (y, t, d, st)], launches
        finally:
            S.CloseOdevec(ode)

    ref, _ = run(False)
    got, launches = run(True)
    assert launches >= 2
    for what, a, b in zip(("y", "t", "dt", "status"), got, ref):
        assert np.array_equal(a, b, equal_nan=True), what
    if max_attempts:
        assert np.sum(ref[3] == 4) >= 0.9 * ncells


@pytest.mark.parametrize("name,network,ncells,precision,staging", [
    ("PRIMORDIAL", "PRIMORDIAL_CSC_FF", 70000, "fp64", 0),
    ("PRIMORDIAL", "PRIMORDIAL_CSC_FF", 70000, "fp32_lu", 0),
    ("OREGO", "OREGO_CSC_CMK", 70000, "fp64", 0),
    ("SYN64", "SYN64_CSC_CMK", 40000, "fp64", 7),   # 32 lanes per cell
])
def test_visit_order_keeps_results(gpu_lib, name, network, ncells, precision, staging):
    """A solve of at least 32,768 cells visits them longest span first (a
    sort inside odevec_solve); the same cells solved as ranges below that
    size keep the given order.  Both give the same bits."""
    import torch
    S = gpu_lib
    wl = W.BUILDERS[name](ncells=ncells, network=network)

    def run(ranges):
        ode = S.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol, MinimalTimestep=wl.dt_min,
                       nvector=1, precision=precision, raise_on_failure=False, staging=staging)
        S.InitOdevec(ode)
        try:
            y = torch.tensor(wl.y, device="cuda")
            t, d, ts = (torch.tensor(a, device="cuda") for a in (wl.t0, wl.dt0, wl.t_stop))
            st = torch.zeros(ncells, dtype=torch.int32, device="cuda")
            for c0, c1 in ranges:
                S.SolveODERange(ode, c0, c1, t, d, ts, y, st)
            torch.cuda.synchronize()
            return [a.cpu().numpy() for a in (y, t, d, st)]
        finally:
            S.CloseOdevec(ode)

    whole = run([(0, ncells)])
    parts = run([(0, 30000), (30000, 60000), (60000, ncells)] if ncells > 60000 else [(0, 30000), (30000, ncells)])
    assert np.all(whole[3] == 0)
    for what, a, b in zip(("y", "t", "dt", "status"), whole, parts):
        assert np.array_equal(a, b, equal_nan=True), what
