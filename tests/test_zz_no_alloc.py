"""The allocation-free solve entry point against the regular one.

odevec_solve_noalloc is for callers that cannot allocate device memory
themselves (a host code handing over its own device arrays from a region
where cudaMalloc is not allowed); it keeps the kernel's only scratch, the
counter that hands out cells, in a static device array shared by all calls.
This test calls it twice in a row through the C ABI -- the second call must
not see the first call's counter -- and checks both results against
odevec_solve on the same inputs, and that the second call leaves the
device's free memory unchanged (nothing allocated).  FP64 without fused
multiply-add is compared bit for bit, as everywhere in the GPU tests;
FP32-LU likewise, since both entry points run the same kernel.  The file is named to be
collected last, so a run that stops at its first failure has run every
other test before it.
"""
import ctypes

import numpy as np
import pytest

from odevec_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _noalloc_fn(S):
    L = S.lib()
    f = L.odevec_solve_noalloc
    f.argtypes = [ctypes.c_char_p, ctypes.POINTER(S._Opts), ctypes.c_int64] + [ctypes.c_void_p] * 8
    f.restype = ctypes.c_int32
    return f


def _solve(S, wl, precision, noalloc, check_free=False):
    import torch
    # the allocation-free entry point has no FP32-LU escalation: compare with
    # the regular entry point without it
    ode = S.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                   MinimalTimestep=wl.dt_min, nvector=wl.group, precision=precision,
                   raise_on_failure=False, escalation=False)
    y = torch.tensor(wl.y, device="cuda")
    t = torch.tensor(wl.t0, device="cuda")
    dt = torch.tensor(wl.dt0, device="cuda")
    ts = torch.tensor(wl.t_stop, device="cuda")
    status = torch.full((wl.ncells,), -1, dtype=torch.int32, device="cuda")
    stats = torch.zeros((wl.ncells, S.OV_NSTATS), dtype=torch.int32, device="cuda")
    ptr = lambda a: ctypes.c_void_p(a.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if noalloc:
        opts = ode._opts()
        fn = _noalloc_fn(S)
        # every input and output exists before the first reading of free memory
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = fn(wl.network.encode(), ctypes.byref(opts), wl.ncells, ptr(y), ptr(t),
                ptr(dt), ptr(ts), None, ptr(status), ptr(stats), stream)
        assert rc == 0, S.lib().odevec_last_error().decode()
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if check_free:
            assert free_after == free_before, \
                "device free memory changed by %d bytes" % (free_before - free_after)
    else:
        S.InitOdevec(ode)
        try:
            S.SolveODE(ode, t, dt, ts, y)
            status, stats = ode.status, ode.stats
        finally:
            S.CloseOdevec(ode)
    torch.cuda.synchronize()
    return [a.cpu().numpy() for a in (y, t, dt, status, stats)]


@pytest.mark.parametrize("precision", ["fp64", "fp32_lu"])
def test_noalloc_matches_regular_entry_twice(gpu_lib, precision):
    wl = W.primordial(ncells=3000, seed=21)
    ref = _solve(gpu_lib, wl, precision, noalloc=False)
    assert np.all(ref[3] == 0)
    for call in range(2):
        # the first call may load the kernel's module (lazy loading) and look
        # up the scratch address; the second must leave device memory as it was
        got = _solve(gpu_lib, wl, precision, noalloc=True, check_free=call == 1)
        for name, a, b in zip(["y", "t", "dt", "status", "stats"], got, ref):
            assert np.array_equal(a, b), "call %d: %s differs" % (call + 1, name)


def test_noalloc_lockstep_and_limits(gpu_lib):
    wl = W.rober(ncells=256)
    ref = _solve(gpu_lib, wl, "fp64", noalloc=False)
    for call in range(2):
        got = _solve(gpu_lib, wl, "fp64", noalloc=True)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
    S = gpu_lib
    opts = S.Odevec(wl.network)._opts()
    fn = _noalloc_fn(S)
    big = (1 << 40) + 1
    rc = fn(wl.network.encode(), ctypes.byref(opts), big, *([ctypes.c_void_p(8)] * 4), None, None,
            None, None)
    assert rc == -6 and b"maximum" in S.lib().odevec_last_error()
