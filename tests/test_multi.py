"""Several networks in one graph launch give the results of separate solves."""
import numpy as np
import pytest

from odevec_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_one_launch_many_networks(gpu_lib):
    import torch
    from odevec_b200.multi import SolveMany
    S = gpu_lib
    wls = [W.rober(ncells=1024), W.orego(ncells=2000), W.primordial(ncells=3000),
           W.syn64(ncells=500)]
    precs = ["fp64", "fp64_fma", "fp32_lu", "fp64"]

    def make(wl, prec):
        ode = S.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                       MinimalTimestep=wl.dt_min, nvector=wl.group, precision=prec, raise_on_failure=False)
        S.InitOdevec(ode)
        arrs = [torch.tensor(a, device="cuda") for a in (wl.t0, wl.dt0, wl.t_stop, wl.y)]
        return (ode, arrs[0], arrs[1], arrs[2], arrs[3])

    alone = []
    for wl, p in zip(wls, precs):
        ode, t, d, ts, y = make(wl, p)
        S.SolveODE(ode, t, d, ts, y)
        alone.append((y.cpu().numpy(), t.cpu().numpy(), d.cpu().numpy()))
        S.CloseOdevec(ode)
    jobs = [make(wl, p) for wl, p in zip(wls, precs)]
    st = SolveMany(jobs).run()
    torch.cuda.synchronize()
    for (ode, t, d, ts, y), ref, s in zip(jobs, alone, st):
        assert int((s != 0).sum()) == 0
        for a, b in zip((y.cpu().numpy(), t.cpu().numpy(), d.cpu().numpy()), ref):
            assert np.array_equal(a, b)
        S.CloseOdevec(ode)


def test_one_kernel_many_networks(gpu_lib):
    """odevec_solve_many: ROBER, PRIMORDIAL and the 64-species network in one
    kernel launch (the compiled serving set), FP64 and FP32-LU, give every
    job's results of its own solve, bit for bit."""
    import torch
    from odevec_b200.multi import SolveMany
    S = gpu_lib
    wls = [W.rober(ncells=700), W.primordial(ncells=3000), W.syn64(ncells=300)]
    for prec in ("fp64", "fp32_lu"):
        def make(wl):
            ode = S.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                           MinimalTimestep=wl.dt_min, nvector=1, precision=prec, raise_on_failure=False,
                           escalation=False, staging=3)
            S.InitOdevec(ode)
            arrs = [torch.tensor(a, device="cuda") for a in (wl.t0, wl.dt0, wl.t_stop, wl.y)]
            return (ode, arrs[0], arrs[1], arrs[2], arrs[3])
        alone = []
        for wl in wls:
            ode, t, d, ts, y = make(wl)
            S.SolveODE(ode, t, d, ts, y)
            alone.append((y.cpu().numpy(), t.cpu().numpy(), d.cpu().numpy(), ode.status.cpu().numpy()))
            S.CloseOdevec(ode)
        jobs = [make(wl) for wl in wls]
        st = SolveMany(jobs, fused=True).run()
        torch.cuda.synchronize()
        for (ode, t, d, ts, y), ref, s in zip(jobs, alone, st):
            got = (y.cpu().numpy(), t.cpu().numpy(), d.cpu().numpy(), s.cpu().numpy())
            for a, b in zip(got, ref):
                assert np.array_equal(a, b), prec
            S.CloseOdevec(ode)


def test_solve_many_rejects(gpu_lib):
    import ctypes
    import torch
    S = gpu_lib
    wl = W.orego(ncells=64)
    ode = S.Odevec(wl.network, nvector=1)
    S.InitOdevec(ode)
    try:
        y = torch.tensor(wl.y, device="cuda")
        t, d, ts = (torch.tensor(a, device="cuda") for a in (wl.t0, wl.dt0, wl.t_stop))
        job = (S._Job * 1)()
        job[0].solver, job[0].ncells = ode.handle, 64
        job[0].y, job[0].t, job[0].dt, job[0].t_stop = y.data_ptr(), t.data_ptr(), d.data_ptr(), ts.data_ptr()
        rc = S.lib().odevec_solve_many(job, 1, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == -5 and b"no multi-network kernel" in S.lib().odevec_last_error()   # OREGO not in a set
        assert S.lib().odevec_solve_many(job, 0, None) == -1
    finally:
        S.CloseOdevec(ode)
