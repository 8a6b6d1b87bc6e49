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
