"""Several networks in one launch.

Cells of different networks (different neq, different generated code) run
different code.  Two ways to put them on the device at once:

* ``fused=True``: one kernel launch (``odevec_solve_many``).  A
  multi-network kernel compiled for a set of variants (odevec_b200/build.py
  MULTI_SETS) gives each job a share of the blocks in proportion to its cells;
  a block whose job has no cells left takes cells of the other jobs, so the
  networks share every SM for the whole launch.  The register budget is that
  of the most demanding network in the set.
* ``fused=False``: one solve per network, each on its own stream forked from
  the capture stream, captured into a single CUDA graph; one replay (one
  cudaGraphLaunch) runs them concurrently, each with 1/k of the resident
  blocks (the serving loop's fair share), joined back into the caller's
  stream.

Results are those of the individual solves either way: every cell is
integrated independently and deterministically.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence

from . import solver as S


class SolveMany:
    """jobs: sequence of (ode, time, dt, t_stop, y) with device tensors of
    matching cell counts (time/dt updated in place, y in place).  Each ode
    must be initialised and must not be shared between jobs."""

    def __init__(self, jobs: Sequence[tuple], share: bool = True, fused: bool = False):
        import torch
        self.torch = torch
        self.fused = fused
        self.jobs: List[tuple] = list(jobs)
        if len({id(j[0]) for j in self.jobs}) != len(self.jobs):
            raise ValueError("every job needs its own Odevec")
        for ode, t, d, ts, y in self.jobs:
            if not all(torch.is_tensor(a) and a.is_cuda for a in (t, d, ts, y)):
                raise ValueError("SolveMany takes CUDA tensors")
            ode.raise_on_failure = False  # no host reads inside the graph
        if share:
            sms = torch.cuda.get_device_properties(self.jobs[0][4].device).multi_processor_count
            k = len(self.jobs)
            for ode, *_ in self.jobs:
                # 1/k of the resident blocks of the staging each solve runs with
                ode.grid_blocks = max(sms, sms * S.BLOCKS_PER_SM.get(ode.staging, 3) // k)
        self.graph = None
        self.statuses = None

    def _launch_all(self):
        torch = self.torch
        main = torch.cuda.current_stream()
        streams = [torch.cuda.Stream() for _ in self.jobs]
        out = []
        for st, (ode, t, d, ts, y) in zip(streams, self.jobs):
            st.wait_stream(main)
            with torch.cuda.stream(st):
                S.SolveODE(ode, t, d, ts, y, want_stats=False, stream=st)
                out.append(ode.status)
        for st in streams:
            main.wait_stream(st)
        return out

    def capture(self):
        """Sizes the library's buffers with an untimed eager pass on copies,
        then captures the solves."""
        torch = self.torch
        saved = [(t.clone(), d.clone(), y.clone()) for _, t, d, _, y in self.jobs]
        self._launch_all()
        torch.cuda.synchronize()
        for (_, t, d, _, y), (t0, d0, y0) in zip(self.jobs, saved):
            t.copy_(t0)
            d.copy_(d0)
            y.copy_(y0)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.statuses = self._launch_all()
        self.graph = g
        return self

    def _launch_fused(self, stream=None):
        torch = self.torch
        n = len(self.jobs)
        arr = (S._Job * n)()
        statuses = []
        for k, (ode, t, d, ts, y) in enumerate(self.jobs):
            o = ode._opts()
            S._check(S.lib().odevec_set_options(ode.handle, ctypes.byref(o)))
            st = torch.empty(y.shape[1], dtype=torch.int32, device=y.device)
            statuses.append(st)
            arr[k].solver = ode.handle
            arr[k].ncells = y.shape[1]
            arr[k].y, arr[k].t, arr[k].dt, arr[k].t_stop = (y.data_ptr(), t.data_ptr(), d.data_ptr(),
                                                             ts.data_ptr())
            arr[k].status = st.data_ptr()
            ode.status = st
        s = stream if stream is not None else torch.cuda.current_stream()
        S._check(S.lib().odevec_solve_many(arr, n, ctypes.c_void_p(s.cuda_stream)))
        return statuses

    def run(self):
        """One launch for all networks (one kernel with fused=True, one graph
        replay otherwise); returns the per-job status tensors."""
        if self.fused:
            self.statuses = self._launch_fused()
            return self.statuses
        if self.graph is None:
            self.capture()
        self.graph.replay()
        return self.statuses


def compare(cells=(65536, 262144, 16384), precision="fp32_lu", repeats=3, seed=7):
    """Times the serving mix's networks (ROBER, PRIMORDIAL, the 64-species
    network; `cells` each) solved together as one fused kernel launch and as
    one graph of concurrent kernels; returns milliseconds per launch (best
    of `repeats`, CUDA events) and whether both gave the same bits."""
    import torch
    from . import workloads as W
    wls = [W.rober(ncells=cells[0], seed=seed), W.primordial(ncells=cells[1], seed=seed),
           W.syn64(ncells=cells[2], seed=seed)]
    out = {"cells": list(cells), "precision": precision}
    results = {}
    for fused in (True, False):
        jobs, init = [], []
        for wl in wls:
            ode = S.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                           MinimalTimestep=wl.dt_min, nvector=1, precision=precision, raise_on_failure=False,
                           escalation=False, staging=3)
            S.InitOdevec(ode)
            arrs = [torch.tensor(a, device="cuda") for a in (wl.t0, wl.dt0, wl.t_stop, wl.y)]
            init.append([a.clone() for a in arrs])
            jobs.append((ode, arrs[0], arrs[1], arrs[2], arrs[3]))
        sm = SolveMany(jobs, fused=fused)
        best = None
        for _ in range(repeats + 1):
            for (ode, t, d, ts, y), a0 in zip(jobs, init):
                t.copy_(a0[0])
                d.copy_(a0[1])
                y.copy_(a0[3])
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            sm.run()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out["fused_ms" if fused else "graph_ms"] = best
        results[fused] = [j[4].cpu().numpy() for j in jobs]
        for ode, *_ in jobs:
            S.CloseOdevec(ode)
    import numpy as np
    out["same_results"] = all(np.array_equal(a, b) for a, b in zip(results[True], results[False]))
    out["fused_over_graph"] = out["graph_ms"] / out["fused_ms"]
    return out


if __name__ == "__main__":
    import json
    import sys
    prec = sys.argv[1] if len(sys.argv) > 1 else "fp32_lu"
    print(json.dumps(compare(precision=prec)))
