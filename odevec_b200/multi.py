"""Several networks in one launch.

Cells of different networks (different neq, different generated code) need
different kernels.  `SolveMany` captures one solve per network, each on its
own stream forked from the capture stream, into a single CUDA graph; one
replay (one cudaGraphLaunch) then runs all of them concurrently on the
device, with the per-request fair block share of the serving loop (each
solve gets 1/k of the resident blocks), and joins them back into the
caller's stream.  Results are those of the individual solves: every cell is
integrated independently and deterministically.
"""
from __future__ import annotations

from typing import List, Sequence

from . import solver as S


class SolveMany:
    """jobs: sequence of (ode, time, dt, t_stop, y) with device tensors of
    matching cell counts (time/dt updated in place, y in place).  Each ode
    must be initialised and must not be shared between jobs."""

    def __init__(self, jobs: Sequence[tuple], share: bool = True):
        import torch
        self.torch = torch
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

    def run(self):
        """One graph launch for all networks; returns the per-job status tensors."""
        if self.graph is None:
            self.capture()
        self.graph.replay()
        return self.statuses
