"""The operator-split caller's formats: mass fractions and t_stop ladders.

A hydro code hands the chemistry its cells once per hydro step.  The
reference's drivers show the two formats this takes:

* mass fractions x and the gas density rho per cell, converted to number
  densities n = rho * x * imass before each solve and back with
  x = n * mass / rho after it (tests/primordial.f90:79-87, 113-140);
* one SolveODE call per entry of a t_stop ladder, the time carried from
  call to call and dt either carried (tests/primordial.f90:67-92) or reset
  before each call (tests/rober.f90:57-62, tests/orego.f90:117-123).

`convert` runs the conversion on the device (odevec_convert).  `Ladder`
runs a whole ladder on device-resident arrays; with ``graph=True`` the
per-call sequence (conversion, t_stop, mask of failed cells, solve, status
bookkeeping, conversion back) is captured once as a CUDA graph of
``chunk`` calls and replayed, so a ladder of thousands of calls costs no
Python or launch overhead per call.  Where the reference stops the program
on a failure, a failed cell here keeps its first nonzero status and is
masked out of the later calls.

`rober_schedule`, `orego_schedule` and `primordial_schedule` give the
reference drivers' ladders and inputs.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional, Sequence

import numpy as np

from . import solver as S

OV_X2N, OV_N2X = 0, 1


def convert(network: str, a, rho, direction: int, out=None, stream=None):
    """Mass fractions -> number densities (OV_X2N) or back (OV_N2X) on the
    device; a: (neq, ncells) CUDA float64 tensor, rho: (ncells,).  Entries
    without a species mass are copied.  Returns out (a new tensor unless given;
    may be a itself)."""
    import torch
    if not (torch.is_tensor(a) and a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()):
        raise ValueError("a must be a contiguous float64 CUDA tensor")
    if not (torch.is_tensor(rho) and rho.is_cuda and rho.dtype == torch.float64 and rho.numel() == a.shape[1]):
        raise ValueError("rho must be a float64 CUDA tensor with one entry per cell")
    if out is None:
        out = torch.empty_like(a)
    st = stream if stream is not None else torch.cuda.current_stream(a.device)
    S._check(S.lib().odevec_convert(network.encode(), a.shape[1], direction, ctypes.c_void_p(a.data_ptr()),
                                    ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(rho.data_ptr()),
                                    ctypes.c_void_p(st.cuda_stream)))
    return out


def x2n(network: str, x, rho, out=None, stream=None):
    return convert(network, x, rho, OV_X2N, out, stream)


def n2x(network: str, n, rho, out=None, stream=None):
    return convert(network, n, rho, OV_N2X, out, stream)


class Ladder:
    """One solve per t_stop on device-resident state.

    ode: an initialised Odevec (its options apply to every call).  y: (neq,
    ncells) CUDA tensor, updated in place: the state itself, or, with rho,
    mass fractions (species rows) and pass-through rows.  time, dt: scalars
    or per-cell tensors (carried from call to call; dt is set to dt_reset
    before each call when given).  run() returns (time, dt, status) tensors.
    """

    def __init__(self, ode: S.Odevec, y, time, dt, t_stops: Sequence[float], rho=None,
                 dt_reset: Optional[float] = None, graph: bool = False, chunk: int = 64):
        import torch
        self.torch = torch
        if ode._h is None:
            raise ValueError("InitOdevec first")
        if not (torch.is_tensor(y) and y.is_cuda and y.dtype == torch.float64 and y.is_contiguous()):
            raise ValueError("y must be a contiguous float64 CUDA tensor")
        self.ode, self.y = ode, y
        self.dev = y.device
        n = y.shape[1]
        self.ncells = n
        f64 = dict(dtype=torch.float64, device=self.dev)
        self.t = S._as_cells(time, n, "time", torch, self.dev).clone()
        self.d = S._as_cells(dt, n, "dt", torch, self.dev).clone()
        self.rho = rho
        self.state = torch.empty_like(y) if rho is not None else y
        self.t_stops = torch.tensor([float(v) for v in t_stops], **f64)
        self.k = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.ts = torch.empty(n, **f64)
        self.mask = torch.ones(n, dtype=torch.uint8, device=self.dev)
        self.status = torch.zeros(n, dtype=torch.int32, device=self.dev)
        self.failed = torch.zeros(n, dtype=torch.int32, device=self.dev)
        self.dt_reset = dt_reset
        self.graph = graph
        self.chunk = max(1, int(chunk))
        self._graphs = {}

    def _call(self):
        """One ladder entry on the current stream; every operation is a
        device operation, so the sequence can be captured."""
        torch = self.torch
        if self.dt_reset is not None:
            self.d.fill_(self.dt_reset)
        self.ts.copy_(self.t_stops.index_select(0, self.k).expand(self.ncells))
        self.k += 1
        self.mask.copy_(self.failed == 0)
        if self.rho is not None:
            x2n(self.ode.network, self.y, self.rho, out=self.state)
        st = torch.cuda.current_stream(self.dev)
        p = lambda a: ctypes.c_void_p(a.data_ptr())
        S._check(S.lib().odevec_solve(self.ode.handle, self.ncells, p(self.state), p(self.t), p(self.d),
                                      p(self.ts), p(self.mask), p(self.status), None,
                                      ctypes.c_void_p(st.cuda_stream)))
        torch.where(self.failed != 0, self.failed, self.status, out=self.failed)
        if self.rho is not None:
            n2x(self.ode.network, self.state, self.rho, out=self.y)

    def _graph_of(self, calls: int):
        """CUDA graph of `calls` ladder entries; the library's buffers are
        sized by an untimed call on scratch copies first."""
        torch = self.torch
        if calls in self._graphs:
            return self._graphs[calls]
        if not self._graphs:
            saved = [a.clone() for a in (self.y, self.t, self.d, self.k, self.failed, self.status)]
            side = torch.cuda.Stream(device=self.dev)
            side.wait_stream(torch.cuda.current_stream(self.dev))
            with torch.cuda.stream(side):
                self._call()
            torch.cuda.current_stream(self.dev).wait_stream(side)
            for a, b in zip((self.y, self.t, self.d, self.k, self.failed, self.status), saved):
                a.copy_(b)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for _ in range(calls):
                self._call()
        self._graphs[calls] = g
        return g

    def run(self):
        S._check(S.lib().odevec_set_options(self.ode.handle, ctypes.byref(self.ode._opts())))
        K = int(self.t_stops.numel())
        self.k.zero_()
        self.failed.zero_()
        if not self.graph:
            for _ in range(K):
                self._call()
        else:
            full, rest = divmod(K, self.chunk)
            if full:
                g = self._graph_of(self.chunk)
                for _ in range(full):
                    g.replay()
            if rest:
                self._graph_of(rest).replay()
        return self.t, self.d, self.failed


# ------------------------------------------------------ reference drivers
@dataclasses.dataclass
class Schedule:
    network: str
    y0: np.ndarray            # (neq, ncells): state, or mass fractions when rho is set
    time: float
    dt: float
    t_stops: List[float]
    rtol: float
    atol: float
    dt_min: float
    dt_reset: Optional[float] = None
    rho: Optional[np.ndarray] = None
    group: int = 1


def _f32(v: float) -> float:
    """A Fortran default-real literal as the double it becomes."""
    return float(np.float32(v))


def rober_schedule(ncells: int = 4096, network: str = "ROBER_DENSE_NONE", group: int = 32) -> Schedule:
    """tests/rober.f90:41-62: rtol 10^(-2-24/4), atol 1e-6 rtol, y = (1, 0, 0),
    t_stop = 1e-10, 1e-9, ... while below the real literal 1e11, dt = 1e-10
    before every call."""
    rtol = 10.0 ** (-2.0 - 24 * 0.25)
    ts, t = [], 1e-10
    while t < _f32(1e11):
        ts.append(t)
        t = t * 1e1
    y0 = np.zeros((3, ncells))
    y0[0] = 1.0
    return Schedule(network, y0, 0.0, 1e-5, ts, rtol, 1e-6 * rtol, 1e-20, dt_reset=1e-10, group=group)


def orego_schedule(ncells: int = 4096, network: str = "OREGO_CSC_CMK", t_end: float = 360.0,
                   dt_min: float = 1e-10) -> Schedule:
    """tests/orego.f90:42-123: rtol 10^(-2-32/4), atol 1e-6 rtol, y = (1, 2, 3),
    t_stop = 1, then + the real literal 0.01 while not above t_end, dt = 1e-10
    before every call (35,901 calls to 360)."""
    rtol = 10.0 ** (-2.0 - 32 * 0.25)
    ts, t = [], 1.0
    while t <= _f32(t_end):
        ts.append(t)
        t = t + _f32(0.01)
    y0 = np.zeros((3, ncells))
    y0[0], y0[1], y0[2] = 1.0, 2.0, 3.0
    return Schedule(network, y0, 0.0, 1e-10, ts, rtol, 1e-6 * rtol, dt_min, dt_reset=1e-10)


def primordial_schedule(ncells: int = 8192, network: str = "PRIMORDIAL_CSC_FF", tgas: float = 1000.0) -> Schedule:
    """tests/primordial.f90:43-92: mass fractions (H 0.75615, He 0.24375,
    e- 4.46406e-8, H+ 8.1967e-5, H2 1.5123e-6, traces 1e-40, the rest 1e-20)
    normalised per cell by their sum taken in index order, rho = 1e-10 g/cm^3,
    t_stop = 1e8, 2e8, ... up to 1e10, dt carried from
    2.2954626201190183E-026, rtol 1e-4, atol 1e-20, dt_min 1e-20.  Every
    real literal of the driver without a d exponent (the fractions, 1e-20,
    rho's 1e-10, the first dt, the loop bound 1e10) is single precision.
    The reference's rate function fixes Tgas at 1000 K; here the temperature
    row passes through the conversion and holds tgas."""
    from .networks import PRIMORDIAL_SPECIES as SP
    x = np.full((16, ncells), _f32(1e-20))
    vals = {"H": 0.75615, "E": 4.46406e-8, "H+": 8.1967e-5, "D": 1.0e-40, "D+": 1.0e-40, "HE": 0.24375,
            "HE+": 1.0e-40, "H2+": 1.0e-40, "H2": 1.5123e-6, "HD": 1.0e-40, "H-": 1.0e-40, "HE++": 1.0e-40}
    for name, v in vals.items():
        x[SP.index(name)] = _f32(v)
    total = x[0].copy()
    for j in range(1, 12):          # sum(x(i,:)) accumulates in index order
        total = total + x[j]
    x[:12] = x[:12] / total
    x[12:] = 0.0
    x[SP.index("Tgas")] = tgas
    ts, t = [], 0.0
    while t < _f32(1e10):
        t = t + 1e8
        ts.append(t)
    return Schedule(network, x, 0.0, _f32(2.2954626201190183e-26), ts, 1e-4, 1e-20, 1e-20,
                    rho=np.full(ncells, _f32(1e-10)))


def run_schedule(sch: Schedule, precision: str = "fp64", graph: bool = False, chunk: int = 64, ode=None):
    """Runs a schedule on the GPU; returns (y, time, dt, status) as NumPy."""
    import torch
    own = ode is None
    if own:
        ode = S.Odevec(sch.network, RelativeTolerance=sch.rtol, AbsoluteTolerance=sch.atol,
                       MinimalTimestep=sch.dt_min, nvector=sch.group, precision=precision,
                       raise_on_failure=False)
        S.InitOdevec(ode)
    try:
        y = torch.tensor(sch.y0, device="cuda")
        rho = None if sch.rho is None else torch.tensor(sch.rho, device="cuda")
        lad = Ladder(ode, y, sch.time, sch.dt, sch.t_stops, rho=rho, dt_reset=sch.dt_reset, graph=graph,
                     chunk=chunk)
        t, d, st = lad.run()
        torch.cuda.synchronize()
        return y.cpu().numpy(), t.cpu().numpy(), d.cpu().numpy(), st.cpu().numpy()
    finally:
        if own:
            S.CloseOdevec(ode)


def main(argv=None):
    """python -m odevec_b200.driver --schedule rober|orego|primordial [--cells N]
    [--graph] [--precision P] [--staging S]: runs a reference driver's ladder
    and prints the wall time per call."""
    import argparse
    import json
    import time
    import torch
    p = argparse.ArgumentParser()
    p.add_argument("--schedule", default="primordial", choices=["rober", "orego", "primordial"])
    p.add_argument("--cells", type=int, default=8192)
    p.add_argument("--graph", action="store_true")
    p.add_argument("--chunk", type=int, default=64)
    p.add_argument("--precision", default="fp64")
    p.add_argument("--t-end", type=float, default=360.0, help="OREGO ladder end")
    p.add_argument("--staging", type=int, default=0, help="launch shape (0: the tuning table)")
    a = p.parse_args(argv)
    if a.schedule == "rober":
        sch = rober_schedule(a.cells)
    elif a.schedule == "orego":
        sch = orego_schedule(a.cells, t_end=a.t_end)
    else:
        sch = primordial_schedule(a.cells)
    ode = S.Odevec(sch.network, RelativeTolerance=sch.rtol, AbsoluteTolerance=sch.atol, MinimalTimestep=sch.dt_min,
                   nvector=sch.group, precision=a.precision, raise_on_failure=False, staging=a.staging)
    S.InitOdevec(ode)
    y0 = torch.tensor(sch.y0, device="cuda")
    y = y0.clone()
    rho = None if sch.rho is None else torch.tensor(sch.rho, device="cuda")
    lad = Ladder(ode, y, sch.time, sch.dt, sch.t_stops, rho=rho, dt_reset=sch.dt_reset, graph=a.graph,
                 chunk=a.chunk)
    t_in, d_in = lad.t.clone(), lad.d.clone()
    lad.run()  # warm-up; with --graph this captures the graphs
    y.copy_(y0)
    lad.t.copy_(t_in)
    lad.d.copy_(d_in)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, _, st = lad.run()
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    st = st.cpu().numpy()
    S.CloseOdevec(ode)
    print(json.dumps({"schedule": a.schedule, "network": sch.network, "cells": a.cells, "calls": len(sch.t_stops),
                      "graph": a.graph, "precision": a.precision, "staging": a.staging, "seconds": el,
                      "ms_per_call": 1e3 * el / len(sch.t_stops), "failed_cells": int((st != 0).sum())}))


if __name__ == "__main__":
    main()
