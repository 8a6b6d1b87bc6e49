"""Serving loop: continuous batching of solve requests on one GPU.

A request is a set of cells of one network, as an operator-split hydro code
hands them over: it is advanced through `steps` successive hydro steps
(t_stop = t0 + k * dt_hydro), and between steps its integrator state --
Nordsieck history, order, step size, error weights -- stays resident on the
device (odevec_solve_resident), so a hydro step costs only the integration
steps it needs.

Continuous batching: requests arrive over time; a request is admitted as
soon as its device memory fits in the HBM budget and an execution slot (a
CUDA stream) is free, not when the previous batch ends.  Every admitted
request advances on its own stream, so the steps of different requests and
networks overlap on the device; a finished step immediately queues the
request's next step.  Cells are independent and every launch is
deterministic, so a request's results are the same alone and in any mix
(tests/test_serving.py).

Latency of a request step = completion time - the time the step became
ready (its arrival for step 0, the previous step's completion after that),
so it includes any wait for admission; service time = completion time -
launch time.

Sharing the device: the solve kernel is persistent (its blocks stay resident
until the request's cells run out), so a launch that takes every SM would
hold back every request behind it.  With fair sharing, the device's
resident blocks are shared by water-filling over the requests in flight:
in order of demand (the blocks a request's cells fill), each request gets
its demand or an equal part of what is left, whichever is smaller -- small
requests get what they can use and the large ones share the rest (never
fewer than one block per SM; everything when a request runs alone).
Requests of at most `small_cells` cells run on a higher-priority stream, so
their blocks are placed first whenever blocks retire; with `chunk_cells` a
large request's step is a series of shorter range launches, so blocks
retire often.

Failures: where the reference stops the program (src/odevec.F90:272-275,
380-390), a cell here gets a nonzero status.  A failed cell keeps its
first nonzero status and is masked out of the request's later hydro steps
(its state stays at the failure); the request still completes, and its
result carries the per-cell status next to the state.

The scheduler is backend-agnostic: GpuBackend drives the CUDA library;
tests drive the same scheduler with a CPU backend built on the oracle.
"""
from __future__ import annotations

import dataclasses
import time
from typing import Dict, List, Optional

import numpy as np


@dataclasses.dataclass
class Request:
    rid: int
    network: str
    y0: np.ndarray            # (neq, ncells)
    dt_hydro: float
    steps: int
    arrival: float            # seconds after the stream starts
    rtol: float
    atol: float
    dt_min: float
    dt_in: float = 1e-10

    @property
    def ncells(self) -> int:
        return self.y0.shape[1]


@dataclasses.dataclass
class StepRecord:
    rid: int
    step: int
    ncells: int
    network: str
    ready: float
    done: float
    launched: float = 0.0

    @property
    def latency(self) -> float:
        return self.done - self.ready

    @property
    def service(self) -> float:
        return self.done - self.launched


@dataclasses.dataclass
class Result:
    y: np.ndarray             # (neq, ncells) state after the last hydro step
    status: np.ndarray        # (ncells,) first nonzero status of each cell, 0 = OK

    @property
    def failed(self) -> int:
        return int(np.count_nonzero(self.status))


class Scheduler:
    """Admission by memory budget and slot count, FIFO by readiness."""

    def __init__(self, backend, hbm_budget: float, slots: int):
        self.backend = backend
        self.budget = float(hbm_budget)
        self.slots = int(slots)

    def run(self, requests: List[Request], realtime: bool = True, poll_s: float = 2e-4):
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        waiting: List[Request] = []            # arrived, not admitted
        active: Dict[int, dict] = {}           # rid -> state
        used = 0.0
        records: List[StepRecord] = []
        results: Dict[int, Result] = {}
        t_start = time.perf_counter()
        now = lambda: time.perf_counter() - t_start
        i = 0
        while i < len(pending) or waiting or active:
            t = now()
            if not realtime and not waiting and not active and i < len(pending):
                t = pending[i].arrival  # jump to the next arrival when idle
                t_start -= max(0.0, t - now())
            while i < len(pending) and pending[i].arrival <= now():
                waiting.append(pending[i])
                i += 1
            # admit in arrival order while memory and slots allow
            while waiting and len(active) < self.slots:
                r = waiting[0]
                need = self.backend.bytes_needed(r)
                if need > self.budget:
                    raise ValueError("request %d needs %.1f GB, more than the budget" % (r.rid, need / 1e9))
                if used + need > self.budget:
                    break
                waiting.pop(0)
                used += need
                h = self.backend.admit(r)
                active[r.rid] = {"req": r, "h": h, "step": 0, "ready": max(r.arrival, 0.0), "need": need,
                                 "launched": now()}
                self.backend.launch(h, 0, [s["req"] for s in active.values()])
            # completions
            done_any = False
            for rid in list(active):
                st = active[rid]
                if self.backend.finished(st["h"]):
                    done_any = True
                    tdone = now()
                    r = st["req"]
                    records.append(StepRecord(rid, st["step"], r.ncells, r.network, st["ready"], tdone,
                                              st["launched"]))
                    st["step"] += 1
                    if st["step"] < r.steps:
                        st["ready"] = tdone
                        st["launched"] = now()
                        self.backend.launch(st["h"], st["step"], [s["req"] for s in active.values()])
                    else:
                        results[rid] = self.backend.release(st["h"])
                        used -= st["need"]
                        del active[rid]
            if not done_any:
                time.sleep(poll_s)
        return records, results


def summarize(records: List[StepRecord], results: Optional[Dict[int, Result]] = None) -> dict:
    lat = np.array([r.latency for r in records]) if records else np.zeros(1)
    svc = np.array([r.service for r in records]) if records else np.zeros(1)
    t0 = min(r.ready for r in records) if records else 0.0
    t1 = max(r.done for r in records) if records else 1.0
    cells = sum(r.ncells for r in records)
    return {"request_steps": len(records), "cells": cells, "seconds": t1 - t0,
            "cells_per_s": cells / max(t1 - t0, 1e-12),
            "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
            "max_ms": 1e3 * float(lat.max()),
            "service_p50_ms": 1e3 * float(np.percentile(svc, 50)),
            "service_p99_ms": 1e3 * float(np.percentile(svc, 99))} | (
        {} if results is None else
        {"failed_cells": sum(results[rid].failed for rid in {r.rid for r in records} if rid in results)})


def water_fill(demands: Dict[int, int], capacity: int) -> Dict[int, int]:
    """Shares of `capacity` blocks: in order of demand (ties by id), each
    gets its demand or an equal part of what is left, whichever is smaller."""
    out = {}
    left, todo = int(capacity), len(demands)
    for rid, d in sorted(demands.items(), key=lambda kv: (kv[1], kv[0])):
        out[rid] = min(int(d), left // todo)
        left -= out[rid]
        todo -= 1
    return out


class GpuBackend:
    """Each admitted request owns device buffers, a resident workspace and a
    CUDA stream; launches are asynchronous and completion is an event."""

    def __init__(self, precision: str = "fp32_lu", device: str = "cuda", fair_share: bool = True,
                 small_cells: int = 16384, staging: int = 3, chunk_cells: int = 0, yield_to_small: bool = True):
        import torch
        from . import solver as S
        self.S = S
        self.torch = torch
        self.precision = precision
        self.device = device
        self.fair_share = fair_share
        self.small_cells = small_cells
        # launch shape for requests: three 128-thread blocks per SM, so blocks
        # of up to three requests share an SM.  The single-solve optimum (one
        # block per SM holding its shared memory) would leave SMs to a single
        # request and most of the device idle under many small requests.
        # staging 3 selects that shape per network (staging_for); any other
        # value is used for every request as given.
        self.staging = staging
        # chunk_cells > 0: a step of a larger request is launched as ranges of
        # at most this many cells, one after another on its stream, so that a
        # short request arriving meanwhile waits for one range, not the step
        self.chunk_cells = chunk_cells
        # yield_to_small: a large request's launch stops starting cells when a
        # new small request arrives (odevec_set_yield), ends once its running
        # cells are done, and is continued from its work counter when that
        # launch has completed (odevec_solve_continue).  The flag is a device
        # word (a flag in pinned host memory made the solve 3x slower), set
        # by a 4-byte copy on a control stream: the copy engine runs it while
        # the large launch holds every SM.
        self.yield_to_small = yield_to_small and not chunk_cells
        self.live: Dict[int, dict] = {}
        if self.yield_to_small:
            lo, hi = torch.cuda.Stream.priority_range()
            self._ctrl = torch.cuda.Stream(device=device, priority=hi)
            self._one = torch.ones(1, dtype=torch.int32).pin_memory()
            self._zero = torch.zeros(1, dtype=torch.int32).pin_memory()
        self.sms = torch.cuda.get_device_properties(device).multi_processor_count

    def staging_for(self, network: str) -> int:
        """The launch shape of a request's solves: staging 3's shape for all
        (three 128-thread blocks per SM), with the history in shared memory
        and soft lockstep (staging 21) where three blocks' histories fit an
        SM (up to 12 solver species), with the state vector in shared memory
        (staging 20) for networks above 32 solver species."""
        if self.staging != 3:
            return self.staging
        nd = (self.S.workspace_doubles(network) - 12) // 8  # 8 doubles per solver species + 12
        if nd > 32:
            return 20
        return 21 if nd <= 12 else 3

    def _solver(self, r: Request):
        # one solver handle per request: each owns its cell counter, so
        # concurrent launches on different streams never share one
        ode = self.S.Odevec(r.network, RelativeTolerance=r.rtol, AbsoluteTolerance=r.atol,
                            MinimalTimestep=r.dt_min, nvector=1, precision=self.precision,
                            raise_on_failure=False, staging=self.staging_for(r.network))
        self.S.InitOdevec(ode)
        return ode

    def bytes_needed(self, r: Request) -> float:
        per_cell = 8 * (r.y0.shape[0] + 3 + self.S.workspace_doubles(r.network)) + 4 + 8 * 8
        return float(per_cell * r.ncells)

    def admit(self, r: Request):
        torch = self.torch
        ode = self._solver(r)
        lo, hi = torch.cuda.Stream.priority_range()  # (lowest, highest): numerically hi <= lo
        stream = torch.cuda.Stream(device=self.device, priority=hi if r.ncells <= self.small_cells else lo)
        with torch.cuda.stream(stream):
            h = {"r": r, "ode": ode, "stream": stream,
                 "y": torch.tensor(r.y0, device=self.device),
                 "t": torch.zeros(r.ncells, dtype=torch.float64, device=self.device),
                 "dt": torch.full((r.ncells,), r.dt_in, dtype=torch.float64, device=self.device),
                 "ts": torch.empty(r.ncells, dtype=torch.float64, device=self.device),
                 "ws": self.S.Workspace(ode, r.ncells, self.device),
                 "failed": torch.zeros(r.ncells, dtype=torch.int32, device=self.device),
                 "mask": torch.ones(r.ncells, dtype=torch.uint8, device=self.device),
                 "ev": None, "flag": None, "running": False}
            if self.yield_to_small and r.ncells > self.small_cells:
                h["flag"] = torch.zeros(1, dtype=torch.int32, device=self.device)
                h["status"] = torch.zeros(r.ncells, dtype=torch.int32, device=self.device)
                self.S.set_yield(ode, h["flag"])
        self.live[r.rid] = h
        return h

    def _launch_whole(self, h, step: int, cont: bool):
        """A large request's step (or its continuation after a yield) as one
        range launch over all its cells, with a persistent status array."""
        torch = self.torch
        r = h["r"]
        with torch.cuda.stream(h["stream"]):
            h["flag"].copy_(self._zero, non_blocking=True)
            if not cont:
                h["status"].zero_()
            self.S.SolveODERange(h["ode"], 0, r.ncells, h["t"], h["dt"], h["ts"], h["y"], h["status"],
                                 Mask=h["mask"], stream=h["stream"], workspace=h["ws"], resume=h["step"] > 0,
                                 cont=cont)
            torch.where(h["failed"] != 0, h["failed"], h["status"], out=h["failed"])
            ev = torch.cuda.Event()
            ev.record(h["stream"])
            h["ev"] = ev
            h["running"] = True

    def share(self, r, active, staging: int) -> int:
        """Blocks for a launch of request r among the requests in flight
        `active` (r included; a count means that many equal requests).
        Water-filling in order of demand; at least one block per SM, since a
        persistent grid keeps its size after the others finish and a
        narrower one would leave SMs idle."""
        capacity = self.sms * self.S.BLOCKS_PER_SM.get(staging, 3)
        if not isinstance(active, (list, tuple)):
            return max(self.sms, capacity // max(int(active), 1))
        bs = self.S.CELLS_PER_BLOCK.get(staging, 128)
        demands = {}
        for p in active:
            n = p.ncells if not self.chunk_cells else min(p.ncells, self.chunk_cells)
            demands[p.rid] = -(-n // bs)
        if r.rid not in demands:
            return capacity  # r runs alone
        return max(self.sms, water_fill(demands, capacity)[r.rid])

    def launch(self, h, step: int, active=1):
        """active: the requests in flight (this one included), or their count."""
        torch = self.torch
        r = h["r"]
        if self.fair_share:
            h["ode"].grid_blocks = self.share(r, active, h["ode"].staging)
        if r.ncells <= self.small_cells and step == 0:
            # a new small request: running large launches stop starting cells
            # and continue, once done, with a share that counts it
            with torch.cuda.stream(self._ctrl):
                for o in self.live.values():
                    if o is not h and o["flag"] is not None and o["running"]:
                        o["flag"].copy_(self._one, non_blocking=True)
        with torch.cuda.stream(h["stream"]):
            h["ts"].fill_(r.dt_hydro * (step + 1))
            if step > 0:
                h["mask"].copy_(h["failed"] == 0)
            if h["flag"] is not None:
                h["step"] = step
                self._launch_whole(h, step, cont=False)
                return
            if self.chunk_cells and r.ncells > self.chunk_cells:
                if "status" not in h:
                    h["status"] = torch.empty(r.ncells, dtype=torch.int32, device=self.device)
                ode = h["ode"]
                for c0 in range(0, r.ncells, self.chunk_cells):
                    c1 = min(r.ncells, c0 + self.chunk_cells)
                    self.S.SolveODERange(ode, c0, c1, h["t"], h["dt"], h["ts"], h["y"], h["status"],
                                         Mask=h["mask"], stream=h["stream"], workspace=h["ws"],
                                         resume=step > 0)
                st = h["status"]
            else:
                self.S.SolveODE(h["ode"], h["t"], h["dt"], h["ts"], h["y"], Mask=h["mask"], stream=h["stream"],
                                want_stats=False, workspace=h["ws"], resume=step > 0)
                st = h["ode"].status
            torch.where(h["failed"] != 0, h["failed"], st, out=h["failed"])
            ev = torch.cuda.Event()
            ev.record(h["stream"])
            h["ev"] = ev

    def finished(self, h) -> bool:
        if h["ev"] is None or not h["ev"].query():
            return False
        if h["flag"] is not None and h["running"]:
            h["running"] = False
            if self.S.cells_started(h["ode"], h["stream"]) < h["r"].ncells:
                # it yielded: start the rest with a share of the requests now in flight
                if self.fair_share:
                    h["ode"].grid_blocks = self.share(h["r"], [o["r"] for o in self.live.values()],
                                                      h["ode"].staging)
                self._launch_whole(h, h["step"], cont=True)
                return False
        return True

    def release(self, h):
        h["stream"].synchronize()
        self.live.pop(h["r"].rid, None)
        if h["flag"] is not None:
            self.S.set_yield(h["ode"], None)
        res = Result(h["y"].cpu().numpy(), h["failed"].cpu().numpy())
        self.S.CloseOdevec(h["ode"])
        return res

    def close(self):
        pass


def make_stream(seed: int = 5, rate: float = 200.0, duration: float = 1.0,
                networks=("ROBER_DENSE_NONE", "PRIMORDIAL_CSC_FF", "SYN64_CSC_CMK"),
                cells=(1000, 262144), dt_hydro=(1e6, 1e11), steps: int = 50,
                max_requests: Optional[int] = None) -> List[Request]:
    """Poisson arrivals of requests drawn uniformly from `networks`, with
    log-uniform cell counts and hydro time steps (the serving configuration:
    200 requests/s, 1k-256k cells, dt 1e6-1e11 s, 50 steps each)."""
    from . import workloads as W
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    rid = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (max_requests is not None and rid >= max_requests):
            break
        net = networks[int(rng.integers(len(networks)))]
        n = int(round(10.0 ** rng.uniform(np.log10(cells[0]), np.log10(cells[1]))))
        name = net.split("_")[0]
        if name not in W.BUILDERS:
            raise ValueError("no workload generator for network %s" % net)
        wl = W.BUILDERS[name](ncells=n, seed=1000 + rid, network=net)
        dth = float(10.0 ** rng.uniform(np.log10(dt_hydro[0]), np.log10(dt_hydro[1])))
        out.append(Request(rid, net, wl.y, dth, steps, t, wl.rtol, wl.atol, wl.dt_min,
                           dt_in=float(wl.dt0[0])))
        rid += 1
    return out


def measure(rate: float = 200.0, duration: float = 0.25, steps: int = 50, cells=(1000, 262144),
            dt_hydro=(1e6, 1e11), networks=("ROBER_DENSE_NONE", "PRIMORDIAL_CSC_FF", "SYN64_CSC_CMK"),
            precisions=("fp32_lu", "fp64"), budget: float = 120e9, slots: int = 16, seed: int = 5,
            isolated: bool = False, fair_share: bool = True, chunk_cells: int = 0,
            staging: int = 3) -> List[dict]:
    """Runs a Poisson request stream through the scheduler on the GPU, per
    precision form; with isolated, every request is run again alone and the
    mix's step latencies are compared with the isolated ones."""
    reqs = make_stream(seed, rate, duration, tuple(networks), tuple(cells), tuple(dt_hydro), steps)
    outs = []
    for prec in precisions:
        be = GpuBackend(prec, fair_share=fair_share, chunk_cells=chunk_cells, staging=staging)
        # warm-up: one small request per network (module load, first launches)
        warm = [Request(10**6 + i, r.network, r.y0[:, :64].copy(), r.dt_hydro, 1, 0.0, r.rtol, r.atol,
                        r.dt_min, r.dt_in) for i, r in enumerate({r.network: r for r in reqs}.values())]
        Scheduler(be, budget, slots).run(warm, realtime=False)
        recs, res = Scheduler(be, budget, slots).run(reqs, realtime=True)
        mix = summarize(recs, res)
        offered = sum(r.ncells * r.steps for r in reqs) / duration
        out = {"form": prec, "requests": len(reqs), "rate": rate, "steps": steps, "chunk_cells": chunk_cells,
               "staging": staging,
               "cells": list(cells), "dt_hydro": list(dt_hydro), "seed": seed,
               "budget_gb": budget / 1e9, "slots": slots, "fair_share": fair_share,
               "mix": mix,
               # offered load: cell-steps asked for per second of arrivals, against
               # the cell-steps per second the device delivered in the mix
               "offered_cell_steps_per_s": offered, "load_factor": offered / mix["cells_per_s"]}
        by_net = {}
        for r in recs:
            by_net.setdefault(r.network, []).append(r)
        out["per_network"] = {k: summarize(v, res) for k, v in by_net.items()}
        if isolated:
            iso = {}
            iso_res = {}
            for r in reqs:
                rr, rs = Scheduler(be, budget, 1).run([dataclasses.replace(r, arrival=0.0)], realtime=False)
                iso_res.update(rs)
                for x in rr:
                    iso[(x.rid, x.step)] = x.latency
            ratio = np.array([x.latency / iso[(x.rid, x.step)] for x in recs])
            iso_l = np.array(list(iso.values()))
            sratio = np.array([x.service / iso[(x.rid, x.step)] for x in recs])
            lat_mix = np.array([x.latency for x in recs])
            # each request's result alone and in the mix
            same = all(np.array_equal(res[k].y, iso_res[k].y, equal_nan=True) and
                       np.array_equal(res[k].status, iso_res[k].status) for k in res)
            out["isolated"] = {"p50_ms": 1e3 * float(np.percentile(iso_l, 50)),
                               "p99_ms": 1e3 * float(np.percentile(iso_l, 99)),
                               "mix_over_isolated_p50": float(np.percentile(ratio, 50)),
                               "mix_over_isolated_p99": float(np.percentile(ratio, 99)),
                               "mix_p99_over_isolated_p99": float(np.percentile(lat_mix, 99)
                                                                  / np.percentile(iso_l, 99)),
                               "service_over_isolated_p50": float(np.percentile(sratio, 50)),
                               "service_over_isolated_p99": float(np.percentile(sratio, 99)),
                               "results_same_alone_and_in_mix": bool(same)}
        outs.append(out)
    return outs


def main(argv=None):
    """Serving measurement: python -m odevec_b200.serving [options]; prints one
    JSON line per precision form."""
    import argparse
    import json
    p = argparse.ArgumentParser()
    p.add_argument("--rate", type=float, default=200.0, help="mean arrivals per second (Poisson)")
    p.add_argument("--duration", type=float, default=0.25, help="seconds of arrivals")
    p.add_argument("--steps", type=int, default=50, help="hydro steps per request")
    p.add_argument("--min-cells", type=int, default=1000)
    p.add_argument("--max-cells", type=int, default=262144)
    p.add_argument("--dt-min", type=float, default=1e6, help="smallest hydro step (s)")
    p.add_argument("--dt-max", type=float, default=1e11, help="largest hydro step (s)")
    p.add_argument("--networks", default="ROBER_DENSE_NONE,PRIMORDIAL_CSC_FF,SYN64_CSC_CMK")
    p.add_argument("--precisions", default="fp32_lu,fp64")
    p.add_argument("--budget", type=float, default=120e9, help="HBM admission budget (bytes)")
    p.add_argument("--slots", type=int, default=16, help="requests in flight")
    p.add_argument("--seed", type=int, default=5)
    p.add_argument("--isolated", action="store_true", help="also time every request alone")
    p.add_argument("--no-fair-share", action="store_true",
                   help="every launch may take the whole device (no 1/k block share, one stream priority)")
    p.add_argument("--chunk-cells", type=int, default=0,
                   help="launch a larger request's step as ranges of at most this many cells (0: whole)")
    p.add_argument("--staging", type=int, default=3, help="launch shape of every request's solves")
    a = p.parse_args(argv)
    for out in measure(a.rate, a.duration, a.steps, (a.min_cells, a.max_cells), (a.dt_min, a.dt_max),
                       a.networks.split(","), a.precisions.split(","), a.budget, a.slots, a.seed,
                       a.isolated, not a.no_fair_share, a.chunk_cells, a.staging):
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
