#!/usr/bin/env python
"""Benchmark of the OdeVec solve path on B200.

Metric: PRIMORDIAL cells/s to t_end at rtol 1e-6 (the 16-species primordial
network, 1,048,576 cells per GPU, per-cell temperature and t_end), reported
for the FP32-LU/FP64-residual form (``value``) beside the FP64 form of the
same kernel (bit-identical to the CPU oracle), the FP64 form with fused
multiply-add, and a plain FP64 port (a thread per cell that takes the next
cell from the work queue on every trip, no batching, no lockstep).  Launch
options come from the autotuner's table
(odevec_b200/tuning.json).  One step = one complete solve of all cells from
the initial state to their t_end; inputs are reset from a device copy before
each step (159 MB of inputs, larger than the 126 MB L2).  ``e2e`` is the same
solve through the C-ABI host entry with pinned host buffers.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference]
                    [--workload PRIMORDIAL|ROBER|OREGO|SYN64 --network TAG]

Multi-GPU (torchrun, one process per GPU): every rank integrates its own
1,048,576 cells (weak scaling; cells are independent, no data exchange);
timing is the maximum over ranks.  ``--impl reference`` times the CPU
restatement of the reference solver (oracle/) on the host cores instead.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PRIMORDIAL cells/s to t_end at rtol 1e-6, FP32-LU vs FP64 path; p50/p99 latency"
WORKLOAD = ("PRIMORDIAL 16-species/38-reaction network, %d cells per GPU, log-uniform n_H 1e-2..1e6, "
            "T 10..1e4 K, t_end 1e8..1e13 s, rtol 1e-6, atol 1e-20")
DATA = "synthetic: seeded inputs with the configuration's distributions (no public data set)"


def parse():
    from odevec_b200 import workloads as W
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="product", choices=["product", "reference"])
    p.add_argument("--ncells", type=int, default=1048576)
    p.add_argument("--network", default="PRIMORDIAL_CSC_FF")
    p.add_argument("--workload", default="PRIMORDIAL", choices=sorted(W.BUILDERS),
                   help="seeded input set (odevec_b200.workloads), solved with its group size; "
                        "the headline is PRIMORDIAL (the accuracy block is PRIMORDIAL only)")
    p.add_argument("--forms", default="fp32_lu,fp64,fp64_fma,plain_fp64",
                   help="fp32_lu | fp64 | fp64_fma | plain_fp64 (FP64, a thread per cell, refilled from "
                        "the work queue on every trip, Jacobian and step-size blocks run where a cell "
                        "needs them)")
    p.add_argument("--staging", type=int, default=0,
                   help="launch shape of the timed forms (0: the tuning table's; see odevec_opts.staging)")
    p.add_argument("--cpu-sample", type=int, default=65536)
    p.add_argument("--accuracy-cells", type=int, default=256)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-configs", action="store_true", help="skip the ROBER/OREGO/SYN64 lines")
    p.add_argument("--serving-duration", type=float, default=8.0,
                   help="seconds of Poisson arrivals in the serving block (0: no serving block)")
    p.add_argument("--serving-rate", type=float, default=1.0, help="mean arrivals per second")
    p.add_argument("--serving-seed", type=int, default=5)
    return p.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class ClockSampler:
    """SM clock and throttle reasons sampled every 100 ms (NVML)."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            names = {
                "hw_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwSlowdown", 0x8),
                "sw_thermal_slowdown": getattr(nv, "nvmlClocksThrottleReasonSwThermalSlowdown", 0x20),
                "hw_thermal_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwThermalSlowdown", 0x40),
                "sw_power_cap": getattr(nv, "nvmlClocksThrottleReasonSwPowerCap", 0x4),
            }
            while not self._stop.is_set():
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                for k, bit in names.items():
                    if r & bit:
                        self.reasons.add(k)
                self._stop.wait(0.1)
        except Exception as e:  # NVML missing: report no samples
            self.reasons.add("nvml_unavailable:%s" % type(e).__name__)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def fma_peaks(torch):
    """Measured FMA throughput (TFLOP/s) of this GPU, FP64 and FP32."""
    import ctypes
    from odevec_b200 import solver as S
    L = S.lib()
    L.odevec_probe_fma.argtypes = [ctypes.c_int32] * 4 + [ctypes.c_void_p] * 2 + [
        ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)]
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    scratch = torch.zeros(sms * 64, dtype=torch.float64, device="cuda")
    out = {}
    for name, fp64, iters in (("fp64", 1, 4096), ("fp32", 0, 8192)):
        best = 0.0
        for _ in range(3):
            ms, fl = ctypes.c_float(), ctypes.c_double()
            S._check(L.odevec_probe_fma(fp64, sms * 8, 512, iters, ctypes.c_void_p(scratch.data_ptr()),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                        ctypes.byref(ms), ctypes.byref(fl)))
            best = max(best, fl.value / (ms.value * 1e-3) / 1e12)
        out[name] = best
    return out


def workload_label(args, n):
    if args.workload == "PRIMORDIAL":
        return WORKLOAD % n
    return "%s seeded synthetic cells (odevec_b200.workloads.%s), %d cells per GPU" % (
        args.workload, args.workload.lower(), n)


def traffic_per_cell():
    """DRAM bytes per cell of the solve kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "bdf_kernel_primordial_ncu.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_cell:"):
            return float(line.split(":")[1])
    return None


def oracle_rate(wl, ncells, threads, fast=True):
    """cells/s of the CPU restatement of the reference (oracle/) on the first
    ncells cells: fast = the -O3 -march=native build with contraction, else
    the parity build (-O2, no contraction, bit-identical to the GPU fp64 form)"""
    from oracle import oracle as O
    sub = slice(0, ncells)
    O.lib(fast=fast)            # build / load outside the timed region
    t0 = time.perf_counter()
    _, _, _, st, _ = O.solve(wl.network, wl.y[:, sub], wl.t0[sub], wl.dt0[sub], wl.t_stop[sub], wl.rtol,
                             wl.atol, wl.dt_min, group=wl.group, nthreads=threads, fast=fast)
    el = time.perf_counter() - t0
    return ncells / el, el, int((st != 0).sum())


def cpu_model():
    from oracle import build as OB
    return OB.cpu_model()


def cpu_baseline(wl, ncells, threads):
    """the reported CPU baseline: the -O3 build timed on ncells cells, the
    parity build beside it"""
    v, el, f = oracle_rate(wl, ncells, threads, fast=True)
    vp, elp, _ = oracle_rate(wl, ncells, threads, fast=False)
    return {"value": v, "unit": "cells/s", "cores": threads, "kind": "port_O3",
            "cpu_model": cpu_model(),
            "sample": "%d cells of the same workload (%.1f s), oracle/ C restatement of src/odevec.F90 "
                      "built -O3 -march=native, OpenMP over cells" % (ncells, el),
            "failed_cells": f,
            "parity_build": {"value": vp, "kind": "port", "sample_s": elp,
                             "build": "-O2 -ffp-contract=off (bit-identical to the GPU fp64 form)"}}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from odevec_b200 import workloads as W
    wl = W.BUILDERS[args.workload](ncells=args.cpu_sample, seed=3, network=args.network)
    threads = host_threads()
    for _ in range(args.warmup):
        oracle_rate(wl, args.cpu_sample, threads)
    times = []
    for _ in range(args.steps):
        _, el, _ = oracle_rate(wl, args.cpu_sample, threads)
        times.append(el)
    value = args.cpu_sample * len(times) / sum(times)
    vp, elp, _ = oracle_rate(wl, args.cpu_sample, threads, fast=False)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA,
        "config": {"workload": workload_label(args, args.ncells), "network": args.network,
                   "sample_cells_per_step": args.cpu_sample},
        "cpu_baseline": {"value": value, "unit": "cells/s", "cores": threads, "kind": "port_O3",
                         "cpu_model": cpu_model(),
                         "sample": "%d of the workload's cells per step, oracle/ (C restatement of "
                                   "src/odevec.F90) built -O3 -march=native, %s, OpenMP over cells" % (
                                       args.cpu_sample, "per-cell control" if wl.group == 1 else
                                       "lockstep groups of %d" % wl.group),
                         "parity_build": {"value": vp, "kind": "port", "sample_s": elp,
                                          "build": "-O2 -ffp-contract=off"}},
        "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_product(args):
    import torch
    import torch.distributed as dist
    from odevec_b200 import metrics, solver as S, workloads as W

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    dev = torch.device("cuda", local_rank)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    wl = W.BUILDERS[args.workload](ncells=args.ncells, seed=3 + rank, network=args.network)
    N = wl.ncells
    y0 = torch.tensor(wl.y, device=dev)
    t0 = torch.tensor(wl.t0, device=dev)
    d0 = torch.tensor(wl.dt0, device=dev)
    ts = torch.tensor(wl.t_stop, device=dev)
    y = torch.empty_like(y0)
    t = torch.empty_like(t0)
    d = torch.empty_like(d0)
    stream = torch.cuda.current_stream(dev)
    forms = args.forms.split(",")
    res = {}
    clocks = None
    for form in forms:
        kw = {}
        if form == "plain_fp64":
            # the reference's loop structure ported one thread per cell: a grid
            # of one thread per cell whose finished lanes take unstarted cells
            # from the work queue on every trip, every Jacobian and step-size
            # block run at once by the lanes that need it (no batching), two
            # 128-thread blocks per SM, no lockstep, arrays thread-local
            kw = dict(jac_batch=1, ss_batch=1, max_wait=-1, staging=1, grid_blocks=(N + 127) // 128)
        if args.staging and form != "plain_fp64":
            kw = dict(staging=args.staging)
        ode = S.Odevec(wl.network, max_cells=N, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                       MinimalTimestep=wl.dt_min, nvector=wl.group, precision="fp64" if form == "plain_fp64" else form,
                       raise_on_failure=False, **kw)
        S.InitOdevec(ode)

        def reset():
            y.copy_(y0)
            t.copy_(t0)
            d.copy_(d0)

        # untimed run with counters: failures and the algorithmic work
        reset()
        S.SolveODE(ode, t, d, ts, y, want_stats=True)
        torch.cuda.synchronize()
        stats = ode.stats.cpu().numpy()
        fails = int((ode.status != 0).sum().item())
        flops = float(metrics.flops_per_cell(wl.network, stats).sum())
        for _ in range(args.warmup):
            reset()
            S.SolveODE(ode, t, d, ts, y, want_stats=False)
        torch.cuda.synchronize()
        barrier()
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
        with ClockSampler(local_rank) as cs:
            for k in range(args.steps):
                ev[k][0].record(stream)
                reset()
                ev[k][1].record(stream)
                S.SolveODE(ode, t, d, ts, y, want_stats=False)
                ev[k][2].record(stream)
            torch.cuda.synchronize()
        barrier()
        total_s = ev[0][0].elapsed_time(ev[-1][2]) / 1e3
        kern = [ev[k][1].elapsed_time(ev[k][2]) / 1e3 for k in range(args.steps)]
        steps_ms = [ev[k][0].elapsed_time(ev[k][2]) for k in range(args.steps)]
        total_s = max_over_ranks(total_s)
        kern_mean = max_over_ranks(sum(kern) / len(kern))

        # end to end through the C-ABI host entry (SolveODE on NumPy arrays ->
        # odevec_solve_host): y, t, dt, t_stop in pinned host memory, which
        # the kernel reads when it sets a cell up and writes when the cell is
        # done (the transfers overlap the solve), status copied back; the
        # call is synchronous, so the wall clock around it is its
        # device-inclusive time
        yh = torch.empty(wl.y.shape, dtype=torch.float64).pin_memory().numpy()
        th = torch.empty(N, dtype=torch.float64).pin_memory().numpy()
        dh = torch.empty(N, dtype=torch.float64).pin_memory().numpy()
        tsh = torch.empty(N, dtype=torch.float64).pin_memory().numpy()
        tsh[:] = wl.t_stop
        e2e_steps = max(1, min(args.steps, 3))
        e2e_times = []
        for k in range(e2e_steps + 1):
            yh[:] = wl.y
            th[:] = wl.t0
            dh[:] = wl.dt0
            barrier()
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            S.SolveODE(ode, th, dh, tsh, yh, want_stats=False, in_place=True)
            w1 = time.perf_counter()
            if k:  # the first call sizes the solver's host-path buffers
                e2e_times.append(w1 - w0)
        e2e_s = max_over_ranks(sum(e2e_times))
        barrier()
        res[form] = {
            "value": world * N * args.steps / total_s,
            "ms_per_step": 1e3 * total_s / args.steps,
            "kernel_ms": 1e3 * kern_mean,
            "step_ms": steps_ms,
            "flops_per_launch": flops,
            "failed_cells": fails,
            "mean_newton_iters": float(stats[:, 4].mean()),
            "mean_jac_evals": float(stats[:, 5].mean()),
            "mean_steps": float(stats[:, 0].mean()),
            "fp64_share": metrics.fp64_fraction(wl.network, stats, form == "fp32_lu"),
            "e2e": world * N * e2e_steps / e2e_s,
            "clocks": cs.summary(),
            # the solve kernel; FP32-LU adds the escalation kernel and the FP64
            # re-solve launch (which returns at once when no cell failed); a
            # per-cell solve of at least 32,768 cells adds the visit order's
            # key kernel and the four kernels of its radix sort
            "launches_per_step": (3 if form == "fp32_lu" else 1) + (5 if wl.group == 1 and N >= 32768 else 0),
        }
        if clocks is None:
            clocks = cs.summary()
        S.CloseOdevec(ode)
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    head = forms[0]
    r = res[head]
    peaks = fma_peaks(torch)
    achieved = r["flops_per_launch"] / (r["kernel_ms"] * 1e-3) / 1e12
    tpc = traffic_per_cell() if args.workload == "PRIMORDIAL" else None
    in_mb = N * (y0.shape[0] + 3) * 8 / 1e6  # species, t, dt, t_stop
    alg_bytes = N * (y0.shape[0] * 8 * 2 + 3 * 8 + 2 * 8 + 4)
    line = {
        # the headline metric for the PRIMORDIAL workload; another workload
        # (--workload) is named by its own cells/s
        "metric": METRIC if args.workload == "PRIMORDIAL" else "%s cells/s to t_end" % args.workload,
        "value": r["value"],
        "unit": "cells/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": r["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 state/residual/control, f32 LU" if head == "fp32_lu" else "f64",
        "data": DATA,
        "config": {"workload": workload_label(args, N), "network": args.network, "form": head,
                   "staging": args.staging or "tuning table",
                   "l2": "inputs %.0f MB per GPU %s 126 MB L2" % (
                       in_mb, ">" if in_mb > 126 else "<= (not flushed between steps)"),
                   "parallelism": "dp%d (independent cell shards, no exchange)" % world},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peaks["fp64"], "unit": "TFLOP/s",
                     "frac": achieved / peaks["fp64"],
                     "traffic": None if tpc is None else tpc * N,
                     "traffic_source": None if tpc is None else
                     "not measured in this run: DRAM bytes per cell of the solve kernel from the ncu "
                     "capture in profiles/bdf_kernel_primordial_ncu.txt (262,144 cells), times the "
                     "cells of one launch",
                     "algorithmic_flops_per_launch": r["flops_per_launch"],
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "achieved_hbm_gbs": alg_bytes / (r["kernel_ms"] * 1e-3) / 1e9,
                     "peak_source": "FP64 FMA-chain probe on this GPU (odevec_probe_fma); "
                                    "MEASURED_PEAKS.json has no FP64 figure",
                     "fp64_share_of_flops": r["fp64_share"], "fp32_peak": peaks["fp32"]},
        "e2e": {"value": r["e2e"], "unit": "cells/s", "h2d_bytes_per_step": N * (y0.shape[0] + 3) * 8,
                "d2h_bytes_per_step": N * ((y0.shape[0] + 2) * 8 + 4),
                "path": "SolveODE on NumPy arrays -> odevec_solve_host; y, t, dt, t_stop in pinned "
                        "host memory read by the kernel at cell set-up and written at cell end "
                        "(transfers inside the solve); status copied back"},
        "gpu_launches": args.steps * r["launches_per_step"],
        "clocks": {k: v for k, v in r["clocks"].items() if k != "samples"},
        "batch_latency_ms": {"p50": float(np.percentile(r["step_ms"], 50)),
                             "p99": float(np.percentile(r["step_ms"], 99))},
        "forms": {f: {k: v for k, v in res[f].items() if k not in ("step_ms", "clocks")} for f in forms},
    }
    if "fp64" in res and "fp32_lu" in res:
        line["fp32lu_over_fp64"] = res["fp32_lu"]["value"] / res["fp64"]["value"]
    if "plain_fp64" in res and "fp32_lu" in res:
        line["fp32lu_over_plain_fp64"] = res["fp32_lu"]["value"] / res["plain_fp64"]["value"]
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(
            W.BUILDERS[args.workload](ncells=args.cpu_sample, seed=3, network=args.network),
            args.cpu_sample, host_threads())
    if world == 1 and args.accuracy_cells > 0 and args.workload == "PRIMORDIAL":
        line["accuracy"] = accuracy(args, wl, S, torch)
    if world == 1 and not args.no_configs:
        line["other_configs"] = other_configs(args, torch, S, W, peaks)
    if world == 1 and args.serving_duration > 0:
        line["serving"] = serving_block(args)
        iso = line["serving"].get("isolated", {})
        line["latency_ms"] = {"p50": line["serving"]["mix"]["p50_ms"], "p99": line["serving"]["mix"]["p99_ms"],
                              "isolated_p99": iso.get("p99_ms"),
                              "p99_over_isolated_p99": iso.get("mix_p99_over_isolated_p99"),
                              "what": "hydro-step latency of the serving stream (serving block)"}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _rel_err(g, ref, mask):
    rel = np.abs(g[mask] - ref[mask]) / np.abs(ref[mask])
    return rel


def accuracy(args, wl, S, torch):
    """Errors of each form at rtol 1e-6 against the oracle at rtol 1e-12 on a
    sample of cells, and where they come from: per species, per abundance
    relative to n_H, under three floors (species above atol/rtol, above atol,
    above 1e-12 n_H), the worst cells, the oracle's own convergence (rtol
    1e-12 against 1e-13) and an rtol sweep of the FP64 form."""
    from oracle import oracle as O
    from odevec_b200 import networks as NW
    from odevec_b200 import workloads as WL
    n = args.accuracy_cells
    sub = slice(0, n)
    thr = host_threads()

    def oracle_at(rtol, fix=True):
        y, _, _, st, _ = O.solve(wl.network, wl.y[:, sub], wl.t0[sub], wl.dt0[sub], wl.t_stop[sub], rtol,
                                 rtol * 1e-14, wl.dt_min, group=1, nthreads=thr, fix_restart=fix)
        return y, int((st != 0).sum())
    ref, f12 = oracle_at(1e-12)
    ref13, f13 = oracle_at(1e-13)
    nh = WL.primordial_invariants(wl.y[:, sub])[0]      # hydrogen nuclei per cell (constant)
    names = list(NW.PRIMORDIAL_SPECIES[:12])
    floors = {"above_atol_over_rtol": np.abs(ref[:12]) > wl.atol / wl.rtol,
              "above_atol": np.abs(ref[:12]) > wl.atol,
              "above_1e-12_nH": np.abs(ref[:12]) > 1e-12 * nh[None, :]}
    selfc = _rel_err(ref[:12], ref13[:12], floors["above_atol_over_rtol"])
    out = {"oracle_rtol": 1e-12, "oracle_fix_restart": True, "cells": n,
           "oracle_failures": f12, "oracle_self_convergence": {
               "what": "oracle at rtol 1e-12 against rtol 1e-13, species above 1e-14",
               "max_rel": float(selfc.max()), "p99_rel": float(np.percentile(selfc, 99)),
               "failures_1e-13": f13}}

    def solve(form, rtol, fix):
        ode = S.Odevec(wl.network, RelativeTolerance=rtol, AbsoluteTolerance=wl.atol,
                       MinimalTimestep=wl.dt_min, nvector=1, precision=form, raise_on_failure=False,
                       fix_restart=fix)
        S.InitOdevec(ode)
        y = torch.tensor(wl.y[:, sub], device="cuda").contiguous()
        S.SolveODE(ode, torch.tensor(wl.t0[sub], device="cuda"), torch.tensor(wl.dt0[sub], device="cuda"),
                   torch.tensor(wl.t_stop[sub], device="cuda"), y)
        g = y.cpu().numpy()
        S.CloseOdevec(ode)
        return g
    forms = [f for f in args.forms.split(",") if f != "plain_fp64"]
    got = {}
    for form in forms:
        for fix in (False, True):
            g = solve(form, wl.rtol, fix)
            got[(form, fix)] = g
            blk = {}
            for fname, m in floors.items():
                rel = _rel_err(g[:12], ref[:12], m)
                blk[fname] = {"max_rel_err": float(rel.max()), "p99_rel_err": float(np.percentile(rel, 99)),
                              "median_rel_err": float(np.median(rel)), "max_over_rtol": float(rel.max() / wl.rtol)}
            out[form + ("+fix_restart" if fix else "")] = blk
    # where the largest errors live (the FP32-LU form as the reference restarts)
    g = got[(forms[0], False)]
    m = floors["above_atol_over_rtol"]
    err = np.where(m, np.abs(g[:12] - ref[:12]) / np.maximum(np.abs(ref[:12]), 1e-300), 0.0)
    out["by_species"] = {names[j]: {"max_rel_err": float(err[j].max()),
                                    "cells_above_10rtol": int((err[j] > 10 * wl.rtol).sum())}
                         for j in range(12)}
    ab = np.abs(ref[:12]) / nh[None, :]
    bins = [(0, 1e-14), (1e-14, 1e-10), (1e-10, 1e-6), (1e-6, 1e-2), (1e-2, 10.0)]
    out["by_abundance_over_nH"] = {"%.0e..%.0e" % (lo, hi): {
        "max_rel_err": float(err[(ab >= lo) & (ab < hi) & m].max()) if np.any((ab >= lo) & (ab < hi) & m) else None,
        "entries": int(np.sum((ab >= lo) & (ab < hi) & m))} for lo, hi in bins}
    worst = np.argsort(err.ravel())[::-1][:5]
    out["worst"] = [{"cell": int(k % n), "species": names[k // n], "rel_err": float(err.ravel()[k]),
                     "abundance_over_nH": float(ab.ravel()[k]), "t_end": float(wl.t_stop[k % n]),
                     "T": float(wl.y[14, k % n])} for k in worst]
    # the global error's scaling: the FP64 form at tighter tolerances
    sweep = {}
    for rt in (1e-6, 1e-7, 1e-8):
        g = solve("fp64", rt, True)
        rel = _rel_err(g[:12], ref[:12], np.abs(ref[:12]) > wl.atol / rt)
        sweep["%.0e" % rt] = {"max_rel_err": float(rel.max()), "max_over_rtol": float(rel.max() / rt),
                              "p99_rel_err": float(np.percentile(rel, 99))}
    out["rtol_sweep_fp64_fix_restart"] = sweep
    # what the FP32 factors add: FP32-LU against the FP64 path at the same rtol
    if ("fp32_lu", False) in got and ("fp64", False) in got:
        a, b = got[("fp32_lu", False)][:12], got[("fp64", False)][:12]
        rel = _rel_err(a, b, np.abs(b) > wl.atol / wl.rtol)
        out["fp32_lu_vs_fp64_same_rtol"] = {"max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
                                            "max_over_rtol": float(rel.max() / wl.rtol)}
    return out


def serving_block(args):
    """A bounded serving run: Poisson arrivals of ROBER, PRIMORDIAL and SYN64
    requests (1k..256k cells, 50 hydro steps each, dt 1e6..1e11 s, 120 GB
    budget) at a rate near the device's capacity, FP32-LU form, and every
    request run again alone; step latencies p50/p99 in the mix and alone."""
    from odevec_b200 import serving as SV
    t0 = time.perf_counter()
    out = SV.measure(rate=args.serving_rate, duration=args.serving_duration, steps=50,
                     precisions=("fp32_lu",), seed=args.serving_seed, isolated=True)[0]
    out["wall_s"] = time.perf_counter() - t0
    out.pop("per_network", None)
    return out


def other_configs(args, torch, S, W, peaks):
    """cells/s of the other configurations (FP64 and FP32-LU), one timed
    solve each after one untimed one, inputs reset from a device copy, with
    the FP64 roofline of the kernel and the CPU baseline on a sample."""
    from odevec_b200 import metrics
    out = {}
    cases = [("ROBER", W.rober(ncells=4096), 4096), ("OREGO", W.orego(ncells=65536), 16384),
             ("SYN64", W.syn64(ncells=262144), 1024)]
    for name, wl, cpu_n in cases:
        row = {"network": wl.network, "cells": wl.ncells, "group": wl.group}
        for form in ("fp64", "fp32_lu"):
            ode = S.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                           MinimalTimestep=wl.dt_min, nvector=wl.group, precision=form, raise_on_failure=False)
            S.InitOdevec(ode)
            y0 = torch.tensor(wl.y, device="cuda")
            t0 = torch.tensor(wl.t0, device="cuda")
            d0 = torch.tensor(wl.dt0, device="cuda")
            ts = torch.tensor(wl.t_stop, device="cuda")
            ms = None
            for k in range(2):
                y, t, d = y0.clone(), t0.clone(), d0.clone()
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                S.SolveODE(ode, t, d, ts, y, want_stats=k == 0)
                e1.record()
                torch.cuda.synchronize()
                if k == 0:
                    stats = ode.stats.cpu().numpy()
                    fails = int((ode.status != 0).sum().item())
                ms = e0.elapsed_time(e1)
            flops = float(metrics.flops_per_cell(wl.network, stats).sum())
            ach = flops / (ms * 1e-3) / 1e12
            row[form] = {"cells_per_s": wl.ncells / (ms * 1e-3), "ms": ms, "failed_cells": fails,
                         "mean_newton_iters": float(stats[:, 4].mean()), "mean_steps": float(stats[:, 0].mean()),
                         "roofline": {"bound": "fp64", "achieved": ach, "peak": peaks["fp64"],
                                      "unit": "TFLOP/s", "frac": ach / peaks["fp64"],
                                      "algorithmic_flops_per_launch": flops,
                                      "fp64_share_of_flops": metrics.fp64_fraction(wl.network, stats,
                                                                                    form == "fp32_lu")}}
            S.CloseOdevec(ode)
        row["fp32lu_over_fp64"] = row["fp32_lu"]["cells_per_s"] / row["fp64"]["cells_per_s"]
        if not args.no_cpu:
            row["cpu_baseline"] = cpu_baseline(wl, min(cpu_n, wl.ncells), host_threads())
        out[name] = row
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_product(args)


if __name__ == "__main__":
    main()
