"""Autotuner for the launch shape of the solve kernel.

What it chooses, per network variant, precision form and GPU model:

* the staging -- where a cell's Nordsieck history and LU live (thread-local
  arrays in registers / local memory, or shared memory), the block size
  (cells per block: 128, 192, 256, 320, 384 or 512 threads), the blocks per
  SM and soft lockstep, or 32, 16 or 8 lanes per cell (stagings 7, 13, 14,
  for the variants that have their tables);
* for staging 1, the batching of the Jacobian and step-size blocks
  (jac_batch, ss_batch, max_wait); the other stagings run those blocks on
  fixed trips.

None of these settings changes a result (every cell runs the same operations whatever the interleaving;
the GPU parity tests check this bit for bit), so tuning only moves time.

The search times every compiled staging (staging 1 with every batch
setting) on a sample of the caller's cells (about fifty short solves).  Results go to a JSON table (``tuning.json`` beside this
file) that InitOdevec consults for options left at 0 (automatic).

    python -m odevec_b200.autotune --network PRIMORDIAL_CSC_FF --precision fp32_lu
"""
from __future__ import annotations

import json
import os
from typing import Callable, Dict, List, Optional, Tuple

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")

STAGINGS = (1, 2, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21)
FP32_STAGINGS = (5,)
BATCHES = ((24, 24, 8), (16, 16, 4), (32, 32, 16), (8, 8, 4), (4, 4, 2), (2, 2, 1), (1, 1, -1))
# the batch options act on staging 1 only; the other stagings run the Jacobian
# and step-size blocks on fixed trips and are timed once
BATCHED_STAGINGS = (1,)
UNBATCHED = ((1, 1, -1),)
FIELDS = ("staging", "jac_batch", "ss_batch", "max_wait")


def key(network: str, precision: str, group: int, device: str) -> str:
    return "%s/%s/G%d/%s" % (network, precision, group, device)


def load(path: str = TABLE) -> Dict[str, dict]:
    if not os.path.exists(path):
        return {}
    with open(path) as fh:
        return json.load(fh)


def save(entries: Dict[str, dict], path: str = TABLE) -> None:
    table = load(path)
    table.update(entries)
    with open(path, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
        fh.write("\n")


def device_name() -> str:
    import torch
    return torch.cuda.get_device_name()


def apply(ode, device: Optional[str] = None, path: str = TABLE) -> bool:
    """Fills the launch options the caller left automatic (0) from the
    table; returns whether an entry was found."""
    if all(getattr(ode, f) != 0 for f in FIELDS):
        return False
    entry = load(path).get(key(ode.network, ode.precision, ode.nvector, device or device_name()))
    if not entry:
        return False
    for f in FIELDS:
        if getattr(ode, f) == 0 and f in entry:
            setattr(ode, f, int(entry[f]))
    return True


def candidates(precision: str) -> List[int]:
    return list(STAGINGS) + (list(FP32_STAGINGS) if precision == "fp32_lu" else [])


def search(time_config: Callable[[dict], Optional[float]], precision: str,
           batches=BATCHES) -> Tuple[dict, List[Tuple[dict, float]]]:
    """Every compiled staging, staging 1 with every batch setting (the
    others schedule the Jacobian and step-size blocks on fixed trips and take
    no batch options); time_config(cfg) returns seconds, or None for a
    configuration that is not compiled for the variant (then the staging is
    skipped)."""
    tried: List[Tuple[dict, float]] = []
    best, best_t = None, None
    for st in candidates(precision):
        for b in (batches if st in BATCHED_STAGINGS else UNBATCHED):
            cfg = {"staging": st, "jac_batch": b[0], "ss_batch": b[1], "max_wait": b[2]}
            t = time_config(cfg)
            if t is None:
                break
            tried.append((cfg, t))
            if best_t is None or t < best_t:
                best, best_t = cfg, t
    if best is None:
        raise RuntimeError("no compiled configuration could be timed")
    return dict(best, seconds=best_t), tried


def tune(network: str, precision: str, y, t, dt, t_stop, rtol: float, atol: float, dt_min: float,
         group: int = 1, reps: int = 2):
    """Times the candidates on the given sample (device tensors or NumPy
    arrays of one workload) and returns (best, tried)."""
    import torch
    from . import solver as S
    y0 = torch.as_tensor(y, device="cuda", dtype=torch.float64).contiguous()
    t0 = torch.as_tensor(t, device="cuda", dtype=torch.float64).contiguous()
    d0 = torch.as_tensor(dt, device="cuda", dtype=torch.float64).contiguous()
    ts = torch.as_tensor(t_stop, device="cuda", dtype=torch.float64).contiguous()

    def time_config(cfg):
        ode = S.Odevec(network, RelativeTolerance=rtol, AbsoluteTolerance=atol, MinimalTimestep=dt_min,
                       nvector=group, precision=precision, raise_on_failure=False, autotune=False, **cfg)
        S.InitOdevec(ode)
        try:
            best = None
            for _ in range(reps):
                yy, tt, dd = y0.clone(), t0.clone(), d0.clone()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                try:
                    S.SolveODE(ode, tt, dd, ts, yy, want_stats=False)
                except S.OdevecError as e:
                    if "not compiled" in str(e):
                        return None
                    raise
                e1.record()
                torch.cuda.synchronize()
                el = e0.elapsed_time(e1) / 1e3
                best = el if best is None else min(best, el)
            return best
        finally:
            S.CloseOdevec(ode)

    return search(time_config, precision)


def main(argv=None):
    import argparse
    from . import workloads as W
    p = argparse.ArgumentParser()
    p.add_argument("--network", action="append", default=None)
    p.add_argument("--precision", action="append", default=None)
    p.add_argument("--cells", type=int, default=262144)
    p.add_argument("--table", default=TABLE)
    a = p.parse_args(argv)
    nets = a.network or ["PRIMORDIAL_CSC_FF", "OREGO_CSC_CMK", "SYN64_CSC_CMK"]
    precs = a.precision or ["fp64", "fp64_fma", "fp32_lu"]
    dev = device_name()
    out = {}
    for net in nets:
        name = net.split("_")[0]
        # SYN64 solves are ~70x slower per cell: half the sample, still
        # several cells per resident lane (a sample smaller than the resident
        # lanes favours the stagings with the most threads, not the fastest)
        n = a.cells if name != "SYN64" else max(1, a.cells // 2)
        wl = W.BUILDERS[name](ncells=n, network=net)
        if wl.group != 1:
            continue  # lockstep groups have a single compiled configuration
        for prec in precs:
            best, tried = tune(net, prec, wl.y, wl.t0, wl.dt0, wl.t_stop, wl.rtol, wl.atol, wl.dt_min)
            out[key(net, prec, 1, dev)] = dict(best, cells=n)
            print(json.dumps({"network": net, "precision": prec, "best": best,
                              "tried": [dict(c, seconds=s) for c, s in tried]}), flush=True)
    save(out, a.table)


if __name__ == "__main__":
    main()
