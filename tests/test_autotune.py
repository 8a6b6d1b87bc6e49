"""Autotuner: coordinate search over stagings and batches, the tuning
table, and the rule that explicit options are never overridden.  The GPU
test checks that a tuned solver gives bit-identical results."""
import types

import numpy as np
import pytest

from odevec_b200 import autotune as A


def test_search_picks_fastest_and_skips_uncompiled():
    cost = {1: 3.0, 2: None, 3: 2.0, 4: 2.5, 6: 1.5, 7: 1.9, 8: 1.7, 9: 1.8, 10: 1.9, 11: 2.2, 12: 1.6, 13: 2.0, 14: 2.1, 15: 1.8, 16: 1.9, 17: 1.65, 18: 1.85, 19: 1.95, 20: 2.05, 21: 2.1, 5: 1.0}

    def timer(cfg):
        base = cost[cfg["staging"]]
        if base is None:
            return None
        if cfg["jac_batch"] == 16:
            return base * 0.4
        return base

    best, tried = A.search(timer, "fp64")
    assert best["staging"] == 1 and best["jac_batch"] == 16 and best["seconds"] == pytest.approx(1.2)
    assert all(c["staging"] != 2 for c, _ in tried)
    # batches are tried on staging 1 only; the others are timed once, unbatched
    assert len(tried) == len(A.BATCHES) + (len(A.STAGINGS) - 2)
    assert all((c["jac_batch"], c["ss_batch"], c["max_wait"]) == (1, 1, -1) for c, _ in tried if c["staging"] != 1)
    cost[1] = 9.0
    best, _ = A.search(timer, "fp64")
    assert best["staging"] == 6 and best["seconds"] == pytest.approx(1.5)
    best32, _ = A.search(timer, "fp32_lu")
    assert best32["staging"] == 5  # FP32-only staging considered for fp32_lu


def test_table_apply_respects_explicit_options(tmp_path):
    path = str(tmp_path / "t.json")
    A.save({A.key("NET", "fp64", 1, "GPU"): {"staging": 6, "jac_batch": 16, "ss_batch": 16, "max_wait": 4}},
           path)
    ode = types.SimpleNamespace(network="NET", precision="fp64", nvector=1, staging=0, jac_batch=0,
                                ss_batch=0, max_wait=0)
    assert A.apply(ode, device="GPU", path=path)
    assert (ode.staging, ode.jac_batch, ode.ss_batch, ode.max_wait) == (6, 16, 16, 4)
    ode2 = types.SimpleNamespace(network="NET", precision="fp64", nvector=1, staging=3, jac_batch=0,
                                 ss_batch=0, max_wait=0)
    A.apply(ode2, device="GPU", path=path)
    assert ode2.staging == 3 and ode2.jac_batch == 16
    ode3 = types.SimpleNamespace(network="NET", precision="fp32_lu", nvector=1, staging=0, jac_batch=0,
                                 ss_batch=0, max_wait=0)
    assert not A.apply(ode3, device="GPU", path=path) and ode3.staging == 0


def test_shipped_table_is_valid():
    for k, v in A.load().items():
        net, prec, grp, dev = k.split("/")
        assert prec in ("fp64", "fp64_fma", "fp32_lu") and grp.startswith("G")
        assert v["staging"] in A.STAGINGS + A.FP32_STAGINGS


@pytest.mark.gpu
def test_tuned_solver_gives_identical_results(gpu_lib):
    from odevec_b200 import workloads as W
    import torch
    wl = W.primordial(ncells=4096)
    best, tried = A.tune(wl.network, "fp64", wl.y, wl.t0, wl.dt0, wl.t_stop, wl.rtol, wl.atol, wl.dt_min,
                         reps=1)
    assert len(tried) >= 5
    out = []
    for cfg in ({}, {k: best[k] for k in A.FIELDS}):
        ode = gpu_lib.Odevec(wl.network, RelativeTolerance=wl.rtol, AbsoluteTolerance=wl.atol,
                             MinimalTimestep=wl.dt_min, nvector=1, precision="fp64", autotune=False, **cfg)
        gpu_lib.InitOdevec(ode)
        y = torch.tensor(wl.y, device="cuda")
        gpu_lib.SolveODE(ode, torch.tensor(wl.t0, device="cuda"), torch.tensor(wl.dt0, device="cuda"),
                         torch.tensor(wl.t_stop, device="cuda"), y)
        out.append(y.cpu().numpy())
        gpu_lib.CloseOdevec(ode)
    assert np.array_equal(out[0], out[1])


def test_c_table_mirrors_tuning_json():
    import re
    from odevec_b200 import build as B
    text = open(B.write_tuning_table()).read()
    rows = re.findall(r'OV_TUNE\("([^"]+)", (\d), (\d+), "([^"]+)", (-?\d+), (-?\d+), (-?\d+), (-?\d+)\)', text)
    table = A.load()
    assert len(rows) == len(table)
    codes = {v: k for k, v in B.PREC_CODE.items()}
    for tag, prec, grp, dev, st, jb, sb, mw in rows:
        v = table[A.key(tag, codes[int(prec)], int(grp), dev)]
        assert (v["staging"], v["jac_batch"], v["ss_batch"], v["max_wait"]) == (int(st), int(jb), int(sb), int(mw))
