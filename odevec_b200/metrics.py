"""Algorithmic work of a solve, from the per-cell counters and the emitter's
static per-call operation counts (csrc/gen/flops.json).

Counted per cell (n = neq; F_* from the emitter):

* per Newton iteration:  F_rhs + F_rates_k + F_lu_solve
                         + 3n (residual) + n (en update) + 2n (y update)
                         + 3n + 2 (weighted norm of the correction) + 6
* per Jacobian refresh:  F_jac + F_rates_k + F_lu_factor
* per predictor / reset pass over one Nordsieck vector: n additions
* per error test:        3n + 2 (norm) + 4n (error weights)
* per accepted step:     4n (Nordsieck update at order 1, a lower bound)
* once:                  F_rhs + F_rates_k + 5n (initial right-hand side,
                         weights and step size)

Step-size/order selection (three norms and three powers every q+1 steps)
and Nordsieck rescaling are not counted, so the count is a lower bound of
the work done.  Rate-law evaluation (once per cell per solve) is not
counted either.
"""
import json
import os

import numpy as np

GEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "gen")


def op_counts(tag):
    with open(os.path.join(GEN, "flops.json")) as fh:
        return json.load(fh)[tag]


def flops_per_cell(tag, stats):
    """FLOPs of each cell from its counters (stats: (ncells, 8) int array)."""
    c = op_counts(tag)
    n = c["neq"]
    st = np.asarray(stats, dtype=np.float64)
    steps, attempts, ltef, convf, newt, jacs, order, ppass = (st[:, i] for i in range(8))
    per_newton = c["rhs"] + c["rates_k"] + c["lu_solve"] + 9 * n + 8
    per_jac = c["jac"] + c["rates_k"] + c["lu_factor"]
    tests = steps + ltef
    return (newt * per_newton + jacs * per_jac + ppass * n + tests * (7 * n + 2) + steps * 4 * n
            + c["rhs"] + c["rates_k"] + 5 * n)


def fp64_fraction(tag, stats, lu_fp32):
    """Share of the counted FLOPs executed in FP64 (the LU factor and solve
    move to FP32 in the FP32-LU form)."""
    c = op_counts(tag)
    st = np.asarray(stats, dtype=np.float64)
    tot = flops_per_cell(tag, st).sum()
    if not lu_fp32:
        return 1.0
    lu = (st[:, 4] * c["lu_solve"] + st[:, 5] * c["lu_factor"]).sum()
    return float((tot - lu) / tot)
