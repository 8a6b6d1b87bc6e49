"""Synthetic 64-species mass-action network, written as a KROME Python dump.

The dump defines ``y`` (state symbols ``y(:,1..64)``), ``rhs`` (a SymPy
column), ``neq`` and ``nrea`` -- the format the preprocessor reads with
``--krome_setupfile`` (as the reference reads KROME dumps,
``pre_odevec.py:97-105``).  The rate coefficients are baked in as
constants.

Construction (seeded): 400 reactions with 1-2 reactants and 1-3 products;
rate coefficients log-uniform in 1e-20..1e-8 (two-body) or 1e-16..1e-6
(one-body).  Every species has an integer "mass" 1..4 and every reaction
conserves mass, so the total mass sum(m_i y_i) is a linear invariant and
the dynamics stay bounded.  Reactants and products of a reaction are drawn
from a window of neighbouring species (index distance at most 2), which
keeps the Jacobian sparse and banded (about 10 % of its 64 x 64 entries).

Regenerate: ``python -m odevec_b200.syn64`` (writes odevec_b200/data/syn64_krome.py).
"""
from __future__ import annotations

import itertools
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DUMP = os.path.join(HERE, "data", "syn64_krome.py")
NEQ, NREA, WINDOW = 64, 400, 2


def masses(neq: int = NEQ) -> np.ndarray:
    return 1 + (np.arange(neq) % 4)


def reactions(seed: int = 64, neq: int = NEQ, nrea: int = NREA, window: int = WINDOW):
    rng = np.random.default_rng(seed)
    m = masses(neq)
    out = []
    seen = set()
    while len(out) < nrea:
        c = int(rng.integers(neq))
        near = [c + d for d in range(-window, window + 1) if 0 <= c + d < neq]
        nr = int(rng.integers(1, 3))
        reac = tuple(sorted(int(rng.choice(near)) for _ in range(nr)))
        total = int(sum(m[r] for r in reac))
        np_ = int(rng.integers(1, 4))
        # products from the window whose masses add up to the reactants' total
        combos = [p for p in itertools.combinations_with_replacement(near, np_)
                  if sum(m[i] for i in p) == total and sorted(p) != sorted(reac)]
        if not combos:
            continue
        prod = tuple(sorted(combos[int(rng.integers(len(combos)))]))
        if (reac, prod) in seen:
            continue
        seen.add((reac, prod))
        if nr == 2:
            k = 10.0 ** rng.uniform(-20.0, -8.0)
        else:
            k = 10.0 ** rng.uniform(-16.0, -6.0)
        out.append((reac, prod, float("%.6e" % k)))
    return out


def dump_text(seed: int = 64) -> str:
    neq = NEQ
    rows = [[] for _ in range(neq)]
    rea = reactions(seed)
    for reac, prod, k in rea:
        flux = "%r*%s" % (k, "*".join("y[%d]" % r for r in reac))
        net = {}
        for s in reac:
            net[s] = net.get(s, 0) - 1
        for s in prod:
            net[s] = net.get(s, 0) + 1
        for s, c in sorted(net.items()):
            if c:
                rows[s].append("%+d*%s" % (c, flux))
    lines = ["# Synthetic 64-species mass-action network (odevec_b200/syn64.py, seed %d)." % seed,
             "# KROME-style Python dump: defines y, rhs, neq, nrea.",
             "neq = %d" % neq, "nrea = %d" % len(rea),
             "y = [Symbol('y(:,%d)' % (i + 1)) for i in range(neq)]",
             "rhs = Matrix(["]
    for r in rows:
        lines.append("    " + (" ".join(r) if r else "0") + ",")
    lines.append("])")
    return "\n".join(lines) + "\n"


def write(path: str = DUMP, seed: int = 64) -> str:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as fh:
        fh.write(dump_text(seed))
    return path


if __name__ == "__main__":
    p = write()
    from . import networks, pre_odevec
    net = networks.load_krome_dump(p, "SYN64")
    s = pre_odevec.build_system(net, "CMK", "CSC")
    print(p, "P nnz", s.p_nnz, "density %.3f" % (s.p_nnz / 64.0 ** 2), "LU nnz", s.nnz)
