"""Tables of the warp-per-cell kernel (odevec_b200/wpc.py) against the
compiled network code.

The warp kernel evaluates the right-hand side from per-species term lists,
the iteration matrix from postfix programs and the LU factorisation and
solves from level-scheduled statement lists.  These tests evaluate the
tables in IEEE doubles in Python and require bit-identical results to the
oracle's compiled straight-line code (right-hand side, P) and to the
statements executed in program order (factorisation, solves)."""
import numpy as np
import pytest

from odevec_b200 import networks, pre_odevec as P, shipped, wpc

VARIANTS = {
    "SYN64_CSC_CMK": lambda: P.build_system(networks.load_krome_dump(shipped.SYN64_DUMP, "SYN64"), "CMK", "CSC"),
    "ROBER_CSC_NONE": lambda: P.build_system(networks.load("ROBER"), "None", "CSC"),
    "OREGO_CSC_CMK": lambda: P.build_system(networks.load("OREGO"), "CMK", "CSC"),
}


@pytest.fixture(scope="module", params=sorted(VARIANTS))
def variant(request):
    s = VARIANTS[request.param]()
    return request.param, s, wpc.tables(s)


def test_parser_follows_c_precedence():
    e = wpc.parse("-2.0*y[0]*y[1] - 3.0*((y[2])*(y[2])) + 4.0")
    assert e == ("+", ("-", ("*", ("*", ("neg", ("num", 2.0)), ("y", 0)), ("y", 1)),
                       ("*", ("num", 3.0), ("*", ("y", 2), ("y", 2)))), ("num", 4.0))
    assert wpc.rhs_terms("-2.0*y[0]*y[1] - 3.0*((y[2])*(y[2])) + 4.0") == [
        (-2.0, [(0, 0), (1, 0)]), (-3.0, [(2, 1)]), (4.0, [])]


def test_rhs_and_matrix_tables_bit_identical(oracle, variant):
    tag, s, t = variant
    rng = np.random.default_rng(11)
    dyn, dpos, kmap = P._reduced(s)
    for _ in range(5):
        y = 10.0 ** rng.uniform(-12, 1, s.neq)
        beta, dt = float(rng.uniform(0.3, 1.0)), float(10.0 ** rng.uniform(-4, 6))
        f, a = oracle.evaluate(tag, y, np.zeros(1), beta, dt)
        for i, sp in enumerate(dyn):
            assert wpc.eval_terms(t["rhs"][i], y) == f[sp]
        packed = [a[kk] for kk in sorted(kmap, key=kmap.get)]
        for e, prog in enumerate(t["progs"]):
            assert wpc.run_program(prog, t["consts"], y, beta, dt) == packed[e]


def _run(ops, order, vals, factor):
    v = dict(vals)
    for i in order:
        k, x, y, z = ops[i]
        if factor:
            v[x] = v[x] / v[y] if k == wpc.DIV else v[x] - v[y] * v[z]
        else:
            v[("d", x)] = (v[("d", x)] / v[("a", z)] if k == wpc.DIV
                           else v[("d", x)] - v[("d", y)] * v[("a", z)])
    return v


def test_level_schedules_equal_program_order(variant):
    tag, s, t = variant
    rng = np.random.default_rng(12)
    nnz = t["nnz"]
    a0 = {i: float(rng.uniform(0.5, 2.0)) for i in range(nnz)}
    seq = _run(t["fops"], range(len(t["fops"])), a0, True)
    lev = _run(t["fops"], [i for l in t["flev"] for i in l], a0, True)
    assert seq == lev
    # within a level: no statement reads or writes another's target
    for l in t["flev"]:
        tg = [t["fops"][i][1] for i in l]
        assert len(set(tg)) == len(tg)
        for i in l:
            k, x, y, z = t["fops"][i]
            assert y not in tg and (k == wpc.DIV or z not in tg)
    d0 = {("d", i): float(rng.normal()) for i in range(s.neq)}
    d0.update({("a", i): seq[i] for i in range(nnz)})
    seq_s = _run(t["sops"], range(len(t["sops"])), d0, False)
    lev_s = _run(t["sops"], [i for l in t["slev"] for i in l], d0, False)
    assert seq_s == lev_s


def test_eligibility():
    assert not wpc.eligible(P.build_system(networks.load("PRIMORDIAL"), "FF", "CSC"))  # rate model
    assert not wpc.eligible(P.build_system(networks.load("ROBER"), "None", "DENSE"))
    assert wpc.eligible(VARIANTS["SYN64_CSC_CMK"]())


def test_table_indices_in_bounds(variant):
    tag, s, t = variant
    wpc.check_bounds(t)
    text = wpc.emit(s, "x")
    assert "ov_wpc_x_sol_op" in text and "NFL = %d" % len(t["flev"]) in text


def test_level_rows_per_lane_count(variant):
    """The rows for K lanes per cell (K = 32, 16, 8) hold at most K
    statements of one level each and keep the level order."""
    tag, s, t = variant
    text = wpc.emit(s, "x")
    for width in wpc.LANES:
        for lev in (t["flev"], t["slev"]):
            rows = wpc.level_rows(lev, width)
            assert all(0 < len(r) <= width for r in rows)
            assert [i for r in rows for i in r] == [i for l in lev for i in l]
            assert len(rows) == sum(-(-len(l) // width) for l in lev)
        if width != 32:
            assert "NFL%d = %d" % (width, len(wpc.level_rows(t["flev"], width))) in text
            assert "ov_wpc_x_sol_op%d" % width in text
