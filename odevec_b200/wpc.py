"""Tables for the warp-per-cell kernel, derived from the emitted network code.

For networks of more than about 32 species one thread cannot keep a cell's
state on chip (SYN64: ~9 KB per cell), so K lanes of a warp (K = 32, 16 or
8; 32/K cells per warp) integrate one cell: lane k of the group holds the
solver-state species k, k+K, ... and the network code runs as tables the
lanes share out.  The tables are produced from exactly the
straight-line C that the thread-per-cell kernel and the CPU oracle compile,
so the warp kernel performs the same IEEE operations in the same order and
its FP64 form is bit-identical to them:

* right-hand side: per species, the terms of its emitted sum in order, each
  a coefficient times up to three factors (a factor is y_a or the square
  (y_a*y_a) that integer powers print as), accumulated left to right;
* iteration matrix P: per packed entry, a postfix program over the emitted
  expression (constants, y_a, beta, dt; +, -, *, /, unary minus);
* LU factorisation and triangular solves: the emitted statement lists,
  level-scheduled: a statement goes one level after the last statement
  that wrote any value it reads, wrote its target, or read its target, so
  the statements of one level are independent and every target keeps its
  program order.

Eligible: constant-coefficient networks (no rate model), LUmethod 1, CSC
packaging.
"""
from __future__ import annotations

import re
from typing import Dict, List, Tuple

LANES = (32, 16, 8)  # lanes per cell the level tables are laid out for

# ------------------------------------------------------------ expression parser
_TOK = re.compile(r"\s*(?:(\d+\.\d*(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+|\d+)|(y\[\d+\])|(beta|dt)|([-+*/()]))")


def _tokens(s: str):
    pos, out = 0, []
    s = s.strip()
    while pos < len(s):
        m = _TOK.match(s, pos)
        if not m or m.end() == pos:
            raise ValueError("cannot parse %r at %d" % (s, pos))
        num, yv, sym, op = m.groups()
        if num is not None:
            out.append(("num", float(num)))
        elif yv is not None:
            out.append(("y", int(yv[2:-1])))
        elif sym is not None:
            out.append(("sym", sym))
        else:
            out.append(("op", op))
        pos = m.end()
    return out


class _Parser:
    """C precedence: unary minus over * and /, over + and -; left-associative."""

    def __init__(self, s):
        self.t = _tokens(s)
        self.i = 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def take(self):
        tok = self.peek()
        self.i += 1
        return tok

    def parse(self):
        e = self.add()
        if self.i != len(self.t):
            raise ValueError("trailing tokens")
        return e

    def add(self):
        e = self.mul()
        while self.peek() in (("op", "+"), ("op", "-")):
            op = self.take()[1]
            e = (op, e, self.mul())
        return e

    def mul(self):
        e = self.unary()
        while self.peek() in (("op", "*"), ("op", "/")):
            op = self.take()[1]
            e = (op, e, self.unary())
        return e

    def unary(self):
        if self.peek() == ("op", "-"):
            self.take()
            return ("neg", self.unary())
        if self.peek() == ("op", "+"):
            self.take()
            return self.unary()
        kind, v = self.take()
        if kind == "op" and v == "(":
            e = self.add()
            if self.take() != ("op", ")"):
                raise ValueError("missing )")
            return e
        if kind in ("num", "y", "sym"):
            return (kind, v)
        raise ValueError("unexpected token %r" % ((kind, v),))


def parse(s: str):
    return _Parser(s).parse()


def evaluate(e, y, beta=0.0, dt=0.0) -> float:
    """Reference evaluation of a parsed expression in IEEE doubles."""
    k = e[0]
    if k == "num":
        return e[1]
    if k == "y":
        return y[e[1]]
    if k == "sym":
        return beta if e[1] == "beta" else dt
    if k == "neg":
        return -evaluate(e[1], y, beta, dt)
    a, b = evaluate(e[1], y, beta, dt), evaluate(e[2], y, beta, dt)
    return {"+": a + b, "-": a - b, "*": a * b, "/": a / b}[k]


# ----------------------------------------------------------- right-hand side
MAXF = 3  # factors per term


def _factor(e):
    """(species, squared) of y_a or (y_a*y_a)."""
    if e[0] == "y":
        return (e[1], 0)
    if e[0] == "*" and e[1][0] == "y" and e[2][0] == "y" and e[1][1] == e[2][1]:
        return (e[1][1], 1)
    raise ValueError("factor %r" % (e,))


def _term(e):
    """coefficient and factors of c*f1*f2*..., left-associated; a unary minus
    on the leading literal or on the whole product negates the coefficient
    (exact)."""
    if e[0] == "neg":
        c, fs = _term(e[1])
        return -c, fs
    chain = []
    while e[0] == "*":
        chain.append(e[2])
        e = e[1]
    chain.append(e)
    chain.reverse()
    if chain[0][0] == "num":
        c = chain[0][1]
        rest = chain[1:]
    elif chain[0][0] == "neg" and chain[0][1][0] == "num":
        c = -chain[0][1][1]
        rest = chain[1:]
    else:
        # no literal coefficient: 1.0 * f1 * ... is the same product
        c = 1.0
        rest = chain
    fs = [_factor(f) for f in rest]
    if len(fs) > MAXF:
        raise ValueError("term with more than %d factors" % MAXF)
    return c, fs


def rhs_terms(expr: str) -> List[Tuple[float, List[Tuple[int, int]]]]:
    """Terms of one emitted right-hand side, in evaluation order, with the
    sign of a subtraction folded into the coefficient (a - t == a + (-t)
    exactly)."""
    e = parse(expr)
    if e == ("num", 0.0):
        return []
    terms = []
    while e[0] in ("+", "-"):
        c, fs = _term(e[2])
        terms.append((c if e[0] == "+" else -c, fs))
        e = e[1]
    terms.append(_term(e))
    terms.reverse()
    return terms


def eval_terms(terms, y) -> float:
    acc = None
    for c, fs in terms:
        v = c
        for s, sq in fs:
            v = v * (y[s] * y[s] if sq else y[s])
        acc = v if acc is None else acc + v
    return 0.0 if acc is None else acc


# --------------------------------------------------------- postfix programs
OP_C, OP_Y, OP_BETA, OP_DT, OP_NEG, OP_ADD, OP_SUB, OP_MUL, OP_DIV = range(9)


def program(e, consts: List[float], out: List[Tuple[int, int]]):
    k = e[0]
    if k == "num":
        out.append((OP_C, len(consts)))
        consts.append(e[1])
    elif k == "y":
        out.append((OP_Y, e[1]))
    elif k == "sym":
        out.append((OP_BETA if e[1] == "beta" else OP_DT, 0))
    elif k == "neg":
        program(e[1], consts, out)
        out.append((OP_NEG, 0))
    else:
        program(e[1], consts, out)
        program(e[2], consts, out)
        out.append(({"+": OP_ADD, "-": OP_SUB, "*": OP_MUL, "/": OP_DIV}[k], 0))


def depth(prog) -> int:
    d = m = 0
    for op, _ in prog:
        d += 1 if op in (OP_C, OP_Y, OP_BETA, OP_DT) else (0 if op == OP_NEG else -1)
        m = max(m, d)
    return m


def run_program(prog, consts, y, beta, dt) -> float:
    st = []
    for op, arg in prog:
        if op == OP_C:
            st.append(consts[arg])
        elif op == OP_Y:
            st.append(y[arg])
        elif op == OP_BETA:
            st.append(beta)
        elif op == OP_DT:
            st.append(dt)
        elif op == OP_NEG:
            st.append(-st.pop())
        else:
            b, a = st.pop(), st.pop()
            st.append({OP_ADD: a + b, OP_SUB: a - b, OP_MUL: a * b, OP_DIV: a / b}[op])
    return st[0]


# ----------------------------------------------------------- statement lists
DIV, SUBMUL = 0, 1
_FDIV = re.compile(r"^a\[(\d+)\] = a\[\1\] / a\[(\d+)\];$")
_FSUB = re.compile(r"^a\[(\d+)\] = a\[\1\] - a\[(\d+)\]\*a\[(\d+)\];$")
_SINIT = re.compile(r"^T d(\d+) = \(T\)\(r\[(\d+)\]\*OV_SC\((\d+)\)\);$")
_SDIV = re.compile(r"^d(\d+) = d\1 / a\[(\d+)\];$")
_SSUB = re.compile(r"^d(\d+) = d\1 - d(\d+)\*a\[(\d+)\];$")
_SOUT = re.compile(r"^x\[(\d+)\] = \(double\)d(\d+)\*OV_ISC\((\d+)\);$")


def factor_ops(lines: List[str]):
    """(kind, target, src1, src2) over the packed LU array."""
    ops = []
    for ln in lines:
        m = _FDIV.match(ln)
        if m:
            ops.append((DIV, int(m.group(1)), int(m.group(2)), -1))
            continue
        m = _FSUB.match(ln)
        if m:
            ops.append((SUBMUL, int(m.group(1)), int(m.group(2)), int(m.group(3))))
            continue
        raise ValueError("factor statement %r" % ln)
    return ops


def solve_ops(lines: List[str]):
    """init map (storage row -> solver index), (kind, target row, src row,
    a index) statements, output map (solver index -> storage row)."""
    init, out, ops = {}, {}, []
    for ln in lines:
        m = _SINIT.match(ln)
        if m:
            init[int(m.group(1))] = int(m.group(2))
            continue
        m = _SDIV.match(ln)
        if m:
            ops.append((DIV, int(m.group(1)), -1, int(m.group(2))))
            continue
        m = _SSUB.match(ln)
        if m:
            ops.append((SUBMUL, int(m.group(1)), int(m.group(2)), int(m.group(3))))
            continue
        m = _SOUT.match(ln)
        if m:
            out[int(m.group(1))] = int(m.group(2))
            continue
        raise ValueError("solve statement %r (the warp kernel needs CSC packaging)" % ln)
    return init, ops, out


def levels(ops, reads_of, write_of) -> List[List[int]]:
    """Level schedule: each statement one level after the last level that
    wrote a value it reads, wrote its target or read its target."""
    last_w: Dict = {}
    last_r: Dict = {}
    lvl = []
    for i, op in enumerate(ops):
        tgt = write_of(op)
        l = 0
        for r in reads_of(op):
            l = max(l, last_w.get(r, -1) + 1)
        l = max(l, last_w.get(tgt, -1) + 1, last_r.get(tgt, -1) + 1)
        lvl.append(l)
        last_w[tgt] = l
        for r in reads_of(op):
            last_r[r] = max(last_r.get(r, -1), l)
    out: List[List[int]] = [[] for _ in range(max(lvl) + 1 if lvl else 0)]
    for i, l in enumerate(lvl):
        out[l].append(i)
    return out


def factor_levels(ops):
    return levels(ops, lambda o: [o[1], o[2]] + ([o[3]] if o[0] == SUBMUL else []), lambda o: o[1])


def solve_levels(ops):
    return levels(ops, lambda o: [("d", o[1]), ("a", o[3])] + ([("d", o[2])] if o[0] == SUBMUL else []),
                  lambda o: ("d", o[1]))


def level_rows(lev: List[List[int]], width: int) -> List[List[int]]:
    """Statement rows for `width` lanes: each level cut into rows of at most
    `width` statements, levels in order."""
    return [idx[r:r + width] for idx in lev for r in range(0, len(idx), width)]


# ------------------------------------------------------------------ emission
def eligible(sysm) -> bool:
    return sysm.packaging == "CSC" and sysm.lu_method == 1 and not sysm.net.rates


def tables(sysm):
    """Every table of the warp kernel for one variant (raises if the
    emitted code has a shape the tables cannot express)."""
    from . import pre_odevec as P
    net = sysm.net
    n = sysm.neq
    dyn, dpos, kmap = P._reduced(sysm)
    ymap = {s: "y[%d]" % i for i, s in enumerate(net.y)}
    pr = P.NetPrinter(ymap)
    rhs = [rhs_terms(P._cexpr(net.rhs[s], pr)) for s in dyn]
    pos = sysm.pos()
    consts: List[float] = []
    progs, rows, cols = [], [], []
    for (i, j), kk in sorted(pos.items(), key=lambda t: t[1]):
        if kk in kmap:
            prog: List[Tuple[int, int]] = []
            program(parse(P._cexpr(sysm.P_order[i, j], pr)), consts, prog)
            progs.append(prog)
            rows.append(dpos[sysm.perm[i]])
            cols.append(dpos[sysm.perm[j]])
    fops = factor_ops([P._remap_a(l, kmap) for l in P._lu_factor_lines(sysm)])
    init, sops, out = solve_ops([P._remap_a(l, kmap) for l in P._lu_solve_lines(sysm, dpos=dpos)])
    return dict(n=n, nd=len(dyn), nnz=len(kmap), dyn=dyn, rhs=rhs, consts=consts, progs=progs, rows=rows,
                cols=cols, fops=fops, flev=factor_levels(fops), init=init, sops=sops, slev=solve_levels(sops),
                out=out)


def check_bounds(t) -> None:
    """Every index the kernel follows lies inside the array it indexes:
    species < neq (state vector, solve vector), packed entries < nnz,
    solver indices < nd, postfix stacks within the declared depth."""
    n, nd, nnz = t["n"], t["nd"], t["nnz"]
    for terms in t["rhs"]:
        for c, fs in terms:
            assert len(fs) <= MAXF and all(0 <= sp < n for sp, _ in fs)
    for prog in t["progs"]:
        d = 0
        for op, arg in prog:
            if op == OP_C:
                assert 0 <= arg < len(t["consts"])
            if op == OP_Y:
                assert 0 <= arg < n
            d += 1 if op in (OP_C, OP_Y, OP_BETA, OP_DT) else (0 if op == OP_NEG else -1)
            assert 1 <= d
        assert d == 1
    assert all(0 <= r < nd and 0 <= c < nd for r, c in zip(t["rows"], t["cols"])) and len(t["rows"]) == nnz
    for k, x, y, z in t["fops"]:
        assert 0 <= x < nnz and 0 <= y < nnz and (k == DIV or 0 <= z < nnz)
    for k, x, y, z in t["sops"]:
        assert 0 <= x < n and 0 <= z < nnz and (k == DIV or 0 <= y < n)
    assert sorted(t["init"].values()) == list(range(nd)) and all(0 <= i < n for i in t["init"])
    assert all(0 <= d < n for d in t["dyn"]) and len(t["dyn"]) == nd
    assert max(nnz, n) < (1 << 20)


def _arr(ctype: str, name: str, vals, per_line: int = 16) -> str:
    vals = list(vals)
    if not vals:
        vals = [0]
    body = ",\n    ".join(", ".join(str(v) for v in vals[i:i + per_line]) for i in range(0, len(vals), per_line))
    return "static __device__ const %s %s[%d] = {\n    %s};" % (ctype, name, len(vals), body)


def _dbl(v: float) -> str:
    return repr(float(v)) if v == v and abs(v) != float("inf") else "0.0"


def emit(sysm, cid: str) -> str:
    """C++ text: the tables as device arrays and a traits struct."""
    t = tables(sysm)
    nd, nnz = t["nd"], t["nnz"]
    check_bounds(t)
    L = ["", "/* warp-per-cell tables (odevec_b200/wpc.py) */"]
    # right-hand side terms
    ptr, coef, fac = [0], [], []
    for terms in t["rhs"]:
        for c, fs in terms:
            coef.append(c)
            enc = []
            for k in range(MAXF):
                if k < len(fs):
                    s, sq = fs[k]
                    enc.append(s * 2 + sq)
                else:
                    enc.append(-1)
            fac.extend(enc)
        ptr.append(len(coef))
    L.append(_arr("int", "ov_wpc_%s_rhs_ptr" % cid, ptr))
    L.append(_arr("double", "ov_wpc_%s_rhs_coef" % cid, [_dbl(c) for c in coef], 4))
    L.append(_arr("int", "ov_wpc_%s_rhs_fac" % cid, fac))
    # iteration-matrix programs
    pptr, code = [0], []
    dmax = 1
    for prog in t["progs"]:
        code.extend(op | (arg << 4) for op, arg in prog)
        pptr.append(len(code))
        dmax = max(dmax, depth(prog))
    L.append(_arr("int", "ov_wpc_%s_jac_ptr" % cid, pptr))
    L.append(_arr("int", "ov_wpc_%s_jac_code" % cid, code))
    L.append(_arr("double", "ov_wpc_%s_jac_const" % cid, [_dbl(c) for c in t["consts"]], 4))
    L.append(_arr("int", "ov_wpc_%s_jac_rc" % cid, [r | (c << 16) for r, c in zip(t["rows"], t["cols"])]))
    # factorisation and solve statements: one row of K slots per level for
    # the K lanes that hold a cell (K = 32, 16, 8); a level of more than K
    # statements takes several rows: its statements are independent, so
    # running them one row after another is the same
    def lev_tables(name, ops, lev, enc, width):
        rows = [[enc(ops[i]) for i in part] + ["-1LL"] * (width - len(part)) for part in level_rows(lev, width)]
        sfx = "" if width == 32 else str(width)
        L.append(_arr("long long", "ov_wpc_%s_%s_op%s" % (cid, name, sfx), [v for row in rows for v in row], 8))
        return len(rows)

    enc = lambda o: "%dLL" % (o[0] | (o[1] << 1) | ((o[2] & 0xfffff) << 21) | ((o[3] & 0xfffff) << 41))
    nlev = {}
    for width in LANES:
        nlev[width] = (lev_tables("fac", t["fops"], t["flev"], enc, width),
                       lev_tables("sol", t["sops"], t["slev"], enc, width))
    nfl, nsl = nlev[32]
    # solver index <-> storage row of the solve vector
    srow = [0] * nd
    for i, j in t["init"].items():
        srow[j] = i
    for j, i in t["out"].items():
        if srow[j] != i:
            raise ValueError("solve maps solver index %d to two rows" % j)
    L.append(_arr("int", "ov_wpc_%s_srow" % cid, srow))
    L.append(_arr("int", "ov_wpc_%s_dyn" % cid, t["dyn"]))
    L.append("struct ov_wpc_%s {" % cid)
    L.append("  static constexpr int NTERM = %d, NPROG = %d, DEPTH = %d, NFL = %d, NSL = %d;"
             % (len(coef), len(t["progs"]), dmax, nfl, nsl))
    for width in LANES[1:]:
        L.append("  static constexpr int NFL%d = %d, NSL%d = %d;" % (width, nlev[width][0], width, nlev[width][1]))
    for nm in ("rhs_ptr", "rhs_fac", "jac_ptr", "jac_code", "jac_rc", "srow", "dyn"):
        L.append("  __device__ static const int* %s() { return ov_wpc_%s_%s; }" % (nm, cid, nm))
    for nm in ("rhs_coef", "jac_const"):
        L.append("  __device__ static const double* %s() { return ov_wpc_%s_%s; }" % (nm, cid, nm))
    for width in LANES:
        sfx = "" if width == 32 else str(width)
        for nm in ("fac_op", "sol_op"):
            L.append("  __device__ static const long long* %s%s() { return ov_wpc_%s_%s%s; }"
                     % (nm, sfx, cid, nm, sfx))
    L.append("};")
    return "\n".join(L) + "\n"
