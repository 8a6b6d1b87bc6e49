#!/usr/bin/env python
"""OdeVec preprocessor: SymPy network -> straight-line C / CUDA network code.

Same command line as the reference (``pre_odevec.py:383-450``): ``--nvector``,
``--example``, ``--krome_setupfile``, ``--LUmethod``, ``--dt_min``,
``--heatcool``, ``--ordering``, ``--packaging``; and the same pipeline
(``pre_odevec.py:463-540``):

1. ``J = rhs.jacobian(y)``                              (``pre_odevec.py:467``)
2. ``P = I - dt*beta*J``                                (``pre_odevec.py:474-475``)
3. reordering CMK / INVERT / FF                         (``pre_odevec.py:265-361``)
4. LU fill pattern of the reordered ``P``                (``pre_odevec.py:494``)
5. CSC arrays ``row_index``, ``u_col_start`` (column starts) and
   ``l_col_start`` (diagonal positions)                 (``pre_odevec.py:523-540``)

Instead of substituting ``#ODEVEC_*`` pragmas in Fortran templates it writes,
per network variant ``<tag>``:

* ``csrc/gen/net_<tag>.h`` - plain C, callable from host and device
  (``OV_HD``): the right-hand side ``f = rhs(y, k)`` in species order and the
  iteration matrix ``P`` at the LU pattern positions in CSC storage order
  (fill-ins written as 0, as ``pre_odevec.py:173-180`` does), plus the
  permutation and CSC arrays as constants.
* ``csrc/gen/net_<tag>.cuh`` - CUDA: a traits struct for the solver kernel and
  the numeric LU factorisation and the two triangular solves unrolled into
  straight-line code over the fill pattern, with the permutation folded into
  the solve's loads and stores.  The operation order is exactly that of the
  reference loops: right-looking Doolittle for DENSE packaging
  (``src/odevec.F90:898-922``, solve ``:797-849``) and left-looking Crout for
  CSC (``src/odevec.F90:929-971``, solve ``:853-891``).  DENSE stores only the
  structurally non-zero entries; the skipped terms are exact zeros, so the
  results equal the full n x n loops.

Expressions are printed term by term without common-subexpression rewriting,
in SymPy's canonical order, which is the order ``fcode`` prints them in the
reference; integer powers are expanded into products as gfortran expands them
(``x*x``, ``x*(x*x)``, ...).  Compiled without floating-point contraction the
emitted code therefore evaluates the same IEEE operations as the reference's
generated Fortran.

The LU pattern is computed structurally (boolean elimination without
pivoting); ``--lu_pattern=symbolic`` instead runs SymPy's symbolic
``LUdecomposition_Simple`` like the reference, which can only drop entries
that cancel exactly.  For the shipped networks both give the reference's
pattern (checked in the tests).
"""
from __future__ import annotations

import argparse
import dataclasses
import os
import re
import sys
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import sympy as sp
from mpmath.libmp import prec_to_dps, to_str as mlib_to_str
from sympy.printing.c import C99CodePrinter

from . import networks

GEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "gen")
MAXORDER = 5  # pre_odevec.py:83


# ----------------------------------------------------------------- ordering
def _pattern_of(P: sp.SparseMatrix) -> np.ndarray:
    n = P.shape[0]
    pat = np.zeros((n, n), dtype=bool)
    for (i, j), v in P.todok().items():
        if v != 0:
            pat[i, j] = True
    return pat


def ordering_cmk(P: sp.SparseMatrix) -> np.ndarray:
    """Reverse Cuthill-McKee of the transposed pattern with SciPy's
    ``reverse_cuthill_mckee(symmetric_mode=False)``, as ``pre_odevec.py:292-302``."""
    from scipy import sparse
    from scipy.sparse import csgraph
    pat = _pattern_of(P)
    rows, cols = np.nonzero(pat)
    # the reference swaps the (row, col) of P.col_list() when building the matrix
    M = sparse.csc_matrix((np.ones(len(rows), dtype=int), (cols, rows)), shape=pat.shape)
    return np.asarray(csgraph.reverse_cuthill_mckee(M, symmetric_mode=False), dtype=int)


def ordering_invert(P: sp.SparseMatrix) -> np.ndarray:
    """Reversed indices (``pre_odevec.py:317-334``)."""
    return np.arange(P.shape[0])[::-1].copy()


def ordering_ff(P: sp.SparseMatrix) -> np.ndarray:
    """Fewest non-zeros first: key = nnz(column i) + nnz(row i) - 1, ascending
    (``pre_odevec.py:337-361``).  Ties keep index order (stable sort)."""
    pat = _pattern_of(P)
    key = pat.sum(axis=0) + pat.sum(axis=1) - 1
    return np.argsort(key, kind="stable").astype(int)


ORDERINGS = {"CMK": ordering_cmk, "INVERT": ordering_invert, "FF": ordering_ff}


# --------------------------------------------------------------- LU pattern
def structural_lu_pattern(pat: np.ndarray) -> np.ndarray:
    """Fill pattern of Gaussian elimination without pivoting."""
    lu = pat.copy()
    n = lu.shape[0]
    for k in range(n):
        rows = np.nonzero(lu[k + 1:, k])[0] + k + 1
        cols = np.nonzero(lu[k, k + 1:])[0] + k + 1
        if len(rows) and len(cols):
            lu[np.ix_(rows, cols)] = True
    return lu


def symbolic_lu_pattern(P_order: sp.Matrix) -> np.ndarray:
    LU, _ = sp.Matrix(P_order).LUdecomposition_Simple()
    n = LU.shape[0]
    pat = np.zeros((n, n), dtype=bool)
    for i in range(n):
        for j in range(n):
            pat[i, j] = LU[i, j] != 0
    return pat


# ------------------------------------------------------------------- system
@dataclasses.dataclass
class System:
    net: networks.Network
    tag: str
    packaging: str            # "DENSE" | "CSC"
    ordering: str             # "None" | "CMK" | "INVERT" | "FF"
    perm: List[int]           # storage row i holds species perm[i]
    P: sp.Matrix              # I - dt*beta*J in species order
    P_order: sp.Matrix        # permuted
    lu_pat: np.ndarray        # bool n x n, storage order
    row_index: List[int]
    u_col_start: List[int]
    l_col_start: List[int]
    p_nnz: int
    nvector: int = 1
    dt_min: float = 1e-10
    lu_method: int = 1
    lu_exprs: Optional[sp.Matrix] = None   # LUmethod 2: symbolic L\U of P_order

    @property
    def neq(self) -> int:
        return self.net.neq

    @property
    def nnz(self) -> int:
        return len(self.row_index)

    def pos(self) -> Dict[Tuple[int, int], int]:
        """(row, col) in storage order -> index into the packed value array."""
        out = {}
        for j in range(self.neq):
            for kk in range(self.u_col_start[j], self.u_col_start[j + 1]):
                out[(self.row_index[kk], j)] = kk
        return out


def build_system(net: networks.Network, ordering: str = "None", packaging: str = "DENSE",
                 lu_pattern: str = "structural", nvector: int = 1, dt_min: float = 1e-10,
                 lu_method: int = 1, tag: Optional[str] = None) -> System:
    packaging = packaging.upper()
    if packaging in ("COO", "CSR"):
        raise SystemExit("# Error: %s packaging is not supported" % packaging)  # pre_odevec.py:515-518
    if packaging not in ("DENSE", "CSC"):
        raise SystemExit("# Error: This format is not known.")
    if lu_method not in (1, 2, 3):
        raise SystemExit("# Error: --LUmethod=%d is not known (1: symbolic Jacobian + numeric LU, "
                         "2: symbolic LU, 3: finite-difference Jacobian + numeric LU)" % lu_method)
    if lu_method == 2 and packaging != "DENSE":
        # the symbolic factors are Doolittle's (unit L); the reference's sparse
        # solve (src/odevec.F90:853-891) expects Crout factors (unit U)
        raise SystemExit("# Error: --LUmethod=2 needs --packaging=DENSE")
    if lu_method == 3 and packaging != "DENSE":
        # src/odevec.F90:509-523: CalcJac_sparse aborts
        raise SystemExit("The Method Flags LUmethod=3 is not supported with sparse matrices, yet. Aborting...")
    if lu_method == 3 and ordering not in (None, "None", "NONE", ""):
        # CalcJac_dense (src/odevec.F90:469-506) fills P in species order, while
        # the solve applies the permutation to the residual
        raise SystemExit("# Error: --LUmethod=3 needs --ordering=None")
    n = net.neq
    if net.heatcool:
        if lu_method == 2:
            raise SystemExit("# Error: --heatcool=1 with --LUmethod=2: the symbolic factors would "
                             "ignore the temperature equation; use --LUmethod=1 or 3")
        if packaging == "DENSE" and lu_method == 1 and ordering not in (None, "None", "NONE", ""):
            # the difference quotients are written at species positions
            # (pre_odevec.py:148-170)
            raise SystemExit("# Error: --heatcool=1 with DENSE packaging needs --ordering=None")
    jac = net.rhs.jacobian(net.y)
    dt, beta = sp.symbols("dt beta")
    P = sp.SparseMatrix(sp.eye(n) - dt * beta * jac)
    if ordering in (None, "None", "NONE", ""):
        ordering = "None"
        perm = np.arange(n)
    else:
        if ordering not in ORDERINGS:
            raise SystemExit("# Error: unknown ordering %r" % ordering)
        perm = ORDERINGS[ordering](P)
    perm = [int(v) for v in perm]
    P_order = sp.zeros(n, n)
    for i in range(n):
        for j in range(n):
            P_order[i, j] = P[perm[i], perm[j]]
    pat = _pattern_of(sp.SparseMatrix(P_order))
    if heatcool_fd(net, packaging, lu_method):
        # the Tgas row over the chemical species and the whole Tgas column
        # are difference quotients (ordering None: storage = species order)
        T = net.neq - 2
        pat[T, :net.nmols] = True
        pat[:, T] = True
    lu_exprs = None
    if lu_method == 3:
        # the difference quotients fill every entry: the rate coefficients of
        # a network may depend on the whole state (PRIMORDIAL's floor on
        # max_j y_j), so a perturbation of one species moves every right-hand
        # side.  Frozen species keep identity rows and columns: their entries
        # never reach a solution (the kernel leaves them out).
        lu = np.ones((n, n), dtype=bool)
        for f in _frozen_of(net):
            lu[f, :] = False
            lu[:, f] = False
            lu[f, f] = True
        pat = lu.copy()
    elif lu_method == 2:
        # the reference's symbolic factorisation (pre_odevec.py:493); its row
        # permutation is dropped there, so a pivot is an error here
        lu_exprs, piv = sp.Matrix(P_order).LUdecomposition_Simple()
        if piv:
            raise SystemExit("# Error: the symbolic LU of P needs row exchanges %s; use --LUmethod=1" % (piv,))
        lu = structural_lu_pattern(pat | np.eye(n, dtype=bool))
        for i in range(n):
            for j in range(n):
                if lu_exprs[i, j] != 0 and not lu[i, j]:
                    raise SystemExit("# Error: symbolic LU entry (%d,%d) outside the fill pattern" % (i, j))
    elif lu_pattern == "symbolic" and packaging == "CSC":
        # the dense factorisation touches every structurally non-zero entry,
        # so DENSE always uses the structural pattern
        lu = symbolic_lu_pattern(P_order)
        lu |= np.eye(n, dtype=bool)
    else:
        lu = structural_lu_pattern(pat | np.eye(n, dtype=bool))
    if (pat & ~lu).any():
        raise SystemExit("# Error: P has entries outside the LU pattern (exact cancellation); "
                         "use --lu_pattern=structural")
    row_index, u_col_start, l_col_start = [], [], []
    for j in range(n):
        u_col_start.append(len(row_index))
        for i in range(n):
            if lu[i, j]:
                if i == j:
                    l_col_start.append(len(row_index))
                row_index.append(i)
    u_col_start.append(len(row_index))
    if tag is None:
        tag = "%s_%s_%s" % (net.name, packaging, ordering.upper())
        if lu_method != 1:
            tag += "_LU%d" % lu_method
    return System(net, tag, packaging, ordering, perm, sp.Matrix(P), P_order, lu,
                  row_index, u_col_start, l_col_start, int(pat.sum()), nvector, dt_min, lu_method, lu_exprs)


# ------------------------------------------------------------------ printer
# addition chain x^n = x^(n-t[n]) * x^t[n] (the way gfortran expands x**n)
_POWI = [0, 1, 1, 2, 2, 3, 3, 4, 4, 6, 5, 6, 6, 10, 7, 9]


class NetPrinter(C99CodePrinter):
    """C printer mapping the reference's symbol names onto array accesses."""

    _sym = re.compile(r"^(y|k)\(:,(\d+)\)$")

    def __init__(self, ymap: Dict[sp.Symbol, str], kname: str = "k"):
        super().__init__()
        self.ymap = ymap
        self.kname = kname

    def _print_Symbol(self, expr):
        if expr in self.ymap:
            return self.ymap[expr]
        m = self._sym.match(expr.name)
        if m and m.group(1) == "k":
            return "%s[%d]" % (self.kname, int(m.group(2)) - 1)
        if expr.name in ("dt", "beta"):
            return expr.name
        raise ValueError("unexpected symbol %s" % expr.name)

    def _print_Float(self, expr):
        # the decimal string fcode writes: the Float's own precision (15
        # significant digits for a double), so the compiled constant is the
        # same double as the reference's generated Fortran constant
        s = mlib_to_str(expr._mpf_, prec_to_dps(expr._prec), strip_zeros=True)
        if s in ("+inf", "inf", "-inf", "nan"):
            raise ValueError("non-finite constant in network expression")
        if "e" not in s and "." not in s:
            s += ".0"
        return s

    def _print_Integer(self, expr):
        return "%d.0" % int(expr)

    def _print_Rational(self, expr):
        return "(%d.0/%d.0)" % (expr.p, expr.q)

    def _powi(self, base: str, n: int) -> str:
        cache = {1: base}

        def rec(m):
            if m in cache:
                return cache[m]
            if m < len(_POWI):
                s = "(%s*%s)" % (rec(m - _POWI[m]), rec(_POWI[m]))
            else:
                s = "(%s*%s)" % (rec(m - 1), base)
            cache[m] = s
            return s
        return rec(n)

    def _print_Pow(self, expr):
        b, e = expr.as_base_exp()
        bs = self.parenthesize(b, 1000)
        if e.is_Integer:
            n = int(e)
            if n > 0:
                return self._powi(bs, n)
            if n < 0:
                return "(1.0/%s)" % self._powi(bs, -n)
            return "1.0"
        if e == sp.Rational(1, 2):
            return "sqrt(%s)" % self._print(b)
        return "ov_pow(%s, %s)" % (self._print(b), self._print(sp.Float(float(e))))


def _cexpr(expr, pr: NetPrinter) -> str:
    expr = sp.sympify(expr)
    if expr == 0:
        return "0.0"
    return pr.doprint(expr)


def _cswitch(vals: Sequence[int]) -> str:
    """constexpr table lookup as a nested conditional (usable on host and device)."""
    expr = str(vals[-1])
    for i in range(len(vals) - 2, -1, -1):
        expr = "i == %d ? %d : (%s)" % (i, vals[i], expr)
    return expr


def _cid(tag: str) -> str:
    return re.sub(r"[^A-Za-z0-9_]", "_", tag).lower()


# ----------------------------------------------------------------- emitters
def emit_c_header(sysm: System) -> str:
    net = sysm.net
    n, nnz = sysm.neq, sysm.nnz
    cid = _cid(sysm.tag)
    ymap = {s: "y[%d]" % i for i, s in enumerate(net.y)}
    pr = NetPrinter(ymap)
    pos = sysm.pos()
    L = []
    g = "OV_NET_%s_H" % cid.upper()
    L.append("/* Generated by odevec_b200.pre_odevec -- do not edit.")
    L.append(" * network %s, packaging %s, ordering %s, neq %d, LU nnz %d (P nnz %d)."
             % (net.name, sysm.packaging, sysm.ordering, n, nnz, sysm.p_nnz))
    L.append(" * rhs(): f = dy/dt in species order (rate array k as in the reference).")
    if sysm.lu_method == 1:
        L.append(" * jac(): P = I - dt*beta*J at the LU pattern positions, CSC storage order")
        L.append(" *        of the permuted matrix; fill-in positions are 0.  */")
    elif sysm.lu_method == 2:
        L.append(" * jac(): LUmethod 2, the symbolic factors L\\U of P (unit L) at the")
        L.append(" *        pattern positions, CSC storage order; no numeric factorisation.  */")
    else:
        L.append(" * jac(): LUmethod 3, empty: P comes from difference quotients of rhs().  */")
    L.append("#ifndef %s" % g)
    L.append("#define %s" % g)
    L.append('#include "../ov_common.h"')
    if net.rates:
        L.append('#include "../rates_%s.h"' % net.rates)
    if net.heatcool:
        L.append('#include "../%s"' % os.path.basename(net.heatcool_header))
    L.append("")
    L.append("#define OV_%s_NEQ %d" % (cid.upper(), n))
    L.append("#define OV_%s_NNZ %d" % (cid.upper(), nnz))
    L.append("#define OV_%s_NREA %d" % (cid.upper(), net.nrea if net.rates else 0))
    L.append("#define OV_%s_DENSE %d" % (cid.upper(), 1 if sysm.packaging == "DENSE" else 0))
    L.append("#define OV_%s_NVECTOR %d" % (cid.upper(), sysm.nvector))
    L.append("#define OV_%s_DT_MIN %r" % (cid.upper(), float(sysm.dt_min)))
    L.append("#define OV_%s_IDX_TGAS %d" % (cid.upper(), net.idx_tgas if net.idx_tgas is not None else -1))

    def arr(name, vals):
        L.append("static const int ov_%s_%s[%d] = {%s};" % (cid, name, len(vals),
                                                          ", ".join(str(v) for v in vals)))
    from . import wpc
    arr("sizes", [n, nnz, net.nrea if net.rates else 0, 1 if sysm.packaging == "DENSE" else 0,
                  net.idx_tgas if net.idx_tgas is not None else -1, n - len(frozen_species(sysm)),
                  sysm.lu_method, 1 if wpc.eligible(sysm) else 0])
    L.append("static const double ov_%s_defaults[2] = {%d.0, %r}; /* nvector, dt_min */"
             % (cid, sysm.nvector, float(sysm.dt_min)))
    # species masses (g) and inverse masses (1/g) for the mass-fraction format;
    # all zero when the network has none
    for name, vals in (("mass", net.masses), ("imass", net.imasses)):
        vals = vals if vals is not None else [0.0] * n
        L.append("static const double ov_%s_%s[%d] = {%s};" % (cid, name, n, ", ".join(repr(float(v)) for v in vals)))
    arr("perm", sysm.perm)
    arr("row_index", sysm.row_index)
    arr("u_col_start", sysm.u_col_start)
    arr("l_col_start", sysm.l_col_start)
    L.append("")
    if net.heatcool:
        L += _hc_function(cid, net)
        L.append("")
    L.append("OV_HD static OV_INLINE void ov_%s_rhs(const double* OV_RESTRICT y, "
             "const double* OV_RESTRICT k, double* OV_RESTRICT f)" % cid)
    L.append("{")
    L.append("  (void)k;")
    body = []
    for i in range(n):
        if net.heatcool and i == n - 2:
            body.append("  f[%d] = ov_%s_hc(y, y[%d], y);  /* heating/cooling */" % (i, cid, i))
        else:
            body.append("  f[%d] = %s;" % (i, _cexpr(net.rhs[i], pr)))
    L += _fenced(body, SCHED_EVERY_RHS, n - len(frozen_species(sysm)) >= SCHED_MIN_ND, "  ")
    L.append("}")
    L.append("")
    hc_note = (" With heating/cooling difference quotients, entries the reference leaves"
               " unwritten keep a[]'s content." if heatcool_fd(net, sysm.packaging, sysm.lu_method) else "")
    L.append("/* P at the pattern positions, CSC storage order.%s */" % hc_note)
    L.append("OV_HD static OV_INLINE void ov_%s_jac(const double* OV_RESTRICT y, "
             "const double* OV_RESTRICT k, double beta, double dt, double* OV_RESTRICT a)" % cid)
    L.append("{")
    L.append("  (void)y; (void)k; (void)beta; (void)dt; (void)a;")
    src = _jac_source(sysm)
    if heatcool_fd(net, sysm.packaging, sysm.lu_method):
        items = [((sysm.row_index[kk], j), kk) for j in range(n)
                 for kk in range(sysm.u_col_start[j], sysm.u_col_start[j + 1])]
        L += _hc_jac_lines(sysm, cid, items, lambda kk, i, j, e: "a[%d] = %s;  /* (%d,%d) */" % (kk, e, i, j),
                           "  ", lambda i, j: _cexpr(src[i, j], pr))
    else:
        for j in range(n):
            for kk in range(sysm.u_col_start[j], sysm.u_col_start[j + 1]):
                i = sysm.row_index[kk]
                if src is not None:
                    L.append("  a[%d] = %s;  /* (%d,%d) */" % (kk, _cexpr(src[i, j], pr), i, j))
    L.append("}")
    L.append("")
    L.append("#endif")
    return "\n".join(L) + "\n"


def _jac_source(sysm: System):
    """What jac() writes: P (LUmethod 1), its symbolic factors (2), nothing (3)."""
    return {1: sysm.P_order, 2: sysm.lu_exprs, 3: None}[sysm.lu_method]


def _lu_factor_lines(sysm: System) -> List[str]:
    """Straight-line numeric LU in the reference's operation order."""
    if sysm.lu_method == 2:
        return []
    n = sysm.neq
    pos = sysm.pos()
    out = []
    if sysm.packaging == "DENSE":
        # right-looking Doolittle (src/odevec.F90:906-921)
        for k in range(n - 1):
            for j in range(k + 1, n):
                if (j, k) in pos:
                    out.append("a[%d] = a[%d] / a[%d];" % (pos[(j, k)], pos[(j, k)], pos[(k, k)]))
            for j in range(k + 1, n):
                if (k, j) not in pos:
                    continue
                for m in range(k + 1, n):
                    if (m, k) in pos:
                        out.append("a[%d] = a[%d] - a[%d]*a[%d];"
                                   % (pos[(m, j)], pos[(m, j)], pos[(m, k)], pos[(k, j)]))
    else:
        # left-looking Crout on the CSC pattern (src/odevec.F90:937-969)
        ri, ucs, lcs = sysm.row_index, sysm.u_col_start, sysm.l_col_start
        for k in range(n):
            colpos = {ri[kk]: kk for kk in range(ucs[k], ucs[k + 1])}
            for kk in range(ucs[k], lcs[k]):
                j = ri[kk]
                out.append("a[%d] = a[%d] / a[%d];" % (kk, kk, lcs[j]))
                for jj in range(lcs[j] + 1, ucs[j + 1]):
                    r = ri[jj]
                    if r in colpos:
                        out.append("a[%d] = a[%d] - a[%d]*a[%d];" % (colpos[r], colpos[r], kk, jj))
    return out


def _lu_solve_lines(sysm: System, dpos: Optional[Dict[int, int]] = None) -> List[str]:
    """Straight-line solve P_order x = r with the permutation folded in:
    reads r[perm[i]] and writes x[perm[i]] (species order), or, with dpos,
    the solver-state index dpos[perm[i]] of the dynamic species only."""
    n = sysm.neq
    pos = sysm.pos()
    p = list(sysm.perm)
    if dpos is None:
        dpos = {s_: s_ for s_ in range(n)}
    live = [i for i in range(n) if p[i] in dpos]
    out = []
    for i in live:
        out.append("T d%d = (T)(r[%d]*OV_SC(%d));" % (i, dpos[p[i]], dpos[p[i]]))
    if sysm.packaging == "DENSE":
        # forward, unit lower (src/odevec.F90:814-826): d_k = r_k - sum_{j<k} L_kj d_j
        for k in live:
            terms = [j for j in range(k) if (k, j) in pos]
            if terms:
                s = "a[%d]*d%d" % (pos[(k, terms[0])], terms[0])
                for j in terms[1:]:
                    s = "(%s + a[%d]*d%d)" % (s, pos[(k, j)], j)
                out.append("d%d = d%d - %s;" % (k, k, s))
        # backward (src/odevec.F90:835-847): x_k = (d_k - sum_{j>k} U_kj x_j) / U_kk
        for k in reversed(live):
            terms = [j for j in range(k + 1, n) if (k, j) in pos]
            if terms:
                s = "a[%d]*d%d" % (pos[(k, terms[0])], terms[0])
                for j in terms[1:]:
                    s = "(%s + a[%d]*d%d)" % (s, pos[(k, j)], j)
                out.append("d%d = (d%d - %s) / a[%d];" % (k, k, s, pos[(k, k)]))
            else:
                out.append("d%d = d%d / a[%d];" % (k, k, pos[(k, k)]))
    else:
        ri, ucs, lcs = sysm.row_index, sysm.u_col_start, sysm.l_col_start
        # forward (src/odevec.F90:864-876)
        for k in live:
            out.append("d%d = d%d / a[%d];" % (k, k, lcs[k]))
            for kk in range(lcs[k] + 1, ucs[k + 1]):
                out.append("d%d = d%d - d%d*a[%d];" % (ri[kk], ri[kk], k, kk))
        # backward (src/odevec.F90:878-889)
        for k in reversed(live):
            for kk in range(ucs[k], lcs[k]):
                out.append("d%d = d%d - d%d*a[%d];" % (ri[kk], ri[kk], k, kk))
    for i in live:
        out.append("x[%d] = (double)d%d*OV_ISC(%d);" % (dpos[p[i]], i, dpos[p[i]]))
    return out


def frozen_species(sysm: System) -> List[int]:
    """Species whose right-hand side is identically zero and that no other
    right-hand side depends on.  Their Newton corrections are exact zeros,
    their state never changes and their rows and columns of P are those of
    the identity, so the CUDA kernel keeps them out of the solver state."""
    return _frozen_of(sysm.net)


def _frozen_of(net: networks.Network) -> List[int]:
    n = net.neq
    J = net.rhs.jacobian(net.y)
    # with --heatcool=1 the temperature has a right-hand side that depends on
    # the chemical species and on itself
    live = set(range(net.nmols)) | {n - 2} if net.heatcool else set()
    out = []
    for i in range(n):
        if i in live:
            continue
        if sp.sympify(net.rhs[i]) == 0 and all(sp.sympify(J[r, i]) == 0 for r in range(n)):
            out.append(i)
    return out


def heatcool_fd(net: networks.Network, packaging: str, lu_method: int) -> bool:
    """whether GetJac writes the heating/cooling difference quotients: DENSE
    packaging with the symbolic Jacobian (pre_odevec.py:146-170); CSC
    packaging keeps the symbolic entries, where the Tgas row is that of the
    network without the heating/cooling term (pre_odevec.py:173-180)"""
    return net.heatcool and packaging.upper() == "DENSE" and lu_method == 1


def _hc_function(cid: str, net: networks.Network) -> List[str]:
    """the gas-temperature right-hand side (pre_odevec.py:556-558):
    ((heating - cooling) * (gamma - 1)) / k_B / sum of the chemical species,
    the sum taken in index order from 0 as gfortran's sum(.., dim=2)"""
    L = ["/* dTgas/dt: heating/cooling term of the temperature row; yv is the state",
         "   heating and cooling see, Tgas their temperature, ys the state whose",
         "   chemical species are summed and whose gamma is taken */",
         "OV_HD static OV_INLINE double ov_%s_hc(const double* OV_RESTRICT yv, double Tgas, "
         "const double* OV_RESTRICT ys)" % cid, "{", "  double s = 0.0;"]
    for j in range(net.nmols):
        L.append("  s = s + ys[%d];" % j)
    L.append("  return (ov_hc_heating(yv, Tgas) - ov_hc_cooling(yv, Tgas)) * (ov_hc_gamma(ys) - 1.0) "
             "/ OV_HC_BOLTZMANN / s;")
    L.append("}")
    return L


def _hc_jac_lines(sysm: "System", cid: str, pos_items, store, indent: str, symbolic) -> List[str]:
    """GetJac with the heating/cooling difference quotients
    (pre_odevec.py:146-170), column by column as the reference writes it:
    the Tgas row of each chemical species column j is
    -(beta*dt*(hc(y + dy_j e_j) - hc(y)))/dy_j with dy_j = y_j*1e-2, written
    only where dy_j > 0 (elsewhere the entry keeps what the matrix storage
    holds); the Tgas column is -(beta*dt*(f_i(yy)/dy_T)) for every row i, 1
    added on the diagonal, where yy is the state of the last species column
    (its species still perturbed) with y_T + dy_T, dy_T = y_T*1e-2 -- f(yy)
    itself, not f(yy) - f(y).  pos_items: ((i, j), kk) in storage order;
    store(kk, i, j, expr) -> line or None; symbolic(i, j) -> expr string."""
    net = sysm.net
    n, T = net.neq, net.neq - 2
    L = [indent + "const double hc_dy0 = ov_%s_hc(y, y[%d], y);" % (cid, T),
         indent + "double hc_yy[%d];" % n]
    col_T = [(i, kk) for (i, j), kk in pos_items if j == T]
    done_T = False
    for (i, j), kk in pos_items:
        if j == T:
            if done_T:
                continue
            done_T = True
            L.append(indent + "{ /* Tgas column */")
            L.append(indent + "  const double dyy = y[%d]*1e-2;" % T)
            L.append(indent + "  hc_yy[%d] = y[%d] + dyy;" % (T, T))
            L.append(indent + "  double dy[%d];" % n)
            L.append(indent + "  ov_%s_rhs(hc_yy, k, dy);" % cid)
            for r, kr in col_T:
                v = "-(beta*dt*(dy[%d]/dyy))" % r
                if r == T:
                    v = "1.0 + (%s)" % v
                ln = store(kr, r, T, v)
                if ln:
                    L.append(indent + "  " + ln)
            L.append(indent + "}")
        elif i == T and j < net.nmols:
            L.append(indent + "{ /* Tgas row, column %d */" % j)
            L.append(indent + "  for (int m = 0; m < %d; ++m) hc_yy[m] = y[m];" % n)
            L.append(indent + "  const double dyy = y[%d]*1e-2;" % j)
            L.append(indent + "  hc_yy[%d] = y[%d] + dyy;" % (j, j))
            L.append(indent + "  const double dy1 = ov_%s_hc(hc_yy, y[%d], y);" % (cid, T))
            ln = store(kk, i, j, "-(beta*dt*(dy1 - hc_dy0)/dyy)")
            if ln:
                L.append(indent + "  if (dyy > 0.0) " + ln)
            L.append(indent + "}")
        else:
            ln = store(kk, i, j, symbolic(i, j))
            if ln:
                L.append(indent + ln)
    return L


def _reduced(sysm: System):
    """Dynamic species, their positions, and the packed-index map of the LU
    pattern restricted to dynamic rows and columns."""
    n = sysm.neq
    fz = set(frozen_species(sysm))
    dyn = [s for s in range(n) if s not in fz]
    dpos = {s: i for i, s in enumerate(dyn)}
    kmap = {}
    for j in range(n):
        for kk in range(sysm.u_col_start[j], sysm.u_col_start[j + 1]):
            i = sysm.row_index[kk]
            if sysm.perm[i] in dpos and sysm.perm[j] in dpos:
                kmap[kk] = len(kmap)
    return dyn, dpos, kmap


_DIV_LINE = re.compile(r"^(\S+) = (.+) / a\[(\d+)\];$")


def reciprocal_pivots(factor: List[str], solve: List[str]):
    """Rewrites the straight-line factorisation and solve so that every
    division x / a[p] becomes ov_divp<T>(x, a[p]), and the factorisation sets
    a[p] = ov_pivot<T>(a[p]) once the pivot a[p] is final: before the first
    factor line that divides by it, or at the end when only the solve does.
    ov_pivot and ov_divp are the identity and a division in FP64, so the FP64
    code divides exactly as the reference; an FP32 LU keeps reciprocals.
    Raises ValueError if a pivot is read other than as a divisor after that
    point (the factorisations emitted here never do)."""
    def rewrite(lines):
        out, used = [], []
        for ln in lines:
            m = _DIV_LINE.match(ln)
            if m:
                p = int(m.group(3))
                used.append(p)
                ln = "%s = ov_divp<T>(%s, a[%d]);" % (m.group(1), m.group(2), p)
            out.append(ln)
        return out, used
    f_out, f_used = rewrite(factor)
    s_out, s_used = rewrite(solve)
    first = {}
    for i, ln in enumerate(factor):
        m = _DIV_LINE.match(ln)
        if m:
            first.setdefault(int(m.group(3)), i)
    at = {}
    for p in dict.fromkeys(f_used + s_used):
        i = first.get(p, len(factor))
        ref = re.compile(r"a\[%d\](?!\d)" % p)
        for ln in factor[i:] + solve:
            m = _DIV_LINE.match(ln)
            rest = "%s = %s" % (m.group(1), m.group(2)) if m else ln
            if ref.search(rest):
                raise ValueError("pivot a[%d] is used other than as a divisor after it is final" % p)
        at.setdefault(i, []).append(p)
    res = []
    for i in range(len(factor) + 1):
        res += ["a[%d] = ov_pivot<T>(a[%d]);" % (p, p) for p in at.get(i, [])]
        if i < len(factor):
            res.append(f_out[i])
    return res, s_out


def _remap_a(line: str, kmap: Dict[int, int]) -> str:
    return re.sub(r"a\[(\d+)\]", lambda m: "a[%d]" % kmap[int(m.group(1))], line)


def _reduce_lines(lines: List[str], kmap: Dict[int, int]) -> List[str]:
    """The factorisation restricted to the dynamic block: a statement that
    writes an entry of a frozen species' row (the heating/cooling Tgas column
    reaches those rows) is left out -- such a row holds the identity's
    pivot, so nothing it computes reaches a dynamic entry; a statement that
    writes a dynamic entry must read dynamic entries only."""
    out = []
    for ln in lines:
        idx = [int(v) for v in re.findall(r"a\[(\d+)\]", ln)]
        if all(i in kmap for i in idx):
            out.append(_remap_a(ln, kmap))
        elif idx and idx[0] not in kmap:
            continue
        else:
            raise ValueError("dynamic entry computed from a frozen one: %s" % ln)
    return out


# Networks above this many solver-state species get a scheduling fence
# (OV_SCHED) every SCHED_EVERY statements of their straight-line code (every
# SCHED_EVERY_RHS species of the right-hand side): their code is long enough
# that the compiler's hoisted loads otherwise spill.
SCHED_MIN_ND = 33
SCHED_EVERY = 16
SCHED_EVERY_RHS = 4


def _fenced(lines: List[str], every: int, on: bool, indent: str = "    ") -> List[str]:
    if not on:
        return lines
    out = []
    for k, ln in enumerate(lines):
        out.append(ln)
        if (k + 1) % every == 0 and k + 1 < len(lines):
            out.append(indent + "OV_SCHED();")
    return out


def emit_cuda_header(sysm: System) -> str:
    net = sysm.net
    cid = _cid(sysm.tag)
    n = sysm.neq
    L = []
    g = "OV_NET_%s_CUH" % cid.upper()
    L.append("/* Generated by odevec_b200.pre_odevec -- do not edit.")
    L.append(" * CUDA traits of network variant %s for the BDF kernel: straight-line" % sysm.tag)
    L.append(" * LU factorisation and solve over the fill pattern (%s). */" %
             ("right-looking Doolittle" if sysm.packaging == "DENSE" else "left-looking Crout, CSC"))
    L.append("#pragma once")
    L.append('#include "net_%s.h"' % cid)
    L.append("")
    dyn, dpos, kmap = _reduced(sysm)
    nd = len(dyn)
    pos = sysm.pos()
    ymap = {sym: "y[%d]" % i for i, sym in enumerate(net.y)}
    pr = NetPrinter(ymap)
    from . import wpc
    has_wpc = wpc.eligible(sysm)
    if has_wpc:
        L.append(wpc.emit(sysm, cid))
    L.append("struct ov_net_%s {" % cid)
    if has_wpc:
        L.append("  /* warp-per-cell tables (staging 7) */")
        L.append("  static constexpr bool HAS_WPC = true;")
        L.append("  using Wpc = ov_wpc_%s;" % cid)
    else:
        L.append("  static constexpr bool HAS_WPC = false;")
        L.append("  using Wpc = void;")
    L.append("  static constexpr int NEQ = %d;   /* all species (state vector) */" % n)
    L.append("  static constexpr int ND = %d;    /* species in the solver state */" % nd)
    L.append("  static constexpr int NNZ = %d;   /* packed LU entries of the dynamic block */" % len(kmap))
    L.append("  static constexpr int NREA = %d;" % (net.nrea if net.rates else 0))
    L.append("  static constexpr int IDX_TGAS = %d;" % (net.idx_tgas if net.idx_tgas is not None else -1))
    L.append("  static constexpr bool DENSE = %s;" % ("true" if sysm.packaging == "DENSE" else "false"))
    L.append("  /* 1: symbolic Jacobian + numeric LU, 2: symbolic LU, 3: difference quotients */")
    L.append("  static constexpr int LU_METHOD = %d;" % sysm.lu_method)
    L.append("  /* the Tgas row is the heating/cooling term (--heatcool=1); HC_FD: GetJac writes")
    L.append("     its difference quotients and leaves some entries as the storage holds them */")
    L.append("  static constexpr bool HEATCOOL = %s;" % ("true" if net.heatcool else "false"))
    L.append("  static constexpr bool HC_FD = %s;" % (
        "true" if heatcool_fd(net, sysm.packaging, sysm.lu_method) else "false"))
    if sysm.lu_method == 3:
        # full pattern, species order: packed index of solver-state entry (i, j)
        for (i, j), kk in pos.items():
            if kk in kmap:
                assert kmap[kk] == dpos[j] * nd + dpos[i]
        L.append("  OV_HD static constexpr int pidx(int i, int j) { return j * ND + i; }")
    L.append('  static constexpr const char* TAG = "%s";' % sysm.tag)
    L.append("  /* dynamic species (solver state index -> species) and frozen ones */")
    L.append("  OV_HD static constexpr int dyn(int i) { return %s; }"
             % _cswitch(dyn))
    fz = [s_ for s_ in range(n) if s_ not in dpos]
    L.append("  static constexpr int NF = %d;" % len(fz))
    L.append("  OV_HD static constexpr int frozen(int i) { return %s; }" % _cswitch(fz if fz else [0]))
    L.append("  OV_HD static OV_INLINE void rhs(const double* y, const double* k, double* f) "
             "{ ov_%s_rhs(y, k, f); }" % cid)
    if net.rates:
        L.append("  static OV_INLINE __device__ void rates_k(const double* y, const double* r, double* k) "
                 "{ ov_rates_%s_k(y, %d, r, k); }" % (net.rates, n))
        L.append("  static __device__ __noinline__ void rates_T(const double* y, double* r) "
                 "{ ov_rates_%s_T(y[%d], r); }" % (net.rates, net.idx_tgas))
    else:
        L.append("  static OV_INLINE __device__ void rates_k(const double*, const double*, double*) {}")
        L.append("  static OV_INLINE __device__ void rates_T(const double*, double*) {}")
    L.append("  /* P = I - dt*beta*J on the dynamic block, packed CSC order */")
    src = _jac_source(sysm)
    L.append("  template <class T, class A> OV_HD static OV_INLINE void jac(const double* OV_RESTRICT y, "
             "const double* OV_RESTRICT k, double beta, double dt, A a) {")
    L.append("    (void)y; (void)k; (void)beta; (void)dt; (void)a;")
    hcfd = heatcool_fd(net, sysm.packaging, sysm.lu_method)
    items = sorted(pos.items(), key=lambda t: t[1])
    if hcfd:
        L += _hc_jac_lines(sysm, cid, items,
                           lambda kk, i, j, e: ("a[%d] = (T)(%s);" % (kmap[kk], e)) if kk in kmap else None,
                           "    ", lambda i, j: _cexpr(src[i, j], pr))
    else:
        L += _fenced(["    a[%d] = (T)(%s);" % (kmap[kk], _cexpr(src[i, j], pr))
                      for (i, j), kk in items if kk in kmap and src is not None], SCHED_EVERY, nd >= SCHED_MIN_ND)
    L.append("  }")
    L.append("  /* a = D P D^-1 rounded to T, D = diag(sc) over solver-state indices */")
    L.append("  template <class T, class A> OV_HD static OV_INLINE void store_scaled(const double* OV_RESTRICT P, "
             "A a, const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {")
    for (i, j), kk in sorted(pos.items(), key=lambda t: t[1]):
        if kk in kmap:
            L.append("    a[%d] = (T)(P[%d]*sc[%d]*isc[%d]);" % (kmap[kk], kmap[kk], dpos[sysm.perm[i]],
                                                              dpos[sysm.perm[j]]))
    L.append("  }")
    L.append("  /* the same, each entry evaluated in FP64, scaled by powers of two and")
    L.append("     rounded to T on the fly */")
    L.append("  template <class T, class A> OV_HD static OV_INLINE void jac_scaled(const double* OV_RESTRICT y, "
             "const double* OV_RESTRICT k, double beta, double dt, A a, "
             "const double* OV_RESTRICT sc, const double* OV_RESTRICT isc) {")
    L.append("    (void)y; (void)k; (void)beta; (void)dt; (void)a; (void)sc; (void)isc;")
    if hcfd:
        L += _hc_jac_lines(sysm, cid, items,
                           lambda kk, i, j, e: ("a[%d] = (T)((%s)*sc[%d]*isc[%d]);" % (
                               kmap[kk], e, dpos[sysm.perm[i]], dpos[sysm.perm[j]])) if kk in kmap else None,
                           "    ", lambda i, j: _cexpr(src[i, j], pr))
    else:
        L += _fenced(["    a[%d] = (T)((%s)*sc[%d]*isc[%d]);" % (kmap[kk], _cexpr(src[i, j], pr),
                                                             dpos[sysm.perm[i]], dpos[sysm.perm[j]])
                      for (i, j), kk in items if kk in kmap and src is not None], SCHED_EVERY, nd >= SCHED_MIN_ND)
    L.append("  }")
    L.append("  /* in-place numeric LU of the packed dynamic block a[0..NNZ-1]; A is a")
    L.append("     pointer or an accessor whose operator[] yields T& */")
    f_lines, s_lines = reciprocal_pivots(_reduce_lines(_lu_factor_lines(sysm), kmap),
                                         [_remap_a(l, kmap) for l in _lu_solve_lines(sysm, dpos=dpos)])
    L.append("  template <class T, class A> OV_HD static OV_INLINE void lu_factor(A a) {")
    L.append("    (void)a;")
    L += _fenced(["    " + ln for ln in f_lines], SCHED_EVERY, nd >= SCHED_MIN_ND)
    L.append("  }")
    L.append("  /* x = P^-1 r on the dynamic block; r, x over solver-state indices.  sc/isc")
    L.append("     scale entry i by sc[i] on the way in and isc[i] on the way out (pass")
    L.append("     nullptr for none); T is the precision of the solve. */")
    L.append("  template <class T, class A> OV_HD static OV_INLINE void lu_solve(A a, "
             "const double* OV_RESTRICT r, double* OV_RESTRICT x, const double* OV_RESTRICT sc, "
             "const double* OV_RESTRICT isc) {")
    L.append("#define OV_SC(i) (sc ? sc[i] : 1.0)")
    L.append("#define OV_ISC(i) (isc ? isc[i] : 1.0)")
    L += _fenced(["    " + ln for ln in s_lines], SCHED_EVERY, nd >= SCHED_MIN_ND)
    L.append("#undef OV_SC")
    L.append("#undef OV_ISC")
    L.append("  }")
    L.append("};")
    return "\n".join(L) + "\n"


def expr_flops(expr) -> int:
    """Binary floating-point operations of an expression as the emitted code
    evaluates it: n-1 per n-term sum or n-factor product (a coefficient of
    -1 is a sign, not an operation), n-1 multiplications for x**n, one per
    division or real power."""
    expr = sp.sympify(expr)
    if expr.is_Atom:
        return 0
    if expr.is_Add:
        return len(expr.args) - 1 + sum(expr_flops(a) for a in expr.args)
    if expr.is_Mul:
        args = [a for a in expr.args if a not in (-1, 1)]
        return max(len(args) - 1, 0) + sum(expr_flops(a) for a in args)
    if expr.is_Pow:
        b, e = expr.as_base_exp()
        if e.is_Integer and int(e) > 0:
            return int(e) - 1 + expr_flops(b)
        return 1 + expr_flops(b)
    return 1 + sum(expr_flops(a) for a in expr.args)


def _line_flops(line: str) -> int:
    rhs = line.split("=", 1)[1]
    return rhs.count("*") + rhs.count("/") + rhs.count(" + ") + rhs.count(" - ")


def flop_counts(sysm: System) -> Dict[str, int]:
    """Static per-call FLOPs of the emitted routines."""
    f_rhs = sum(expr_flops(e) for e in sysm.net.rhs)
    pos = sysm.pos()
    f_k = (4 + sysm.net.nrea) if sysm.net.rates else 0
    src = _jac_source(sysm)
    if src is not None:
        f_jac = sum(expr_flops(src[i, j]) for (i, j) in pos)
    else:
        # difference quotients: ND + 1 right-hand sides, the norm of f, and per
        # column the increment (6) and ND differences times the factor
        nd = sysm.neq - len(frozen_species(sysm))
        f_jac = (nd + 1) * (f_rhs + f_k) + 3 * nd + 4 + nd * (6 + 2 * nd) + nd
    f_lu = sum(_line_flops(l) for l in _lu_factor_lines(sysm))
    f_solve = sum(_line_flops(l) for l in _lu_solve_lines(sysm) if not l.startswith(("T d", "x[")))
    # rates_k of the PRIMORDIAL rate model: 3 mul + 1 div for the floor, one add per rate
    return {"neq": sysm.neq, "nnz": sysm.nnz, "rhs": f_rhs, "jac": f_jac, "lu_factor": f_lu,
            "lu_solve": f_solve, "rates_k": f_k}


def write_variant(sysm: System, outdir: str = GEN_DIR) -> Tuple[str, str]:
    os.makedirs(outdir, exist_ok=True)
    cid = _cid(sysm.tag)
    h = os.path.join(outdir, "net_%s.h" % cid)
    cu = os.path.join(outdir, "net_%s.cuh" % cid)
    text_h, text_cu = emit_c_header(sysm), emit_cuda_header(sysm)
    with open(h, "w") as fh:
        fh.write(text_h)
    with open(cu, "w") as fh:
        fh.write(text_cu)
    import json
    fpath = os.path.join(outdir, "flops.json")
    table = json.load(open(fpath)) if os.path.exists(fpath) else {}
    table[sysm.tag] = flop_counts(sysm)
    with open(fpath, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    write_registry(outdir)
    return h, cu


def write_registry(outdir: str = GEN_DIR) -> str:
    """X-macro list of every emitted variant: OV_NET(cid, "TAG")."""
    tags = []
    for f in sorted(os.listdir(outdir)):
        m = re.match(r"net_(.*)\.cuh$", f)
        if m:
            txt = open(os.path.join(outdir, f)).read()
            t = re.search(r'TAG = "([^"]+)"', txt).group(1)
            tags.append((m.group(1), t))
    path = os.path.join(outdir, "registry.inc")
    with open(path, "w") as fh:
        fh.write("/* Generated by odevec_b200.pre_odevec: every emitted network variant. */\n")
        for cid, t in tags:
            fh.write('OV_NET(%s, "%s")\n' % (cid, t))
    with open(os.path.join(outdir, "includes.inc"), "w") as fh:
        fh.write("/* Generated by odevec_b200.pre_odevec. */\n")
        for cid, _ in tags:
            fh.write('#include "net_%s.cuh"\n' % cid)
    with open(os.path.join(outdir, "includes_c.inc"), "w") as fh:
        fh.write("/* Generated by odevec_b200.pre_odevec. */\n")
        for cid, _ in tags:
            fh.write('#include "net_%s.h"\n' % cid)
    return path


# ---------------------------------------------------------------------- CLI
def parse_args(argv=None):
    p = argparse.ArgumentParser(
        description="Preprocessor for OdeVec on B200: emits straight-line C/CUDA network code.")
    p.add_argument("--example", default="PRIMORDIAL", help="ROBER | OREGO | PRIMORDIAL | KROME")
    p.add_argument("--krome_setupfile", default=None, help="python dump of a KROME network")
    p.add_argument("--LUmethod", type=int, default=1,
                   help="1: symbolic Jacobian + numeric LU; 2: symbolic LU (DENSE); "
                        "3: finite-difference Jacobian + numeric LU (DENSE, no ordering)")
    p.add_argument("--dt_min", default=1e-10, help="default minimal time step")
    p.add_argument("--nvector", type=int, required=True,
                   help="default lockstep group size (1 = per-cell control, 32 = one warp)")
    p.add_argument("--heatcool", type=int, default=0,
                   help="1: the Tgas row (species neq-1 of a KROME layout) follows heating and cooling")
    p.add_argument("--heatcool_header", default=None,
                   help="header in odevec_b200/csrc defining ov_hc_heating, ov_hc_cooling, ov_hc_gamma, "
                        "OV_HC_BOLTZMANN and OV_HC_NMOLS for --heatcool=1")
    p.add_argument("--equilibrium_H", type=int, default=0)
    p.add_argument("--ordering", default="None", help="CMK | INVERT | FF | None")
    p.add_argument("--packaging", default="DENSE", help="DENSE | CSC")
    p.add_argument("--lu_pattern", default="structural", help="structural | symbolic")
    p.add_argument("--name", default=None, help="network name used in the variant tag")
    p.add_argument("--outdir", default=GEN_DIR)
    p.add_argument("--sparsity_structure", default=False)
    return p.parse_args(argv)


def main(argv=None) -> System:
    args = parse_args(argv)
    if args.krome_setupfile is not None:
        args.example = "KROME"
    if args.heatcool and not args.heatcool_header:
        raise SystemExit("# Error: --heatcool=1 needs --heatcool_header=<file> with the heating and "
                         "cooling functions (KROME's heating/cooling are not part of this build)")
    if args.equilibrium_H == 1 and args.packaging != "DENSE":   # pre_odevec.py:455-460
        raise SystemExit("args.equilibrium_H is only allowed with DENSE packaging.")
    if args.equilibrium_H == 1 and args.ordering != "None":
        raise SystemExit("args.equilibrium_H is only allowed without ordering.")
    if args.equilibrium_H == 1 and args.LUmethod != 3:
        raise SystemExit("args.equilibrium_H is currently only usable with LUmethod==3.")
    print("#  Setting up system..")
    print('#  Vector length "nvector":', args.nvector)
    net = networks.load(args.example, args.krome_setupfile)
    if args.name:
        net.name = args.name
    if args.heatcool:
        hdr = os.path.join(os.path.dirname(GEN_DIR), os.path.basename(args.heatcool_header))
        if not os.path.exists(hdr):
            raise SystemExit("# Error: heating/cooling header %s not found (it must be in odevec_b200/csrc)" % hdr)
        networks.enable_heatcool(net, hdr)
    sysm = build_system(net, args.ordering, args.packaging, args.lu_pattern, args.nvector,
                        float(args.dt_min), args.LUmethod)
    n = net.neq
    print("#  Permutation list", np.array(sysm.perm))
    print("#  NNZs in Jacobian: %d | Sparsity: %s" % (sysm.p_nnz, 1 - sysm.p_nnz / (n * n)))
    print("#  NNZs in LU-Matrix: %d | Sparsity: %s" % (sysm.nnz, 1 - sysm.nnz / (n * n)))
    h, cu = write_variant(sysm, args.outdir)
    print("#  Wrote out file: " + h)
    print("#  Wrote out file: " + cu)
    if str(args.sparsity_structure) == "True":
        for i in range(n):
            print("".join("X" if sysm.lu_pat[i, j] else "." for j in range(n)))
    return sysm


if __name__ == "__main__":
    main()
