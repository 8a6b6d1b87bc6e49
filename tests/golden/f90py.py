"""Mechanical translator of a Fortran 95 subset into Python/NumPy.

TEST INFRASTRUCTURE ONLY.  It exists to run the reference's own generated
solver modules (``build/odevec.f90`` and ``build/odevec_commons.f90``, which
``pre_odevec.py`` writes from ``src/odevec.F90`` and
``src/odevec_commons.F90``) where no Fortran compiler is available, so that
their outputs can pin the CPU oracle.  The translation is statement by
statement; nothing of the solver's logic is restated by hand.  Nothing it
produces is committed: only numbers computed by running it.

Semantics reproduced (those of gfortran -O2 on x86-64 without -ffast-math):

* IEEE binary64 ``double precision`` / ``real*8`` and binary32 ``real``
  arithmetic, left-to-right evaluation of ``a*b*c`` and ``a+b+c``, no fused
  multiply-add; a real literal without a ``d`` exponent is single precision
  (``1.3`` is the float nearest 1.3, widened when it meets a double);
  integer division truncates.
* ``x**n`` with an integer constant ``n`` is expanded into multiplications
  along the optimal power tree (the table gfortran's front end uses),
  negative ``n`` as its reciprocal; ``x**c`` with a real constant ``c`` equal
  to -1, 0, 1 or 2 is expanded the same way (the middle end does that
  without -ffast-math), every other real power calls the C library's
  ``pow``; ``x**n`` with an integer variable follows libgcc's ``__powidf2``.
* ``exp``/``log``/``log10``/``pow`` call the C library (Python's ``math``),
  ``sqrt`` is correctly rounded; ``sum(a, dim)`` accumulates in index order.
* Arguments are passed by reference: scalar variables, derived-type
  components and array elements are passed as reference cells, arrays as
  views, so a callee that writes ``order`` writes ``this%order``; array
  dummies take the caller's storage with their own declared bounds.
* ``where``/``elsewhere``, ``spread``, ``any``/``all``, ``maxval``/``minval``
  with ``mask``, ``maxloc``, ``reshape``/``transpose``, array constructors
  with implied do, named ``do`` loops with ``cycle``/``exit`` by name,
  generic interfaces resolved by argument type and rank, optional arguments
  and ``present``, ``save`` variables, ``allocate`` (zero-filled, as fresh
  pages are) and ``stop`` (raised as :class:`FortranStop`).

Execution counters: every procedure entry is counted (:data:`CALLS`), and a
caller may register statement probes (counted when a statement of a given
procedure with a given text executes) and entry hooks.
"""
from __future__ import annotations

import math
import re

import numpy as np

np.seterr(all="ignore")


# ====================================================================== runtime
class FortranStop(Exception):
    pass


class _Cycle(Exception):
    def __init__(self, label):
        super().__init__(label)
        self.label = label


class _Exit(Exception):
    def __init__(self, label):
        super().__init__(label)
        self.label = label


class Ref:
    """A scalar variable: what a Fortran dummy argument refers to."""
    __slots__ = ("v",)

    def __init__(self, v):
        self.v = v


class FieldRef:
    """A scalar component of a derived-type object passed by reference."""
    __slots__ = ("o", "n")

    def __init__(self, o, n):
        self.o = o
        self.n = n

    @property
    def v(self):
        return getattr(self.o, self.n)

    @v.setter
    def v(self, x):
        setattr(self.o, self.n, x)


class ElemRef:
    """An array element passed by reference."""
    __slots__ = ("a", "i")

    def __init__(self, a, i):
        self.a = a
        self.i = i

    @property
    def v(self):
        return self.a[self.i]

    @v.setter
    def v(self, x):
        self.a[self.i] = x


class FArray:
    """A Fortran array: NumPy storage (column-major) with lower bounds.
    Subscripts are Fortran subscripts; a slice(lo, hi, step) is the
    inclusive section lo:hi:step."""
    __slots__ = ("a", "lb")

    def __init__(self, a, lb=None):
        self.a = a
        self.lb = tuple(lb) if lb is not None else (1,) * a.ndim

    def _ix(self, idx):
        out = []
        for s, lb in zip(idx, self.lb):
            if isinstance(s, slice):
                st = 1 if s.step is None else s.step
                if st < 0:
                    raise NotImplementedError("negative section stride")
                lo = None if s.start is None else s.start - lb
                hi = None if s.stop is None else s.stop - lb + 1
                out.append(slice(lo, hi, st))
            else:
                out.append(int(s) - lb)
        return tuple(out)

    def __getitem__(self, idx):
        return self.a[self._ix(idx)]

    def __setitem__(self, idx, val):
        self.a[self._ix(idx)] = val


_DT = {"r8": np.float64, "r4": np.float32, "i": np.int64, "l": np.bool_}
FILL = {"value": 0.0}


def _alloc(t, dims):
    shape = [max(int(hi) - int(lo) + 1, 0) for lo, hi in dims]
    if t in ("r8", "r4"):
        a = np.full(shape, FILL["value"], dtype=_DT[t], order="F")
    else:
        a = np.zeros(shape, dtype=_DT[t], order="F")
    return FArray(a, [int(lo) for lo, _ in dims])


def _dummy(x, dims):
    """An explicit-shape array dummy: the actual's storage with the dummy's
    bounds (sequence association when the shapes differ)."""
    if x is None:
        return None
    a = x.a if isinstance(x, FArray) else np.asarray(x)
    if dims is None:
        return FArray(a)
    shape = tuple(max(int(hi) - int(lo) + 1, 0) for lo, hi in dims)
    if a.shape != shape:
        flat = a.reshape(-1, order="F")
        n = int(np.prod(shape))
        if not np.shares_memory(flat, a) and a.size:
            raise ValueError("sequence association needs contiguous storage")
        a = flat[:n].reshape(shape, order="F")
    return FArray(a, [int(lo) for lo, _ in dims])


def _sect(view):
    return FArray(np.asarray(view))


def _val(v):
    return v.a if isinstance(v, FArray) else v


def _idiv(a, b):
    if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        a = np.asarray(a)
        b = np.asarray(b)
        q = np.abs(a) // np.abs(b)
        return np.where((a < 0) != (b < 0), -q, q)
    q = abs(a) // abs(b)
    return -q if (a < 0) != (b < 0) else q


def _imod(a, b):
    return a - _idiv(a, b) * b


# optimal power tree (Knuth; the table gfortran's front end and GCC use):
# x^n = x^(n - T[n]) * x^T[n]
_POWI_TABLE = [0, 1, 1, 2, 2, 3, 3, 4, 4, 6, 5, 6, 6, 10, 7, 9, 8, 16, 9, 16, 10, 12, 11, 13,
               12, 17, 13, 18, 14, 24, 15, 26]


def _powi(x, n):
    if n == 0:
        return (np.ones_like(x) if isinstance(x, np.ndarray) else type(x)(1))
    neg = n < 0
    n = -n if neg else n
    cache = {1: x}

    def rec(m):
        if m in cache:
            return cache[m]
        if m >= len(_POWI_TABLE):
            # binary method beyond the table (not reached by the modules run here)
            v = rec(m >> 1)
            v = v * v
            if m & 1:
                v = v * x
        else:
            v = rec(m - _POWI_TABLE[m]) * rec(_POWI_TABLE[m])
        cache[m] = v
        return v
    r = rec(n)
    if neg:
        one = np.ones_like(r) if isinstance(r, np.ndarray) else type(r)(1)
        r = one / r
    return r


def _powidf2(x, m):
    """libgcc __powidf2: real ** integer variable."""
    n = -m if m < 0 else m
    y = x if n % 2 else type(x)(1)
    while True:
        n >>= 1
        if not n:
            break
        x = x * x
        if n % 2:
            y = y * x
    return (type(y)(1) / y) if m < 0 else y


def _map1(f, x, t):
    if isinstance(x, np.ndarray):
        flat = [f(float(v)) for v in x.ravel(order="K")]
        return np.array(flat, dtype=_DT[t]).reshape(x.shape)
    return _DT[t](f(float(x)))


def _libm_pow(a, b):
    try:
        return math.pow(a, b)
    except (OverflowError, ValueError):
        if a < 0 and not float(b).is_integer():
            return math.nan
        if a == 0:
            return math.inf
        return math.inf if abs(a) > 1 else 0.0


def _fpow(x, y, t):
    if isinstance(x, np.ndarray) or isinstance(y, np.ndarray):
        xb, yb = np.broadcast_arrays(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64))
        out = np.array([_libm_pow(float(a), float(b)) for a, b in zip(xb.ravel(), yb.ravel())],
                       dtype=np.float64).reshape(xb.shape)
        return out.astype(_DT[t])
    return _DT[t](_libm_pow(float(x), float(y)))


def _libm(name, x, t):
    f = {"exp": math.exp, "log": math.log, "log10": math.log10}[name]

    def g(v):
        try:
            return f(v)
        except OverflowError:
            return math.inf
        except ValueError:
            if name != "exp" and v == 0:
                return -math.inf
            return math.nan
    return _map1(g, x, t)


def _fmax(*a):
    r = a[0]
    for b in a[1:]:
        if isinstance(r, np.ndarray) or isinstance(b, np.ndarray):
            r = np.where(b > r, b, r)
        else:
            r = b if b > r else r
    return r


def _fmin(*a):
    r = a[0]
    for b in a[1:]:
        if isinstance(r, np.ndarray) or isinstance(b, np.ndarray):
            r = np.where(b < r, b, r)
        else:
            r = b if b < r else r
    return r


def _seqsum(x, axis):
    x = np.moveaxis(np.asarray(x), axis, 0)
    acc = np.zeros(x.shape[1:], dtype=x.dtype)
    for j in range(x.shape[0]):
        acc = acc + x[j]
    return acc


def _sum(x, dim=None, mask=None):
    x = np.asarray(x)
    if mask is not None:
        x = np.where(np.broadcast_to(mask, x.shape), x, x.dtype.type(0))
    if dim is None:
        acc = x.dtype.type(0)
        for v in x.ravel(order="F"):
            acc = acc + v
        return acc
    return _seqsum(x, int(dim) - 1)


def _maxval(x, dim=None, mask=None, minimum=False):
    x = np.asarray(x)
    if dim is not None:
        raise NotImplementedError("maxval with dim")
    m = np.ones(x.shape, bool) if mask is None else np.broadcast_to(np.asarray(mask), x.shape)
    sel = x[m]
    if sel.size == 0:
        fi = np.finfo(x.dtype) if x.dtype.kind == "f" else np.iinfo(x.dtype)
        return x.dtype.type(fi.max if minimum else -fi.max)
    # gfortran: NaNs are skipped unless every element is NaN
    ok = sel[~np.isnan(sel)] if x.dtype.kind == "f" else sel
    if ok.size == 0:
        return x.dtype.type(np.nan)
    return ok.min() if minimum else ok.max()


def _maxloc(x, dim=None):
    x = np.asarray(x)
    i = int(np.argmax(x)) + 1
    return i if dim is not None else np.array([i], dtype=np.int64)


def _spread(s, dim, n):
    s = np.asarray(s)
    return np.repeat(np.expand_dims(s, int(dim) - 1), int(n), axis=int(dim) - 1)


def _ctor(items, t):
    parts = []
    for it in items:
        a = np.atleast_1d(np.asarray(_val(it)))
        parts.append(a.ravel(order="F"))
    out = np.concatenate(parts) if parts else np.zeros(0)
    return out.astype(_DT[t])


def _nint(x):
    if isinstance(x, np.ndarray):
        return np.where(x >= 0, np.floor(x + 0.5), -np.floor(-x + 0.5)).astype(np.int64)
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def _where_set(view, rhs, mask):
    r = np.broadcast_to(np.asarray(rhs), view.shape)
    view[mask] = r[mask]


PRINTED = []
CALLS = {}
HITS = {}
HOOKS = {}


def _print(*items):
    PRINTED.append(" ".join(str(_val(i)) for i in items))


def _enter(name, frame):
    CALLS[name] = CALLS.get(name, 0) + 1
    h = HOOKS.get(name)
    if h is not None:
        h(frame)


def reset_counters():
    CALLS.clear()
    HITS.clear()


# ==================================================================== front end
def preprocess(text, defines=()):
    """The cpp directives the generated modules use (#ifdef/#ifndef/#else/
    #endif), comments removed, continuation lines joined, lower case outside
    string literals.  Returns a list of (statement, original line number)."""
    out_lines = []
    stack = []
    for ln, line in enumerate(text.split("\n"), 1):
        s = line.strip()
        if s.startswith("#"):
            m = re.match(r"#\s*(ifdef|ifndef|else|endif)\s*(\w*)", s)
            if not m:
                raise ValueError("unsupported directive at %d: %s" % (ln, s))
            d, name = m.groups()
            if d == "ifdef":
                stack.append(name in defines)
            elif d == "ifndef":
                stack.append(name not in defines)
            elif d == "else":
                stack[-1] = not stack[-1]
            else:
                stack.pop()
            out_lines.append(("", ln))
            continue
        if stack and not all(stack):
            out_lines.append(("", ln))
            continue
        out_lines.append((_strip_comment(line), ln))
    stmts = []
    buf, start = "", None
    for s, ln in out_lines:
        t = s.strip()
        if not t and not buf:
            continue
        if buf and t.startswith("&"):
            t = t[1:]
        if start is None:
            start = ln
        if t.endswith("&"):
            buf += t[:-1]
            continue
        buf += t
        for part in _split_semicolons(buf):
            if part.strip():
                stmts.append((_lower(part.strip()), start))
        buf, start = "", None
    return stmts


def _strip_comment(line):
    q = None
    for i, ch in enumerate(line):
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "!":
            return line[:i]
    return line


def _split_semicolons(s):
    parts, q, cur = [], None, ""
    for ch in s:
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == ";":
            parts.append(cur)
            cur = ""
            continue
        cur += ch
    parts.append(cur)
    return parts


def _lower(s):
    out, q = [], None
    for ch in s:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        else:
            out.append(ch.lower())
    return "".join(out)


_DOTOPS = ("eq", "ne", "lt", "le", "gt", "ge", "and", "or", "not", "eqv", "neqv", "true", "false")
_TOKRE = re.compile(r"""
  (?P<ws>\s+)
 |(?P<str>'[^']*'|"[^"]*")
 |(?P<dot>\.(?:eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv|true|false)\.)
 |(?P<num>(?:\d+\.\d*|\.\d+)(?:[ed][+-]?\d+)?(?:_\w+)?|\d+[ed][+-]?\d+(?:_\w+)?|\d+(?:_\w+)?)
 |(?P<name>[a-z_][a-z0-9_]*)
 |(?P<op>\*\*|//|==|/=|<=|>=|\(/|/\)|[-+*/<>=(),:%])
""", re.X)


def tokenize(s):
    toks = []
    i = 0
    while i < len(s):
        m = _TOKRE.match(s, i)
        if not m:
            raise SyntaxError("cannot tokenize at %r" % s[i:])
        kind = m.lastgroup
        text = m.group(kind)
        if kind == "num" and "." in text and re.match(r"\d+\.", text):
            # '1.eq.x': the dot belongs to an operator
            rest = s[m.start() + text.index(".") + 1:]
            dm = re.match(r"(%s)\." % "|".join(_DOTOPS), rest)
            if dm:
                text = text[:text.index(".")]
                toks.append(("num", text))
                i = m.start() + len(text)
                continue
        i = m.end()
        if kind == "ws":
            continue
        toks.append((kind, text))
    return _fix_ctor_tokens(toks)


def _fix_ctor_tokens(toks):
    # '(/' only opens a constructor where an operand may start; '/)' closes
    # one only inside a constructor.  Elsewhere split them back into '(' '/'
    # and '/' ')'.
    out = []
    depth = 0
    for k, t in toks:
        if k == "op" and t == "(/":
            prev = out[-1] if out else None
            operand_start = prev is None or (prev[0] in ("op", "dot") and prev[1] not in (")", "/)"))
            if operand_start:
                depth += 1
                out.append((k, t))
            else:
                out.append(("op", "("))
                out.append(("op", "/"))
            continue
        if k == "op" and t == "/)":
            if depth:
                depth -= 1
                out.append((k, t))
            else:
                out.append(("op", "/"))
                out.append(("op", ")"))
            continue
        out.append((k, t))
    return out


# AST: tuples
#   ('num', text)  ('str', text)  ('bool', True|False)  ('paren', x)
#   ('des', [(name, args|None), ...])          designator / call
#   ('bin', op, l, r)  ('un', op, x)  ('ctor', items)  ('ido', expr, var, lo, hi, step)
#   ('slice', lo, hi, step)  ('kw', name, expr)
class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, text=None):
        tok = self.peek()
        if text is not None and tok[1] != text:
            raise SyntaxError("expected %r, got %r in %r" % (text, tok, self.t))
        self.i += 1
        return tok

    def at(self, text):
        return self.peek()[1] == text

    def done(self):
        return self.i >= len(self.t)

    def expr(self):
        x = self.or_()
        while self.peek()[1] in (".eqv.", ".neqv."):
            op = self.take()[1]
            x = ("bin", op, x, self.or_())
        return x

    def or_(self):
        x = self.and_()
        while self.at(".or."):
            self.take()
            x = ("bin", ".or.", x, self.and_())
        return x

    def and_(self):
        x = self.not_()
        while self.at(".and."):
            self.take()
            x = ("bin", ".and.", x, self.not_())
        return x

    def not_(self):
        if self.at(".not."):
            self.take()
            return ("un", ".not.", self.not_())
        return self.rel()

    _REL = {"==": "==", ".eq.": "==", "/=": "!=", ".ne.": "!=", "<": "<", ".lt.": "<",
            "<=": "<=", ".le.": "<=", ">": ">", ".gt.": ">", ">=": ">=", ".ge.": ">="}

    def rel(self):
        x = self.add()
        if self.peek()[1] in self._REL:
            op = self._REL[self.take()[1]]
            x = ("bin", op, x, self.add())
        return x

    def add(self):
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            x = self.mul()
            x = ("un", op, x)
        else:
            x = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            x = ("bin", op, x, self.mul())
        return x

    def mul(self):
        x = self.pow_()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            x = ("bin", op, x, self.pow_())
        return x

    def pow_(self):
        x = self.primary()
        if self.at("**"):
            self.take()
            if self.peek()[1] in ("+", "-"):   # x**-n (an extension gfortran accepts)
                op = self.take()[1]
                return ("bin", "**", x, ("un", op, self.pow_()))
            return ("bin", "**", x, self.pow_())
        return x

    def primary(self):
        k, t = self.peek()
        if k == "num":
            self.take()
            return ("num", t)
        if k == "str":
            self.take()
            return ("str", t[1:-1])
        if t in (".true.", ".false."):
            self.take()
            return ("bool", t == ".true.")
        if t == "(/":
            self.take()
            items = []
            if not self.at("/)"):
                items.append(self.ctor_item())
                while self.at(","):
                    self.take()
                    items.append(self.ctor_item())
            self.take("/)")
            return ("ctor", items)
        if t == "(":
            self.take()
            x = self.expr()
            self.take(")")
            return ("paren", x)
        if k == "name":
            return self.designator()
        raise SyntaxError("unexpected %r in %r" % (t, self.t))

    def ctor_item(self):
        if self.at("("):
            # implied do?  '(' expr ',' name '=' ...
            depth, j = 0, self.i
            while j < len(self.t):
                tt = self.t[j][1]
                if tt in ("(", "(/"):
                    depth += 1
                elif tt in (")", "/)"):
                    depth -= 1
                    if depth == 0:
                        break
                elif depth == 1 and tt == "," and j + 2 < len(self.t) and \
                        self.t[j + 1][0] == "name" and self.t[j + 2][1] == "=":
                    self.take("(")
                    body = self.expr()
                    self.take(",")
                    var = self.take()[1]
                    self.take("=")
                    lo = self.expr()
                    self.take(",")
                    hi = self.expr()
                    step = None
                    if self.at(","):
                        self.take()
                        step = self.expr()
                    self.take(")")
                    return ("ido", body, var, lo, hi, step)
                j += 1
        return self.expr()

    def designator(self):
        parts = []
        while True:
            name = self.take()[1]
            args = None
            if self.at("("):
                self.take()
                args = []
                if not self.at(")"):
                    args.append(self.arg())
                    while self.at(","):
                        self.take()
                        args.append(self.arg())
                self.take(")")
            parts.append((name, args))
            if self.at("%"):
                self.take()
                continue
            return ("des", parts)

    def arg(self):
        if self.peek()[0] == "name" and self.peek(1)[1] == "=":
            name = self.take()[1]
            self.take("=")
            return ("kw", name, self.expr())
        if self.at(":"):
            return self.section(None)
        x = self.expr()
        if self.at(":"):
            return self.section(x)
        return x

    def section(self, lo):
        self.take(":")
        hi = None
        step = None
        if not (self.at(",") or self.at(")") or self.at(":")):
            hi = self.expr()
        if self.at(":"):
            self.take()
            step = self.expr()
        return ("slice", lo, hi, step)


def parse_expr(s):
    p = Parser(tokenize(s))
    x = p.expr()
    if not p.done():
        raise SyntaxError("trailing tokens in %r: %r" % (s, p.t[p.i:]))
    return x


def split_top(s, sep=","):
    parts, depth, q, cur = [], 0, None, ""
    for ch in s:
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == sep and depth == 0:
            parts.append(cur)
            cur = ""
            continue
        cur += ch
    parts.append(cur)
    return [p.strip() for p in parts]


def match_paren(s, i):
    """index of the ')' matching the '(' at s[i]"""
    depth, q = 0, None
    for j in range(i, len(s)):
        ch = s[j]
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                return j
    raise SyntaxError("unbalanced parentheses in %r" % s)


def top_assign(s):
    """position of the assignment '=' at parenthesis depth 0, or -1"""
    depth, q = 0, None
    for j, ch in enumerate(s):
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0:
            prev = s[j - 1] if j else ""
            nxt = s[j + 1] if j + 1 < len(s) else ""
            if prev not in "=/<>" and nxt != "=":
                return j
    return -1


# ------------------------------------------------------------------ declarations
class Var:
    def __init__(self, name, t, dims=None, attrs=(), init=None, tname=None):
        self.name = name
        self.t = t            # 'r8' 'r4' 'i' 'l' 'c' 'd' 'proc'
        self.tname = tname    # derived type name
        self.dims = dims      # list of (lo_ast|None, hi_ast|None) or None
        self.attrs = set(attrs)
        self.init = init

    @property
    def rank(self):
        return len(self.dims) if self.dims else 0


_TYPESPEC = re.compile(r"^(double\s*precision|real\s*\*\s*8|real\s*\(\s*(?:kind\s*=\s*)?8\s*\)|real|"
                       r"integer(?:\s*\*\s*\d+)?|logical|character(?:\s*\([^)]*\))?|"
                       r"type\s*\(\s*\w+\s*\))(?![\w])")


def parse_typespec(s):
    m = _TYPESPEC.match(s)
    if not m:
        return None
    ts = re.sub(r"\s+", "", m.group(1))
    if ts.startswith("double") or ts in ("real*8", "real(8)", "real(kind=8)"):
        t, tn = "r8", None
    elif ts == "real":
        t, tn = "r4", None
    elif ts.startswith("integer"):
        t, tn = "i", None
    elif ts == "logical":
        t, tn = "l", None
    elif ts.startswith("character"):
        t, tn = "c", None
    else:
        t, tn = "d", re.match(r"type\((\w+)\)", ts).group(1)
    return t, tn, s[m.end():]


def parse_dims(s):
    dims = []
    for d in split_top(s):
        if ":" in d:
            lo, hi = d.split(":", 1)
            dims.append((parse_expr(lo) if lo.strip() else None, parse_expr(hi) if hi.strip() else None))
        else:
            dims.append((("num", "1"), parse_expr(d)))
    return dims


def parse_decl(s):
    """type-spec [, attr]... [::] entity-list -> [Var]"""
    r = parse_typespec(s)
    if r is None:
        return None
    t, tn, rest = r
    rest = rest.strip()
    attrs, dims = [], None
    if "::" in rest:
        head, ents = rest.split("::", 1)
        for a in split_top(head.lstrip(",")):
            a = a.strip()
            if not a:
                continue
            m = re.match(r"dimension\s*\((.*)\)$", a)
            if m:
                dims = parse_dims(m.group(1))
                continue
            m = re.match(r"intent\s*\(\s*(\w+)\s*\)$", a)
            if m:
                attrs.append("intent_" + m.group(1))
                continue
            attrs.append(a)
    else:
        ents = rest
    out = []
    for e in split_top(ents):
        if not e:
            continue
        init = None
        j = top_assign(e)
        if j >= 0:
            init = parse_expr(e[j + 1:])
            e = e[:j].strip()
        edims = dims
        m = re.match(r"(\w+)\s*\((.*)\)$", e)
        if m:
            e = m.group(1)
            edims = parse_dims(m.group(2))
        out.append(Var(e, t, edims, attrs, init, tn))
    return out


# ------------------------------------------------------------------- structure
class Proc:
    def __init__(self, name, kind, params, result=None):
        self.name = name
        self.kind = kind          # 'subroutine' | 'function'
        self.params = params
        self.result = result or name
        self.vars = {}
        self.body = []            # list of (stmt, line)


class Module:
    def __init__(self):
        self.types = {}           # name -> {comp: Var}
        self.type_order = {}
        self.generics = {}        # name -> [specific]
        self.procs = {}


def structure(stmts, mod=None):
    """Splits preprocessed statements into derived types, interfaces and
    module procedures."""
    mod = mod or Module()
    i = 0
    n = len(stmts)
    while i < n:
        s, ln = stmts[i]
        m = re.match(r"^type\s*(?:,\s*\w+\s*)?(?:::)?\s*(\w+)$", s)
        if m and not s.startswith("type("):
            name = m.group(1)
            comps = {}
            order = []
            i += 1
            while not re.match(r"^end\s*type", stmts[i][0]):
                for v in parse_decl(stmts[i][0]) or []:
                    comps[v.name] = v
                    order.append(v.name)
                i += 1
            mod.types[name] = comps
            mod.type_order[name] = order
            i += 1
            continue
        m = re.match(r"^interface\s+(\w+)$", s)
        if m:
            g = m.group(1)
            specs = []
            i += 1
            while not re.match(r"^end\s*interface", stmts[i][0]):
                mm = re.match(r"^module\s+procedure\s+(.*)$", stmts[i][0])
                if mm:
                    specs += [x.strip() for x in mm.group(1).split(",")]
                i += 1
            mod.generics[g] = specs
            i += 1
            continue
        m = re.match(r"^(?:(?:pure|elemental|recursive)\s+)*(subroutine|function)\s+(\w+)\s*(?:\((.*?)\))?"
                     r"\s*(?:result\s*\(\s*(\w+)\s*\))?$", s)
        if m:
            kind, name, params, res = m.groups()
            params = [p.strip() for p in params.split(",")] if params and params.strip() else []
            p = Proc(name, kind, params, res)
            i += 1
            while True:
                t, l2 = stmts[i]
                if re.match(r"^end\s*(subroutine|function)\b", t) or t == "end":
                    break
                p.body.append((t, l2))
                i += 1
            i += 1
            _split_spec(p)
            mod.procs[name] = p
            continue
        i += 1
    return mod


_ATTR_STMT = re.compile(r"^(intent\s*\(\s*(\w+)\s*\)|optional|external|save|allocatable|pointer|"
                        r"value|dimension)\s*(?:::)?\s*(.*)$")


def _split_spec(p):
    body = []
    spec_done = False
    for s, ln in p.body:
        if not spec_done:
            if s.startswith("implicit") or s.startswith("use "):
                continue
            d = parse_decl(s)
            if d is not None:
                for v in d:
                    if v.name in p.vars:
                        old = p.vars[v.name]
                        old.t, old.tname = v.t, v.tname
                        if v.dims:
                            old.dims = v.dims
                        old.attrs |= v.attrs
                        if v.init is not None:
                            old.init = v.init
                    else:
                        p.vars[v.name] = v
                continue
            m = _ATTR_STMT.match(s)
            if m:
                attr = m.group(1)
                for nm in split_top(m.group(3)):
                    if not nm:
                        continue
                    dims = None
                    mm = re.match(r"(\w+)\s*\((.*)\)$", nm)
                    if mm:
                        nm, dims = mm.group(1), parse_dims(mm.group(2))
                    v = p.vars.setdefault(nm, Var(nm, None))
                    if attr.startswith("intent"):
                        v.attrs.add("intent_" + m.group(2))
                    elif attr == "external":
                        v.attrs.add("external")
                        v.t = v.t or "proc"
                    elif attr == "dimension":
                        v.dims = dims
                    else:
                        v.attrs.add(attr)
                continue
            spec_done = True
        body.append((s, ln))
    p.body = body
    for nm, v in p.vars.items():
        if v.t is None:
            raise ValueError("%s: no type for %s" % (p.name, nm))


# ===================================================================== back end
def _promote(a, b):
    if "r8" in (a, b):
        return "r8"
    if "r4" in (a, b):
        return "r4"
    if a == "i" and b == "i":
        return "i"
    return a if a == b else "r8"


def _conv_code(code, frm, to, rank):
    if frm == to or to is None or frm in ("c", "d", "proc") or to in ("c", "d", "proc"):
        return code
    if rank:
        return "(%s).astype(%s)" % (code, {"r8": "np.float64", "r4": "np.float32", "i": "np.int64",
                                           "l": "np.bool_"}[to])
    if to == "r8":
        return "np.float64(%s)" % code
    if to == "r4":
        return "np.float32(%s)" % code
    if to == "i":
        return "int(%s)" % code
    if to == "l":
        return "bool(%s)" % code
    return code


def _f32_literal(text):
    """The binary32 value nearest the decimal literal (correct rounding)."""
    from fractions import Fraction
    exact = Fraction(text)
    c = np.float32(float(text))
    best = c
    for cand in (np.nextafter(c, np.float32(-np.inf)), c, np.nextafter(c, np.float32(np.inf))):
        if abs(Fraction(float(cand)) - exact) < abs(Fraction(float(best)) - exact):
            best = cand
    return best


class Emitter:
    def __init__(self, mod, probes=None):
        self.mod = mod
        self.consts = {}
        self.probes = probes or {}
        self.saves = []

    # ------------------------------------------------------------ constants
    def const(self, text):
        t = text.lower()
        kind = None
        if "_" in t:
            t, kind = t.split("_", 1)
        if re.fullmatch(r"\d+", t):
            return t, "i"
        if "d" in t or kind == "8":
            v = np.float64(float(t.replace("d", "e")))
            typ = "r8"
        else:
            v = _f32_literal(t)
            typ = "r4"
        key = (typ, float(v).hex())
        if key not in self.consts:
            self.consts[key] = "_K%d" % len(self.consts)
        return self.consts[key], typ

    def const_value(self, node):
        """numeric value of a literal (or a signed one), else None"""
        if node is None:
            return None
        if node[0] == "num":
            code, t = self.const(node[1])
            if t == "i":
                return int(code), t
            for (typ, hx), nm in self.consts.items():
                if nm == code:
                    return float.fromhex(hx), t
        if node[0] == "un" and node[1] in "+-":
            r = self.const_value(node[2])
            if r is not None:
                return (-r[0] if node[1] == "-" else r[0]), r[1]
        if node[0] == "paren":
            return self.const_value(node[1])
        return None

    def var(self, p, name):
        if p is not None and name in p.vars:
            return p.vars[name]
        return None

    # ------------------------------------------------------------ expressions
    def ex(self, p, node):
        """-> (code, type, rank)"""
        k = node[0]
        if k == "num":
            code, t = self.const(node[1])
            return code, t, 0
        if k == "str":
            return repr(node[1]), "c", 0
        if k == "bool":
            return ("True" if node[1] else "False"), "l", 0
        if k == "paren":
            c, t, r = self.ex(p, node[1])
            return "(%s)" % c, t, r
        if k == "un":
            c, t, r = self.ex(p, node[2])
            if node[1] == ".not.":
                return ("np.logical_not(%s)" % c if r else "(not %s)" % c), "l", r
            return ("(-%s)" % c if node[1] == "-" else c), t, r
        if k == "bin":
            return self.binop(p, node)
        if k == "ctor":
            items = []
            ts = []
            for it in node[1]:
                if it[0] == "ido":
                    c, t = self.ido(p, it)
                else:
                    c, t, _ = self.ex(p, it)
                items.append(c)
                ts.append(t)
            t = ts[0]
            for u in ts[1:]:
                t = _promote(t, u)
            return "_ctor([%s], %r)" % (", ".join(items), t), t, 1
        if k == "des":
            return self.des_value(p, node)
        raise SyntaxError("cannot emit %r" % (node,))

    def ido(self, p, node):
        _, body, var, lo, hi, step = node
        # the implied-do variable is a statement entity: a Python name of its own
        inner = "_ido_" + var
        saved = p.vars.get(var)
        p.vars[var] = Var(var, "i", attrs=("ido",))
        c, t, _ = self.ex(p, body)
        if saved is not None:
            p.vars[var] = saved
        else:
            del p.vars[var]
        lc = self.ex(p, lo)[0]
        hc = self.ex(p, hi)[0]
        sc = self.ex(p, step)[0] if step is not None else "1"
        return ("[%s for %s in range(%s, (%s) + (1 if (%s) > 0 else -1), %s)]"
                % (c, inner, lc, hc, sc, sc)), t

    def binop(self, p, node):
        _, op, l, r = node
        if op == "**":
            return self.power(p, l, r)
        lc, lt, lr = self.ex(p, l)
        rc, rt, rr = self.ex(p, r)
        rank = max(lr, rr)
        if op in (".and.", ".or.", ".eqv.", ".neqv."):
            if rank:
                f = {".and.": "np.logical_and", ".or.": "np.logical_or", ".eqv.": "np.equal",
                     ".neqv.": "np.not_equal"}[op]
                return "%s(%s, %s)" % (f, lc, rc), "l", rank
            pop = {".and.": "and", ".or.": "or", ".eqv.": "==", ".neqv.": "!="}[op]
            return "(%s %s %s)" % (lc, pop, rc), "l", 0
        if lt == "c" or rt == "c":
            return "(%s %s %s)" % (lc, op, rc), "l", rank
        t = _promote(lt, rt)
        lc = _conv_code(lc, lt, t, lr)
        rc = _conv_code(rc, rt, t, rr)
        if op in ("==", "!=", "<", "<=", ">", ">="):
            return "(%s %s %s)" % (lc, op, rc), "l", rank
        if op == "/" and t == "i":
            return "_idiv(%s, %s)" % (lc, rc), "i", rank
        return "(%s %s %s)" % (lc, op, rc), t, rank

    def power(self, p, l, r):
        lc, lt, lr = self.ex(p, l)
        cv = self.const_value(r)
        if lt == "i":
            rc, rt, rr = self.ex(p, r)
            if rt == "i":
                return "(%s ** %s)" % (lc, rc), "i", max(lr, rr)
            lc = _conv_code(lc, "i", rt, lr)
            lt = rt
        if cv is not None and cv[1] == "i":
            return "_powi(%s, %d)" % (lc, cv[0]), lt, lr
        rc, rt, rr = self.ex(p, r)
        if rt == "i":
            return "_powidf2(%s, %s)" % (lc, rc), lt, lr
        t = _promote(lt, rt)
        if cv is not None and float(cv[0]).is_integer() and -1 <= cv[0] <= 2:
            return "_powi(%s, %d)" % (_conv_code(lc, lt, t, lr), int(cv[0])), t, lr
        return ("_fpow(%s, %s, %r)" % (_conv_code(lc, lt, t, lr), _conv_code(rc, rt, t, rr), t), t,
                max(lr, rr))

    # designators -----------------------------------------------------------
    def resolve(self, p, node):
        """-> dict(cat=..., code=..., t, tname, rank) or None (not a variable)"""
        parts = node[1]
        name, args = parts[0]
        v = self.var(p, name)
        if v is None:
            return None
        if "ido" in v.attrs and len(parts) == 1 and args is None:
            return {"cat": "ido", "code": "_ido_" + name, "t": "i", "rank": 0}
        if v.t == "proc" or "external" in v.attrs:
            return {"cat": "proc", "code": "v_" + name, "t": "proc", "rank": 0}
        return self._walk(p, "v_" + name, v, args, parts[1:], top=True)

    def _walk(self, p, base, v, args, rest, top):
        if v.dims:
            if args is None:
                info = {"cat": "array", "code": base, "t": v.t, "tname": v.tname, "rank": v.rank}
            else:
                idx, rank = self.subscripts(p, args)
                if rank == 0:
                    info = {"cat": "elem", "code": base, "idx": idx, "t": v.t, "tname": v.tname, "rank": 0}
                else:
                    info = {"cat": "section", "code": base, "idx": idx, "t": v.t, "tname": v.tname,
                            "rank": rank}
        elif v.t == "d":
            info = {"cat": "derived", "code": base, "t": "d", "tname": v.tname, "rank": 0}
        else:
            info = {"cat": "scalar" if top else "field", "code": base, "t": v.t, "rank": 0}
        if not rest:
            return info
        if info["cat"] != "derived":
            raise NotImplementedError("component of an array of derived type")
        comps = self.mod.types[v.tname]
        cname, cargs = rest[0]
        return self._walk(p, "%s.%s" % (base, cname), comps[cname], cargs, rest[1:], top=False)

    def subscripts(self, p, args):
        out = []
        rank = 0
        for a in args:
            if a[0] == "slice":
                lo = self.ex(p, a[1])[0] if a[1] is not None else "None"
                hi = self.ex(p, a[2])[0] if a[2] is not None else "None"
                st = self.ex(p, a[3])[0] if a[3] is not None else "None"
                out.append("slice(%s, %s, %s)" % (lo, hi, st))
                rank += 1
            else:
                c, t, r = self.ex(p, a)
                if r:
                    raise NotImplementedError("vector subscript")
                out.append(c)
        return "(%s,)" % ", ".join(out), rank

    def des_value(self, p, node):
        info = self.resolve(p, node)
        if info is None:
            return self.call_value(p, node)
        c = info["cat"]
        if c == "ido":
            return info["code"], "i", 0
        if c == "scalar":
            return info["code"] + ".v", info["t"], 0
        if c == "field":
            return info["code"], info["t"], 0
        if c == "array":
            return info["code"] + ".a", info["t"], info["rank"]
        if c in ("elem", "section"):
            return "%s[%s]" % (info["code"], info["idx"]), info["t"], info["rank"]
        if c == "derived":
            return info["code"], "d", 0
        if c == "proc":
            return info["code"], "proc", 0
        raise AssertionError(c)

    def des_ref(self, p, node):
        """code passing the actual argument `node` by reference:
        (code, type, rank, derived type name)"""
        if node[0] == "des":
            info = self.resolve(p, node)
            if info is None:
                name = node[1][0][0]
                if len(node[1]) == 1 and node[1][0][1] is None and name in self.mod.procs:
                    return "p_" + name, "proc", 0, None
                c, t, r = self.call_value(p, node)
                return ("_sect(%s)" % c if r else "Ref(%s)" % c), t, r, None
            c = info["cat"]
            if c == "scalar":
                return info["code"], info["t"], 0, None
            if c == "field":
                obj, attr = info["code"].rsplit(".", 1)
                return "FieldRef(%s, %r)" % (obj, attr), info["t"], 0, None
            if c == "elem":
                return "ElemRef(%s, %s)" % (info["code"], info["idx"]), info["t"], 0, None
            if c == "array":
                return info["code"], info["t"], info["rank"], None
            if c == "section":
                return "_sect(%s[%s])" % (info["code"], info["idx"]), info["t"], info["rank"], None
            if c == "derived":
                return info["code"], "d", 0, info["tname"]
            if c == "proc":
                return info["code"], "proc", 0, None
            if c == "ido":
                return "Ref(%s)" % info["code"], "i", 0, None
        cc, t, r = self.ex(p, node)
        return ("_sect(%s)" % cc if r else "Ref(%s)" % cc), t, r, None

    # calls -------------------------------------------------------------------
    def pick_specific(self, p, gname, args):
        acts = [self.des_ref(p, a) for a in args if a[0] != "kw"]
        for sname in self.mod.generics[gname]:
            sp = self.mod.procs[sname]
            if len(acts) > len(sp.params):
                continue
            ok = True
            for (code, t, r, tn), pname in zip(acts, sp.params):
                pv = sp.vars[pname]
                if pv.t == "d":
                    ok &= t == "d" and tn == pv.tname
                elif pv.t == "proc" or "external" in pv.attrs:
                    ok &= t == "proc"
                else:
                    ok &= t != "d" and r == pv.rank
            nreq = sum(1 for q in sp.params if "optional" not in sp.vars[q].attrs)
            if ok and len(acts) >= nreq:
                return sname
        raise TypeError("no specific of %s matches %r" % (gname, args))

    def user_call(self, p, name, args):
        if name in self.mod.generics:
            name = self.pick_specific(p, name, args or [])
        if name in self.mod.procs:
            callee = "p_" + name
            sp = self.mod.procs[name]
        else:
            v = self.var(p, name)
            if v is None or not (v.t == "proc" or "external" in v.attrs):
                return None
            callee = "v_" + name
            sp = None
        parts = []
        for a in args or []:
            if a[0] == "kw":
                parts.append("%s=%s" % ("v_" + a[1], self.des_ref(p, a[2])[0]))
            else:
                parts.append(self.des_ref(p, a)[0])
        return "%s(%s)" % (callee, ", ".join(parts)), sp

    def call_value(self, p, node):
        parts = node[1]
        if len(parts) != 1:
            raise NotImplementedError("call through a component: %r" % (node,))
        name, args = parts[0]
        r = self.user_call(p, name, args)
        if r is not None:
            code, sp = r
            if sp is None:
                raise TypeError("function %s has no interface" % name)
            rv = sp.vars[sp.result]
            return code, rv.t, rv.rank
        return self.intrinsic(p, name, args or [])

    def intrinsic(self, p, name, args):
        pos = [a for a in args if a[0] != "kw"]
        kw = {a[1]: a[2] for a in args if a[0] == "kw"}

        def E(a):
            return self.ex(p, a)

        def arg(key, i):
            return kw.get(key, pos[i] if len(pos) > i else None)
        if name == "abs":
            c, t, r = E(pos[0])
            return ("np.abs(%s)" % c if t != "i" else "abs(%s)" % c), t, r
        if name in ("sqrt", "dsqrt"):
            c, t, r = E(pos[0])
            return "np.sqrt(%s)" % _conv_code(c, t, "r8" if t == "i" else t, r), t, r
        if name in ("exp", "dexp", "log", "dlog", "alog", "log10", "dlog10", "alog10"):
            base = {"dexp": "exp", "dlog": "log", "alog": "log", "dlog10": "log10",
                    "alog10": "log10"}.get(name, name)
            c, t, r = E(pos[0])
            return "_libm(%r, %s, %r)" % (base, c, t), t, r
        if name in ("max", "min", "dmax1", "dmin1", "amax1", "amin1", "max0", "min0"):
            xs = [E(a) for a in pos]
            t = xs[0][1]
            for x in xs[1:]:
                t = _promote(t, x[1])
            rank = max(x[2] for x in xs)
            f = "_fmax" if name.startswith(("max", "dmax", "amax")) else "_fmin"
            return "%s(%s)" % (f, ", ".join(_conv_code(c, tt, t, rr) for c, tt, rr in xs)), t, rank
        if name in ("maxval", "minval", "sum"):
            c, t, r = E(pos[0])
            dim, mask = arg("dim", 1), arg("mask", 2)
            dc = self.ex(p, dim)[0] if dim is not None else "None"
            mc = self.ex(p, mask)[0] if mask is not None else "None"
            rank = r - 1 if dim is not None else 0
            if name == "sum":
                return "_sum(%s, %s, %s)" % (c, dc, mc), t, rank
            return "_maxval(%s, %s, %s, minimum=%s)" % (c, dc, mc, name == "minval"), t, rank
        if name in ("any", "all"):
            c, t, r = E(pos[0])
            dim = arg("dim", 1)
            f = "np.any" if name == "any" else "np.all"
            if dim is None:
                return "bool(%s(%s))" % (f, c), "l", 0
            return "%s(%s, axis=(%s) - 1)" % (f, c, self.ex(p, dim)[0]), "l", r - 1
        if name == "spread":
            c, t, r = E(arg("source", 0))
            d = self.ex(p, arg("dim", 1))[0]
            n = self.ex(p, arg("ncopies", 2))[0]
            return "_spread(%s, %s, %s)" % (c, d, n), t, r + 1
        if name == "maxloc":
            c, t, r = E(pos[0])
            dim = arg("dim", 1)
            if dim is not None:
                return "_maxloc(%s, %s)" % (c, self.ex(p, dim)[0]), "i", 0
            return "_maxloc(%s)" % c, "i", 1
        if name == "size":
            c, t, r = E(pos[0])
            dim = arg("dim", 1)
            if dim is None:
                return "int(np.asarray(%s).size)" % c, "i", 0
            return "int(np.asarray(%s).shape[(%s) - 1])" % (c, self.ex(p, dim)[0]), "i", 0
        if name in ("real", "float", "sngl", "dble", "dfloat"):
            c, t, r = E(pos[0])
            to = "r8" if name in ("dble", "dfloat") else "r4"
            k = arg("kind", 1)
            if k is not None:
                kv = self.const_value(k)
                to = "r8" if kv and kv[0] == 8 else "r4"
            return _conv_code(c, t, to, r), to, r
        if name in ("int", "idint", "ifix"):
            c, t, r = E(pos[0])
            if r:
                return "np.trunc(%s).astype(np.int64)" % c, "i", r
            return "int(%s)" % c, "i", 0
        if name == "nint":
            c, t, r = E(pos[0])
            return "_nint(%s)" % c, "i", r
        if name == "mod":
            (a, ta, ra), (b, tb, rb) = E(pos[0]), E(pos[1])
            t = _promote(ta, tb)
            if t == "i":
                return "_imod(%s, %s)" % (a, b), "i", max(ra, rb)
            return "np.fmod(%s, %s)" % (_conv_code(a, ta, t, ra), _conv_code(b, tb, t, rb)), t, max(ra, rb)
        if name == "transpose":
            c, t, r = E(pos[0])
            return "np.asarray(%s).T" % c, t, 2
        if name == "reshape":
            src, shp = arg("source", 0), arg("shape", 1)
            c, t, r = E(src)
            s, _, _ = E(shp)
            n = len(shp[1]) if shp[0] == "ctor" else 2
            return "np.reshape(%s, tuple(int(v) for v in %s), order='F')" % (c, s), t, n
        if name == "present":
            return "(v_%s is not None)" % pos[0][1][0][0], "l", 0
        if name in ("allocated", "associated"):
            info = self.resolve(p, pos[0])
            return "(%s is not None)" % info["code"], "l", 0
        if name == "huge":
            c, t, r = E(pos[0])
            return ("np.finfo(%s).max" % {"r8": "np.float64", "r4": "np.float32"}[t] if t != "i"
                    else "2147483647"), t, 0
        if name == "epsilon":
            c, t, r = E(pos[0])
            return "np.finfo(%s).eps" % {"r8": "np.float64", "r4": "np.float32"}[t], t, 0
        if name == "sign":
            (a, ta, ra), (b, tb, rb) = E(pos[0]), E(pos[1])
            return "np.copysign(%s, %s)" % (a, b), ta, max(ra, rb)
        raise NotImplementedError("intrinsic or unknown function %s" % name)

    # ------------------------------------------------------------- statements
    def emit_proc(self, p):
        L = []
        params = []
        for nm in p.params:
            v = p.vars[nm]
            params.append("v_%s=None" % nm if "optional" in v.attrs else "v_" + nm)
        L.append("def p_%s(%s):" % (p.name, ", ".join(params)))
        body = []
        for nm in p.params:
            v = p.vars[nm]
            if v.dims:
                if v.dims[0][1] is None:      # assumed shape
                    body.append("v_%s = _dummy(v_%s, None)" % (nm, nm))
                else:
                    body.append("v_%s = _dummy(v_%s, %s)" % (nm, nm, self.dims_code(p, v.dims)))
        for nm, v in p.vars.items():
            if nm in p.params or v.t == "proc" or "external" in v.attrs:
                continue
            if "save" in v.attrs or (v.init is not None and "parameter" not in v.attrs):
                gname = "S_%s_%s" % (p.name, nm)
                self.saves.append((gname, v, p))
                body.append("v_%s = %s" % (nm, gname))
                continue
            if v.dims:
                if v.dims[0][1] is None:
                    body.append("v_%s = None" % nm)
                else:
                    body.append("v_%s = _alloc(%r, %s)" % (nm, v.t, self.dims_code(p, v.dims)))
            elif v.t == "d":
                body.append("v_%s = T_%s()" % (nm, v.tname))
            else:
                init = {"r8": "np.float64(0.0)", "r4": "np.float32(0.0)", "i": "0", "l": "False",
                        "c": "''"}[v.t]
                if v.init is not None:
                    c, t, _ = self.ex(p, v.init)
                    init = _conv_code(c, t, v.t, 0)
                body.append("v_%s = Ref(%s)" % (nm, init))
        body.append("_enter(%r, locals())" % p.name)
        self.block(p, p.body, 0, len(p.body), body, 0, [])
        if p.kind == "function":
            body.append(self.ret_code(p))
        for b in body:
            L.append("    " + b)
        return L

    def ret_code(self, p):
        if p.kind != "function":
            return "return"
        rv = p.vars[p.result]
        return "return v_%s.a" % p.result if rv.dims else "return v_%s.v" % p.result

    def dims_code(self, p, dims):
        out = []
        for lo, hi in dims:
            lc = self.ex(p, lo)[0] if lo is not None else "1"
            hc = self.ex(p, hi)[0]
            out.append("(%s, %s)" % (lc, hc))
        return "[%s]" % ", ".join(out)

    def block(self, p, stmts, i, j, out, ind, loops):
        """emits statements[i:j] at indentation ind; loops: enclosing labels"""
        pad = "    " * ind
        k = i
        start_len = len(out)
        while k < j:
            s, ln = stmts[k]
            for label, (pn, text) in self.probes.items():
                if pn == p.name and re.sub(r"\s+", "", text.lower()) == re.sub(r"\s+", "", s):
                    out.append(pad + "HITS[%r] = HITS.get(%r, 0) + 1" % (label, label))
            m = re.match(r"^(?:(\w+)\s*:\s*)?do\b\s*(.*)$", s)
            if m:
                label, rest = m.group(1), m.group(2).strip()
                end = self.find_end(stmts, k, j, "do")
                self.emit_do(p, label, rest, stmts, k + 1, end, out, ind, loops)
                k = end + 1
                continue
            if re.match(r"^if\s*\(", s):
                o = s.index("(")
                c = match_paren(s, o)
                cond = s[o + 1:c]
                rest = s[c + 1:].strip()
                if rest == "then":
                    end, branches = self.find_if(stmts, k, j)
                    for bi, (kind, bcond, b0, b1) in enumerate(branches):
                        if kind == "else":
                            out.append(pad + "else:")
                        else:
                            out.append(pad + ("if %s:" if bi == 0 else "elif %s:") % self.cond(p, bcond))
                        self.block(p, stmts, b0, b1, out, ind + 1, loops)
                    k = end + 1
                    continue
                out.append(pad + "if %s:" % self.cond(p, cond))
                self.block(p, [(rest, ln)], 0, 1, out, ind + 1, loops)
                k += 1
                continue
            if re.match(r"^where\s*\(", s):
                o = s.index("(")
                c = match_paren(s, o)
                mask = s[o + 1:c]
                rest = s[c + 1:].strip()
                mv = "_wm%d" % ln
                out.append(pad + "%s = np.asarray(%s, dtype=bool)" % (mv, self.ex(p, parse_expr(mask))[0]))
                if rest:
                    self.where_assign(p, rest, mv, out, pad)
                    k += 1
                    continue
                end = self.find_end(stmts, k, j, "where")
                cur = mv
                for kk in range(k + 1, end):
                    t, _ = stmts[kk]
                    mm = re.match(r"^else\s*where\s*(?:\((.*)\))?$", t)
                    if mm:
                        if mm.group(1):
                            out.append(pad + "%s_e = np.logical_and(np.logical_not(%s), %s)" % (
                                mv, mv, self.ex(p, parse_expr(mm.group(1)))[0]))
                        else:
                            out.append(pad + "%s_e = np.logical_not(%s)" % (mv, mv))
                        cur = mv + "_e"
                        continue
                    self.where_assign(p, t, cur, out, pad)
                k = end + 1
                continue
            self.simple(p, s, out, pad, loops)
            k += 1
        if len(out) == start_len:
            out.append(pad + "pass")

    def cond(self, p, text):
        c, t, r = self.ex(p, parse_expr(text))
        return "bool(%s)" % c

    def where_assign(self, p, s, mask, out, pad):
        j = top_assign(s)
        lhs = parse_expr(s[:j])
        rc, rt, rr = self.ex(p, parse_expr(s[j + 1:]))
        info = self.resolve(p, lhs)
        if info["cat"] == "array":
            view = info["code"] + ".a"
        elif info["cat"] == "section":
            view = "%s[%s]" % (info["code"], info["idx"])
        else:
            raise NotImplementedError("where on %r" % s)
        out.append(pad + "_where_set(%s, %s, %s)" % (view, _conv_code(rc, rt, info["t"], rr), mask))

    def emit_do(self, p, label, rest, stmts, b0, b1, out, ind, loops):
        pad = "    " * ind
        m = re.match(r"^while\s*\((.*)\)$", rest)
        body = []
        if m:
            head = "while %s:" % self.cond(p, m.group(1))
        elif rest == "":
            head = "while True:"
        else:
            mm = re.match(r"^(\w+)\s*=\s*(.*)$", rest)
            var = mm.group(1)
            bounds = split_top(mm.group(2))
            lo = self.ex(p, parse_expr(bounds[0]))[0]
            hi = self.ex(p, parse_expr(bounds[1]))[0]
            st = self.ex(p, parse_expr(bounds[2]))[0] if len(bounds) > 2 else "1"
            info = self.resolve(p, ("des", [(var, None)]))
            target = info["code"] + ".v" if info["cat"] == "scalar" else info["code"]
            head = "for %s in range(%s, (%s) + (1 if (%s) > 0 else -1), %s):" % (target, lo, hi, st, st)
        self.block(p, stmts, b0, b1, body, 0, loops + [label])
        if label:
            out.append(pad + "try:")
            out.append(pad + "    " + head)
            out.append(pad + "        try:")
            for b in body:
                out.append(pad + "            " + b)
            out.append(pad + "        except _Cycle as _e:")
            out.append(pad + "            if _e.label != %r:" % label)
            out.append(pad + "                raise")
            out.append(pad + "except _Exit as _e:")
            out.append(pad + "    if _e.label != %r:" % label)
            out.append(pad + "        raise")
        else:
            out.append(pad + head)
            for b in body:
                out.append(pad + "    " + b)

    def find_end(self, stmts, k, j, kw):
        depth = 0
        for kk in range(k, j):
            s = stmts[kk][0]
            if kw == "do":
                if re.match(r"^(?:\w+\s*:\s*)?do\b", s):
                    depth += 1
                elif re.match(r"^end\s*do\b", s):
                    depth -= 1
            elif kw == "where":
                if re.match(r"^where\s*\(", s):
                    o = s.index("(")
                    if not s[match_paren(s, o) + 1:].strip():
                        depth += 1
                elif re.match(r"^end\s*where", s):
                    depth -= 1
            if depth == 0:
                return kk
        raise SyntaxError("unterminated %s at %r" % (kw, stmts[k]))

    def find_if(self, stmts, k, j):
        depth = 0
        branches = []
        s0 = stmts[k][0]
        o = s0.index("(")
        cur = ["if", s0[o + 1:match_paren(s0, o)], k + 1]
        for kk in range(k, j):
            s = stmts[kk][0]
            if re.match(r"^if\s*\(", s):
                o = s.index("(")
                if s[match_paren(s, o) + 1:].strip() == "then":
                    depth += 1
                    continue
            if re.match(r"^end\s*if\b", s):
                depth -= 1
                if depth == 0:
                    branches.append((cur[0], cur[1], cur[2], kk))
                    return kk, branches
                continue
            if depth == 1:
                if re.match(r"^else\s*if\s*\(", s):
                    o = s.index("(")
                    branches.append((cur[0], cur[1], cur[2], kk))
                    cur = ["elif", s[o + 1:match_paren(s, o)], kk + 1]
                    continue
                if re.match(r"^else$", s):
                    branches.append((cur[0], cur[1], cur[2], kk))
                    cur = ["else", None, kk + 1]
        raise SyntaxError("unterminated if")

    def simple(self, p, s, out, pad, loops):
        m = re.match(r"^(cycle|exit)\s*(\w*)$", s)
        if m:
            kind, label = m.groups()
            innermost = loops[-1] if loops else None
            if not label or label == innermost:
                out.append(pad + ("continue" if kind == "cycle" else "break"))
            else:
                out.append(pad + "raise %s(%r)" % ("_Cycle" if kind == "cycle" else "_Exit", label))
            return
        if s == "return":
            out.append(pad + self.ret_code(p))
            return
        if s == "continue":
            out.append(pad + "pass")
            return
        m = re.match(r"^stop\b\s*(.*)$", s)
        if m:
            out.append(pad + "raise FortranStop(%r)" % m.group(1))
            return
        m = re.match(r"^print\s*\*\s*,?(.*)$", s) or re.match(r"^write\s*\([^)]*\)\s*(.*)$", s)
        if m:
            items = [self.ex(p, parse_expr(x))[0] for x in split_top(m.group(1)) if x]
            out.append(pad + "_print(%s)" % ", ".join(items))
            return
        m = re.match(r"^call\s+(\w+)\s*(?:\((.*)\))?$", s)
        if m:
            name = m.group(1)
            args = []
            if m.group(2) and m.group(2).strip():
                args = Parser(tokenize("x(%s)" % m.group(2))).designator()[1][0][1]
            r = self.user_call(p, name, args)
            if r is None:
                raise NotImplementedError("call of unknown %s" % name)
            out.append(pad + r[0])
            return
        m = re.match(r"^(allocate|deallocate|nullify)\s*\((.*)\)$", s)
        if m:
            self.alloc(p, m.group(1), m.group(2), out, pad)
            return
        j = top_assign(s)
        if j < 0:
            raise NotImplementedError("statement %r in %s" % (s, p.name))
        self.assign(p, s[:j].strip(), s[j + 1:].strip(), out, pad)

    def alloc(self, p, kind, text, out, pad):
        for item in split_top(text):
            mm = re.match(r"^stat\s*=\s*(\w+)$", item)
            if mm:
                info = self.resolve(p, ("des", [(mm.group(1), None)]))
                out.append(pad + "%s.v = 0" % info["code"])
                continue
            parts = parse_expr(item)[1]
            if kind in ("deallocate", "nullify"):
                info = self.resolve(p, ("des", [(n, None) for n, _ in parts]))
                out.append(pad + "%s = None" % info["code"])
                continue
            info = self.resolve(p, ("des", [(n, None) for n, _ in parts]))
            dims = []
            for a in parts[-1][1]:
                if a[0] == "slice":
                    dims.append("(%s, %s)" % (self.ex(p, a[1])[0], self.ex(p, a[2])[0]))
                else:
                    dims.append("(1, %s)" % self.ex(p, a)[0])
            out.append(pad + "%s = _alloc(%r, [%s])" % (info["code"], info["t"], ", ".join(dims)))

    def assign(self, p, lhs, rhs, out, pad):
        rc, rt, rr = self.ex(p, parse_expr(rhs))
        info = self.resolve(p, parse_expr(lhs))
        if info is None:
            raise NameError("assignment to undeclared %r in %s" % (lhs, p.name))
        c = info["cat"]
        if c == "scalar":
            out.append(pad + "%s.v = %s" % (info["code"], _conv_code(rc, rt, info["t"], 0)))
        elif c == "field":
            out.append(pad + "%s = %s" % (info["code"], _conv_code(rc, rt, info["t"], 0)))
        elif c == "elem":
            out.append(pad + "%s[%s] = %s" % (info["code"], info["idx"], _conv_code(rc, rt, info["t"], 0)))
        elif c == "section":
            out.append(pad + "%s[%s] = %s" % (info["code"], info["idx"], rc))
        elif c == "array":
            out.append(pad + "%s.a[...] = %s" % (info["code"], rc))
        elif c == "derived":
            out.append(pad + "%s = %s" % (info["code"], rc))
        else:
            raise NotImplementedError("assignment to %r" % lhs)

    # ---------------------------------------------------------------- module
    def emit_module(self):
        L = []
        for tname, comps in self.mod.types.items():
            L.append("class T_%s:" % tname)
            L.append("    def __init__(self):")
            for cn in self.mod.type_order[tname]:
                v = comps[cn]
                if v.dims:
                    L.append("        self.%s = None" % cn)
                elif v.t == "d":
                    L.append("        self.%s = T_%s()" % (cn, v.tname))
                elif v.init is not None:
                    c, t, _ = self.ex(None, v.init)
                    L.append("        self.%s = %s" % (cn, _conv_code(c, t, v.t, 0)))
                else:
                    L.append("        self.%s = %s" % (cn, {"r8": "np.float64(0.0)", "r4": "np.float32(0.0)",
                                                             "i": "0", "l": "False", "c": "''"}[v.t]))
            L.append("")
        for name, p in self.mod.procs.items():
            L += self.emit_proc(p)
            L.append("")
        saves = []
        for gname, v, p in self.saves:
            if v.dims:
                saves.append("%s = _alloc(%r, %s)" % (gname, v.t, self.dims_code(None, v.dims)))
            else:
                init = {"r8": "np.float64(0.0)", "r4": "np.float32(0.0)", "i": "0", "l": "False"}[v.t]
                if v.init is not None:
                    c, t, _ = self.ex(p, v.init)
                    init = _conv_code(c, t, v.t, 0)
                saves.append("%s = Ref(%s)" % (gname, init))
        head = ["# generated by f90py: do not edit"]
        for (typ, hx), nm in self.consts.items():
            head.append("%s = %s(float.fromhex(%r))" % (nm, "np.float64" if typ == "r8" else "np.float32", hx))
        return "\n".join(head + saves + L) + "\n"


def translate(sources, defines=(), probes=None):
    """sources: Fortran texts (modules in dependency order).  Returns
    (python_source, namespace) with the module procedures as p_<name> and
    derived types as T_<name>."""
    mod = Module()
    for src in sources:
        structure(preprocess(src, defines), mod)
    py = Emitter(mod, probes).emit_module()
    ns = {"np": np, "math": math}
    for k, v in list(globals().items()):
        if (k.startswith("_") and not k.startswith("__")) or k in (
                "Ref", "FieldRef", "ElemRef", "FArray", "FortranStop", "HITS", "CALLS", "HOOKS", "PRINTED"):
            ns[k] = v
    exec(compile(py, "<f90py>", "exec"), ns)
    return py, ns
