#!/usr/bin/env python
"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run in a container where the reference sources are mounted (read-only) at
``REF`` (default /root/reference); the GPU machines never run this script,
they only read the JSON it writes.

What it does:

1. Copies the reference to a temporary directory and applies four shims that
   its preprocessor needs under SymPy 1.14 outside a git checkout:
   ``example_systems.py`` uses ``symbols``/``Matrix``/``k`` without defining
   them (``pre_odevec/example_systems.py:27,33,37,65-69``); ``fcode`` cannot
   print NumPy arrays (``pre_odevec.py:193,220-224``); ``git rev-parse`` needs
   a checkout (``pre_odevec.py:372-373``).
2. Runs ``pre_odevec.py`` for each (example, packaging, ordering) case and
   parses the generated Fortran: the permutation, the CSC pattern
   (``row_index``, ``u_col_start``, ``l_col_start``, 1-based in the Fortran,
   stored 0-based here), ``nnz``, and the generated ``rhs(:,i)`` and
   ``jac(:,i,j)`` / ``jac%sdata(:,i)`` expressions, and for LUmethod 2 the
   ``LU(:,i,j)`` expressions of the generated GetLU.
3. Evaluates those expressions at seeded random points with Python floats.
   Python float arithmetic is IEEE binary64 without fused multiply-add and
   evaluates ``a*b*c`` and ``a+b+c`` left to right, like gfortran -O2 on
   x86-64; integer powers ``x**2``/``x**3`` are expanded into products the way
   gfortran expands them (``x*x``, ``x*(x*x)``).
4. Evaluates the 38 PRIMORDIAL rate laws of the reference's ``coe`` function
   (``src/odevec_commons.F90:101-384``) from its Fortran source text on a
   temperature grid, with Fortran literal kinds honoured (a real literal
   without a ``d`` exponent is single precision) and ``small`` set to 0.

Only numbers are written (inputs and outputs as hex floats), no generated
source.  Usage: ``python tests/golden/make_golden.py [REF]``.
"""
import json
import math
import os
import re
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"

CASES = [
    ("ROBER", "DENSE", "None"),
    ("ROBER", "CSC", "None"),
    ("OREGO", "DENSE", "None"),
    ("OREGO", "CSC", "CMK"),
    ("PRIMORDIAL", "DENSE", "None"),
    ("PRIMORDIAL", "CSC", "None"),
    ("PRIMORDIAL", "CSC", "FF"),
    ("PRIMORDIAL", "CSC", "CMK"),
    ("PRIMORDIAL", "CSC", "INVERT"),
    # LUmethod 2: the generated GetLU (symbolic factors), dense only
    ("ROBER", "DENSE", "None", 2),
    ("OREGO", "DENSE", "None", 2),
]
NSAMPLES = 6


def shim_copy(dst):
    shutil.copytree(REF, dst)
    for root, dirs, files in os.walk(dst):
        for f in files + dirs:
            os.chmod(os.path.join(root, f), 0o755)
    ex = os.path.join(dst, "pre_odevec", "example_systems.py")
    src = open(ex).read().split("\n")
    src.insert(1, "from sympy import *\nk = 0")
    open(ex, "w").write("\n".join(src))
    pp = os.path.join(dst, "pre_odevec.py")
    src = open(pp).read()
    src = src.replace('commit = check_output("git rev-parse --short HEAD", shell=True).rstrip()',
                      'commit = b"nogit"')
    src = src.replace('''dirty = check_output("git diff --quiet || echo 'dirty'", shell=True).rstrip()''',
                      'dirty = b""')
    src = src.replace("from pre_odevec.example_systems import *", '''from pre_odevec.example_systems import *
_fcode_orig = fcode
def fcode(e, **kw):
    import numpy as _np
    if isinstance(e, _np.ndarray):
        return "(/ " + ", ".join(str(int(v)) for v in e.ravel()) + " /)"
    return _fcode_orig(e, **kw)
''')
    open(pp, "w").write(src)


def join_continuations(text):
    # free-form continuation: trailing '&' joins with the next line's text
    return re.sub(r"&\s*\n\s*", "", text)


def int_list(text, name):
    m = re.search(r"%s\s*=\s*&?\s*\(/(.*?)/\)" % re.escape(name), text, re.S)
    return [int(v) for v in m.group(1).split(",")]


def fortran_expr_to_python(e):
    e = re.sub(r"\b(y|k)\s*\(\s*:\s*,\s*(\d+)\s*\)", lambda m: "%s[%d]" % (m.group(1), int(m.group(2)) - 1), e)
    e = re.sub(r"(\d\.?\d*)d([+-]?\d+)", r"\1e\2", e)
    # gfortran expands small integer powers into multiplications
    e = re.sub(r"((?:y|k)\[\d+\]|\bbeta|\bdt)\*\*2\b", r"(\1*\1)", e)
    e = re.sub(r"((?:y|k)\[\d+\]|\bbeta|\bdt)\*\*3\b", r"(\1*(\1*\1))", e)
    if "**" in e:
        raise ValueError("unhandled power in %s" % e)
    return e


def parse_generated(build):
    solver = join_continuations(open(os.path.join(build, "odevec.f90")).read())
    common = join_continuations(open(os.path.join(build, "odevec_commons.f90")).read())
    out = {}
    out["perm"] = [v - 1 for v in int_list(solver, "this%Perm")]
    out["nnz"] = int(re.search(r"integer :: nnz=(\d+)", solver).group(1))
    out["neq"] = int(re.search(r"integer :: neq=(\d+)", solver).group(1))
    if "this%LU%row_index" in solver:
        out["row_index"] = [v - 1 for v in int_list(solver, "this%LU%row_index")]
        out["u_col_start"] = [v - 1 for v in int_list(solver, "this%LU%u_col_start")]
        out["l_col_start"] = [v - 1 for v in int_list(solver, "this%LU%l_col_start")]
    rhs, jac, lu = {}, {}, {}
    for line in common.split("\n"):
        s = line.strip()
        m = re.match(r"LU\(:,(\d+),(\d+)\)\s*=\s*(.*)$", s)
        if m:
            lu[(int(m.group(1)) - 1, int(m.group(2)) - 1)] = fortran_expr_to_python(m.group(3))
            continue
        m = re.match(r"rhs\(:,(\d+)\)\s*=\s*(.*)$", s)
        if m:
            rhs[int(m.group(1)) - 1] = fortran_expr_to_python(m.group(2))
            continue
        m = re.match(r"jac\(:,(\d+),(\d+)\)\s*=\s*(.*)$", s)
        if m:
            jac[(int(m.group(1)) - 1, int(m.group(2)) - 1)] = fortran_expr_to_python(m.group(3))
            continue
        m = re.match(r"jac%sdata\(:,(\d+)\)\s*=\s*(.*)$", s)
        if m:
            jac[int(m.group(1)) - 1] = fortran_expr_to_python(m.group(2))
    return out, rhs, jac, lu


def hexs(vals):
    return [float(v).hex() for v in vals]


def sample_inputs(rng, neq, nrea):
    y = list(10.0 ** rng.uniform(-8, 2, neq))
    k = list(10.0 ** rng.uniform(-20, -8, nrea)) if nrea else []
    beta = float(rng.uniform(0.35, 1.0))
    dt = float(10.0 ** rng.uniform(-6, 8))
    return y, k, beta, dt


def run_cases(work):
    results = {}
    rng = np.random.default_rng(20240611)
    for case in CASES:
        ex, pack, order = case[:3]
        lum = case[3] if len(case) > 3 else 1
        for d in ("build",):
            os.makedirs(os.path.join(work, d), exist_ok=True)
        cmd = [sys.executable, "pre_odevec.py", "--nvector=32", "--example=%s" % ex,
               "--packaging=%s" % pack, "--ordering=%s" % order, "--LUmethod=%d" % lum]
        log = subprocess.run(cmd, cwd=work, capture_output=True, text=True, check=True).stdout
        meta, rhs, jac, lu = parse_generated(os.path.join(work, "build"))
        m = re.search(r"NNZs in Jacobian: (\d+)", log)
        meta["p_nnz"] = int(m.group(1))
        neq = meta["neq"]
        nrea = 38 if ex == "PRIMORDIAL" else 0
        samples = []
        for _ in range(NSAMPLES):
            y, k, beta, dt = sample_inputs(rng, neq, nrea)
            env = {"y": y, "k": k, "beta": beta, "dt": dt}
            f = [eval(rhs[i], {}, env) for i in range(neq)]
            if pack == "DENSE":
                # row-major n x n of the (permuted) iteration matrix P
                P = [eval(jac[(i, j)], {}, env) for i in range(neq) for j in range(neq)]
            else:
                P = [eval(jac[i], {}, env) for i in range(meta["nnz"])]
            smp = {"y": hexs(y), "k": hexs(k), "beta": beta.hex(), "dt": dt.hex(),
                   "rhs": hexs(f), "P": hexs(P)}
            if lum == 2:
                # row-major n x n of the symbolic factors; entries GetLU does not
                # write stay at their initial 0
                smp["LU"] = hexs([eval(lu[(i, j)], {}, env) if (i, j) in lu else 0.0
                                  for i in range(neq) for j in range(neq)])
            samples.append(smp)
        meta["samples"] = samples
        results["%s_%s_%s" % (ex, pack, order) + ("_LU%d" % lum if lum != 1 else "")] = meta
        print(ex, pack, order, "nnz", meta["nnz"], "perm", meta["perm"])
    return results


# ---------------------------------------------------------------- rate laws
def f32(x):
    return float(np.float32(x))


def powi(x, n):
    """x**n for a small positive integer n as gfortran expands it
    (addition chain x^n = x^(n-t[n]) * x^t[n])."""
    table = [0, 1, 1, 2, 2, 3, 3, 4, 4, 6, 5, 6, 6, 10, 7, 9]
    cache = {1: x}

    def rec(m):
        if m in cache:
            return cache[m]
        v = rec(m - table[m]) * rec(table[m])
        cache[m] = v
        return v
    return rec(n)


def coe_to_python(expr):
    e = expr.replace("dexp(", "exp(")
    # Fortran real literals: with a d exponent -> double; otherwise single
    def lit(m):
        s = m.group(0)
        if "d" in s.lower():
            return repr(float(s.lower().replace("d", "e")))
        if "." in s or "e" in s.lower():
            return repr(f32(float(s)))
        return s
    e = re.sub(r"(?<![\w.])(\d+\.\d*(?:[dDeE][+-]?\d+)?|\d*\.\d+(?:[dDeE][+-]?\d+)?|\d+[dDeE][+-]?\d+)",
               lit, e)
    # powers are resolved in eval_fortran (integer exponent -> powi)
    return e.replace("**", "^^")


def parse_coe(path):
    text = join_continuations(open(path).read())
    body = text[text.index("function coe(this)"):text.index("end function coe")]
    laws = {}
    cond = None
    for line in body.split("\n"):
        s = line.strip()
        m = re.match(r"where\s*\((.*)\)\s*$", s)
        if m:
            cond = m.group(1)
            continue
        if s.startswith("end where"):
            cond = None
            continue
        m = re.match(r"vec_k\(:,(\d+)\)\s*=\s*small\s*\+\s*(.*)$", s)
        if m:
            laws[int(m.group(1))] = (cond, m.group(2))
    return laws


def eval_fortran(expr, env):
    # '^^' marks a real power: rewrite a^^b with Python's float pow,
    # which calls the C library pow() like gfortran does.
    py = expr
    while "^^" in py:
        i = py.index("^^")
        # right operand: parenthesised group or literal/identifier
        j = i + 2
        if py[j] == "(":
            depth = 0
            for jj in range(j, len(py)):
                depth += py[jj] == "("
                depth -= py[jj] == ")"
                if depth == 0:
                    break
            right_end = jj + 1
        else:
            m = re.match(r"[-+]?[\w.]+(?:e[-+]?\d+)?", py[j:])
            right_end = j + m.end()
        # left operand
        k = i - 1
        if py[k] == ")":
            depth = 0
            for kk in range(k, -1, -1):
                depth += py[kk] == ")"
                depth -= py[kk] == "("
                if depth == 0:
                    break
            left_start = kk
            # include a function name before the parenthesis
            m = re.search(r"[A-Za-z_][A-Za-z0-9_]*$", py[:left_start])
            if m:
                left_start = m.start()
        else:
            m = re.search(r"[\w.]+$", py[:i])
            left_start = m.start()
        right = py[i + 2:right_end]
        fn = "powi" if re.fullmatch(r"\d+", right) else "fpow"
        py = (py[:left_start] + fn + "(" + py[left_start:i] + "," + right + ")"
              + py[right_end:])
    return eval(py, {"exp": math.exp, "log": math.log, "log10": math.log10, "sqrt": math.sqrt,
                     "powi": powi, "fpow": lambda a, b: math.pow(float(a), float(b))}, env)


def tgas_conditions(cond, T):
    c = cond.replace("Tgas", "T").replace(".LE.", "<=").replace(".LT.", "<").replace(
        ".GE.", ">=").replace(".GT.", ">")
    c = re.sub(r"(\d\.?\d*)d([+-]?\d+)", r"\1e\2", c)
    return eval(c, {}, {"T": T})


def run_rates():
    laws = parse_coe(os.path.join(REF, "src", "odevec_commons.F90"))
    assert sorted(laws) == list(range(1, 39)), sorted(laws)
    temps = sorted(set(list(np.geomspace(10.0, 1.0e4, 37)) +
                       [50.0, 200.0, 300.0, 617.0, 1160.0, 2000.0, 3480.0, 5500.0, 6700.0, 9280.0,
                        299.0, 301.0, 1159.5, 1160.5, 5499.0, 5501.0, 9279.0, 9281.0, 1000.0]))
    rows = []
    for T in temps:
        Te = T * 8.617343e-5
        env = {"Tgas": T, "Te": Te, "lnTe": math.log(Te), "T32": T * f32(0.0033333333333333335),
               "invT": 1.0 / T, "invTe": 1.0 / Te, "sqrTgas": math.sqrt(T)}
        vals = []
        for i in range(1, 39):
            cond, expr = laws[i]
            if cond is not None and not tgas_conditions(cond, T):
                vals.append(0.0)
            else:
                vals.append(float(eval_fortran(coe_to_python(expr), env)))
        rows.append({"T": T.hex() if isinstance(T, float) else float(T).hex(), "k": hexs(vals)})
    return rows


def main():
    work = tempfile.mkdtemp(prefix="odevec_ref_")
    try:
        shim_copy(os.path.join(work, "ref"))
        pre = run_cases(os.path.join(work, "ref"))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    with open(os.path.join(HERE, "ref_preproc.json"), "w") as fh:
        json.dump(pre, fh, indent=0, sort_keys=True)
    rates = run_rates()
    with open(os.path.join(HERE, "ref_rates.json"), "w") as fh:
        json.dump({"note": "PRIMORDIAL rate laws of the reference coe() with small=0",
                   "rows": rates}, fh, indent=0)
    print("wrote", os.path.join(HERE, "ref_preproc.json"), os.path.join(HERE, "ref_rates.json"))


if __name__ == "__main__":
    main()
