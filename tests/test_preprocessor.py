"""Preprocessor and emitted network code against the reference's own output.

tests/golden/ref_preproc.json holds, for nine (example, packaging, ordering)
cases, what the reference preprocessor produced (permutation, LU nnz, CSC
arrays) and the values of its generated Fortran right-hand sides and
iteration matrices at seeded points, plus, for two dense LUmethod=2 cases,
the values of its generated symbolic factors (tests/golden/make_golden.py).
"""
import json
import os
import re
import subprocess
import sys

import numpy as np
import pytest
import sympy as sp

from odevec_b200 import networks, pre_odevec

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "ref_preproc.json")))
h2f = lambda l: np.array([float.fromhex(v) for v in l])


@pytest.fixture(scope="module")
def systems():
    out = {}
    for key in GOLDEN:
        ex, pack, order, lum = _case(key)
        out[key] = pre_odevec.build_system(networks.load(ex), order, pack, lu_method=lum)
    return out


def _case(key):
    parts = key.split("_")
    return parts[0], parts[1], parts[2], int(parts[3][2:]) if len(parts) > 3 else 1


@pytest.mark.parametrize("key", sorted(GOLDEN))
def test_permutation_and_pattern_match_reference(systems, key):
    g, s = GOLDEN[key], systems[key]
    assert s.perm == g["perm"]
    assert s.nnz == g["nnz"]
    assert s.p_nnz == g["p_nnz"]
    if "row_index" in g:
        assert s.row_index == g["row_index"]
        assert s.u_col_start == g["u_col_start"]
        assert s.l_col_start == g["l_col_start"]


@pytest.mark.parametrize("key", ["PRIMORDIAL_CSC_FF", "PRIMORDIAL_CSC_CMK", "OREGO_CSC_CMK"])
def test_symbolic_lu_pattern_equals_structural(key):
    ex, pack, order = key.split("_")
    a = pre_odevec.build_system(networks.load(ex), order, pack, lu_pattern="structural")
    b = pre_odevec.build_system(networks.load(ex), order, pack, lu_pattern="symbolic")
    assert a.row_index == b.row_index and a.u_col_start == b.u_col_start


@pytest.mark.parametrize("key", [k for k in sorted(GOLDEN)])
def test_emitted_code_bit_identical_to_reference_expressions(oracle, key):
    tag = key.upper()
    if tag not in oracle.tags():
        pytest.skip("variant not compiled into the oracle")
    info = oracle.netinfo(tag)
    n = info["neq"]
    for smp in GOLDEN[key]["samples"]:
        f, a = oracle.evaluate(tag, h2f(smp["y"]), h2f(smp["k"]), float.fromhex(smp["beta"]),
                               float.fromhex(smp["dt"]))
        assert np.array_equal(f, h2f(smp["rhs"]))
        # LUmethod 2: jac() writes the symbolic factors, pinned by GetLU's values
        P = h2f(smp["LU"] if "LU" in smp else smp["P"])
        if "DENSE" in key:
            full = np.zeros((n, n))
            for c in range(n):
                for kk in range(info["u_col_start"][c], info["u_col_start"][c + 1]):
                    full[info["row_index"][kk], c] = a[kk]
            assert np.array_equal(full.ravel(), P)
        else:
            assert np.array_equal(a, P)


def test_primordial_rhs_equals_reference_table():
    # the reaction-list construction gives the reference's hand-expanded rhs:
    # compare against the golden values for every species at every sample
    net = networks.load_primordial()
    f = sp.lambdify([net.y, net.k], list(net.rhs), "math")
    for smp in GOLDEN["PRIMORDIAL_DENSE_None"]["samples"]:
        got = np.array(f(list(h2f(smp["y"])), list(h2f(smp["k"]))), dtype=float)
        ref = h2f(smp["rhs"])
        assert np.allclose(got, ref, rtol=1e-13, atol=0.0)


def test_frozen_species():
    s = pre_odevec.build_system(networks.load_primordial(), "FF", "CSC")
    assert pre_odevec.frozen_species(s) == [12, 13, 14, 15]
    s = pre_odevec.build_system(networks.load_rober(), "None", "DENSE")
    assert pre_odevec.frozen_species(s) == []


def test_dense_always_uses_structural_pattern():
    a = pre_odevec.build_system(networks.load_orego(), "None", "DENSE", lu_pattern="symbolic")
    b = pre_odevec.build_system(networks.load_orego(), "None", "DENSE", lu_pattern="structural")
    assert a.row_index == b.row_index


def test_flop_counts():
    s = pre_odevec.build_system(networks.load_primordial(), "None", "DENSE")
    c = pre_odevec.flop_counts(s)
    assert c["lu_factor"] == 975  # 2n^3/3-type count over the natural-order fill
    assert c["rhs"] > 300 and c["jac"] > 500


def test_krome_dump_loader(tmp_path):
    dump = tmp_path / "rober_krome.py"
    dump.write_text(
        "neq = 3\nnrea = 3\n"
        "y = [Symbol('y(:,%d)' % (i + 1)) for i in range(3)]\n"
        "rhs = Matrix([-0.04*y[0] + 1e4*y[1]*y[2],\n"
        "              0.04*y[0] - 3e7*y[1]*y[1] - 1e4*y[1]*y[2],\n"
        "              3e7*y[1]*y[1]])\n")
    a = networks.load_krome_dump(str(dump))
    b = networks.load_rober()
    assert a.neq == 3 and list(a.rhs) == list(b.rhs)


def test_cli_writes_variant(tmp_path):
    out = subprocess.run([sys.executable, "-m", "odevec_b200.pre_odevec", "--nvector=32", "--example=ROBER",
                          "--packaging=CSC", "--ordering=INVERT", "--outdir=%s" % tmp_path],
                         capture_output=True, text=True, cwd=os.path.dirname(HERE))
    assert out.returncode == 0, out.stderr
    assert (tmp_path / "net_rober_csc_invert.h").exists()
    assert (tmp_path / "net_rober_csc_invert.cuh").exists()
    reg = (tmp_path / "registry.inc").read_text()
    assert 'OV_NET(rober_csc_invert, "ROBER_CSC_INVERT")' in reg
    assert "Permutation list [2 1 0]" in out.stdout


@pytest.mark.parametrize("argv,msg", [
    (["--packaging=COO"], "COO packaging is not supported"),
    (["--packaging=CSR"], "CSR packaging is not supported"),
    (["--packaging=XYZ"], "This format is not known"),
    (["--heatcool=1"], "heating/cooling"),
    (["--heatcool=1", "--heatcool_header=heatcool_hctoy.h"], "KROME species layout"),
    (["--heatcool=1", "--heatcool_header=no_such_header.h"], "not found"),
    (["--LUmethod=2", "--packaging=CSC"], "LUmethod=2 needs --packaging=DENSE"),
    (["--LUmethod=3", "--packaging=CSC"], "not supported with sparse matrices"),
    (["--LUmethod=3", "--ordering=CMK"], "LUmethod=3 needs --ordering=None"),
    (["--LUmethod=4"], "is not known"),
    (["--equilibrium_H=1", "--packaging=CSC"], "only allowed with DENSE"),
])
def test_cli_rejects(tmp_path, argv, msg):
    out = subprocess.run([sys.executable, "-m", "odevec_b200.pre_odevec", "--nvector=1", "--example=ROBER",
                          "--outdir=%s" % tmp_path] + argv, capture_output=True, text=True,
                         cwd=os.path.dirname(HERE))
    assert out.returncode != 0
    assert msg in out.stderr + out.stdout


def test_lumethod3_pattern_is_full_dynamic_block():
    s = pre_odevec.build_system(networks.load("PRIMORDIAL"), "None", "DENSE", lu_method=3)
    assert s.tag == "PRIMORDIAL_DENSE_NONE_LU3"
    fz = pre_odevec.frozen_species(s)
    nd = s.neq - len(fz)
    dyn = [i for i in range(s.neq) if i not in fz]
    assert s.lu_pat[np.ix_(dyn, dyn)].all()
    for f in fz:
        assert s.lu_pat[f].sum() == 1 and s.lu_pat[:, f].sum() == 1 and s.lu_pat[f, f]
    assert s.nnz == nd * nd + len(fz)
    fl = pre_odevec.flop_counts(s)
    assert fl["jac"] > (nd + 1) * fl["rhs"] and fl["lu_factor"] > 0


def test_lumethod2_factors_are_lu_of_p():
    # the emitted factors multiply back to P at a point
    s = pre_odevec.build_system(networks.load("OREGO"), "None", "DENSE", lu_method=2)
    pt = {**{sym: v for sym, v in zip(s.net.y, (0.3, 1.7, 2.2))}, sp.Symbol("dt"): 0.01, sp.Symbol("beta"): 0.8}
    LU = s.lu_exprs.subs(pt).evalf()
    n = s.neq
    L = sp.eye(n) + sp.Matrix(n, n, lambda i, j: LU[i, j] if i > j else 0)
    U = sp.Matrix(n, n, lambda i, j: LU[i, j] if i <= j else 0)
    P = s.P_order.subs(pt).evalf()
    assert max(abs(float(v)) for v in (L * U - P)) < 1e-12


def _run_lines(lines, a, r, recip):
    """Evaluates emitted factor/solve lines in Python doubles; with recip the
    pivots are reciprocals (the FP32 convention of ov_pivot / ov_divp)."""
    env = {"a": a, "r": r, "x": [0.0] * len(r),
           "piv": (lambda p: 1.0 / p) if recip else (lambda p: p),
           "divp": (lambda v, p: v * p) if recip else (lambda v, p: v / p)}
    for ln in lines:
        ln = re.sub(r"OV_I?SC\(\d+\)", "1.0", ln.rstrip(";"))
        ln = ln.replace("ov_divp<T>(", "divp(").replace("ov_pivot<T>(", "piv(")
        ln = ln.replace("(T)", "").replace("(double)", "")
        if ln.startswith("T "):
            ln = ln[2:]
        exec(ln, env)
    return np.array(env["x"])


@pytest.mark.parametrize("example,order,pack", [("PRIMORDIAL", "FF", "CSC"), ("PRIMORDIAL", "CMK", "CSC"),
                                                ("PRIMORDIAL", "None", "DENSE"), ("ROBER", "None", "DENSE"),
                                                ("OREGO", "CMK", "CSC")])
def test_reciprocal_pivots_solve_the_same_system(example, order, pack):
    # the FP32 LU's pivot reciprocals are placed where each pivot is final:
    # factor + solve with reciprocals gives the solution of the divisions
    s = pre_odevec.build_system(networks.load(example), order, pack)
    fl, sl = pre_odevec._lu_factor_lines(s), pre_odevec._lu_solve_lines(s)
    rf, rs = pre_odevec.reciprocal_pivots(fl, sl)
    assert sum("ov_pivot" in l for l in rf) == s.neq
    rng = np.random.default_rng(7)
    a0 = rng.uniform(-1.0, 1.0, s.nnz)
    for (i, j), k in s.pos().items():
        if i == j:
            a0[k] += 2.0 * s.neq
    r = list(rng.uniform(-1.0, 1.0, s.neq))
    x_div = _run_lines(fl + sl, list(a0), r, recip=False)
    x_rec = _run_lines(rf + rs, list(a0), r, recip=True)
    assert np.max(np.abs(x_rec - x_div)) <= 1e-13 * np.max(np.abs(x_div))
    # and the rewritten lines with FP64 pivots are the original arithmetic
    assert np.array_equal(_run_lines(rf + rs, list(a0), r, recip=False), x_div)


def test_reciprocal_pivots_rejects_a_pivot_read_after_it_is_final():
    with pytest.raises(ValueError, match="other than as a divisor"):
        pre_odevec.reciprocal_pivots(["a[1] = a[1] / a[0];", "a[2] = a[2] - a[0]*a[1];"], [])


@pytest.mark.parametrize("example,order,pack,lum", [("PRIMORDIAL", "FF", "CSC", 1), ("ROBER", "None", "DENSE", 2),
                                                    ("PRIMORDIAL", "None", "DENSE", 3)])
def test_cuda_header_divides_only_through_pivot_helpers(example, order, pack, lum):
    # every division of the emitted factorisation and solves goes through
    # ov_divp, every pivot gets ov_pivot, so the FP32 LU uses reciprocals
    s = pre_odevec.build_system(networks.load(example), order, pack, lu_method=lum)
    text = pre_odevec.emit_cuda_header(s)
    body = text[text.index("void lu_factor("):]
    assert "ov_pivot<T>(" in body and "ov_divp<T>(" in body
    assert not re.search(r"/ a\[\d+\]", body)


def test_heatcool_structure():
    """--heatcool=1 (pre_odevec.py:146-190): the Tgas row becomes the
    heating/cooling term, GetJac fills the Tgas row over the chemical species
    and the whole Tgas column with difference quotients (DENSE), the
    temperature and every chemical species stay in the solver state, and a
    network whose rates depend on the temperature is refused."""
    hdr = os.path.join(os.path.dirname(HERE), "odevec_b200", "csrc", "heatcool_hctoy.h")
    dump = os.path.join(os.path.dirname(HERE), "odevec_b200", "data", "hctoy_krome.py")
    net = networks.enable_heatcool(networks.load_krome_dump(dump, "HCTOY"), hdr)
    s = pre_odevec.build_system(net, "None", "DENSE")
    T = net.neq - 2
    assert net.idx_tgas == T and net.nmols == 5
    assert all(s.lu_pat[T, j] for j in range(net.nmols)) and all(s.lu_pat[:, T])
    assert pre_odevec.frozen_species(s) == [5, 6, 8]
    h = pre_odevec.emit_c_header(s)
    assert "f[7] = ov_hctoy_dense_none_hc(y, y[7], y);" in h
    assert h.count("if (dyy > 0.0)") == net.nmols and "ov_hctoy_dense_none_rhs(hc_yy, k, dy);" in h
    cu = pre_odevec.emit_cuda_header(s)
    assert "static constexpr bool HC_FD = true;" in cu
    # CSC packaging keeps the symbolic P (pre_odevec.py:173-180): no difference quotients
    c = pre_odevec.emit_c_header(pre_odevec.build_system(net, "CMK", "CSC"))
    assert "dyy" not in c and "ov_hctoy_csc_cmk_hc(y, y[7], y)" in c
    with pytest.raises(SystemExit, match="ordering=None"):
        pre_odevec.build_system(net, "CMK", "DENSE")
    with pytest.raises(SystemExit, match="temperature"):
        networks.enable_heatcool(networks.load("PRIMORDIAL"), hdr)
