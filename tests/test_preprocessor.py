"""Preprocessor and emitted network code against the reference's own output.

tests/golden/ref_preproc.json holds, for nine (example, packaging, ordering)
cases, what the reference preprocessor produced (permutation, LU nnz, CSC
arrays) and the values of its generated Fortran right-hand sides and
iteration matrices at seeded points (tests/golden/make_golden.py).
"""
import json
import os
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
        ex, pack, order = key.split("_")
        out[key] = pre_odevec.build_system(networks.load(ex), order, pack)
    return out


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
        P = h2f(smp["P"])
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
    (["--LUmethod=2"], "LUmethod=2"),
    (["--equilibrium_H=1", "--packaging=CSC"], "only allowed with DENSE"),
])
def test_cli_rejects(tmp_path, argv, msg):
    out = subprocess.run([sys.executable, "-m", "odevec_b200.pre_odevec", "--nvector=1", "--example=ROBER",
                          "--outdir=%s" % tmp_path] + argv, capture_output=True, text=True,
                         cwd=os.path.dirname(HERE))
    assert out.returncode != 0
    assert msg in out.stderr + out.stdout
