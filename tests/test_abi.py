"""The C ABI library: it loads without a GPU, exports every function that
include/odevec_b200.h declares, and rejects bad arguments with the
documented codes before touching the GPU (no compute call needs a device
here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "odevec_b200.h")


@pytest.fixture(scope="module")
def L():
    from odevec_b200 import build, solver
    if not os.path.exists(solver.LIBPATH):
        build.build()
    return solver.lib()


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:int32_t|const char\*)\s+(odevec_\w+)\(", text, re.M)))


def test_exports_every_declared_function(L):
    names = declared()
    assert "odevec_solve" in names and "odevec_solve_noalloc" in names and len(names) >= 11
    for n in names:
        assert hasattr(L, n), n


def test_network_registry(L):
    from odevec_b200 import solver
    tags = solver.networks()
    for t in ("ROBER_DENSE_NONE", "OREGO_CSC_CMK", "PRIMORDIAL_CSC_FF", "PRIMORDIAL_DENSE_NONE"):
        assert t in tags
    info = solver.network_info("PRIMORDIAL_CSC_FF")
    assert info["neq"] == 16 and info["nnz"] == 88 and info["nrea"] == 38 and info["idx_tgas"] == 14
    assert solver.network_info("ROBER_DENSE_NONE")["nvector"] == 32
    with pytest.raises(solver.OdevecError, match="unknown network"):
        solver.network_info("NOPE")


def _opts(**kw):
    from odevec_b200 import solver
    o = solver._Opts()
    o.rtol, o.atol, o.dt_min = 1e-6, 1e-20, -1.0
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def test_init_argument_errors(L):
    h = ctypes.c_void_p()
    assert L.odevec_init(b"NOPE", 10, ctypes.byref(_opts()), ctypes.byref(h)) == -2
    assert L.odevec_init(b"ROBER_DENSE_NONE", -1, ctypes.byref(_opts()), ctypes.byref(h)) == -1
    assert L.odevec_init(b"ROBER_DENSE_NONE", 10, ctypes.byref(_opts(rtol=0.0)), ctypes.byref(h)) == -1
    assert b"rtol" in L.odevec_last_error()
    assert L.odevec_init(b"ROBER_DENSE_NONE", 10, ctypes.byref(_opts(group_size=7)), ctypes.byref(h)) == -1
    assert L.odevec_init(b"ROBER_DENSE_NONE", 10, ctypes.byref(_opts(precision=9)), ctypes.byref(h)) == -1
    assert L.odevec_init(b"ROBER_DENSE_NONE", 10, ctypes.byref(_opts(block_threads=256)),
                         ctypes.byref(h)) == -1
    assert L.odevec_init(b"ROBER_DENSE_NONE", 10, ctypes.byref(_opts(staging=22)), ctypes.byref(h)) == -1
    assert L.odevec_init(b"ROBER_DENSE_NONE", 10, ctypes.byref(_opts()), None) == -1


def test_solve_argument_errors(L):
    assert L.odevec_solve(None, 10, None, None, None, None, None, None, None, None) == -1
    assert L.odevec_solve_host(None, 10, None, None, None, None, None, None, None) == -1
    assert L.odevec_close(None) == 0


def test_yield_and_continue_argument_errors(L):
    """Interruptible-solve entry points reject a null solver, a bad resume
    code and a resume without workspace before touching the GPU."""
    P = ctypes.c_void_p(16)
    n = ctypes.c_int64(0)
    assert L.odevec_set_yield(None, None) == -1
    assert L.odevec_cells_started(None, None, ctypes.byref(n)) == -1
    cont = L.odevec_solve_continue
    assert cont(None, 10, 10, P, P, P, P, None, None, None, None, 0, None) == -1
    assert cont(None, 10, 10, P, P, P, P, None, None, None, None, 3, None) == -1
    assert b"resume" in L.odevec_last_error()
    assert cont(None, 10, 10, P, P, P, P, None, None, None, None, 1, None) == -1
    assert b"workspace" in L.odevec_last_error()
    rng = L.odevec_solve_range
    assert rng(None, 10, 10, P, P, P, P, None, None, None, None, 0, None) == -1


def test_noalloc_argument_errors(L):
    f = L.odevec_solve_noalloc
    from odevec_b200 import solver
    f.argtypes = [ctypes.c_char_p, ctypes.POINTER(solver._Opts), ctypes.c_int64] + [ctypes.c_void_p] * 8
    P = ctypes.c_void_p(16)
    o = _opts()
    assert f(b"NOPE", ctypes.byref(o), 10, P, P, P, P, None, None, None, None) == -2
    assert f(b"ROBER_DENSE_NONE", ctypes.byref(o), -1, P, P, P, P, None, None, None, None) == -1
    assert f(b"ROBER_DENSE_NONE", ctypes.byref(o), (1 << 40) + 1, P, P, P, P, None, None, None, None) == -6
    assert f(b"ROBER_DENSE_NONE", ctypes.byref(o), 0, P, P, P, P, None, None, None, None) == 0
    assert f(b"ROBER_DENSE_NONE", ctypes.byref(o), 64, None, P, P, P, None, None, None, None) == -1
    bad = _opts(rtol=-1.0)
    assert f(b"ROBER_DENSE_NONE", ctypes.byref(bad), 64, P, P, P, P, None, None, None, None) == -1


def test_probe_argument_errors(L):
    assert L.odevec_probe_fma(1, 0, 0, 0, None, None, None, None) == -1
