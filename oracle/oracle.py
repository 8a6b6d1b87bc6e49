"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Used by tests/, by ``__graft_entry__.smoke()`` as the checker and by
``bench.py`` for the CPU baseline; never by the product path.
"""
import ctypes
import os

import numpy as np

from . import build as _build

OV_NSTATS = 8
_libs = {}


def lib(libm: bool = False, fast: bool = False):
    """The oracle library; libm=True: the variant calling the C library's
    exp/log/log10/pow (as the reference's Fortran does) instead of the
    library's own, for bit-for-bit comparison with the reference's solver;
    fast=True: the -O3 -march=native build timed as the CPU baseline."""
    key = (libm, fast)
    if key not in _libs:
        path = _build.build(libm=libm, fast=fast)
        L = ctypes.CDLL(path)
        d, i64, i32 = ctypes.c_double, ctypes.c_int64, ctypes.c_int
        P = ctypes.c_void_p
        L.ov_oracle_solve.argtypes = [ctypes.c_char_p, i64, i32, d, d, d, i32, i32, i64, P, P, P, P,
                                      P, P, P, i32, P, i32]
        L.ov_oracle_ws_doubles.argtypes = [ctypes.c_char_p, i64, i32]
        L.ov_oracle_ws_doubles.restype = i64
        L.ov_oracle_solve.restype = i32
        L.ov_oracle_eval.argtypes = [ctypes.c_char_p, P, P, d, d, P, P]
        L.ov_oracle_rates.argtypes = [d, P]
        L.ov_oracle_rates_k.argtypes = [P, i32, P, P]
        L.ov_oracle_netinfo.argtypes = [ctypes.c_char_p, P, P, P, P, P]
        L.ov_oracle_num_nets.restype = i32
        L.ov_oracle_net_tag.restype = ctypes.c_char_p
        L.ov_oracle_net_tag.argtypes = [i32]
        for f in ("ov_oracle_exp", "ov_oracle_log", "ov_oracle_exp_sel", "ov_oracle_log_sel"):
            getattr(L, f).argtypes = [d]
            getattr(L, f).restype = d
        for f in ("ov_oracle_pow", "ov_oracle_pow_sel"):
            getattr(L, f).argtypes = [d, d]
            getattr(L, f).restype = d
        L.ov_oracle_convert.argtypes = [ctypes.c_char_p, i64, i32, P, P, P]
        L.ov_oracle_convert.restype = i32
        _libs[key] = L
    return _libs[key]


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def netinfo(tag):
    L = lib()
    info = np.zeros(5, dtype=np.int32)
    if L.ov_oracle_netinfo(tag.encode(), _p(info), None, None, None, None) != 0:
        raise KeyError(tag)
    neq, nnz = int(info[0]), int(info[1])
    perm = np.zeros(neq, np.int32)
    ri = np.zeros(nnz, np.int32)
    ucs = np.zeros(neq + 1, np.int32)
    lcs = np.zeros(neq, np.int32)
    L.ov_oracle_netinfo(tag.encode(), _p(info), _p(perm), _p(ri), _p(ucs), _p(lcs))
    return {"neq": neq, "nnz": nnz, "nrea": int(info[2]), "dense": bool(info[3]),
            "idx_tgas": int(info[4]), "perm": perm, "row_index": ri, "u_col_start": ucs,
            "l_col_start": lcs}


def tags():
    L = lib()
    return [L.ov_oracle_net_tag(i).decode() for i in range(L.ov_oracle_num_nets())]


def solve(tag, y, t, dt, t_stop, rtol, atol, dt_min, group=1, check_negatives=False,
          mask=None, max_attempts=1000000, nthreads=0, fix_restart=False, ws=None, resume=False,
          libm=False, fast=False):
    """SolveODE on all cells.  y: (neq, ncells) float64, modified copy returned
    with t, dt, status, stats.  ws: a workspace from workspace() to save the
    integrator state into (and, with resume, to continue from); resume
    "en_old" (or 2): a fresh start keeping the previous call's last Newton
    correction from ws, as the reference's solver object does.  libm: the
    oracle variant with the C library's exp/log/log10/pow; fast: the -O3
    -march=native build (CPU baseline timing only)."""
    y = np.ascontiguousarray(y, dtype=np.float64).copy()
    ncells = y.shape[1]
    t = np.ascontiguousarray(np.broadcast_to(t, (ncells,)), dtype=np.float64).copy()
    dt = np.ascontiguousarray(np.broadcast_to(dt, (ncells,)), dtype=np.float64).copy()
    t_stop = np.ascontiguousarray(np.broadcast_to(t_stop, (ncells,)), dtype=np.float64).copy()
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    status = np.zeros(ncells, np.int32)
    stats = np.zeros((ncells, OV_NSTATS), np.int32)
    rc = lib(libm, fast).ov_oracle_solve(tag.encode(), ncells, group, rtol, atol, dt_min,
                               int(bool(check_negatives)), int(bool(fix_restart)), max_attempts,
                               _p(y), _p(t), _p(dt),
                               _p(t_stop), _p(m), _p(status), _p(stats), nthreads, _p(ws),
                               {False: 0, True: 1, 2: 2, "en_old": 2}[resume])
    if rc != 0:
        raise ValueError("oracle solve failed rc=%d" % rc)
    return y, t, dt, status, stats


def evaluate(tag, y, k, beta, dt):
    info = netinfo(tag)
    y = np.ascontiguousarray(y, np.float64)
    k = np.ascontiguousarray(k if len(k) else [0.0], np.float64)
    f = np.zeros(info["neq"])
    a = np.zeros(info["nnz"])
    lib().ov_oracle_eval(tag.encode(), _p(y), _p(k), beta, dt, _p(f), _p(a))
    return f, a


def rates(T):
    r = np.zeros(38)
    lib().ov_oracle_rates(float(T), _p(r))
    return r


def workspace(tag, ncells, group=1):
    n = lib().ov_oracle_ws_doubles(tag.encode(), ncells, group)
    if n < 0:
        raise ValueError("bad workspace request")
    return np.zeros(n, np.float64)


def convert(tag, a, rho, direction):
    """Mass fractions -> number densities (direction 0) or back (1),
    tests/primordial.f90:117-140; a: (neq, ncells)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    out = np.empty_like(a)
    rc = lib().ov_oracle_convert(tag.encode(), a.shape[1], direction, _p(a), _p(out), _p(rho))
    if rc:
        raise ValueError("convert(%s): code %d" % (tag, rc))
    return out


def ladder(tag, y, time, dt, t_stops, rtol, atol, dt_min, rho=None, dt_reset=None, group=1,
           nthreads=0):
    """The reference drivers' loop (tests/rober.f90:57-62, tests/orego.f90:
    117-123, tests/primordial.f90:76-92): one SolveODE per entry of t_stops,
    time and dt carried from call to call (dt set to dt_reset before each
    call when given), and, with rho, the state kept as mass fractions and
    converted to number densities around each call.  Where the reference
    stops the program, a failed cell here keeps its first status and is
    masked out of the later calls.  Returns (y, time, dt, status)."""
    y = np.array(y, dtype=np.float64)
    ncells = y.shape[1]
    t = np.broadcast_to(np.asarray(time, dtype=np.float64), (ncells,)).copy()
    d = np.broadcast_to(np.asarray(dt, dtype=np.float64), (ncells,)).copy()
    failed = np.zeros(ncells, np.int32)
    for k, ts in enumerate(t_stops):
        if dt_reset is not None:
            d[:] = dt_reset
        n = convert(tag, y, rho, 0) if rho is not None else y
        mask = None if k == 0 else (failed == 0).astype(np.uint8)
        n, t, d, st, _ = solve(tag, n, t, d, np.full(ncells, ts), rtol, atol, dt_min, group=group,
                               mask=mask, nthreads=nthreads)
        failed = np.where(failed != 0, failed, st).astype(np.int32)
        y = convert(tag, n, rho, 1) if rho is not None else n
    return y, t, d, failed
