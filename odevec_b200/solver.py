"""Python host side of the solve path: ctypes over libodevec_b200.so.

Mirrors the reference's Fortran interface (src/odevec.F90):

* ``Odevec`` - the ``type(odevec)`` object, with the caller-set fields
  ``RelativeTolerance``, ``AbsoluteTolerance``, ``MinimalTimestep`` and
  ``CheckNegatives`` (``src/odevec.F90:48-52``), plus ``nvector`` (the
  lockstep group size, 1 or 32), ``neq`` and the precision form;
* ``InitOdevec(ode)`` (``:94-154``), ``SolveODE(ode, time, dt, t_stop, y,
  Mask=None)`` (``:158-214``) and ``CloseOdevec(ode)`` (``:1058-1074``).

``SolveODE`` takes ``y`` as an ``(ncells, neq)`` or ``(neq, ncells)`` view
of the reference's ``y(nvector, neq)`` array - species-major storage,
``y[s * ncells + c]`` - either as a torch CUDA tensor (solved in place on
the device, on torch's current stream) or as a NumPy array (copied to the
GPU and back through ``odevec_solve_host``).  ``time`` and ``dt`` are
updated like the Fortran ``intent(inout)`` arguments; scalars are broadcast
to all cells.

Where the reference stops the program (``print`` + ``stop``) this raises
``OdevecError`` carrying the per-cell status codes, unless
``raise_on_failure`` is False.  The product path always runs the CUDA
kernels: importing this module or creating a solver fails loudly when the
library is missing or no GPU is visible.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libodevec_b200.so")

OV_OK = 0
STATUS_NAMES = {
    0: "OK",
    1: "DT_MIN_PREDICTOR",
    2: "CONV_FAILURES",
    3: "DT_MIN_CONV",
    4: "MAX_STEPS",
    5: "ORDER",
    6: "GROUP_MISMATCH",
}
OV_NSTATS = 8
STAT_NAMES = ["steps", "attempts", "lte_fails", "conv_fails", "newton_iters", "jac_evals",
              "order", "reserved"]
PREC = {"fp64": 0, "fp64_fma": 1, "fp32_lu": 2}


class OdevecError(RuntimeError):
    def __init__(self, msg, status=None):
        super().__init__(msg)
        self.status = status


class _Opts(ctypes.Structure):
    _fields_ = [("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("dt_min", ctypes.c_double),
                ("check_negatives", ctypes.c_int32), ("group_size", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("max_attempts", ctypes.c_int32),
                ("jac_batch", ctypes.c_int32), ("ss_batch", ctypes.c_int32), ("max_wait", ctypes.c_int32),
                ("staging", ctypes.c_int32), ("block_threads", ctypes.c_int32), ("grid_blocks", ctypes.c_int32),
                ("fix_restart", ctypes.c_int32), ("no_escalation", ctypes.c_int32)]


class _Job(ctypes.Structure):
    """odevec_job (include/odevec_b200.h)"""
    _fields_ = [("solver", ctypes.c_void_p), ("ncells", ctypes.c_int64), ("y", ctypes.c_void_p),
                ("t", ctypes.c_void_p), ("dt", ctypes.c_void_p), ("t_stop", ctypes.c_void_p),
                ("mask", ctypes.c_void_p), ("status", ctypes.c_void_p), ("stats", ctypes.c_void_p),
                ("workspace", ctypes.c_void_p), ("resume", ctypes.c_int32)]


_lib = None


def lib():
    """The loaded C-ABI library (built in-tree by odevec_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise OdevecError("libodevec_b200.so not found at %s: run `python -m odevec_b200.build`"
                              % LIBPATH)
        L = ctypes.CDLL(LIBPATH)
        P, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        L.odevec_num_networks.restype = i32
        L.odevec_network_tag.restype = ctypes.c_char_p
        L.odevec_network_tag.argtypes = [i32]
        L.odevec_network_info.argtypes = [ctypes.c_char_p, P]
        L.odevec_network_info.restype = i32
        L.odevec_init.argtypes = [ctypes.c_char_p, i64, ctypes.POINTER(_Opts), ctypes.POINTER(P)]
        L.odevec_init.restype = i32
        L.odevec_set_options.argtypes = [P, ctypes.POINTER(_Opts)]
        L.odevec_set_options.restype = i32
        L.odevec_solve.argtypes = [P, i64, P, P, P, P, P, P, P, P]
        L.odevec_solve.restype = i32
        L.odevec_solve_host.argtypes = [P, i64, P, P, P, P, P, P, P]
        L.odevec_solve_host.restype = i32
        L.odevec_workspace_doubles.argtypes = [ctypes.c_char_p, ctypes.POINTER(i64)]
        L.odevec_workspace_doubles.restype = i32
        L.odevec_solve_resident.argtypes = [P, i64, P, P, P, P, P, P, P, P, i32, P]
        L.odevec_solve_resident.restype = i32
        L.odevec_close.argtypes = [P]
        L.odevec_close.restype = i32
        L.odevec_convert.argtypes = [ctypes.c_char_p, i64, i32, P, P, P, P]
        L.odevec_convert.restype = i32
        L.odevec_last_error.restype = ctypes.c_char_p
        L.odevec_solve_range.argtypes = [P, i64, i64, P, P, P, P, P, P, P, P, i32, P]
        L.odevec_solve_range.restype = i32
        L.odevec_solve_many.argtypes = [ctypes.POINTER(_Job), i32, P]
        L.odevec_solve_many.restype = i32
        L.odevec_set_yield.argtypes = [P, P]
        L.odevec_set_yield.restype = i32
        L.odevec_solve_continue.argtypes = [P, i64, i64, P, P, P, P, P, P, P, P, i32, P]
        L.odevec_solve_continue.restype = i32
        L.odevec_cells_started.argtypes = [P, P, ctypes.POINTER(i64)]
        L.odevec_cells_started.restype = i32
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise OdevecError("odevec: %s (code %d)" % (lib().odevec_last_error().decode(), rc))


def networks():
    L = lib()
    return [L.odevec_network_tag(i).decode() for i in range(L.odevec_num_networks())]


def network_info(tag):
    info = np.zeros(6, np.int32)
    _check(lib().odevec_network_info(tag.encode(), info.ctypes.data_as(ctypes.c_void_p)))
    return {"neq": int(info[0]), "nnz": int(info[1]), "nrea": int(info[2]), "dense": bool(info[3]),
            "idx_tgas": int(info[4]), "nvector": int(info[5])}


# resident blocks per SM of each staging (block size x blocks: the launch
# shape the kernel is compiled for; 0 = the library's automatic choice, 3)
BLOCKS_PER_SM = {0: 3, 1: 2, 2: 1, 3: 3, 4: 4, 5: 1, 6: 1, 7: 3, 8: 1, 9: 1, 10: 1, 11: 1, 12: 1, 13: 2, 14: 1, 15: 1, 16: 1, 17: 1, 18: 1, 19: 1, 20: 3, 21: 3}
# cells one block of each staging holds at a time (thread per cell: the block
# size; 32, 16 or 8 lanes per cell: 8, 16 or 32 cells in 8 warps)
CELLS_PER_BLOCK = {0: 128, 1: 128, 2: 128, 3: 128, 4: 128, 5: 192, 6: 384, 7: 8, 8: 384, 9: 256, 10: 320, 11: 192,
                   12: 384, 13: 16, 14: 32, 15: 256, 16: 512, 17: 384, 18: 256, 19: 384, 20: 128, 21: 128}


class Odevec:
    """The solver object (``type(odevec)``, src/odevec.F90:33-74)."""

    def __init__(self, network: str, max_cells: int = 0, RelativeTolerance: float = 1e-4,
                 AbsoluteTolerance: float = 1e-20, MinimalTimestep: Optional[float] = None,
                 CheckNegatives: bool = False, nvector: Optional[int] = None,
                 precision: str = "fp64", max_attempts: int = 0, raise_on_failure: bool = True,
                 jac_batch: int = 0, ss_batch: int = 0, max_wait: int = 0, staging: int = 0,
                 block_threads: int = 0, grid_blocks: int = 0, fix_restart: bool = False,
                 escalation: bool = True, autotune: bool = True):
        info = network_info(network)
        self.network = network
        self.neq = info["neq"]
        self.nnz = info["nnz"]
        self.nrea = info["nrea"]
        self.idx_tgas = info["idx_tgas"]
        self.nvector = info["nvector"] if nvector is None else int(nvector)
        self.max_cells = int(max_cells)
        self.RelativeTolerance = RelativeTolerance
        self.AbsoluteTolerance = AbsoluteTolerance
        self.MinimalTimestep = MinimalTimestep
        self.CheckNegatives = CheckNegatives
        self.precision = precision
        self.max_attempts = max_attempts
        self.raise_on_failure = raise_on_failure
        self.jac_batch = jac_batch
        self.ss_batch = ss_batch
        self.max_wait = max_wait
        self.staging = staging
        self.block_threads = block_threads
        self.grid_blocks = grid_blocks
        self.fix_restart = fix_restart
        self.escalation = escalation
        # launch options left at 0 are taken from the autotuner's table at
        # InitOdevec (odevec_b200/autotune.py); they never change results
        self.autotune = autotune
        self.status = None
        self.stats = None
        self._h = None

    def _opts(self):
        o = _Opts()
        o.rtol = float(self.RelativeTolerance)
        o.atol = float(self.AbsoluteTolerance)
        o.dt_min = -1.0 if self.MinimalTimestep is None else float(self.MinimalTimestep)
        o.check_negatives = 1 if self.CheckNegatives else 0
        o.group_size = int(self.nvector)
        if self.precision not in PREC:
            raise ValueError("precision must be one of %s" % list(PREC))
        o.precision = PREC[self.precision]
        o.max_attempts = int(self.max_attempts)
        o.jac_batch = int(self.jac_batch)
        o.ss_batch = int(self.ss_batch)
        o.max_wait = int(self.max_wait)
        o.staging = int(self.staging)
        o.block_threads = int(self.block_threads)
        o.grid_blocks = int(self.grid_blocks)
        o.fix_restart = 1 if self.fix_restart else 0
        o.no_escalation = 0 if self.escalation else 1
        return o

    @property
    def handle(self):
        if self._h is None:
            raise OdevecError("InitOdevec has not been called")
        return self._h


def InitOdevec(ode: Odevec) -> Odevec:
    """Creates the device-side solver (src/odevec.F90:94-154)."""
    import torch
    if not torch.cuda.is_available():
        raise OdevecError("odevec_b200 needs a CUDA GPU; none is visible")
    torch.cuda.init()
    if ode.autotune:
        from . import autotune
        autotune.apply(ode)
    h = ctypes.c_void_p()
    o = ode._opts()
    _check(lib().odevec_init(ode.network.encode(), ode.max_cells, ctypes.byref(o), ctypes.byref(h)))
    ode._h = h
    return ode


def CloseOdevec(ode: Odevec) -> None:
    """Frees the device-side solver (src/odevec.F90:1058-1074)."""
    if ode._h is not None:
        lib().odevec_close(ode._h)
        ode._h = None


def _as_cells(a, ncells, name, torch_mod=None, device=None):
    if torch_mod is not None:
        if not torch_mod.is_tensor(a):
            a = torch_mod.full((ncells,), float(a), dtype=torch_mod.float64, device=device)
        elif a.dim() == 0 or a.numel() == 1:
            a = a.reshape(1).to(device=device, dtype=torch_mod.float64).expand(ncells).contiguous()
        if a.dtype != torch_mod.float64 or not a.is_contiguous() or a.numel() != ncells:
            raise ValueError("%s must be a contiguous float64 tensor of %d cells" % (name, ncells))
        return a
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 0 or a.size == 1:
        return np.full(ncells, float(a), np.float64)
    if a.size != ncells:
        raise ValueError("%s must have %d entries" % (name, ncells))
    return np.ascontiguousarray(a)


def workspace_doubles(network: str) -> int:
    n = ctypes.c_int64()
    _check(lib().odevec_workspace_doubles(network.encode(), ctypes.byref(n)))
    return int(n.value)


def Workspace(ode: Odevec, ncells: int, device=None):
    """Device buffer for the resident integrator state of ncells cells."""
    import torch
    return torch.zeros(workspace_doubles(ode.network) * ncells, dtype=torch.float64,
                       device=device or "cuda")


def SolveODE(ode: Odevec, time, dt, t_stop, y, Mask=None, stream=None, want_stats=True,
             workspace=None, resume=False, in_place=False):
    """Integrates every cell from ``time`` to ``t_stop`` (src/odevec.F90:158-214).

    ``y``: species-major storage of ``ncells x neq`` values: a torch CUDA
    tensor or NumPy array of shape ``(neq, ncells)`` (C order), solved in
    place.  ``time``/``dt``: scalars or per-cell arrays; returns
    ``(time, dt)`` after the solve (``time == t_stop``).  ``Mask``: optional
    per-cell booleans.  Per-cell status and statistics are left in
    ``ode.status`` / ``ode.stats``.

    ``workspace`` (from :func:`Workspace`) keeps each cell's integrator state
    between calls.  ``resume``: False/0 starts fresh and saves the state;
    True/1 continues from the saved state; ``"en_old"``/2 starts fresh but
    keeps the previous call's last Newton correction, as the reference's
    solver object does between SolveODE calls (this%en_old is never reset).

    NumPy arrays go through ``odevec_solve_host``; those in pinned host
    memory are read and written by the kernel in place (no copies).
    ``in_place`` (NumPy only): ``time`` and ``dt`` are per-cell float64
    arrays updated in place, as the Fortran SolveODE's intent(inout)
    arguments are, instead of returned copies.
    """
    resume_code = {False: 0, True: 1, 2: 2, "en_old": 2}[resume]
    h = ode.handle
    is_torch = False
    try:
        import torch
        is_torch = torch.is_tensor(y)
    except ImportError:
        torch = None
    if y.ndim != 2 or y.shape[0] != ode.neq:
        raise ValueError("y must have shape (neq=%d, ncells)" % ode.neq)
    ncells = int(y.shape[1])
    o = ode._opts()
    _check(lib().odevec_set_options(h, ctypes.byref(o)))
    if is_torch:
        if not y.is_cuda or y.dtype != torch.float64 or not y.is_contiguous():
            raise ValueError("y must be a contiguous float64 CUDA tensor")
        dev = y.device
        t = _as_cells(time, ncells, "time", torch, dev)
        d = _as_cells(dt, ncells, "dt", torch, dev)
        ts = _as_cells(t_stop, ncells, "t_stop", torch, dev)
        m = None
        if Mask is not None:
            m = torch.as_tensor(Mask, device=dev).to(torch.uint8).contiguous()
        status = torch.empty(ncells, dtype=torch.int32, device=dev)
        stats = torch.empty((ncells, OV_NSTATS), dtype=torch.int32, device=dev) if want_stats else None
        st = stream if stream is not None else torch.cuda.current_stream(dev)
        ptr = lambda a: None if a is None else ctypes.c_void_p(a.data_ptr())
        with torch.cuda.device(dev):
            if workspace is None:
                _check(lib().odevec_solve(h, ncells, ptr(y), ptr(t), ptr(d), ptr(ts), ptr(m),
                                          ptr(status), ptr(stats), ctypes.c_void_p(st.cuda_stream)))
            else:
                if workspace.numel() < workspace_doubles(ode.network) * ncells or not workspace.is_cuda:
                    raise ValueError("workspace too small: use Workspace(ode, ncells)")
                _check(lib().odevec_solve_resident(h, ncells, ptr(y), ptr(t), ptr(d), ptr(ts), ptr(m),
                                                   ptr(status), ptr(stats), ptr(workspace),
                                                   resume_code,
                                                   ctypes.c_void_p(st.cuda_stream)))
        ode.status, ode.stats = status, stats
        if ode.raise_on_failure:
            bad = int((status != 0).sum().item())
            if bad:
                raise OdevecError("SolveODE: %d cells failed (first status %s)"
                                  % (bad, STATUS_NAMES.get(int(status[status != 0][0].item()))), status)
        return t, d
    # host arrays: copy in, solve, copy out (odevec_solve_host)
    if not isinstance(y, np.ndarray) or y.dtype != np.float64 or not y.flags.c_contiguous:
        raise ValueError("y must be a C-contiguous float64 NumPy array or a CUDA tensor")
    if ncells > ode.max_cells:
        raise ValueError("ncells %d > max_cells %d given at InitOdevec" % (ncells, ode.max_cells))
    if in_place:
        for a, nm in ((time, "time"), (dt, "dt")):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
                    and a.flags.writeable and a.shape == (ncells,)):
                raise ValueError("in_place needs %s as a writable C-contiguous float64 array of %d cells"
                                 % (nm, ncells))
        t, d = time, dt
    else:
        t = _as_cells(time, ncells, "time").copy()
        d = _as_cells(dt, ncells, "dt").copy()
    ts = _as_cells(t_stop, ncells, "t_stop")
    m = None if Mask is None else np.ascontiguousarray(Mask, dtype=np.uint8)
    status = np.zeros(ncells, np.int32)
    stats = np.zeros((ncells, OV_NSTATS), np.int32) if want_stats else None
    p = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
    _check(lib().odevec_solve_host(h, ncells, p(y), p(t), p(d), p(ts), p(m), p(status), p(stats)))
    ode.status, ode.stats = status, stats
    if ode.raise_on_failure and np.any(status != 0):
        bad = int(np.sum(status != 0))
        raise OdevecError("SolveODE: %d cells failed (first status %s)"
                          % (bad, STATUS_NAMES.get(int(status[status != 0][0]))), status)
    return t, d


def SolveODERange(ode: Odevec, c0: int, c1: int, t, dt, t_stop, y, status, Mask=None, stream=None,
                  workspace=None, resume=False, cont=False):
    """SolveODE on cells [c0, c1) of full-size CUDA tensors (odevec_solve_range):
    y (neq, ncells), t, dt, t_stop, status (int32) and Mask (uint8, or None)
    with one entry per cell, workspace from :func:`Workspace` for all ncells
    (or None).  Only the range is read and written; a large solve cut into
    ranges gives the results of the whole solve.  Asynchronous on `stream`.
    ``cont``: continue the previous call on the same range after it yielded
    (odevec_solve_continue; see :func:`set_yield`)."""
    import torch
    ncells = int(y.shape[1])
    if not (0 <= c0 <= c1 <= ncells):
        raise ValueError("range [%d, %d) outside %d cells" % (c0, c1, ncells))
    for a in (y, t, dt, t_stop, status) + ((Mask,) if Mask is not None else ()):
        if not (torch.is_tensor(a) and a.is_cuda and a.is_contiguous()):
            raise ValueError("SolveODERange takes contiguous CUDA tensors")
    o = ode._opts()
    _check(lib().odevec_set_options(ode.handle, ctypes.byref(o)))
    off = lambda a, k: None if a is None else ctypes.c_void_p(a.data_ptr() + k * a.element_size())
    st = stream if stream is not None else torch.cuda.current_stream(y.device)
    with torch.cuda.device(y.device):
        fn = lib().odevec_solve_continue if cont else lib().odevec_solve_range
        _check(fn(ode.handle, c1 - c0, ncells, off(y, c0), off(t, c0), off(dt, c0),
                                        off(t_stop, c0), off(Mask, c0), off(status, c0), None,
                                        off(workspace, c0), {False: 0, True: 1, 2: 2, "en_old": 2}[resume],
                                        ctypes.c_void_p(st.cuda_stream)))


def set_yield(ode: Odevec, flag=None):
    """Registers a yield flag (a one-element int32 CUDA tensor, or None;
    set it from another stream with a copy, e.g. ``flag.copy_(one_pinned,
    non_blocking=True)``, so that no SM is needed to write it):
    while it holds a nonzero value, the kernels of this solver's later solves
    start no new cells and their launch ends once the running cells are done
    (odevec_set_yield).  The solver keeps the pointer: keep the tensor alive."""
    ode._yield_flag = flag
    _check(lib().odevec_set_yield(ode.handle, None if flag is None else ctypes.c_void_p(flag.data_ptr())))


def cells_started(ode: Odevec, stream=None) -> int:
    """Cells the current solve has started (>= ncells: all); synchronises
    `stream` (odevec_cells_started)."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    n = ctypes.c_int64(0)
    _check(lib().odevec_cells_started(ode.handle, ctypes.c_void_p(st.cuda_stream), ctypes.byref(n)))
    return int(n.value)
