"""CPU backend of the serving scheduler on the oracle (test infrastructure).

It has the interface of odevec_b200.serving.GpuBackend, and each step runs
synchronously on the CPU oracle, so the scheduler's admission, masking and
continuation logic can be tested without a GPU.
"""
import numpy as np

from odevec_b200.serving import Request, Result


class OracleBackend:
    """CPU stand-in with the same interface: each step runs synchronously on
    the oracle (used to test the scheduler without a GPU)."""

    def __init__(self, nthreads: int = 1):
        from oracle import oracle as O
        self.O = O
        self.nthreads = nthreads

    def bytes_needed(self, r: Request) -> float:
        return float(8 * r.y0.size + 8 * self.O.lib().ov_oracle_ws_doubles(r.network.encode(), r.ncells, 1))

    def admit(self, r: Request):
        return {"r": r, "y": r.y0.copy(), "t": np.zeros(r.ncells), "dt": np.full(r.ncells, r.dt_in),
                "ws": self.O.workspace(r.network, r.ncells), "failed": np.zeros(r.ncells, np.int32),
                "done": False}

    def launch(self, h, step: int, active: int = 1):
        r = h["r"]
        mask = None if step == 0 else (h["failed"] == 0).astype(np.uint8)
        y, t, dt, st, _ = self.O.solve(r.network, h["y"], h["t"], h["dt"], r.dt_hydro * (step + 1), r.rtol,
                                       r.atol, r.dt_min, mask=mask, ws=h["ws"], resume=step > 0,
                                       nthreads=self.nthreads)
        h["failed"] = np.where(h["failed"] != 0, h["failed"], st).astype(np.int32)
        h["y"], h["t"], h["dt"], h["done"] = y, t, dt, True

    def finished(self, h) -> bool:
        return h["done"]

    def release(self, h):
        return Result(h["y"], h["failed"])

    def close(self):
        pass
