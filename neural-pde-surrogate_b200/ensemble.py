"""Batched ensemble of independent grids on the GPU (fv_ensemble_* in include/fv.h).

The reference runs the solver once per trajectory, as separate processes (data/generate.py:60-105,
experiments/solver_baseline.py:116-117).  Here many members of uneven sizes advance together, each
with its own CFL dt, and each is bit-identical to its own single-grid run.

    ens = Ensemble(grids, "hllc", "vanleer")
    ens.set_state(k, U_k)                 # (ny_k, nx_k, 4) float64
    t, steps, status = ens.advance_to(0.25)
    U = ens.get_state(k)
"""
import ctypes as C

import numpy as np

from ._lib import FV_ERR_NONPHYSICAL, FVError, StreamOrder, check, device_ptr, lib
from .solver import FLUXES, LIMITERS


class Ensemble:
    def __init__(self, grids, flux="hllc", limiter="vanleer", cfl=0.5, stream=None):
        """grids: list of solver.Grid (or objects with nx, ny, x_min, x_max, y_min, y_max, bc_x, bc_y)."""
        self.grids = list(grids)
        n = len(self.grids)
        nx = (C.c_int * n)(*[g.nx for g in self.grids])
        ny = (C.c_int * n)(*[g.ny for g in self.grids])
        bx = (C.c_int * n)(*[g.bc_x for g in self.grids])
        by = (C.c_int * n)(*[g.bc_y for g in self.grids])
        bounds = (C.c_double * (4 * n))(*[v for g in self.grids for v in (g.x_min, g.x_max, g.y_min, g.y_max)])
        h = C.c_void_p()
        check(lib().fv_ensemble_create(n, nx, ny, bounds, bx, by, FLUXES[flux], LIMITERS[limiter], float(cfl),
                                       C.c_void_p(stream) if stream else None, C.byref(h)))
        self._h = h
        self.count = n
        self._order = StreamOrder(lib().fv_ensemble_get_stream, h)

    def close(self):
        if getattr(self, "_h", None):
            lib().fv_ensemble_destroy(self._h)
            self._h = None

    __del__ = close

    def __len__(self):
        return self.count

    def set_state(self, k, U):
        g = self.grids[k]
        if hasattr(U, "data_ptr") and getattr(U, "is_cuda", False):
            ptr = device_ptr(U, (g.ny, g.nx, 4), what=f"member {k} state")
            self._order.before()
            check(lib().fv_ensemble_set_state_device(self._h, int(k), ptr))
            return
        U = np.ascontiguousarray(U, np.float64)
        if U.shape != (g.ny, g.nx, 4):
            raise ValueError(f"member {k}: state must have shape {(g.ny, g.nx, 4)}")
        check(lib().fv_ensemble_set_state(self._h, int(k), C.c_void_p(U.ctypes.data)))

    def set_all(self, U):
        """All members from one CUDA float64 tensor holding their states back to back in member order
        (e.g. shape (count, ny, nx, 4) when all members have one size)."""
        ptr = device_ptr(U, numel=4 * sum(g.nx * g.ny for g in self.grids), what="states")
        self._order.before()  # U may still be being written on torch's stream
        check(lib().fv_ensemble_set_all_device(self._h, ptr))

    def get_all(self, out):
        """All members' states into a CUDA float64 tensor (layout of set_all)."""
        ptr = device_ptr(out, numel=4 * sum(g.nx * g.ny for g in self.grids), what="out")
        self._order.before()  # torch may still be reading out's previous contents
        check(lib().fv_ensemble_get_all_device(self._h, ptr))
        self._order.after()  # torch work on out waits for the copy
        return out

    def get_state(self, k):
        g = self.grids[k]
        out = np.empty((g.ny, g.nx, 4), np.float64)
        check(lib().fv_ensemble_get_state(self._h, int(k), C.c_void_p(out.ctypes.data)))
        return out

    def advance_to(self, t_next, raise_on_nonphysical=True):
        """Advance every member to t_next (a scalar or one value per member).  Returns
        (t, steps, status) arrays; status 3 marks a member stopped at a non-physical state."""
        tn = np.ascontiguousarray(np.broadcast_to(np.asarray(t_next, np.float64), (self.count,)))
        t = np.empty(self.count, np.float64)
        steps = np.empty(self.count, np.int64)
        status = np.empty(self.count, np.int32)
        rc = lib().fv_ensemble_advance_to(self._h, C.c_void_p(tn.ctypes.data), C.c_void_p(t.ctypes.data),
                                          C.c_void_p(steps.ctypes.data), C.c_void_p(status.ctypes.data))
        if rc == FV_ERR_NONPHYSICAL and not raise_on_nonphysical:
            return t, steps, status
        check(rc)
        return t, steps, status

    def launch_count(self):
        n = C.c_longlong()
        check(lib().fv_ensemble_launch_count(self._h, C.byref(n)))
        return n.value


__all__ = ["Ensemble", "FVError"]
