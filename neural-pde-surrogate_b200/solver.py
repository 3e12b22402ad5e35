"""Python mirror of the reference solver's interface, running on the B200 through libfv.

The reference (GusGus2004/neural-pde-surrogate, solver/src) exposes

    Grid g = make_grid(nx, ny, x_min, x_max, y_min, y_max, bc_x, bc_y);   // grid2d.hpp:30-39
    Solver solver(g, hllc_flux, van_leer, cfl);                          // solver2d.hpp:61-64
    double dt = solver.compute_dt(U);                                    // solver2d.hpp:67-83
    solver.step(U, dt);                                                  // solver2d.hpp:86-103

with the flux and limiter chosen by name in the driver (main2d.cpp:145-155).  Here the same names
map onto one libfv handle whose state lives in device memory; compute_dt/step take the state as an
optional argument, so code written against the reference (U passed in, updated in place) runs
unchanged, while code that keeps the state on the GPU simply omits it.

State arrays: float64, shape (ny, nx, 4) -- (rho, rho*u, rho*v, E) of the interior cells.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import BadCell, StreamOrder, check, device_ptr, host_out_ptr, lib

FLUXES = {"rusanov": 0, "hllc": 1}            # main2d.cpp:145-148
LIMITERS = {"none": 0, "unlimited": 1, "minmod": 2, "vanleer": 3}  # main2d.cpp:150-155


class BC:
    """grid2d.hpp:7"""
    Transmissive = 0
    Periodic = 1
    names = {"transmissive": 0, "periodic": 1}


@dataclass
class Grid:
    """grid2d.hpp:12-28 (the ghost ring is implicit: boundaries are applied inside the kernels)."""
    nx: int
    ny: int
    x_min: float = 0.0
    x_max: float = 1.0
    y_min: float = 0.0
    y_max: float = 1.0
    bc_x: int = BC.Transmissive
    bc_y: int = BC.Transmissive

    @property
    def dx(self):
        return (self.x_max - self.x_min) / self.nx

    @property
    def dy(self):
        return (self.y_max - self.y_min) / self.ny

    def xc(self, i):
        return self.x_min + (np.asarray(i) + 0.5) * self.dx

    def yc(self, j):
        return self.y_min + (np.asarray(j) + 0.5) * self.dy


def make_grid(nx, ny, x_min, x_max, y_min, y_max, bc_x, bc_y):
    """grid2d.hpp:30-39.  bc_x/bc_y: BC.* or 'periodic'/'transmissive'."""
    bc_x = BC.names[bc_x] if isinstance(bc_x, str) else int(bc_x)
    bc_y = BC.names[bc_y] if isinstance(bc_y, str) else int(bc_y)
    return Grid(int(nx), int(ny), float(x_min), float(x_max), float(y_min), float(y_max), bc_x, bc_y)


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class Solver:
    """Solver(grid, flux, limiter, cfl): flux in {'hllc','rusanov'}, limiter in {'none','minmod',
    'vanleer','unlimited'} (the driver's option names, main2d.cpp:25-28)."""

    def __init__(self, grid, flux="hllc", limiter="vanleer", cfl=0.5, stream=None):
        if flux not in FLUXES:
            raise ValueError(f"Unknown scheme '{flux}' (use rusanov or hllc)")
        if limiter not in LIMITERS:
            raise ValueError(f"Unknown limiter '{limiter}'")
        self.grid, self.flux, self.limiter, self.cfl = grid, flux, limiter, float(cfl)
        h = C.c_void_p()
        check(lib().fv_create(grid.nx, grid.ny, grid.x_min, grid.x_max, grid.y_min, grid.y_max, grid.bc_x,
                              grid.bc_y, FLUXES[flux], LIMITERS[limiter], self.cfl,
                              C.c_void_p(stream) if stream else None, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().fv_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def shape(self):
        return (self.grid.ny, self.grid.nx, 4)

    # --- state ---------------------------------------------------------------------------------
    def set_state(self, U):
        """U: host ndarray (ny, nx, 4) float64, or a CUDA torch tensor of that shape."""
        if hasattr(U, "data_ptr") and getattr(U, "is_cuda", False):
            ptr = device_ptr(U, self.shape, what="state")
            self._order().before()
            check(lib().fv_set_state_device(self._h, ptr))
            return
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != self.shape:
            raise ValueError(f"state must have shape {self.shape}, got {U.shape}")
        check(lib().fv_set_state(self._h, _ptr(U)))

    def _order(self):
        if getattr(self, "_stream_order", None) is None:
            self._stream_order = StreamOrder(lib().fv_get_stream, self._h)
        return self._stream_order

    def set_primitive(self, rho, u, v, p):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, v, p)]
        for a in arrs:
            if a.shape != self.shape[:2]:
                raise ValueError(f"primitive fields must have shape {self.shape[:2]}")
        check(lib().fv_set_primitive(self._h, *[_ptr(a) for a in arrs]))

    def get_state(self, out=None):
        if out is not None and hasattr(out, "data_ptr") and getattr(out, "is_cuda", False):
            ptr = device_ptr(out, self.shape, what="out")
            self._order().before()
            check(lib().fv_get_state_device(self._h, ptr))
            self._order().after()
            return out
        out = np.empty(self.shape, np.float64) if out is None else out
        check(lib().fv_get_state(self._h, host_out_ptr(out, self.shape, np.float64)))
        return out

    def set_time(self, t):
        check(lib().fv_set_time(self._h, float(t)))

    def time(self):
        t, n = C.c_double(), C.c_longlong()
        check(lib().fv_get_time(self._h, C.byref(t), C.byref(n)))
        return t.value, n.value

    # --- the reference interface -------------------------------------------------------------------
    def compute_dt(self, U=None):
        """solver2d.hpp:67-83; raises NonPhysicalError where the reference exits."""
        if U is not None:
            self.set_state(U)
        dt, bad = C.c_double(), BadCell()
        check(lib().fv_compute_dt(self._h, C.byref(dt), C.byref(bad)), bad)
        return dt.value

    def step(self, U=None, dt=None):
        """solver2d.hpp:86-103.  step(U, dt) updates the host array U in place, like the reference;
        step(dt=...) or step(None, dt) advances the device-resident state."""
        if dt is None:
            U, dt = None, U
        if U is not None:
            self.set_state(U)
        check(lib().fv_step(self._h, float(dt)))
        if U is not None:
            self.get_state(out=U)

    def advance_to(self, t_next):
        """main2d.cpp:237-242 on the device.  Returns (t, total steps)."""
        t, n, bad = C.c_double(), C.c_longlong(), BadCell()
        check(lib().fv_advance_to(self._h, float(t_next), C.byref(t), C.byref(n), C.byref(bad)), bad)
        return t.value, n.value

    def block_average(self, factor, out=None):
        """trajectory.hpp:31-51 for one level: (4, ny/f, nx/f) float32."""
        shape = (4, self.grid.ny // factor, self.grid.nx // factor)
        if out is not None and hasattr(out, "data_ptr") and getattr(out, "is_cuda", False):
            ptr = device_ptr(out, shape, dtype="torch.float32", what="out")
            self._order().before()
            check(lib().fv_block_average_device(self._h, int(factor), ptr))
            self._order().after()
            return out
        out = np.empty(shape, np.float32) if out is None else out
        check(lib().fv_block_average(self._h, int(factor), host_out_ptr(out, shape, np.float32)))
        return out

    def run_trajectory(self, t_end, t_start=0.0, nout=1, sizes=None):
        """The driver in --traj mode (main2d.cpp:224-246): returns (times (nout+1,),
        {size: (nout+1, 4, ny_c, size) float32}, steps).  sizes default: [nx] (main2d.cpp:201)."""
        sizes = [self.grid.nx] if sizes is None else list(sizes)
        for m in sizes:  # trajectory.hpp:19-28
            if m <= 0 or self.grid.nx % m:
                raise ValueError(f"save size {m} does not divide nx = {self.grid.nx}")
            if self.grid.ny % (self.grid.nx // m):
                raise ValueError(f"save size {m} does not divide ny evenly")
        outs = {m: np.empty((nout + 1, 4, self.grid.ny // (self.grid.nx // m), m), np.float32) for m in sizes}
        times = np.empty(nout + 1, np.float64)
        arr = (C.c_int * len(sizes))(*sizes)
        ptrs = (C.c_void_p * len(sizes))(*[o.ctypes.data for o in outs.values()])
        steps, bad = C.c_longlong(), BadCell()
        check(lib().fv_run_trajectory(self._h, float(t_start), float(t_end), int(nout), arr, len(sizes), ptrs,
                                      _ptr(times), C.byref(steps), C.byref(bad)), bad)
        return times, outs, steps.value

    def synchronize(self):
        check(lib().fv_synchronize(self._h))


def riemann_flux(flux, UL, UR, face="x"):
    """Face fluxes on the GPU (riemann2d.hpp:8 FluxFn, or flux_y_face :42-44 for face='y').
    UL, UR: (..., 4) conserved states; returns F of the same shape."""
    UL = np.ascontiguousarray(UL, np.float64)
    UR = np.ascontiguousarray(UR, np.float64)
    if UL.shape != UR.shape or UL.ndim == 0 or UL.shape[-1] != 4:
        raise ValueError(f"UL and UR must have the same shape (..., 4), got {UL.shape} and {UR.shape}")
    F = np.empty_like(UL)
    check(lib().fv_riemann_flux(FLUXES[flux], 1 if face == "y" else 0, UL.size // 4, _ptr(UL), _ptr(UR), _ptr(F)))
    return F


DIVISIONS = {"general": 0, "gm1": 1, "zero": 2, "back": 3}  # FV_DIV_* of include/fv.h


def eval_division(a, b, kind="general"):
    """Elementwise quotients computed on the GPU by one of the stage kernels' division sequences
    (fv_eval_division_kind): 'general' is a / b at every general division site (IEEE in the parity
    build, the Newton-Raphson sequence in the tolerance build); 'gm1' is a / (GAMMA - 1) (b unused);
    'zero' is a / b with the zero-numerator fast path; 'back' is RN(RN(a*b)/a), a face state's
    velocity after the conserved/primitive round trip (a = rho, b = u)."""
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(np.zeros_like(a) if b is None else b, np.float64)
    if a.shape != b.shape:
        raise ValueError(f"a and b must have the same shape, got {a.shape} and {b.shape}")
    q = np.empty_like(a)
    check(lib().fv_eval_division_kind(DIVISIONS[kind], a.size, _ptr(a), _ptr(b), _ptr(q)))
    return q


def division_sweep(kind, n, seed=0):
    """Draws n operand pairs on the GPU and counts the quotients of division sequence `kind` that
    differ in any bit from IEEE division (fv_division_sweep).  Returns (mismatches, max ulps)."""
    mism, ulps = C.c_longlong(), C.c_longlong()
    check(lib().fv_division_sweep(DIVISIONS[kind], int(n), int(seed), C.byref(mism), C.byref(ulps)))
    return mism.value, ulps.value


def fill_ghosts(U, bc_x, bc_y):
    """(ny+4, nx+4, 4) ghosted array apply_bcs would build (grid2d.hpp:43-66), made on the GPU."""
    U = np.ascontiguousarray(U, np.float64)
    if U.ndim != 3 or U.shape[2] != 4:
        raise ValueError(f"U must have shape (ny, nx, 4), got {U.shape}")
    ny, nx = U.shape[:2]
    bc_x = BC.names[bc_x] if isinstance(bc_x, str) else int(bc_x)
    bc_y = BC.names[bc_y] if isinstance(bc_y, str) else int(bc_y)
    Ug = np.empty((ny + 4, nx + 4, 4), np.float64)
    check(lib().fv_fill_ghosts(nx, ny, bc_x, bc_y, _ptr(U), _ptr(Ug)))
    return Ug


def profile(solver, enable=True):
    """Bracket every stage-kernel launch of `solver` with CUDA events (fv_profile)."""
    check(lib().fv_profile(solver._h, 1 if enable else 0))


def profile_read(solver):
    """(mean ms of stage-1 launches, mean ms of stage-2 launches, steps timed) since profile(), for
    steps taken by the per-stage kernels (fv_step, or fv_advance_to with FV_STEPPER=0)."""
    a, b, n = C.c_double(), C.c_double(), C.c_longlong()
    check(lib().fv_profile_read(solver._h, C.byref(a), C.byref(b), C.byref(n)))
    return a.value, b.value, n.value


def profile_steps(solver):
    """(mean device ms per step, steps timed, stepper launches timed) since profile(), over both
    kernel paths (fv_profile_steps)."""
    ms, n, k = C.c_double(), C.c_longlong(), C.c_longlong()
    check(lib().fv_profile_steps(solver._h, C.byref(ms), C.byref(n), C.byref(k)))
    return ms.value, n.value, k.value


def stepper_tile(solver):
    """(tile width, height, threads) of the handle's persistent stepper; zeros before its first use."""
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    check(lib().fv_stepper_tile(solver._h, C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


def stepper_launch(solver):
    """(shape index, CTAs per SM, CTAs) of the handle's persistent stepper; (-1, 0, 0) before its
    first use."""
    v, per_sm, ctas = C.c_int(), C.c_int(), C.c_int()
    check(lib().fv_stepper_launch(solver._h, C.byref(v), C.byref(per_sm), C.byref(ctas)))
    return v.value, per_sm.value, ctas.value


def launch_count(solver):
    n = C.c_longlong()
    check(lib().fv_launch_count(solver._h, C.byref(n)))
    return n.value


def tile_variants():
    """[(tile width, tile height, threads)] of the stage-kernel tile shapes (fv_tile_variant)."""
    out = []
    k = 0
    while True:
        tx, ty, nt = C.c_int(), C.c_int(), C.c_int()
        if lib().fv_tile_variant(k, C.byref(tx), C.byref(ty), C.byref(nt)) != 0:
            return out
        out.append((tx.value, ty.value, nt.value))
        k += 1


def set_tile(solver, variant):
    check(lib().fv_set_tile(solver._h, int(variant)))


def get_tile(solver):
    v = C.c_int()
    check(lib().fv_get_tile(solver._h, C.byref(v)))
    return v.value


def autotune(solver, steps=8):
    """Re-time every tile shape on a copy of the solver's state; returns the chosen index."""
    v = C.c_int()
    check(lib().fv_autotune(solver._h, int(steps), C.byref(v)))
    return v.value
