"""ctypes wrappers for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU legs, as the checker.  Two
implementations share one interface:

* ``OracleSolver`` -- the plain-C restatement in oracle/fv_oracle.c (always available once built);
* ``RefSolver``    -- the reference's own solver core compiled in oracle/_ref (ref_harness.cpp).

State arrays are numpy float64 of shape (ny, nx, 4): (rho, rho*u, rho*v, E) per cell, row-major,
interior cells only -- the same layout the CUDA library takes.
"""
import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_D = C.c_double
_I = C.c_int
_P = C.c_void_p
_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)
_LLP = C.POINTER(C.c_longlong)

FLUX = {"rusanov": 0, "hllc": 1}
LIMITER = {"none": 0, "unlimited": 1, "minmod": 2, "vanleer": 3}
BC = {"transmissive": 0, "periodic": 1}


class NonPhysical(RuntimeError):
    """Raised where the reference prints 'Non-physical state in cell (i, j)' and exits."""

    def __init__(self, i, j, rho, p):
        super().__init__(f"Non-physical state in cell ({i}, {j}): rho = {rho:g}, p = {p:g}")
        self.i, self.j, self.rho, self.p = i, j, rho, p


def _dp(a):
    return a.ctypes.data_as(_DP)


_libs = {}


def _load(which):
    if which in _libs:
        return _libs[which]
    if which == "oracle":
        path = HERE / "libfvoracle.so"
        if not path.exists():
            from . import build_oracle  # noqa: F401  (package-relative when imported as oracle.oracle)
        lib = C.CDLL(str(path))
        pre = "orc_"
        lib.orc_create.restype = _P
        lib.orc_create.argtypes = [_I, _I, _D, _D, _D, _D, _I, _I, _I, _I, _D]
        lib.orc_primitive_to_state.argtypes = [_I, _DP, _DP, _DP, _DP, _DP]
        lib.orc_apply_bcs_ghosted.argtypes = [_I, _I, _I, _I, _DP]
        lib.orc_flux_x_physical.argtypes = [_DP, _DP]
        lib.orc_to_conserved.argtypes = [_DP, _DP]
        lib.orc_frame_time.restype = _D
        lib.orc_frame_time.argtypes = [_D, _D, _I, _I]
        lib.orc_dx.restype = _D
        lib.orc_dx.argtypes = [_P]
        lib.orc_dy.restype = _D
        lib.orc_dy.argtypes = [_P]
    else:
        path = HERE / "_ref" / "libfvref.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (reference tree absent when oracle/build_oracle.py ran)")
        lib = C.CDLL(str(path))
        pre = "ref_"
        lib.ref_create.restype = _P
        lib.ref_create.argtypes = [_I, _I, _D, _D, _D, _D, _I, _I, _I, _I, _D]
    getattr(lib, pre + "destroy").argtypes = [_P]
    getattr(lib, pre + "set_state").argtypes = [_P, _DP]
    getattr(lib, pre + "get_state").argtypes = [_P, _DP]
    getattr(lib, pre + "compute_dt").argtypes = [_P, _DP, _IP, _IP, _DP, _DP]
    getattr(lib, pre + "step").argtypes = [_P, _D]
    getattr(lib, pre + "advance_to").argtypes = [_P, _D, _DP, _LLP, _IP, _IP, _DP, _DP]
    getattr(lib, pre + "block_average").argtypes = [_P, _I, _FP]
    getattr(lib, pre + "apply_bcs_ghosted").argtypes = [_I, _I, _I, _I, _DP]
    getattr(lib, pre + "flux").argtypes = [_I, _DP, _DP, _DP]
    getattr(lib, pre + "flux_y").argtypes = [_I, _DP, _DP, _DP]
    getattr(lib, pre + "hllc_1d").argtypes = [_DP, _DP, _DP]
    getattr(lib, pre + "max_threads").restype = _I
    _libs[which] = (lib, pre)
    return _libs[which]


def ref_available():
    return (HERE / "_ref" / "libfvref.so").exists()


class _Base:
    which = "oracle"

    def __init__(self, nx, ny, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, bc_x="periodic", bc_y="periodic",
                 flux="hllc", limiter="vanleer", cfl=0.5):
        self._lib, self._pre = _load(self.which)
        self.nx, self.ny = int(nx), int(ny)
        self.dx = (x_max - x_min) / nx
        self.dy = (y_max - y_min) / ny
        self._h = self._f("create")(self.nx, self.ny, x_min, x_max, y_min, y_max, BC[bc_x], BC[bc_y],
                                    FLUX[flux], LIMITER[limiter], cfl)
        self.t = 0.0
        self.steps = 0

    def _f(self, name):
        return getattr(self._lib, self._pre + name)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._f("destroy")(h)
            self._h = None

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (self.ny, self.nx, 4)
        self._f("set_state")(self._h, _dp(U))

    def get_state(self):
        out = np.empty((self.ny, self.nx, 4), np.float64)
        self._f("get_state")(self._h, _dp(out))
        return out

    def compute_dt(self):
        dt, bi, bj, br, bp = _D(), _I(), _I(), _D(), _D()
        if self._f("compute_dt")(self._h, C.byref(dt), C.byref(bi), C.byref(bj), C.byref(br), C.byref(bp)):
            raise NonPhysical(bi.value, bj.value, br.value, bp.value)
        return dt.value

    def step(self, dt):
        self._f("step")(self._h, float(dt))

    def advance_to(self, t_next):
        t, n = _D(self.t), C.c_longlong(self.steps)
        bi, bj, br, bp = _I(), _I(), _D(), _D()
        rc = self._f("advance_to")(self._h, float(t_next), C.byref(t), C.byref(n), C.byref(bi), C.byref(bj),
                                   C.byref(br), C.byref(bp))
        self.t, self.steps = t.value, n.value
        if rc:
            raise NonPhysical(bi.value, bj.value, br.value, bp.value)
        return self.t

    def block_average(self, f):
        out = np.empty((4, self.ny // f, self.nx // f), np.float32)
        self._f("block_average")(self._h, int(f), out.ctypes.data_as(_FP))
        return out

    def run(self, t_end, t_start=0.0, nout=1, save=()):
        """Driver time loop (main2d.cpp:224-246): spin up to t_start, then nout frames to t_end.
        Returns (frame times, {size: (frames, 4, nyc, nxc) float32})."""
        times, levels = [], {m: [] for m in save}
        while self.t < t_start:
            self.advance_to(t_start)
        def out():
            times.append(self.t)
            for m in save:
                levels[m].append(self.block_average(self.nx // m))
        out()
        for k in range(1, nout + 1):
            self.advance_to(t_start + (t_end - t_start) * k / nout)
            out()
        return np.array(times), {m: np.stack(v) for m, v in levels.items()}

    def max_threads(self):
        return self._f("max_threads")()


class OracleSolver(_Base):
    which = "oracle"


class RefSolver(_Base):
    which = "ref"


def flux(face, scheme, UL, UR, which="oracle"):
    """One face flux: face 'x' -> flux(UL, UR); 'y' -> flux_y_face (riemann2d.hpp:42-44)."""
    lib, pre = _load(which)
    UL = np.ascontiguousarray(UL, np.float64)
    UR = np.ascontiguousarray(UR, np.float64)
    F = np.empty(4, np.float64)
    getattr(lib, pre + ("flux" if face == "x" else "flux_y"))(FLUX[scheme], _dp(UL), _dp(UR), _dp(F))
    return F


def hllc_1d(UL, UR, which="oracle"):
    lib, pre = _load(which)
    UL = np.ascontiguousarray(UL, np.float64)
    UR = np.ascontiguousarray(UR, np.float64)
    F = np.empty(3, np.float64)
    getattr(lib, pre + "hllc_1d")(_dp(UL), _dp(UR), _dp(F))
    return F


def apply_bcs_ghosted(Ug, bc_x, bc_y, which="oracle"):
    """Ug: (ny+4, nx+4, 4) ghosted array, filled in place (grid2d.hpp:43-66)."""
    lib, pre = _load(which)
    ny, nx = Ug.shape[0] - 4, Ug.shape[1] - 4
    assert Ug.dtype == np.float64 and Ug.flags.c_contiguous
    getattr(lib, pre + "apply_bcs_ghosted")(nx, ny, BC[bc_x], BC[bc_y], _dp(Ug))
    return Ug


def to_conserved(rho, u, v, p):
    """Vectorised to_conserved via the oracle (bit-exact with state2d.hpp:16-19)."""
    lib, _ = _load("oracle")
    rho, u, v, p = (np.ascontiguousarray(a, np.float64) for a in (rho, u, v, p))
    out = np.empty(rho.shape + (4,), np.float64)
    lib.orc_primitive_to_state(rho.size, _dp(rho), _dp(u), _dp(v), _dp(p), _dp(out))
    return out


def frame_time(t_start, t_end, k, nout):
    lib, _ = _load("oracle")
    return lib.orc_frame_time(t_start, t_end, k, nout)
