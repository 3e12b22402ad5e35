"""fv_step_noalloc: the step for callers that cannot allocate device memory when they step (a host
inside another framework's memory pool, or a driver loop that forbids allocation after start-up).
It keeps its scratch in a fixed array compiled into libfv instead of calling cudaMalloc.

Checked through the C-ABI against the handle API (fv_step) on two calls in a row, bit for bit --
the tolerance every solver parity test here uses -- so that the second call also shows the shared
scratch, which keeps the first call's contents, does not leak into the result.  This file is
collected last so that a run stopping at its first failure has already run every other test; it
passes alone in a fresh process as well."""
import ctypes as C
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

fv = importlib.import_module("neural-pde-surrogate_b200")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")

MAX_CELLS = 128 * 128  # FV_NOALLOC_MAX_CELLS in include/fv.h


def _noalloc():
    f = fv.lib().fv_step_noalloc
    f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                  C.c_int, C.c_void_p, C.c_double, C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.parametrize("nx,ny,bcs,flux,lim", [(64, 48, (1, 0), "hllc", "vanleer"),
                                                (128, 128, (1, 1), "rusanov", "minmod"),
                                                (37, 5, (0, 1), "hllc", "unlimited")])
def test_noalloc_step_matches_handle_step(cuda_ok, nx, ny, bcs, flux, lim):
    import torch
    rng = np.random.default_rng(nx * 1000 + ny)
    rho = 0.5 + rng.random((ny, nx))
    u, v = rng.uniform(-1, 1, (ny, nx)), rng.uniform(-1, 1, (ny, nx))
    p = 0.3 + rng.random((ny, nx))
    U0 = ic.to_conserved(rho, u, v, p)
    names = ("transmissive", "periodic")
    ref = fv.Solver(fv.make_grid(nx, ny, 0.0, 1.0, 0.0, 0.8, names[bcs[0]], names[bcs[1]]), flux, lim, 0.5)
    ref.set_state(U0)
    d_U = torch.from_numpy(U0.copy()).cuda()
    step = _noalloc()
    for call in range(2):  # two calls in a row share (and must clear) the scratch
        dt = ref.compute_dt()
        ref.step(dt=dt)
        expected = ref.get_state()
        rc = step(nx, ny, 0.0, 1.0, 0.0, 0.8, bcs[0], bcs[1], fv.FLUXES[flux], fv.LIMITERS[lim],
                  C.c_void_p(d_U.data_ptr()), dt, None)
        assert rc == 0, fv.lib().fv_last_error()
        torch.cuda.synchronize()
        got = d_U.cpu().numpy()
        assert got.tobytes() == expected.tobytes(), f"call {call}: differs from fv_step"


def test_noalloc_rejects_grids_beyond_the_limit(cuda_ok):
    import torch
    d_U = torch.zeros((MAX_CELLS + 1) * 4, dtype=torch.float64, device="cuda")
    rc = _noalloc()(MAX_CELLS + 1, 1, 0.0, 1.0, 0.0, 1.0, 1, 1, 1, 3, C.c_void_p(d_U.data_ptr()), 1e-3, None)
    assert rc == 1
    assert b"FV_NOALLOC_MAX_CELLS" in fv.lib().fv_last_error()


def _rejects(args, needle):
    """Calls the entry point on a 64 x 64 state with one argument replaced (`offset`: bytes added to
    the state's address, inside the buffer, which has two spare doubles) and checks it is refused."""
    import torch
    d_U = torch.zeros(64 * 64 * 4 + 2, dtype=torch.float64, device="cuda")
    a = dict(nx=64, ny=64, x0=0.0, x1=1.0, y0=0.0, y1=1.0, bcx=1, bcy=1, flux=1, lim=3, offset=0, null=False,
             dt=1e-3)
    a.update(args)
    ptr = None if a["null"] else C.c_void_p(d_U.data_ptr() + a["offset"])
    before = d_U.clone()
    rc = _noalloc()(a["nx"], a["ny"], a["x0"], a["x1"], a["y0"], a["y1"], a["bcx"], a["bcy"], a["flux"], a["lim"],
                    ptr, a["dt"], None)
    torch.cuda.synchronize()
    assert rc == 1, rc
    assert needle in fv.lib().fv_last_error()
    assert torch.equal(before, d_U)  # rejected before any kernel ran


@pytest.mark.parametrize("args,needle", [
    (dict(flux=7), b"unknown flux/limiter/bc"), (dict(lim=-1), b"unknown flux/limiter/bc"),
    (dict(lim=4), b"unknown flux/limiter/bc"), (dict(bcx=2), b"unknown flux/limiter/bc"),
    (dict(bcy=-1), b"unknown flux/limiter/bc"), (dict(x1=0.0), b"empty domain"), (dict(y0=2.0), b"empty domain"),
    (dict(nx=0), b"must be positive"), (dict(ny=-3), b"must be positive"), (dict(null=True), b"NULL"),
])
def test_noalloc_rejects_invalid_arguments(cuda_ok, args, needle):
    _rejects(args, needle)


def test_noalloc_rejects_a_misaligned_state(cuda_ok):
    """A state 8 bytes off a 16-byte boundary (a view at an odd double offset) is refused with
    FV_ERR_ARG, not handed to kernels that load each cell as two 16-byte words."""
    _rejects(dict(offset=8), b"16-byte aligned")
