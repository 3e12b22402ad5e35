"""The division sequences of the stage kernels against IEEE division, and the tolerance build
(libfv_tol.so: FMA contraction and a Newton-Raphson division) against the reference.

Parity build: every division sequence it uses in place of IEEE `/` (div_gm1, div_z, div_back) must
return the IEEE quotient bit for bit, on 2^31 operand pairs drawn on the device per kind and on
chosen edge operands.

Tolerance build: 1e-12 relative per step and 1e-9 per run of the reference, each field's maximum
absolute difference over its maximum magnitude; its general division within 1 ulp of IEEE.  It loads
per process (FV_BUILD=tolerance), so its runs happen in child processes that write .npz files; the
parity build and the reference run here.
"""
import importlib
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from cases import cpu_solver
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
fv = importlib.import_module("neural-pde-surrogate_b200")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")
SWEEP = 1 << 31


def operands(n=1 << 20, seed=3):
    rng = np.random.default_rng(seed)
    a = np.ldexp(1.0 + rng.random(n), rng.integers(-60, 60, n)) * rng.choice([-1.0, 1.0], n)
    b = np.ldexp(1.0 + rng.random(n), rng.integers(-60, 60, n)) * rng.choice([-1.0, 1.0], n)
    # zeros of both signs, extremes, subnormal and infinite divisors take the IEEE path
    a[:10] = [0.0, -0.0, 1.0, -1.0, 1e-300, 1e300, 3.0, 7.0, -0.0, 0.0]
    b[:10] = [2.0, 2.0, 3.0, 3.0, 3.0, 3.0, 1e-310, np.inf, -5.0, -np.inf]
    return a, b


def ulps(x, y):
    def ordered(v):
        i = v.view(np.int64)
        return np.where(i < 0, np.int64(-(2 ** 63)) - i, i)
    return np.abs(ordered(x) - ordered(y))


def same_sign(x, y):
    return bool((np.signbit(x) == np.signbit(y)).all())


def _child(code, out, *args):
    env = dict(os.environ, FV_BUILD="tolerance")
    r = subprocess.run([sys.executable, "-c", code, str(ROOT), str(out), *map(str, args)], env=env,
                       capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stderr
    return np.load(out)


# ---- parity build: the exact division sequences ------------------------------------------------

def test_parity_general_division_is_ieee(cuda_ok):
    a, b = operands()
    q = fv.eval_division(a, b)
    assert q.tobytes() == (a / b).tobytes()


@pytest.mark.parametrize("kind", ["gm1", "zero", "back"])
def test_parity_division_sequences_are_ieee_on_device_draws(cuda_ok, kind):
    mism, worst = fv.division_sweep(kind, SWEEP, seed=11 + len(kind))
    assert mism == 0, (kind, mism, worst)


def test_parity_division_sequences_on_edge_operands(cuda_ok):
    gm1 = 1.4 - 1.0
    p = np.array([0.0, -0.0, 5e-324, -1e-310, 1e-300, 0.1, 2.5, 1e300, -1e308, np.inf, -np.inf, np.ldexp(1.0, -900),
                  np.ldexp(1.0, 900), np.nextafter(np.ldexp(1.0, -900), 0), 1.0, np.nextafter(1.0, 2.0), np.nextafter(2.0, 0.0)])
    assert fv.eval_division(p, None, kind="gm1").tobytes() == (p / gm1).tobytes()
    a, b = operands()
    q = fv.eval_division(a, b, kind="zero")
    assert q.tobytes() == (a / b).tobytes()
    # div_back: rho and u with edge mantissas (powers of two, all-ones), zeros, signs, extremes
    rho = np.array([1.0, 0.5, 3.0, np.nextafter(2.0, 0.0), 1e-300, np.ldexp(1.0, -301), np.ldexp(1.0, 299), 0.0, -1.0, 7.25,
                    np.nextafter(1.0, 2.0), 0.1])
    u = np.array([0.1, -0.3, 1.0, -2.0, np.nextafter(4.0, 0.0), 0.0, -0.0, 1e-290, 3.7e290, -np.ldexp(1.0, -301),
                  np.nextafter(1.0, 2.0), 5e-324])
    R, V = np.meshgrid(rho, u)
    R, V = R.ravel(), V.ravel()
    with np.errstate(all="ignore"):
        ref = (R * V) / R
    got = fv.eval_division(R, V, kind="back")
    nan = np.isnan(ref)
    assert (np.isnan(got) == nan).all()
    assert got[~nan].tobytes() == ref[~nan].tobytes()


# ---- tolerance build ---------------------------------------------------------------------------

DIV = r"""
import importlib, sys
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
fv = importlib.import_module("neural-pde-surrogate_b200")
assert b"tolerance build" in fv.lib().fv_version()
from test_gpu_tolerance import operands, SWEEP
a, b = operands()
out = {"q": fv.eval_division(a, b)}
for kind in ("general", "gm1", "zero", "back"):
    out["sweep_" + kind] = np.array(fv.division_sweep(kind, SWEEP, seed=5))
np.savez(sys.argv[2], **out)
"""


def test_tolerance_division_within_one_ulp(cuda_ok, tmp_path):
    a, b = operands()
    r = _child(DIV, tmp_path / "q.npz")
    q = r["q"]
    d = ulps(q, a / b)
    assert d.max() <= 1, (int(d.max()), float((d > 0).mean()))
    assert same_sign(q, a / b)  # signed zeros keep IEEE's sign
    assert int(r["sweep_gm1"][0]) == 0  # p / (GAMMA - 1) stays exact in the tolerance build
    for kind in ("general", "zero", "back"):
        mism, worst = (int(x) for x in r["sweep_" + kind])
        assert worst <= 1, (kind, mism, worst)


RUN = r"""
import importlib, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
fv = importlib.import_module("neural-pde-surrogate_b200")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")
assert b"tolerance build" in fv.lib().fv_version()
fam, idx, n, flux, lim = sys.argv[3], int(sys.argv[4]), int(sys.argv[5]), sys.argv[6], sys.argv[7]
rho, u, v, p, t_end, _ = ic.sample(fam, idx, n)
s = fv.Solver(fv.make_grid(n, n, 0, 1, 0, 1, "periodic", "periodic"), flux, lim, 0.5)
U0 = ic.to_conserved(rho, u, v, p)
s.set_state(U0)
dt0 = s.compute_dt()
s.step(dt=dt0)
one = s.get_state()
s.set_state(U0)
s.advance_to(0.5 * t_end)
mid = s.get_state()
dtm = s.compute_dt()
s.step(dt=dtm)
mid1 = s.get_state()
s.set_state(U0)
t, steps = s.advance_to(t_end)
np.savez(sys.argv[2], dt0=dt0, one=one, mid=mid, dtm=dtm, mid1=mid1, final=s.get_state(), t=t, steps=steps)
"""


def rel(a, b):
    a, b = a.reshape(-1, 4), b.reshape(-1, 4)
    return float((np.abs(a - b).max(axis=0) / np.abs(b).max(axis=0)).max())


@pytest.mark.parametrize("fam,idx,n,flux,lim", [
    ("riemann", 0, 256, "hllc", "vanleer"),   # the four-quadrant Riemann configuration at its size
    ("blast", 3, 512, "hllc", "vanleer"),     # the bench's blast configuration at its size
    ("blast", 3, 512, "hllc", "minmod"),
    ("blast", 3, 512, "rusanov", "minmod"),
    ("blast", 3, 512, "rusanov", "vanleer"),
    ("blast", 1, 128, "hllc", "vanleer"),
])
def test_tolerance_build_within_the_stated_tolerances(cuda_ok, tmp_path, fam, idx, n, flux, lim):
    if not orc.ref_available():
        pytest.fail("oracle/_ref/libfvref.so is missing")
    r = _child(RUN, tmp_path / "run.npz", fam, idx, n, flux, lim)
    rho, u, v, p, t_end, _ = ic.sample(fam, idx, n)
    U0 = ic.to_conserved(rho, u, v, p)
    ref = cpu_solver("ref", dict(nx=n, ny=n, bc_x="periodic", bc_y="periodic"), flux, lim)
    ref.set_state(U0)
    dt0 = ref.compute_dt()
    assert abs(float(r["dt0"]) - dt0) <= 1e-12 * dt0
    ref.step(float(r["dt0"]))  # one step from the same state with the same dt
    assert rel(r["one"], ref.get_state()) <= 1e-12
    ref.set_state(r["mid"])  # one step from the tolerance build's own mid-run state (shocks formed)
    ref.step(float(r["dtm"]))
    assert rel(r["mid1"], ref.get_state()) <= 1e-12
    ref.set_state(U0)
    ref.advance_to(t_end)
    assert float(r["t"]) == t_end
    assert rel(r["final"], ref.get_state()) <= 1e-9
