"""GPU checks of the tolerance build (libfv_tol.so: FMA contraction and the Newton-Raphson division).

Staged: pytest collects only test_*.py, so these run once this file is renamed to
test_gpu_tolerance.py, after they have passed on a B200.

The tolerance build loads per process (FV_BUILD=tolerance), so its runs happen in child processes
that write their results to .npz files; the parity build and the oracle run here.
Tolerances: 1e-12 relative per step and 1e-9 per run, each field's maximum absolute difference over
its maximum magnitude.
"""
import importlib
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
fv = importlib.import_module("neural-pde-surrogate_b200")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")


def operands(n=1 << 20, seed=3):
    rng = np.random.default_rng(seed)
    a = np.ldexp(1.0 + rng.random(n), rng.integers(-60, 60, n)) * rng.choice([-1.0, 1.0], n)
    b = np.ldexp(1.0 + rng.random(n), rng.integers(-60, 60, n)) * rng.choice([-1.0, 1.0], n)
    a[:8] = [0.0, -0.0, 1.0, -1.0, 1e-300, 1e300, 3.0, 7.0]  # zeros and extremes take the IEEE path
    b[:8] = [2.0, 2.0, 3.0, 3.0, 3.0, 3.0, 1e-310, np.inf]
    return a, b


def ulps(x, y):
    def ordered(v):
        i = v.view(np.int64)
        return np.where(i < 0, np.int64(-(2 ** 63)) - i, i)
    return np.abs(ordered(x) - ordered(y))


def _child(code, out, *args):
    env = dict(os.environ, FV_BUILD="tolerance")
    r = subprocess.run([sys.executable, "-c", code, str(ROOT), str(out), *map(str, args)], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    return np.load(out)


DIV = r"""
import importlib, sys
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
fv = importlib.import_module("neural-pde-surrogate_b200")
assert b"tolerance build" in fv.lib().fv_version()
from pending_gpu_tolerance import operands
a, b = operands()
np.savez(sys.argv[2], q=fv.eval_division(a, b))
"""


def test_parity_division_is_ieee(cuda_ok):
    a, b = operands()
    assert fv.eval_division(a, b).tobytes() == (a / b).tobytes()


def test_tolerance_division_within_one_ulp(cuda_ok, tmp_path):
    a, b = operands()
    q = _child(DIV, tmp_path / "q.npz")["q"]
    d = ulps(q, a / b)
    assert d.max() <= 1, (int(d.max()), float((d > 0).mean()))


RUN = r"""
import importlib, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
fv = importlib.import_module("neural-pde-surrogate_b200")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")
assert b"tolerance build" in fv.lib().fv_version()
fam, idx, n, lim = sys.argv[3], int(sys.argv[4]), int(sys.argv[5]), sys.argv[6]
rho, u, v, p, t_end, _ = ic.sample(fam, idx, n)
s = fv.Solver(fv.make_grid(n, n, 0, 1, 0, 1, "periodic", "periodic"), "hllc", lim, 0.5)
U0 = ic.to_conserved(rho, u, v, p)
s.set_state(U0)
dt = s.compute_dt()
s.step(dt=dt)
one = s.get_state()
s.set_state(U0)
t, steps = s.advance_to(t_end)
np.savez(sys.argv[2], dt=dt, one=one, final=s.get_state(), t=t, steps=steps)
"""


def rel(a, b):
    a, b = a.reshape(-1, 4), b.reshape(-1, 4)
    return float((np.abs(a - b).max(axis=0) / np.abs(b).max(axis=0)).max())


@pytest.mark.parametrize("fam,idx,n,lim", [("blast", 1, 128, "vanleer"), ("blast", 3, 128, "minmod"),
                                           ("riemann", 2, 128, "vanleer")])
def test_tolerance_build_within_the_stated_tolerances(cuda_ok, tmp_path, fam, idx, n, lim):
    from oracle.oracle import OracleSolver
    r = _child(RUN, tmp_path / "run.npz", fam, idx, n, lim)
    rho, u, v, p, t_end, _ = ic.sample(fam, idx, n)
    U0 = ic.to_conserved(rho, u, v, p)
    o = OracleSolver(n, n, 0, 1, 0, 1, "periodic", "periodic", "hllc", lim, 0.5)
    o.set_state(U0)
    dt = o.compute_dt()
    assert abs(float(r["dt"]) - dt) <= 1e-12 * dt
    o.step(float(r["dt"]))  # the same dt: one step from the same state
    assert rel(r["one"], o.get_state()) <= 1e-12
    o.set_state(U0)
    o.advance_to(t_end)
    assert float(r["t"]) == t_end
    assert rel(r["final"], o.get_state()) <= 1e-9
