"""Generate the golden fixtures in this folder from the REFERENCE solver core.

  python tests/golden/make_golden.py

Runs oracle/_ref/libfvref.so -- the reference's own headers (solver/src of
GusGus2004/neural-pde-surrogate) compiled by oracle/build_oracle.py -- on small seeded cases and
stores inputs and outputs as .npz.  The tests compare the C oracle and the CUDA library against
these files, so they also work where the reference tree is absent.
"""
import importlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import build_oracle  # noqa: E402
from oracle.oracle import RefSolver  # noqa: E402

ic = importlib.import_module("neural-pde-surrogate_b200.ic")
OUT = Path(__file__).resolve().parent

# (name, grid kwargs, flux, limiter, U0 builder, t_end, nout, save sizes)
def cases():
    rng = np.random.default_rng(20261203)
    out = []
    # every flux x limiter on a small non-square grid with mixed boundaries, 6 steps via advance_to
    g = dict(nx=20, ny=12, x_min=0.0, x_max=1.0, y_min=0.0, y_max=0.6, bc_x="periodic", bc_y="transmissive")
    rho = 1.0 + 0.5 * rng.random((12, 20))
    u = rng.uniform(-0.5, 0.5, (12, 20))
    v = rng.uniform(-0.5, 0.5, (12, 20))
    p = 0.5 + rng.random((12, 20))
    U0 = ic.to_conserved(rho, u, v, p)
    for flux in ("hllc", "rusanov"):
        for lim in ("none", "unlimited", "minmod", "vanleer"):
            out.append((f"mixed_{flux}_{lim}", g, flux, lim, U0, 0.02, 2, ()))
    # four-quadrant Riemann (periodic) at 32^2, HLLC + van Leer
    rho, u, v, p, _, _ = ic.sample("riemann", 7, 32)
    out.append(("riemann32_hllc_vanleer", dict(nx=32, ny=32, bc_x="periodic", bc_y="periodic"), "hllc", "vanleer",
                ic.to_conserved(rho, u, v, p), 0.05, 2, (16, 8)))
    # blast + bubbles at 32^2, all four graded combos
    rho, u, v, p, _, _ = ic.sample("blast", 3, 32)
    for flux in ("hllc", "rusanov"):
        for lim in ("minmod", "vanleer"):
            out.append((f"blast32_{flux}_{lim}", dict(nx=32, ny=32, bc_x="periodic", bc_y="periodic"), flux, lim,
                        ic.to_conserved(rho, u, v, p), 0.01, 2, (16, 8)))
    # Sod along x, 200 x 4, transmissive (test_solver2d.cpp:55-71)
    gk, t_end, U0 = ic.test_problem("sod_x", 200)
    out.append(("sod_x200", gk, "hllc", "vanleer", U0, t_end, 1, ()))
    return out


def main():
    build_oracle.build()
    for name, g, flux, lim, U0, t_end, nout, save in cases():
        s = RefSolver(g["nx"], g["ny"], g.get("x_min", 0.0), g.get("x_max", 1.0), g.get("y_min", 0.0),
                      g.get("y_max", 1.0), g["bc_x"], g["bc_y"], flux, lim, 0.5)
        s.set_state(U0)
        dt0 = s.compute_dt()
        times, levels = s.run(t_end, 0.0, nout, save)
        np.savez_compressed(OUT / f"{name}.npz", U0=U0, U=s.get_state(), times=times, steps=s.steps, dt0=dt0,
                            flux=flux, limiter=lim, t_end=t_end, nout=nout, cfl=0.5,
                            grid=np.array([g["nx"], g["ny"]]),
                            bounds=np.array([g.get("x_min", 0.0), g.get("x_max", 1.0), g.get("y_min", 0.0),
                                             g.get("y_max", 1.0)]),
                            bcs=np.array([g["bc_x"], g["bc_y"]]),
                            **{f"level_{m}": a for m, a in levels.items()})
        print(f"{name}: {s.steps} steps, t = {s.t:.6f}")


if __name__ == "__main__":
    main()
