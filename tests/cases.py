"""Shared helpers: load a golden fixture, build a solver of any implementation for it."""
import importlib
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden_names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name):
    z = np.load(GOLDEN / f"{name}.npz")
    d = {k: z[k] for k in z.files}
    nx, ny = (int(v) for v in d["grid"])
    x0, x1, y0, y1 = (float(v) for v in d["bounds"])
    d["g"] = dict(nx=nx, ny=ny, x_min=x0, x_max=x1, y_min=y0, y_max=y1, bc_x=str(d["bcs"][0]), bc_y=str(d["bcs"][1]))
    d["flux"], d["limiter"] = str(d["flux"]), str(d["limiter"])
    d["save"] = sorted((int(k[6:]) for k in d if k.startswith("level_")), reverse=True)
    return d


def cpu_solver(kind, g, flux, limiter, cfl=0.5):
    """kind: 'oracle' (C restatement) or 'ref' (reference build)."""
    from oracle.oracle import OracleSolver, RefSolver
    cls = OracleSolver if kind == "oracle" else RefSolver
    return cls(g["nx"], g["ny"], g.get("x_min", 0.0), g.get("x_max", 1.0), g.get("y_min", 0.0), g.get("y_max", 1.0),
               g["bc_x"], g["bc_y"], flux, limiter, cfl)


def gpu_solver(g, flux, limiter, cfl=0.5):
    fv = importlib.import_module("neural-pde-surrogate_b200")
    grid = fv.make_grid(g["nx"], g["ny"], g.get("x_min", 0.0), g.get("x_max", 1.0), g.get("y_min", 0.0),
                        g.get("y_max", 1.0), g["bc_x"], g["bc_y"])
    return fv.Solver(grid, flux, limiter, cfl)


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and a.tobytes() == b.tobytes()


def max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
