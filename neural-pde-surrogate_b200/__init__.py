"""B200-native (sm_100a) finite-volume step of the 2D compressible-Euler solver of
GusGus2004/neural-pde-surrogate, behind the C-ABI in include/fv.h.

The directory name is not a Python identifier; import it with
``importlib.import_module("neural-pde-surrogate_b200")``.
"""
from ._lib import FVError, NonPhysicalError, lib  # noqa: F401
from .solver import BC, FLUXES, LIMITERS, Grid, Solver, division_sweep, eval_division, fill_ghosts, make_grid, riemann_flux  # noqa: F401

__all__ = ["BC", "FLUXES", "LIMITERS", "Grid", "Solver", "make_grid", "riemann_flux", "eval_division", "division_sweep", "fill_ghosts", "FVError", "NonPhysicalError", "lib"]
