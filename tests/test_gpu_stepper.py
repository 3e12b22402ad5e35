"""The persistent stepper (fv_advance_to's device loop) against the per-stage kernels and the oracle.

Each case runs in two child processes, one with FV_STEPPER=0 (the per-stage kernels, two launches
per step) and one with the stepper, and both must be bit-identical to the CPU oracle: grids with
partial edge tiles (whose halos reach two tiles away through a periodic wrap), grids of one tile,
grids with fewer tiles than resident CTAs, every boundary combination, a run stopped by a
non-physical cell, fv_step mixed with fv_advance_to, and runs across several launches.
"""
import importlib
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from cases import bits_equal, cpu_solver
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
fv = importlib.import_module("neural-pde-surrogate_b200")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")

CHILD = r"""
import importlib, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
fv = importlib.import_module("neural-pde-surrogate_b200")
solver = importlib.import_module("neural-pde-surrogate_b200.solver")
z = np.load(sys.argv[2])
nx, ny = int(z["nx"]), int(z["ny"])
s = fv.Solver(fv.make_grid(nx, ny, 0.0, 1.0, 0.0, float(z["ly"]), str(z["bcx"]), str(z["bcy"])),
              str(z["flux"]), str(z["lim"]), 0.5)
s.set_state(z["U0"])
out = {}
for k, t in enumerate(z["targets"]):
    if k == 1 and bool(z["mix_step"]):
        s.step(dt=s.compute_dt())  # one fixed step between two device loops
    try:
        tt, n = s.advance_to(float(t))
        out[f"t{k}"], out[f"n{k}"] = tt, n
    except fv.NonPhysicalError as e:
        out["bad"] = np.array([e.i, e.j, k])
        out[f"n{k}"] = s.time()[1]
        break
out["U"] = s.get_state()
out["tile"] = np.array(solver.stepper_tile(s))
np.savez(sys.argv[3], **out)
"""


def _run(tmp_path, stepper, tile=None, **case):
    inp, out = tmp_path / "case.npz", tmp_path / f"out{stepper}.npz"
    np.savez(inp, **case)
    env = dict(os.environ, FV_STEPPER=str(stepper))
    if tile is not None:
        env["FV_STEPPER_TILE"] = str(tile)
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT), str(inp), str(out)], env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    return dict(np.load(out))


def _oracle(case):
    g = dict(nx=int(case["nx"]), ny=int(case["ny"]), x_min=0.0, x_max=1.0, y_min=0.0, y_max=float(case["ly"]),
             bc_x=str(case["bcx"]), bc_y=str(case["bcy"]))
    o = cpu_solver("oracle", g, str(case["flux"]), str(case["lim"]))
    o.set_state(case["U0"])
    out = {}
    for k, t in enumerate(case["targets"]):
        if k == 1 and case["mix_step"]:
            o.step(o.compute_dt())
            o.steps += 1
        try:
            o.advance_to(float(t))
            out[f"t{k}"], out[f"n{k}"] = o.t, o.steps
        except orc.NonPhysical as e:
            out["bad"] = np.array([e.i, e.j, k])
            out[f"n{k}"] = o.steps
            break
    out["U"] = o.get_state()
    return out


def _random(nx, ny, seed):
    rng = np.random.default_rng(seed)
    rho = 0.5 + rng.random((ny, nx))
    u, v = rng.uniform(-1, 1, (ny, nx)), rng.uniform(-1, 1, (ny, nx))
    p = 0.3 + rng.random((ny, nx))
    return ic.to_conserved(rho, u, v, p)


CASES = [
    # (nx, ny, bcx, bcy, flux, lim, targets, mix_step): partial edge tiles, one tile, few tiles, every BC pair
    (65, 33, "periodic", "periodic", "hllc", "vanleer", (0.02, 0.05), False),
    (70, 45, "periodic", "transmissive", "rusanov", "minmod", (0.03,), True),
    (17, 3, "transmissive", "periodic", "hllc", "minmod", (0.01, 0.04, 0.05), True),
    (1, 5, "periodic", "transmissive", "hllc", "none", (0.05,), False),
    (33, 17, "transmissive", "transmissive", "rusanov", "vanleer", (0.04,), False),
    (256, 100, "periodic", "periodic", "hllc", "vanleer", (0.01, 0.02), True),
]


@pytest.mark.parametrize("nx,ny,bcx,bcy,flux,lim,targets,mix", CASES)
def test_stepper_bitexact_vs_per_stage_and_oracle(cuda_ok, tmp_path, nx, ny, bcx, bcy, flux, lim, targets, mix):
    case = dict(nx=nx, ny=ny, ly=0.7, bcx=bcx, bcy=bcy, flux=flux, lim=lim, targets=np.array(targets),
                mix_step=mix, U0=_random(nx, ny, nx * 131 + ny))
    a, b, o = _run(tmp_path, 0, **case), _run(tmp_path, 1, **case), _oracle(case)
    assert tuple(b["tile"]) != (0, 0, 0) and tuple(a["tile"]) == (0, 0, 0)  # which path ran
    for k in range(len(targets)):
        assert a[f"n{k}"] == b[f"n{k}"] == o[f"n{k}"], (k, a[f"n{k}"], b[f"n{k}"], o[f"n{k}"])
        assert a[f"t{k}"] == b[f"t{k}"] == o[f"t{k}"]
    assert bits_equal(a["U"], o["U"]) and bits_equal(b["U"], o["U"])


def test_stepper_stops_at_the_first_bad_cell_like_the_reference(cuda_ok, tmp_path):
    """Unlimited slopes on a strong blast go non-physical; the stepper must stop at the same step and
    report the same first bad cell as the per-stage kernels and the oracle."""
    n = 64
    rho, u, v, p, _, _ = ic.sample("blast", 1, n)
    case = dict(nx=n, ny=n, ly=1.0, bcx="periodic", bcy="periodic", flux="hllc", lim="unlimited",
                targets=np.array([0.2]), mix_step=False, U0=ic.to_conserved(rho, u, v, p))
    a, b, o = _run(tmp_path, 0, **case), _run(tmp_path, 1, **case), _oracle(case)
    assert "bad" in o, "the case was meant to go non-physical"
    assert (a["bad"] == o["bad"]).all() and (b["bad"] == o["bad"]).all()
    assert a["n0"] == b["n0"] == o["n0"]
    assert bits_equal(b["U"], o["U"])


def test_stepper_long_run_spans_several_launches(cuda_ok, tmp_path):
    """A 128^2 Riemann run to t = 0.25 in 20 frames: 20 advance_to calls, each a stepper launch that
    must stop by itself exactly at its frame time (its step budget is larger than the steps needed)."""
    n = 128
    rho, u, v, p, t_end, _ = ic.sample("riemann", 5, n)
    case = dict(nx=n, ny=n, ly=1.0, bcx="periodic", bcy="periodic", flux="hllc", lim="vanleer",
                targets=np.linspace(0.0125, t_end, 20), mix_step=False, U0=ic.to_conserved(rho, u, v, p))
    b, o = _run(tmp_path, 1, **case), _oracle(case)
    for k in range(20):
        assert b[f"n{k}"] == o[f"n{k}"] and b[f"t{k}"] == o[f"t{k}"]
    assert bits_equal(b["U"], o["U"])


# (tile width, height, threads) of each stepper shape, in the library's order
STEPPER_SHAPES = [(16, 14, 256), (16, 16, 256), (32, 8, 256), (16, 7, 128), (32, 16, 512), (16, 7, 128),
                  (32, 14, 512)]


@pytest.mark.parametrize("shape", range(len(STEPPER_SHAPES)))
def test_every_stepper_shape_is_bitexact(cuda_ok, tmp_path, shape):
    """Each tile shape of the stepper (FV_STEPPER_TILE fixes it instead of the autotuner) on a grid
    with partial edge tiles in both directions and a transmissive boundary, against the oracle."""
    nx, ny = 70, 45
    case = dict(nx=nx, ny=ny, ly=45 / 70, bcx="periodic", bcy="transmissive", flux="hllc", lim="vanleer",
                U0=_random(nx, ny, 40 + shape), targets=np.array([0.02, 0.03]), mix_step=False)
    got = _run(tmp_path, 1, tile=shape, **case)
    assert tuple(int(x) for x in got["tile"]) == STEPPER_SHAPES[shape]
    ref = _oracle(case)
    for k in range(2):
        assert float(got[f"t{k}"]) == ref[f"t{k}"] and int(got[f"n{k}"]) == ref[f"n{k}"]
    assert bits_equal(got["U"], ref["U"])
