"""Parity at the benchmarked sizes, against the reference's own solver core (oracle/_ref/libfvref.so,
its headers compiled from source) rather than the C restatement.

* The bench's workload: the 512^2 blast + bubble problem run in trajectory mode to t = 0.2 with 20
  frames saved at 128^2 and 64^2, for each of the four flux x limiter combinations the bench times.
  Step counts, frame times, every saved frame and the final state must be bit-identical.
* The batched-ensemble workload: 256 members of sizes {64^2, 128^2, 256^2, 512^2}, alternately
  Riemann and blast initial conditions, each to t = 0.25 with its own CFL dt.  Every member must be
  bit-identical to its own single-grid run, and 16 members (four of each size) to the reference.

The reference runs on all host cores (OpenMP; bit-identical for any thread count).
"""
import importlib

import numpy as np
import pytest

from cases import bits_equal, cpu_solver, gpu_solver
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
fv = importlib.import_module("neural-pde-surrogate_b200")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")
ens_mod = importlib.import_module("neural-pde-surrogate_b200.ensemble")

BENCH_N, BENCH_NOUT, BENCH_T_END, BENCH_SAVE = 512, 20, 0.2, (128, 64)
BENCH_IC = 3  # bench.py's initial condition of the first timed step (blast index 3 on rank 0)
PERIODIC = dict(bc_x="periodic", bc_y="periodic")


@pytest.fixture(autouse=True)
def _gpu(cuda_ok):
    if not orc.ref_available():
        pytest.fail("oracle/_ref/libfvref.so is missing: build it with oracle/build_oracle.py where the "
                    "reference sources are present; the built file travels with the repository")


@pytest.mark.parametrize("flux,lim", [("hllc", "minmod"), ("hllc", "vanleer"), ("rusanov", "minmod"),
                                      ("rusanov", "vanleer")])
def test_bench_trajectory_matches_the_reference(flux, lim):
    n = BENCH_N
    rho, u, v, p, _, _ = ic.sample("blast", BENCH_IC, n)
    g = dict(nx=n, ny=n, **PERIODIC)
    ref = cpu_solver("ref", g, flux, lim)
    gpu = gpu_solver(g, flux, lim)
    ref.set_state(ic.to_conserved(rho, u, v, p))
    gpu.set_primitive(rho, u, v, p)  # the bench's e2e path: to_conserved on the device
    t_ref, lv_ref = ref.run(BENCH_T_END, 0.0, BENCH_NOUT, BENCH_SAVE)
    t_gpu, lv_gpu, steps = gpu.run_trajectory(BENCH_T_END, 0.0, BENCH_NOUT, BENCH_SAVE)
    assert steps == ref.steps and steps > 1000
    assert bits_equal(t_ref, t_gpu)
    for m in BENCH_SAVE:
        assert lv_gpu[m].shape == (BENCH_NOUT + 1, 4, m, m)
        assert bits_equal(lv_ref[m], lv_gpu[m]), f"frames at {m}^2 differ"
    assert bits_equal(ref.get_state(), gpu.get_state())


def _single_run(n, U0, t_end):
    s = gpu_solver(dict(nx=n, ny=n, **PERIODIC), "hllc", "vanleer")
    s.set_state(U0)
    t, steps = s.advance_to(t_end)
    return t, steps, s.get_state()


def test_ensemble_workload_matches_single_runs_and_the_reference():
    t_end = 0.25
    spec = ic.ensemble_spec(256)
    states = [ic.to_conserved(*ic.sample(fam, idx, n)[:4]) for fam, idx, n in spec]
    grids = [fv.make_grid(n, n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic") for _, _, n in spec]
    ens = ens_mod.Ensemble(grids, "hllc", "vanleer")
    for k, U in enumerate(states):
        ens.set_state(k, U)
    t, steps, status = ens.advance_to(t_end)
    assert (status == 0).all() and (t == t_end).all()
    finals = [ens.get_state(k) for k in range(len(spec))]
    for k, ((_, _, n), U0) in enumerate(zip(spec, states)):  # every member against its own run
        ts, st, Us = _single_run(n, U0, t_end)
        assert ts == t[k] and st == steps[k], f"member {k}: steps {steps[k]} vs {st}"
        assert bits_equal(finals[k], Us), f"member {k} ({n}^2) differs from its single-grid run"
    checked = {}
    for k, (_, _, n) in enumerate(spec):  # the first four members of each size against the reference
        if checked.get(n, 0) >= 4:
            continue
        checked[n] = checked.get(n, 0) + 1
        ref = cpu_solver("ref", dict(nx=n, ny=n, **PERIODIC), "hllc", "vanleer")
        ref.set_state(states[k])
        ref.advance_to(t_end)
        assert ref.steps == steps[k] and ref.t == t[k], f"member {k}: {ref.steps} reference steps"
        assert bits_equal(ref.get_state(), finals[k]), f"member {k} ({n}^2) differs from the reference"
    assert sum(checked.values()) == 16
