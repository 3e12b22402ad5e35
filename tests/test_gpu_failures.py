"""Failure detection on the GPU without a GPU fault: the library's bounded waits give up and report.

Every TMA copy of the stage kernels and every tensor-core batch of the correction network is waited
for with a time-limited mbarrier wait.  fv_wait_selftest runs that wait on a barrier nothing arrives
at (10 ms limit): it must come back with FV_ERR_TIMEOUT, and the context must stay usable -- the next
solver run still matches the oracle bit for bit."""
import importlib

import pytest

from cases import bits_equal, cpu_solver, gpu_solver

pytestmark = pytest.mark.gpu
_lib = importlib.import_module("neural-pde-surrogate_b200._lib")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")


@pytest.fixture(autouse=True)
def _gpu(cuda_ok):
    pass


def test_bounded_wait_gives_up_and_the_context_survives():
    for _ in range(2):
        assert _lib.lib().fv_wait_selftest() == 4  # FV_ERR_TIMEOUT
    n = 48
    rho, u, v, p, _, _ = ic.sample("riemann", 7, n)
    U0 = ic.to_conserved(rho, u, v, p)
    grid = dict(nx=n, ny=n, bc_x="periodic", bc_y="periodic")
    g = gpu_solver(grid, "hllc", "vanleer")
    g.set_state(U0)
    g.advance_to(0.01)
    c = cpu_solver("oracle", grid, "hllc", "vanleer")
    c.set_state(U0)
    c.advance_to(0.01)
    assert bits_equal(g.get_state(), c.get_state())


def test_stepper_waits_give_up_and_the_context_survives():
    """The persistent stepper's waits (for a step's publication, for neighbour tiles' flags) are
    bounded: run against blocks nothing publishes they give up, record FV_ERR_TIMEOUT, and a CTA
    waiting on the same block leaves at once; afterwards the stepper still matches the oracle."""
    for _ in range(2):
        assert _lib.lib().fv_stepper_wait_selftest() == 4  # FV_ERR_TIMEOUT
    n = 64
    rho, u, v, p, _, _ = ic.sample("blast", 4, n)
    U0 = ic.to_conserved(rho, u, v, p)
    grid = dict(nx=n, ny=n, bc_x="periodic", bc_y="periodic")
    g = gpu_solver(grid, "rusanov", "minmod")
    g.set_state(U0)
    g.advance_to(0.02)
    c = cpu_solver("oracle", grid, "rusanov", "minmod")
    c.set_state(U0)
    c.advance_to(0.02)
    assert bits_equal(g.get_state(), c.get_state())
