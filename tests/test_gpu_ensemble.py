"""Batched ensemble: every member must match its single-trajectory run bit for bit (same steps,
same time, same state), whatever the other members do."""
import importlib

import numpy as np
import pytest

from cases import bits_equal, gpu_solver

pytestmark = pytest.mark.gpu
fv = importlib.import_module("neural-pde-surrogate_b200")
ic = importlib.import_module("neural-pde-surrogate_b200.ic")
ens_mod = importlib.import_module("neural-pde-surrogate_b200.ensemble")


@pytest.fixture(autouse=True)
def _gpu(cuda_ok):
    pass


def _members():
    rng = np.random.default_rng(3)
    out = []
    for k, (n, m, fam, bcs) in enumerate([(64, 64, "riemann", ("periodic", "periodic")),
                                          (128, 128, "blast", ("periodic", "periodic")),
                                          (96, 64, None, ("periodic", "transmissive")),
                                          (33, 17, None, ("transmissive", "periodic")),
                                          (1, 5, None, ("periodic", "transmissive")),
                                          (64, 64, "blast", ("periodic", "periodic")),
                                          (256, 256, "riemann", ("periodic", "periodic")),
                                          (16, 48, None, ("transmissive", "transmissive"))]):
        if fam:
            rho, u, v, p, _, _ = ic.sample(fam, k, n)
        else:
            rho = 0.5 + rng.random((m, n))
            u, v = rng.uniform(-1, 1, (m, n)), rng.uniform(-1, 1, (m, n))
            p = 0.3 + rng.random((m, n))
        g = fv.make_grid(n, m, 0.0, 1.0, 0.0, m / n if fam is None else 1.0, *bcs)
        out.append((g, ic.to_conserved(rho, u, v, p)))
    return out


def _single(g, U0, flux, lim, t_next):
    s = gpu_solver(dict(nx=g.nx, ny=g.ny, x_min=g.x_min, x_max=g.x_max, y_min=g.y_min, y_max=g.y_max,
                        bc_x=("transmissive", "periodic")[g.bc_x], bc_y=("transmissive", "periodic")[g.bc_y]),
                   flux, lim)
    s.set_state(U0)
    t, steps = s.advance_to(t_next)
    return t, steps, s.get_state()


@pytest.mark.parametrize("flux,lim", [("hllc", "vanleer"), ("rusanov", "minmod")])
def test_members_bitexact_vs_single_runs(flux, lim):
    members = _members()
    ens = ens_mod.Ensemble([g for g, _ in members], flux, lim)
    for k, (_, U0) in enumerate(members):
        ens.set_state(k, U0)
    t_next = np.array([0.05, 0.02, 0.03, 0.04, 0.05, 0.01, 0.03, 0.02])
    t, steps, status = ens.advance_to(t_next)
    assert (status == 0).all()
    for k, (g, U0) in enumerate(members):
        ts, ns, Us = _single(g, U0, flux, lim, t_next[k])
        assert t[k] == ts and steps[k] == ns, k
        assert bits_equal(ens.get_state(k), Us), k
    assert ens.launch_count() > 0


def test_two_advances_equal_one_run():
    members = _members()[:4]
    ens = ens_mod.Ensemble([g for g, _ in members], "hllc", "vanleer")
    for k, (_, U0) in enumerate(members):
        ens.set_state(k, U0)
    ens.advance_to(0.01)
    t, steps, _ = ens.advance_to(0.025)
    for k, (g, U0) in enumerate(members):
        s = gpu_solver(dict(nx=g.nx, ny=g.ny, x_min=g.x_min, x_max=g.x_max, y_min=g.y_min, y_max=g.y_max,
                            bc_x=("transmissive", "periodic")[g.bc_x], bc_y=("transmissive", "periodic")[g.bc_y]),
                       "hllc", "vanleer")
        s.set_state(U0)
        s.advance_to(0.01)
        ts, ns = s.advance_to(0.025)
        assert t[k] == ts and steps[k] == ns and bits_equal(ens.get_state(k), s.get_state())


def test_nonphysical_member_stops_alone():
    """With unlimited slopes the blast member goes non-physical (like the reference, which would
    exit); it stops exactly where its single run stops, while the smooth members finish."""
    n = 64
    rho, u, v, p, _, _ = ic.sample("blast", 1, n)
    blast = ic.to_conserved(rho, u, v, p)
    gk, _, sine = ic.test_problem("sine2d", n)
    g = fv.make_grid(n, n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic")
    ens = ens_mod.Ensemble([g, g, g], "hllc", "unlimited")
    for k, U0 in enumerate((sine, blast, sine)):
        ens.set_state(k, U0)
    t, steps, status = ens.advance_to(0.2, raise_on_nonphysical=False)
    assert list(status) == [0, 3, 0]
    single = gpu_solver(dict(nx=n, ny=n, bc_x="periodic", bc_y="periodic"), "hllc", "unlimited")
    single.set_state(blast)
    with pytest.raises(fv.NonPhysicalError):
        single.advance_to(0.2)
    assert steps[1] == single.time()[1] and bits_equal(ens.get_state(1), single.get_state())
    ts, ns, Us = _single(g, sine, "hllc", "unlimited", 0.2)
    assert steps[0] == ns and bits_equal(ens.get_state(0), Us) and bits_equal(ens.get_state(2), Us)
    with pytest.raises(fv.FVError):
        ens.advance_to(0.3)


def test_device_buffers_are_ordered_against_torchs_stream():
    """The ensemble queues its copies on its own non-blocking stream.  A tensor whose last write on
    torch's current stream is still queued behind a long matmul must still reach the ensemble intact
    (set_all waits for torch's stream), and torch must see get_all's copy (it waits for the library's
    stream) -- without either wait the copy would move stale data."""
    import torch
    B, n = 4, 64
    g = fv.make_grid(n, n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic")
    e = ens_mod.Ensemble([g] * B, "hllc", "vanleer")
    U = torch.stack([torch.from_numpy(ic.to_conserved(*ic.sample("riemann", k, n)[:4])) for k in range(B)]).cuda()
    x = torch.zeros_like(U)
    big = torch.randn(6144, 6144, device="cuda")
    out = torch.zeros_like(U)
    torch.cuda.synchronize()
    for _ in range(3):
        y = big @ big  # milliseconds of queued work on torch's stream
        x.copy_(U + 0.0 * y[0, 0].double())  # x is final only after the matmul
        e.set_all(x)
        e.get_all(out)
        res = out * 1.0  # torch work on out, queued right behind get_all
        torch.cuda.synchronize()
        assert torch.equal(res, U)
        x.zero_()
        out.zero_()
