"""Pins the CPU oracle (oracle/fv_oracle.c) to the reference before anything is checked against it:
the reference's own unit programs, bit-for-bit agreement with the reference build on random cases,
the golden fixtures, and the reference's known answers."""
import subprocess
import zlib

import numpy as np
import pytest

from cases import bits_equal, cpu_solver, golden_names, load_golden
import known_answers as ka
from oracle import oracle as orc
from oracle.build_oracle import REF_OUT, build_oracle

build_oracle()
ref = pytest.mark.skipif(not orc.ref_available(), reason="oracle/_ref not built (reference tree absent)")


@ref
@pytest.mark.parametrize("prog", ["test_riemann2d", "test_grid2d", "test_solver2d"])
def test_reference_unit_programs_pass(prog):
    exe = REF_OUT / prog
    if not exe.exists():
        pytest.skip(f"{exe} not built")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "ALL PASSED" in r.stdout, r.stdout


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_golden(name):
    d = load_golden(name)
    s = cpu_solver("oracle", d["g"], d["flux"], d["limiter"], float(d["cfl"]))
    s.set_state(d["U0"])
    assert s.compute_dt() == float(d["dt0"])
    times, levels = s.run(float(d["t_end"]), 0.0, int(d["nout"]), d["save"])
    assert s.steps == int(d["steps"])
    assert bits_equal(times, d["times"])
    assert bits_equal(s.get_state(), d["U"])
    for m in d["save"]:
        assert bits_equal(levels[m], d[f"level_{m}"])


def _random_case(rng, nx, ny, bcx, bcy):
    rho = 0.5 + rng.random((ny, nx))
    u = rng.uniform(-1, 1, (ny, nx))
    v = rng.uniform(-1, 1, (ny, nx))
    p = 0.3 + rng.random((ny, nx))
    from known_answers import ic
    g = dict(nx=nx, ny=ny, x_min=-0.5, x_max=0.5 + 0.1 * nx, y_min=0.0, y_max=0.7, bc_x=bcx, bc_y=bcy)
    return g, ic.to_conserved(rho, u, v, p)


@ref
@pytest.mark.parametrize("flux", ["hllc", "rusanov"])
@pytest.mark.parametrize("lim", ["none", "unlimited", "minmod", "vanleer"])
@pytest.mark.parametrize("shape,bcs", [((1, 5), ("periodic", "transmissive")), ((2, 3), ("transmissive", "periodic")),
                                       ((37, 21), ("periodic", "periodic")), ((21, 37), ("transmissive", "transmissive"))])
def test_oracle_bitexact_vs_reference(flux, lim, shape, bcs):
    rng = np.random.default_rng(zlib.crc32(repr((flux, lim, shape)).encode()))
    g, U0 = _random_case(rng, shape[0], shape[1], *bcs)
    a = cpu_solver("oracle", g, flux, lim, 0.45)
    b = cpu_solver("ref", g, flux, lim, 0.45)
    a.set_state(U0)
    b.set_state(U0)
    for _ in range(3):
        da, db = a.compute_dt(), b.compute_dt()
        assert da == db
        a.step(da)
        b.step(db)
    assert bits_equal(a.get_state(), b.get_state())
    outcome = []
    for s in (a, b):
        try:
            s.run(0.05, 0.0, 2, ())
            outcome.append(None)
        except orc.NonPhysical as e:  # unlimited slopes may blow up: both must stop at the same cell
            outcome.append((e.i, e.j))
    assert outcome[0] == outcome[1]
    assert a.steps == b.steps and bits_equal(a.get_state(), b.get_state())


@ref
def test_oracle_block_average_vs_reference():
    from known_answers import ic
    rho, u, v, p, _, _ = ic.sample("blast", 11, 64)
    g = dict(nx=64, ny=64, bc_x="periodic", bc_y="periodic")
    a, b = cpu_solver("oracle", g, "hllc", "minmod"), cpu_solver("ref", g, "hllc", "minmod")
    U0 = ic.to_conserved(rho, u, v, p)
    for s in (a, b):
        s.set_state(U0)
        s.advance_to(0.004)
    for f in (1, 2, 4, 8, 16):
        assert bits_equal(a.block_average(f), b.block_average(f))


@ref
@pytest.mark.parametrize("index", [1, 2, 4])
def test_oracle_nonphysical_report_matches_reference(index):
    """Unlimited slopes on a blast drive rho or p negative (the reference's results.md:40,45-46 reports
    the same for Sod at CFL 0.8); both report the same first bad cell, after the same number of steps,
    instead of exiting."""
    from known_answers import ic
    rho, u, v, p, _, _ = ic.sample("blast", index, 64)
    U0 = ic.to_conserved(rho, u, v, p)
    g = dict(nx=64, ny=64, bc_x="periodic", bc_y="periodic")
    out = []
    for kind in ("oracle", "ref"):
        s = cpu_solver(kind, g, "hllc", "unlimited")
        s.set_state(U0)
        with pytest.raises(orc.NonPhysical) as e:
            s.advance_to(0.2)
        out.append((e.value.i, e.value.j, e.value.rho, e.value.p, s.steps, s.get_state().tobytes()))
    assert out[0] == out[1]


@ref
@pytest.mark.parametrize("bcs", [("transmissive", "transmissive"), ("periodic", "periodic"), ("periodic", "transmissive")])
def test_ghost_fill_matches_reference(bcs):
    """test_grid2d.cpp:26-63 on the 5x3 grid: the ghost ring the oracle builds is the reference's."""
    nx, ny = 5, 3
    Ug = np.zeros((ny + 4, nx + 4, 4))
    for j in range(ny):
        for i in range(nx):
            Ug[j + 2, i + 2] = (1.0, i, j, 0.0)
    a = orc.apply_bcs_ghosted(Ug.copy(), *bcs, which="oracle")
    b = orc.apply_bcs_ghosted(Ug.copy(), *bcs, which="ref")
    assert bits_equal(a, b)


def test_ghost_fill_known_answers():
    """test_grid2d.cpp:40-63 restated on the oracle."""
    nx, ny = 5, 3
    def fill(bcx, bcy):
        Ug = np.zeros((ny + 4, nx + 4, 4))
        for j in range(ny):
            for i in range(nx):
                Ug[j + 2, i + 2] = (1.0, i, j, 0.0)
        return orc.apply_bcs_ghosted(Ug, bcx, bcy)
    def src(U, i, j):
        c = U[j + 2, i + 2]
        return (c[1], c[2])
    U = fill("transmissive", "transmissive")
    assert src(U, -1, 1) == (0, 1) and src(U, -2, 1) == (0, 1)
    assert src(U, 5, 2) == (4, 2) and src(U, 6, 2) == (4, 2)
    assert src(U, 3, -1) == (3, 0) and src(U, 3, -2) == (3, 0)
    assert src(U, 3, 3) == (3, 2) and src(U, 3, 4) == (3, 2)
    assert src(U, -2, -2) == (0, 0) and src(U, 6, 4) == (4, 2)
    U = fill("periodic", "periodic")
    assert src(U, -1, 1) == (4, 1) and src(U, -2, 1) == (3, 1)
    assert src(U, 5, 1) == (0, 1) and src(U, 6, 1) == (1, 1)
    assert src(U, 2, -1) == (2, 2) and src(U, 2, -2) == (2, 1)
    assert src(U, 2, 3) == (2, 0) and src(U, 2, 4) == (2, 1)
    assert src(U, -1, -1) == (4, 2) and src(U, 5, 3) == (0, 0)
    U = fill("periodic", "transmissive")
    assert src(U, -1, 1) == (4, 1) and src(U, 2, 3) == (2, 2)


@pytest.mark.parametrize("which", ["oracle", pytest.param("ref", marks=ref)])
def test_riemann_known_answers(which):
    """test_riemann2d.cpp:17-47."""
    from known_answers import ic
    for s in ka.RIEMANN_STATES:
        L = ic.to_conserved(np.array(s[0]), np.array(s[1]), np.array(0.0), np.array(s[2]))
        R = ic.to_conserved(np.array(s[3]), np.array(s[4]), np.array(0.0), np.array(s[5]))
        F2 = orc.flux("x", "hllc", L, R, which)
        L1 = np.array([s[0], s[0] * s[1], s[2] / (1.4 - 1.0) + 0.5 * s[0] * s[1] * s[1]])
        R1 = np.array([s[3], s[3] * s[4], s[5] / (1.4 - 1.0) + 0.5 * s[3] * s[4] * s[4]])
        F1 = orc.hllc_1d(L1, R1, which)
        assert ka.close(F2[0], F1[0]) and ka.close(F2[1], F1[1]) and ka.close(F2[3], F1[2])
        assert ka.close(F2[2], 0.0)
        Ly = ic.to_conserved(np.array(s[0]), np.array(0.0), np.array(s[1]), np.array(s[2]))
        Ry = ic.to_conserved(np.array(s[3]), np.array(0.0), np.array(s[4]), np.array(s[5]))
        Fy = orc.flux("y", "hllc", Ly, Ry, which)
        assert ka.close(Fy[0], F2[0]) and ka.close(Fy[2], F2[1]) and ka.close(Fy[3], F2[3])
    U = ic.to_conserved(np.array(1.3), np.array(0.4), np.array(-0.7), np.array(2.1))
    F = orc.flux("x", "hllc", U, U, which)
    u = U[1] / U[0]
    p = (1.4 - 1.0) * (U[3] - 0.5 * U[0] * (u * u + (U[2] / U[0]) ** 2))
    Fp = np.array([U[1], U[1] * u + p, U[2] * u, u * (U[3] + p)])
    assert ka.close(F[1], Fp[1]) and ka.close(F[2], Fp[2]) and ka.close(F[3], Fp[3])


def test_solver_known_answers_on_oracle():
    """test_solver2d.cpp:35-108 restated on the oracle."""
    mk = lambda g, f, l, c: cpu_solver("oracle", g, f, l, c)
    assert ka.free_stream(mk) < 1e-13
    r = ka.check_sod(mk)
    assert r["same_steps"]
    assert r["rows_identical"] == 0.0 and r["my_zero"] == 0.0 and r["transpose"] == 0.0
    assert r["mass"] < 1e-13 and r["energy"] < 1e-13
    rho, p, u = r["plateau"]
    assert abs(rho - 0.26557) < 1e-3 and abs(p - 0.30313) < 1e-3 and abs(u - 0.92745) < 1e-3


def test_exact_sod_star_state():
    """README.md:38 / results.md:23: p* = 0.30313, u* = 0.92745."""
    from oracle.exact_riemann import star_state
    ps, us = star_state((1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    assert round(ps, 5) == 0.30313 and round(us, 5) == 0.92745


def test_kh_growth_rates_match_the_reference_validation():
    """README.md:66-69 / experiments/results.md:98-102: the seeded KH mode decays at 16^2 and grows at
    1.20, 2.41 and 2.71 at 32^2, 64^2 and 128^2 (HLLC + van Leer, fit over 0.6 <= t <= 1.2); its
    amplitude at t = 2 is 0.193 at 64^2 and 0.225 at 128^2."""
    mk = lambda g, f, l, c: cpu_solver("oracle", g, f, l, c)
    assert ka.kh_growth_rate(mk, 16)[0] < 0.0
    for n, published in ((32, 1.20), (64, 2.41), (128, 2.71)):
        rate, amps = ka.kh_growth_rate(mk, n)
        assert abs(rate - published) < 0.01, (n, rate, published)
        assert amps[0] == pytest.approx(0.01)  # the seeded amplitude, v = 0.01 sin(4 pi x)
    for n, published in ((64, "0.193"), (128, "0.225")):  # the final mode amplitude at t = 2
        assert f"{ka.kh_final_amplitude(mk, n):.3f}" == published


@pytest.mark.parametrize("n,limiter,published", [(32, "none", "9.024e-02"), (32, "vanleer", "1.088e-02"),
                                                 (64, "none", "5.862e-02"), (64, "vanleer", "3.203e-03"),
                                                 (128, "none", "3.379e-02"), (128, "vanleer", "8.531e-04")])
def test_sine2d_errors_match_the_published_table(n, limiter, published):
    """experiments/results.md section 3: the reference's published L1 errors, to every printed digit."""
    mk = lambda g, f, l, c: cpu_solver("oracle", g, f, l, c)
    assert f"{ka.sine2d_l1(mk, n, limiter):.3e}" == published


def test_lax_liu3_symmetric_to_the_published_level():
    """README.md:64: Lax-Liu configuration 3 at 256^2, t = 0.3 (HLLC + van Leer) is symmetric about
    x = y to 3e-14 (density; the oracle gives 2.4e-14)."""
    g, t_end, U0 = ka.ic.test_problem("lax_liu3", 256)
    s = cpu_solver("oracle", g, "hllc", "vanleer", 0.5)
    s.set_state(U0)
    s.advance_to(t_end)
    U = s.get_state()
    assert t_end == 0.3 and np.abs(U[..., 0] - U[..., 0].T).max() < 3e-14
    assert max(np.abs(U[..., 1] - U[..., 2].T).max(), np.abs(U[..., 3] - U[..., 3].T).max()) < 1e-13
