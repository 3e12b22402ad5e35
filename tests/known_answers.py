"""The reference's own known-answer checks, restated once and run against any implementation.

Sources (GusGus2004/neural-pde-surrogate): solver/src/test_solver2d.cpp:35-108,
test_riemann2d.cpp:17-47, test_grid2d.cpp:33-63, README.md:36-69 (validation numbers: Sod errors, Lax-Liu symmetry,
Kelvin-Helmholtz growth rates).
Each function takes a factory make(g, flux, limiter, cfl) returning an object with set_state /
get_state / compute_dt / step (the interface shared by oracle.OracleSolver and the GPU Solver).
"""
import importlib

import numpy as np

ic = importlib.import_module("neural-pde-surrogate_b200.ic")


def run_to(s, t_end):
    """test_solver2d.cpp:23-33: while (t < t_end) { dt = min(compute_dt, t_end - t); step; }"""
    t, steps = 0.0, 0
    while t < t_end:
        dt = s.compute_dt()
        dt = (t_end - t) if (t_end - t) < dt else dt
        s.step(dt)
        t += dt
        steps += 1
    return steps


def free_stream(make):
    """test_solver2d.cpp:37-53: a uniform moving state stays uniform (< 1e-13)."""
    g = dict(nx=16, ny=12, bc_x="periodic", bc_y="periodic")
    U0 = ic.to_conserved(np.array(1.3), np.array(0.7), np.array(-0.4), np.array(2.0))
    U = np.broadcast_to(U0, (12, 16, 4)).copy()
    s = make(g, "hllc", "vanleer", 0.5)
    s.set_state(U)
    run_to(s, 0.5)
    return float(np.max(np.abs(s.get_state() - U0)))


def sod_pair(make, flux="hllc", limiter="vanleer"):
    """test_solver2d.cpp:55-71: Sod along x (200x4) and along y (4x200)."""
    gx, t_end, Ux = ic.test_problem("sod_x", 200)
    gy, _, Uy = ic.test_problem("sod_y", 200)
    sx = make(gx, flux, limiter, 0.5)
    sy = make(gy, flux, limiter, 0.5)
    sx.set_state(Ux)
    sy.set_state(Uy)
    nsx, nsy = run_to(sx, t_end), run_to(sy, t_end)
    return nsx, nsy, Ux, sx.get_state(), sy.get_state()


def total(U, q, dx, dy):
    """test_solver2d.cpp:15-20: row-major sum times dx*dy."""
    s = 0.0
    for v in U[..., q].ravel():
        s += float(v)
    return s * dx * dy


def check_sod(make):
    """All of test_solver2d.cpp 2-2e; returns a dict of named results."""
    nsx, nsy, U0, X, Y = sod_pair(make)
    N, M = 200, 4
    dx, dy = 1.0 / N, (float(M) / N) / M
    res = {}
    res["same_steps"] = nsx == nsy
    res["rows_identical"] = float(np.max(np.abs(X[1:, :, 0] - X[0:1, :, 0])))
    res["my_zero"] = float(np.max(np.abs(X[..., 2])))
    sym = 0.0
    for q_x, q_y in ((0, 0), (1, 2), (2, 1), (3, 3)):
        sym = max(sym, float(np.max(np.abs(X[..., q_x] - Y[..., q_y].T))))
    res["transpose"] = sym
    res["mass"] = abs(total(X, 0, dx, dy) - total(U0, 0, dx, dy))
    res["energy"] = abs(total(X, 3, dx, dy) - total(U0, 3, dx, dy))
    c = X[0, int(0.78 * N)]
    u = c[1] / c[0]
    p = (1.4 - 1.0) * (c[3] - 0.5 * c[0] * (u * u + (c[2] / c[0]) ** 2))
    res["plateau"] = (c[0], p, u)
    res["steps"] = nsx
    return res


RIEMANN_STATES = [(1.0, 0.0, 1.0, 0.125, 0.0, 0.1), (1.0, 0.75, 1.0, 0.125, 0.0, 0.1),
                  (1.0, 2.0, 0.4, 1.0, -2.0, 0.4)]  # test_riemann2d.cpp:17-19


def close(a, b, tol=1e-13):
    """test_riemann2d.cpp:10-13"""
    return abs(a - b) <= tol * (1.0 + abs(b))


def sod_l1(U, n):
    """L1 density error against the exact Sod solution at t = 0.2 on x-cells (plot_sod.py:73-76)."""
    from oracle.exact_riemann import exact_riemann
    x = (np.arange(n) + 0.5) / n
    exact, _, _ = exact_riemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), x, 0.5, 0.2)
    return float(np.sum(np.abs(U[0, :, 0] - exact[:, 0])) * (1.0 / n))


def kh_mode_amplitude(U, n):
    """Amplitude of the seeded sin(4 pi x) mode of v near the two shear layers: the diagnostic of
    McNally, Lyra & Passy (2012), eqs. 4-7, applied as experiments/kh_growth.py:17-27 applies it."""
    x = ic.cell_centres(n)
    X, Y = np.meshgrid(x, x)
    v = U[..., 2] / U[..., 0]
    w = np.exp(-4.0 * np.pi * np.where(Y < 0.5, np.abs(Y - 0.25), np.abs(0.75 - Y)))
    s = np.sum(v * np.sin(4.0 * np.pi * X) * w) / np.sum(w)
    c = np.sum(v * np.cos(4.0 * np.pi * X) * w) / np.sum(w)
    return 2.0 * float(np.hypot(s, c))


def kh_growth_rate(make, n, nout=20, t_end=2.0, window=(0.6, 1.2)):
    """Exponential growth rate of the seeded KH mode (the driver's `kh` test, HLLC + van Leer):
    frames at the driver's times t_end * k / nout (main2d.cpp:236-242), the slope of log amplitude
    fitted over `window` (experiments/kh_growth.py:38-40)."""
    g, _, U0 = ic.test_problem("kh", n)
    s = make(g, "hllc", "vanleer", 0.5)
    s.set_state(U0)
    t, ts, amps = 0.0, [0.0], [kh_mode_amplitude(U0, n)]
    for k in range(1, nout + 1):
        t_next = 0.0 + ((t_end - 0.0) * k) / nout
        if t_next > window[1] + 1e-12:
            break
        while t < t_next:
            dt = s.compute_dt()
            dt = (t_next - t) if (t_next - t) < dt else dt
            s.step(dt)
            t += dt
        ts.append(t)
        amps.append(kh_mode_amplitude(s.get_state(), n))
    ts, amps = np.array(ts), np.array(amps)
    sel = (ts >= window[0] - 1e-12) & (ts <= window[1] + 1e-12)
    return float(np.polyfit(ts[sel], np.log(amps[sel]), 1)[0]), amps


def sine2d_l1(make, n, limiter):
    """experiments/results.md section 3 (2D diagonal advection, HLLC, CFL 0.5, t = 1): the L1 density
    error against the exact solution sampled at cell centres, sum |err| dx dy, as
    experiments/convergence_sine2d.py:18-26 computes it; one run to t = 1."""
    g, t_end, U0 = ic.test_problem("sine2d", n)
    s = make(g, "hllc", limiter, 0.5)
    s.set_state(U0)
    run_to(s, t_end)
    x = ic.cell_centres(n)
    X, Y = np.meshgrid(x, x)
    exact = 1.0 + 0.2 * np.sin(2.0 * np.pi * (X + Y - 2.0 * t_end))
    return float(np.abs(s.get_state()[..., 0] - exact).sum() * (x[1] - x[0]) * (x[1] - x[0]))


def kh_final_amplitude(make, n, nout=20):
    """experiments/results.md:98-102: the seeded KH mode's amplitude at the driver's end time t = 2
    (the `kh` test, HLLC + van Leer, frames every t_end / nout)."""
    g, t_end, U0 = ic.test_problem("kh", n)
    s = make(g, "hllc", "vanleer", 0.5)
    s.set_state(U0)
    t = 0.0
    for k in range(1, nout + 1):
        t_next = 0.0 + ((t_end - 0.0) * k) / nout
        while t < t_next:
            dt = s.compute_dt()
            dt = (t_next - t) if (t_next - t) < dt else dt
            s.step(dt)
            t += dt
    return kh_mode_amplitude(s.get_state(), n)
