"""Initial conditions: the driver's built-in test problems and the seeded random families.

Built-in tests (main2d.cpp:52-135): sod_x, sod_y, lax_liu3, sine2d, kh -> ``test_problem(name, n)``.

Random families, each fully determined by (family, index) through
``numpy.random.default_rng([crc32(family), index])`` (the seeding scheme of data/families.py:16-19),
with the parameter distributions of this build's workloads:

* ``riemann`` -- periodic [0,1]^2; corner (x0, y0) ~ U(0.2, 0.8)^2; each quadrant constant with
  rho ~ U(0.1, 2), p ~ U(0.1, 2), u, v ~ U(-1, 1); t_end = 0.25.
* ``blast``   -- periodic; background rho = 1, u = v = 0, p = 0.1; 1-3 blasts with p ~ U(5, 50) in
  discs of radius U(0.03, 0.1) at uniform centres (pressure only); 0-3 density bubbles with
  rho ~ U(0.1, 5), radius U(0.05, 0.15), density only (pressure balance kept).  Disc edges are the
  smooth tanh profile of width 0.005 with the periodic distance (data/families.py:70-79); t_end = 0.2.
* ``kh``      -- periodic Kelvin-Helmholtz: rho = 1 outside and 2 inside 0.25 < y < 0.75 with tanh
  edges of width w ~ U(0.02, 0.05); u = +0.5 outside, -0.5 inside; p = 2.5;
  v = A sin(4 pi x) with A ~ U(0.005, 0.02); recording starts at t_start ~ U(0, 1), t_end =
  t_start + 0.25.

All fields are float64 arrays of shape (n, n) indexed [j, i] (y first), like data/ic.py.
"""
import zlib

import numpy as np

PI = 3.14159265358979323846  # main2d.cpp:89


def cell_centres(n, lo=0.0, hi=1.0):
    """data/ic.py:13-15 / Grid::xc (grid2d.hpp:26)."""
    dx = (hi - lo) / n
    return lo + (np.arange(n) + 0.5) * dx


def rng_for(family, index):
    """A generator seeded only by the family name and the index (data/families.py:16-19)."""
    return np.random.default_rng([zlib.crc32(family.encode()), int(index)])


def periodic_distance(X, Y, cx, cy):
    """Shortest distance on the unit periodic box (data/families.py:70-74)."""
    dx = (X - cx + 0.5) % 1.0 - 0.5
    dy = (Y - cy + 0.5) % 1.0 - 0.5
    return np.sqrt(dx ** 2 + dy ** 2)


def smooth_disc(r, radius, width):
    """1 inside, 0 outside, tanh edge (data/families.py:77-79)."""
    return 0.5 * (1.0 - np.tanh((r - radius) / width))


def riemann(rng, n):
    xs, ys = rng.uniform(0.2, 0.8), rng.uniform(0.2, 0.8)
    # quadrant k = 0 bottom-left, 1 bottom-right, 2 top-left, 3 top-right; columns rho, u, v, p
    states = np.array([[rng.uniform(0.1, 2.0), rng.uniform(-1.0, 1.0), rng.uniform(-1.0, 1.0),
                        rng.uniform(0.1, 2.0)] for _ in range(4)])
    x = cell_centres(n)
    X, Y = np.meshgrid(x, x)
    quadrant = (X > xs).astype(int) + 2 * (Y > ys).astype(int)
    rho, u, v, p = (np.ascontiguousarray(states[quadrant, q]) for q in range(4))
    return rho, u, v, p, 0.25, {"split_x": xs, "split_y": ys, "states": states}


BLAST_EDGE = 0.005


def blast(rng, n):
    x = cell_centres(n)
    X, Y = np.meshgrid(x, x)
    rho = np.full((n, n), 1.0)
    p = np.full((n, n), 0.1)
    blasts, bubbles = [], []
    for _ in range(int(rng.integers(1, 4))):
        cx, cy = rng.uniform(0.0, 1.0, size=2)
        R = rng.uniform(0.03, 0.1)
        pb = rng.uniform(5.0, 50.0)
        w = smooth_disc(periodic_distance(X, Y, cx, cy), R, BLAST_EDGE)
        p = p + w * (pb - p)
        blasts.append([cx, cy, R, pb])
    for _ in range(int(rng.integers(0, 4))):
        cx, cy = rng.uniform(0.0, 1.0, size=2)
        R = rng.uniform(0.05, 0.15)
        rb = rng.uniform(0.1, 5.0)
        w = smooth_disc(periodic_distance(X, Y, cx, cy), R, BLAST_EDGE)
        rho = rho * (1.0 + w * (rb - 1.0))
        bubbles.append([cx, cy, R, rb])
    u = np.zeros((n, n))
    v = np.zeros((n, n))
    params = {"blasts": np.array(blasts).reshape(-1, 4), "bubbles": np.array(bubbles).reshape(-1, 4)}
    return rho, u, v, p, 0.2, params


def kh(rng, n):
    w = rng.uniform(0.02, 0.05)
    A = rng.uniform(0.005, 0.02)
    t_start = rng.uniform(0.0, 1.0)
    x = cell_centres(n)
    X, Y = np.meshgrid(x, x)
    inside = 0.5 * (np.tanh((Y - 0.25) / w) - np.tanh((Y - 0.75) / w))  # ~1 in the band, ~0 outside
    rho = 1.0 + inside
    u = 0.5 - inside
    v = A * np.sin(4.0 * PI * X)
    p = np.full((n, n), 2.5)
    return rho, u, v, p, t_start + 0.25, {"width": w, "amp": A, "t_start": t_start}


FAMILIES = {"riemann": riemann, "blast": blast, "kh": kh}


def sample(family, index, n):
    """(rho, u, v, p, t_end, params) for one member of a family (data/families.py:176-182)."""
    if family not in FAMILIES:
        raise ValueError(f"unknown family '{family}' (have: {', '.join(FAMILIES)})")
    rho, u, v, p, t_end, params = FAMILIES[family](rng_for(family, index), n)
    return rho, u, v, p, t_end, {"family": family, "index": int(index), **params}


def ensemble_spec(count=256, sizes=(64, 128, 256, 512), seed=2026):
    """Members of the batched-ensemble workload: `count` periodic trajectories, alternately a
    four-quadrant Riemann and a blast + bubble initial condition (member k is index k // 2 of its
    family), each with a grid size drawn uniformly from `sizes` by a generator seeded with `seed`.
    Returns a list of (family, index, n)."""
    rng = np.random.default_rng(seed)
    return [("riemann" if k % 2 == 0 else "blast", k // 2, int(sizes[int(rng.integers(len(sizes)))]))
            for k in range(count)]


def to_conserved(rho, u, v, p):
    """state2d.hpp:16-19 elementwise, same association (numpy rounds every operation separately,
    like the reference's build without FMA contraction).  Returns (ny, nx, 4)."""
    E = p / (1.4 - 1.0) + 0.5 * rho * (u * u + v * v)
    return np.ascontiguousarray(np.stack([rho, rho * u, rho * v, E], axis=-1))


def test_problem(name, n):
    """The driver's built-in tests (main2d.cpp:52-135).  Returns (grid kwargs, t_end, U (ny,nx,4))."""
    if name in ("sod_x", "sod_y"):
        m = 4
        along_x = name == "sod_x"
        if along_x:
            g = dict(nx=n, ny=m, x_min=0.0, x_max=1.0, y_min=0.0, y_max=float(m) / n,
                     bc_x="transmissive", bc_y="transmissive")
        else:
            g = dict(nx=m, ny=n, x_min=0.0, x_max=float(m) / n, y_min=0.0, y_max=1.0,
                     bc_x="transmissive", bc_y="transmissive")
        xc = g["x_min"] + (np.arange(g["nx"]) + 0.5) * ((g["x_max"] - g["x_min"]) / g["nx"])
        yc = g["y_min"] + (np.arange(g["ny"]) + 0.5) * ((g["y_max"] - g["y_min"]) / g["ny"])
        X, Y = np.meshgrid(xc, yc)
        s = X if along_x else Y
        left = s < 0.5
        rho = np.where(left, 1.0, 0.125)
        p = np.where(left, 1.0, 0.1)
        z = np.zeros_like(rho)
        return g, 0.2, to_conserved(rho, z, z, p)
    if name == "lax_liu3":
        g = dict(nx=n, ny=n, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, bc_x="transmissive", bc_y="transmissive")
        x = cell_centres(n)
        X, Y = np.meshgrid(x, x)
        right, top = X > 0.5, Y > 0.5
        q1, q2 = (1.5, 0.0, 0.0, 1.5), (0.5323, 1.206, 0.0, 0.3)
        q3, q4 = (0.138, 1.206, 1.206, 0.029), (0.5323, 0.0, 1.206, 0.3)
        fields = []
        for q in range(4):
            fields.append(np.where(top, np.where(right, q1[q], q2[q]), np.where(right, q4[q], q3[q])))
        return g, 0.3, to_conserved(*fields)
    if name == "sine2d":
        g = dict(nx=n, ny=n, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, bc_x="periodic", bc_y="periodic")
        x = cell_centres(n)
        X, Y = np.meshgrid(x, x)
        rho = 1.0 + 0.2 * np.sin(2.0 * PI * (X + Y))
        one = np.ones_like(rho)
        return g, 1.0, to_conserved(rho, one, one, one)
    if name == "kh":
        g = dict(nx=n, ny=n, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, bc_x="periodic", bc_y="periodic")
        x = cell_centres(n)
        X, Y = np.meshgrid(x, x)
        rho1, rho2 = 1.0, 2.0
        rhom = 0.5 * (rho1 - rho2)
        u1, u2 = 0.5, -0.5
        um = 0.5 * (u1 - u2)
        L = 0.025
        rho = np.where(Y < 0.25, rho1 - rhom * np.exp((Y - 0.25) / L),
              np.where(Y < 0.5, rho2 + rhom * np.exp((0.25 - Y) / L),
              np.where(Y < 0.75, rho2 + rhom * np.exp((Y - 0.75) / L), rho1 - rhom * np.exp((0.75 - Y) / L))))
        u = np.where(Y < 0.25, u1 - um * np.exp((Y - 0.25) / L),
            np.where(Y < 0.5, u2 + um * np.exp((0.25 - Y) / L),
            np.where(Y < 0.75, u2 + um * np.exp((Y - 0.75) / L), u1 - um * np.exp((0.75 - Y) / L))))
        v = 0.01 * np.sin(4.0 * PI * X)
        return g, 2.0, to_conserved(rho, u, v, np.full_like(rho, 2.5))
    raise ValueError(f"Unknown test '{name}' (use sod_x, sod_y, lax_liu3, sine2d or kh)")
