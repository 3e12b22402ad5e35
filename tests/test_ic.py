"""Initial conditions on the CPU: the seeded families' determinism and parameter ranges, and the
driver's built-in test problems (main2d.cpp:52-135)."""
import importlib

import numpy as np
import pytest

ic = importlib.import_module("neural-pde-surrogate_b200.ic")


@pytest.mark.parametrize("family", ["riemann", "blast", "kh"])
def test_a_member_depends_on_family_and_index_only(family):
    a = ic.sample(family, 17, 32)
    b = ic.sample(family, 17, 32)
    for x, y in zip(a[:4], b[:4]):
        assert x.tobytes() == y.tobytes()
    assert a[4] == b[4]
    c = ic.sample(family, 18, 32)
    assert any(x.tobytes() != y.tobytes() for x, y in zip(a[:4], c[:4]))
    # the resolution does not enter the seed: the same problem at another size
    d = ic.sample(family, 17, 64)
    for k, v in a[5].items():
        assert np.array_equal(np.asarray(v), np.asarray(d[5][k])), k
    for f in a[:4]:
        assert f.shape == (32, 32) and f.dtype == np.float64 and f.flags.c_contiguous


def test_families_use_distinct_streams():
    r = ic.rng_for("riemann", 5).uniform()
    assert r != ic.rng_for("blast", 5).uniform()
    assert r == ic.rng_for("riemann", 5).uniform()


def test_riemann_quadrants():
    for k in range(200):
        rho, u, v, p, t_end, prm = ic.sample("riemann", k, 16)
        assert t_end == 0.25
        assert 0.2 <= prm["split_x"] <= 0.8 and 0.2 <= prm["split_y"] <= 0.8
        st = prm["states"]
        assert st.shape == (4, 4)
        assert np.all((st[:, 0] >= 0.1) & (st[:, 0] <= 2.0)) and np.all((st[:, 3] >= 0.1) & (st[:, 3] <= 2.0))
        assert np.all(np.abs(st[:, 1:3]) <= 1.0)
        # every cell holds exactly its quadrant's state
        x = ic.cell_centres(16)
        X, Y = np.meshgrid(x, x)
        q = (X > prm["split_x"]).astype(int) + 2 * (Y > prm["split_y"]).astype(int)
        for f, col in zip((rho, u, v, p), range(4)):
            assert np.array_equal(f, st[q, col])


def test_blast_discs_and_bubbles():
    nblast, nbub = set(), set()
    for k in range(200):
        rho, u, v, p, t_end, prm = ic.sample("blast", k, 32)
        assert t_end == 0.2
        B, D = prm["blasts"], prm["bubbles"]
        nblast.add(len(B))
        nbub.add(len(D))
        assert 1 <= len(B) <= 3 and 0 <= len(D) <= 3
        assert np.all((B[:, 2] >= 0.03) & (B[:, 2] <= 0.1)) and np.all((B[:, 3] >= 5.0) & (B[:, 3] <= 50.0))
        if len(D):
            assert np.all((D[:, 2] >= 0.05) & (D[:, 2] <= 0.15)) and np.all((D[:, 3] >= 0.1) & (D[:, 3] <= 5.0))
        assert np.all((B[:, :2] >= 0.0) & (B[:, :2] <= 1.0))
        assert not u.any() and not v.any()
        # pressure from the blasts alone: bubbles change density only (pressure balance)
        x = ic.cell_centres(32)
        X, Y = np.meshgrid(x, x)
        pp = np.full((32, 32), 0.1)
        for cx, cy, R, pb in B:
            w = ic.smooth_disc(ic.periodic_distance(X, Y, cx, cy), R, ic.BLAST_EDGE)
            pp = pp + w * (pb - pp)
        assert np.array_equal(p, pp)
        assert p.min() >= 0.1 - 1e-15 and p.max() <= B[:, 3].max() + 1e-12
        assert rho.min() > 0.0
        if not len(D):
            assert np.all(rho == 1.0)
    assert nblast == {1, 2, 3} and nbub == {0, 1, 2, 3}


def test_kh_band():
    for k in range(100):
        rho, u, v, p, t_end, prm = ic.sample("kh", k, 64)
        assert 0.02 <= prm["width"] <= 0.05 and 0.005 <= prm["amp"] <= 0.02 and 0.0 <= prm["t_start"] <= 1.0
        assert t_end == prm["t_start"] + 0.25
        assert np.all((rho > 1.0 - 1e-12) & (rho < 2.0 + 1e-12))
        assert np.allclose(u + rho, 1.5, atol=1e-14)  # u = +0.5 where rho = 1, -0.5 where rho = 2
        assert np.all(p == 2.5)
        assert np.abs(v).max() <= prm["amp"] + 1e-15
        assert rho[32, 0] > 1.99 and rho[0, 0] < 1.01  # the band is around y = 0.5


def test_periodic_distance_wraps():
    assert ic.periodic_distance(np.array(0.01), np.array(0.5), 0.99, 0.5) == pytest.approx(0.02)
    assert ic.periodic_distance(np.array(0.5), np.array(0.02), 0.5, 0.98) == pytest.approx(0.04)
    assert ic.periodic_distance(np.array(0.3), np.array(0.3), 0.3, 0.3) == 0.0


def test_unknown_family():
    with pytest.raises(ValueError, match="unknown family 'sedov'"):
        ic.sample("sedov", 0, 16)


def test_to_conserved_follows_the_reference_association():
    rng = np.random.default_rng(3)
    rho, u, v, p = (rng.uniform(0.1, 2.0, (5, 7)) for _ in range(4))
    U = ic.to_conserved(rho, u, v, p)
    assert U.shape == (5, 7, 4) and U.flags.c_contiguous
    gm1 = 1.4 - 1.0
    for j in range(5):
        for i in range(7):
            r, a, b, q = float(rho[j, i]), float(u[j, i]), float(v[j, i]), float(p[j, i])
            want = (r, r * a, r * b, q / gm1 + 0.5 * r * (a * a + b * b))  # state2d.hpp:16-19, one rounding per op
            assert tuple(U[j, i]) == want


def test_built_in_problems():
    g, t_end, U = ic.test_problem("sod_x", 64)
    assert (g["nx"], g["ny"], t_end, g["bc_x"]) == (64, 4, 0.2, "transmissive") and U.shape == (4, 64, 4)
    assert U[0, 0, 0] == 1.0 and U[0, -1, 0] == 0.125
    gy, _, Uy = ic.test_problem("sod_y", 64)
    assert (gy["nx"], gy["ny"]) == (4, 64) and np.array_equal(Uy[:, 0, 0], U[0, :, 0])
    g, t_end, U = ic.test_problem("lax_liu3", 32)
    assert t_end == 0.3 and U[-1, -1, 0] == 1.5 and U[0, 0, 0] == 0.138
    g, t_end, U = ic.test_problem("sine2d", 32)
    assert g["bc_x"] == "periodic" and t_end == 1.0 and np.all(U[..., 1] == U[..., 0])
    g, t_end, U = ic.test_problem("kh", 32)
    assert t_end == 2.0 and np.all(U[..., 0] >= 1.0) and np.all(U[..., 0] <= 2.0)
    with pytest.raises(ValueError, match="Unknown test 'orszag'"):
        ic.test_problem("orszag", 32)
