"""The euler2d host driver (the reference's main2d.cpp over the C-ABI).

CPU: option handling before any device call, the .npz layer both ways (C++ writes -> numpy reads,
numpy.savez writes -> C++ reads), initial-condition validation (io_hdf5.hpp:197-204).
GPU: --traj and snapshot runs bit-identical to the oracle's driver loop (main2d.cpp:224-246), and a
restart from a snapshot (read_initial_condition accepts snapshots, io_hdf5.hpp:166-169).
"""
import importlib
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "neural-pde-surrogate_b200"
EXE = PKG / "host" / "euler2d"


@pytest.fixture(scope="module")
def exe():
    importlib.import_module("neural-pde-surrogate_b200.build").build()
    assert EXE.exists()
    return str(EXE)


def run(exe, *args, cwd=None):
    return subprocess.run([exe, *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=600)


@pytest.mark.parametrize("args,msg", [
    (["--bogus", "1"], "Unknown option --bogus"),
    (["--n"], "Expected '--key value', got '--n'"),
    (["--scheme", "roe"], "Unknown scheme 'roe' (use rusanov or hllc)"),
    (["--limiter", "superbee"], "Unknown limiter 'superbee'"),
    (["--n", "0"], "n, nout and cfl must be positive"),
    (["--cfl", "-1"], "n, nout and cfl must be positive"),
    (["--test", "orszag"], "Unknown test 'orszag' (use sod_x, sod_y, lax_liu3, sine2d or kh)"),
    (["--test", "sod_x", "--tend", "-2"], "tend must be positive"),
])
def test_driver_rejects_bad_options(exe, args, msg):
    r = run(exe, *args)
    assert r.returncode == 1 and msg in r.stderr, (r.returncode, r.stderr)


NPZ_HARNESS = r"""
#include "npz_io.hpp"
#include <iostream>
int main(int argc, char** argv) {
    if (std::string(argv[1]) == "write") {
        std::vector<double> a(6); for (int k = 0; k < 6; ++k) a[k] = 0.1 * k - 0.25;
        std::vector<float> b(2 * 4 * 3 * 5); for (size_t k = 0; k < b.size(); ++k) b[k] = float(k) / 7.0f;
        npz::write(argv[2], {{"a", npz::f64({2, 3}, a.data())}, {"b", npz::f32({2, 4, 3, 5}, b.data())},
                             {"t", npz::scalar(0.125)}, {"n", npz::scalar_int(-42)}, {"s", npz::string("periodic")},
                             {"v", npz::f64({6}, a.data())}});
        return 0;
    }
    auto f = npz::read(argv[2]);
    std::cout << "{";
    bool first = true;
    for (auto& kv : f) {
        std::cout << (first ? "" : ", ") << "\"" << kv.first << "\": {\"descr\": \"" << kv.second.descr << "\", \"shape\": [";
        for (size_t k = 0; k < kv.second.shape.size(); ++k) std::cout << (k ? ", " : "") << kv.second.shape[k];
        std::cout << "], \"value\": ";
        if (kv.second.descr[1] == 'U') std::cout << "\"" << kv.second.str() << "\"";
        else { auto v = kv.second.doubles(); double s = 0; for (double x : v) s += x; std::cout.precision(17); std::cout << s; }
        std::cout << "}";
        first = false;
    }
    std::cout << "}\n";
    return 0;
}
"""


@pytest.fixture(scope="module")
def npz_tool(tmp_path_factory):
    d = tmp_path_factory.mktemp("npz")
    src = d / "npz_tool.cpp"
    src.write_text(NPZ_HARNESS)
    out = d / "npz_tool"
    subprocess.run(["g++", "-O1", "-std=c++17", f"-I{PKG / 'host'}", "-o", str(out), str(src)], check=True)
    return str(out)


def test_npz_written_by_the_driver_reads_in_numpy(npz_tool, tmp_path):
    f = tmp_path / "w.npz"
    subprocess.run([npz_tool, "write", str(f)], check=True)
    z = np.load(f)
    a = 0.1 * np.arange(6) - 0.25
    assert z["a"].dtype == np.float64 and z["a"].shape == (2, 3) and np.array_equal(z["a"].ravel(), a)
    b = (np.arange(120, dtype=np.float32) / np.float32(7.0)).reshape(2, 4, 3, 5)
    assert z["b"].dtype == np.float32 and np.array_equal(z["b"], b)
    assert z["t"].shape == () and float(z["t"]) == 0.125
    assert z["n"].dtype == np.int32 and int(z["n"]) == -42
    assert str(z["s"]) == "periodic"
    assert z["v"].shape == (6,)


def test_npz_written_by_numpy_reads_in_the_driver(npz_tool, tmp_path):
    f = tmp_path / "r.npz"
    rng = np.random.default_rng(0)
    arrays = dict(rho=rng.random((3, 5)), u=rng.random((3, 5)).astype(np.float32), nx=np.int64(5),
                  ny=np.array(3, np.int32), bc_x=np.array("transmissive"), t_end=np.float64(0.25))
    np.savez(f, **arrays)
    out = json.loads(subprocess.run([npz_tool, "read", str(f)], check=True, capture_output=True, text=True).stdout)
    assert out["rho"]["shape"] == [3, 5] and out["rho"]["value"] == float(arrays["rho"].sum())
    assert out["u"]["descr"] == "<f4" and abs(out["u"]["value"] - float(arrays["u"].astype(np.float64).sum())) < 1e-12
    assert out["nx"]["value"] == 5 and out["ny"]["value"] == 3 and out["t_end"]["value"] == 0.25
    assert out["bc_x"]["value"] == "transmissive"


def test_npz_reader_rejects_compressed_archives(npz_tool, tmp_path):
    f = tmp_path / "c.npz"
    np.savez_compressed(f, x=np.zeros(100))
    r = subprocess.run([npz_tool, "read", str(f)], capture_output=True, text=True)
    assert r.returncode != 0 and "numpy.savez" in r.stderr


def write_ic(path, rho, u, v, p, t_end=0.05, bc="periodic", test="riemann", box=(0.0, 1.0, 0.0, 1.0)):
    ny, nx = rho.shape
    np.savez(path, rho=rho, u=u, v=v, p=p, nx=np.int32(nx), ny=np.int32(ny), x_min=box[0], x_max=box[1],
             y_min=box[2], y_max=box[3], bc_x=np.array(bc), bc_y=np.array(bc), t_end=np.float64(t_end),
             test=np.array(test))


def test_init_file_with_nonpositive_density_is_rejected(exe, tmp_path):
    rho = np.ones((8, 8))
    rho[3, 4] = 0.0
    write_ic(tmp_path / "ic.npz", rho, np.zeros_like(rho), np.zeros_like(rho), np.ones_like(rho))
    r = run(exe, "--init", tmp_path / "ic.npz")
    assert r.returncode == 1
    assert "initial condition has non-positive density or pressure" in r.stderr


def test_init_file_missing_attribute(exe, tmp_path):
    np.savez(tmp_path / "ic.npz", rho=np.ones((4, 4)))
    r = run(exe, "--init", tmp_path / "ic.npz")
    assert r.returncode == 1 and "missing attribute nx" in r.stderr


def _ic_arrays(n=8, rho=None):
    one = np.ones((n, n))
    return dict(rho=one if rho is None else rho, u=0 * one, v=0 * one, p=one, nx=np.int32(n), ny=np.int32(n),
                x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, bc_x=np.array("periodic"),
                bc_y=np.array("periodic"), t_end=np.float64(0.1), test=np.array("riemann"))


def test_malformed_init_files_fail_cleanly(exe, tmp_path):
    """Every unreadable IC file ends the driver with status 1 and a message, before any GPU work."""
    import zipfile
    (tmp_path / "garbage.npz").write_bytes(b"garbage")
    np.savez(tmp_path / "full.npz", **_ic_arrays())
    whole = (tmp_path / "full.npz").read_bytes()
    (tmp_path / "truncated.npz").write_bytes(whole[: len(whole) // 2])
    np.savez(tmp_path / "shape.npz", **_ic_arrays(rho=np.ones((4, 8))))
    np.savez(tmp_path / "dtype.npz", **_ic_arrays(rho=np.ones((8, 8), np.complex128)))
    with zipfile.ZipFile(tmp_path / "header.npz", "w") as z:
        z.writestr("rho.npy", b"\x93NUMPY\x01\x00\x10\x00{'descr': '<f8',   ")
    expected = {"garbage": "is not an .npz archive", "truncated": "is not an .npz archive",
                "shape": "dataset rho has the wrong size", "dtype": "unsupported dtype <c16",
                "header": ".npy header lacks fortran_order"}
    for name, msg in expected.items():
        r = run(exe, "--init", tmp_path / f"{name}.npz")
        assert r.returncode == 1 and msg in r.stderr, (name, r.returncode, r.stderr)


# ---------------------------------------------------------------- GPU: bit-identical runs


def _oracle(g, flux="hllc", limiter="vanleer"):
    from oracle.oracle import OracleSolver
    return OracleSolver(g["nx"], g["ny"], g["x_min"], g["x_max"], g["y_min"], g["y_max"], g["bc_x"], g["bc_y"],
                        flux, limiter, 0.5)


def _to_primitive(U):  # state2d.hpp:21-25 in numpy (no FMA): same bits as the driver's snapshot writer
    u = U[..., 1] / U[..., 0]
    v = U[..., 2] / U[..., 0]
    p = (1.4 - 1.0) * (U[..., 3] - 0.5 * U[..., 0] * (u * u + v * v))  # GAMMA - 1.0, not 0.4
    return U[..., 0], u, v, p


@pytest.mark.gpu
def test_traj_mode_matches_oracle(exe, tmp_path, cuda_ok):
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    g, t_end, U0 = ic.test_problem("sod_x", 64)
    r = run(exe, "--test", "sod_x", "--n", 64, "--scheme", "rusanov", "--limiter", "minmod", "--nout", 5,
            "--traj", tmp_path / "t.npz", "--save", "64,16")
    assert r.returncode == 0, r.stderr
    z = np.load(tmp_path / "t.npz")
    o = _oracle(g, "rusanov", "minmod")
    o.set_state(U0)
    times, levels = o.run(t_end, nout=5, save=(64, 16))
    assert z["t"].tobytes() == times.tobytes()
    assert z["U_64"].tobytes() == levels[64].tobytes() and z["U_16"].tobytes() == levels[16].tobytes()
    assert int(z["steps"]) == o.steps and int(z["frames"]) == 6
    assert str(z["scheme"]) == "rusanov" and str(z["bc_x"]) == "transmissive" and int(z["solver_nx"]) == 64


@pytest.mark.gpu
def test_init_and_tstart_match_oracle(exe, tmp_path, cuda_ok):
    """The generator's path: an IC file with t_end, spin-up to --tstart, nout frames at two sizes."""
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    rho, u, v, p, _, _ = ic.sample("riemann", 3, 64)
    write_ic(tmp_path / "ic.npz", rho, u, v, p, t_end=0.06)
    r = run(exe, "--init", tmp_path / "ic.npz", "--nout", 4, "--tstart", 0.01, "--traj", tmp_path / "t.npz",
            "--save", "64,32")
    assert r.returncode == 0, r.stderr
    z = np.load(tmp_path / "t.npz")
    o = _oracle(dict(nx=64, ny=64, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, bc_x="periodic", bc_y="periodic"))
    o.set_state(ic.to_conserved(rho, u, v, p))
    times, levels = o.run(0.06, t_start=0.01, nout=4, save=(64, 32))
    assert z["t"].tobytes() == times.tobytes()
    assert z["U_64"].tobytes() == levels[64].tobytes() and z["U_32"].tobytes() == levels[32].tobytes()
    assert str(z["test"]) == "riemann" and float(z["t_start"]) == 0.01


@pytest.mark.gpu
def test_snapshots_and_restart_match_oracle(exe, tmp_path, cuda_ok):
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    g, t_end, U0 = ic.test_problem("lax_liu3", 32)
    r = run(exe, "--test", "lax_liu3", "--n", 32, "--nout", 2, "--out", tmp_path)
    assert r.returncode == 0, r.stderr
    d = tmp_path / "lax_liu3_hllc_vanleer_N32"
    o = _oracle(g)
    o.set_state(U0)
    snaps = []
    for k in range(3):
        if k:
            o.advance_to(0.0 + (t_end - 0.0) * k / 2)
        z = np.load(d / f"snap_{k:04d}.npz")
        want = _to_primitive(o.get_state())
        for name, w in zip(("rho", "u", "v", "p"), want):
            assert z[name].tobytes() == np.ascontiguousarray(w).tobytes(), (k, name)
        assert float(z["t"]) == o.t and int(z["step"]) == (o.steps if k else 0)
        snaps.append(z)
    # restart from snapshot 1 (its primitives become the new initial state) to the original t_end
    r = run(exe, "--init", d / "snap_0001.npz", "--tend", t_end, "--nout", 1, "--traj", tmp_path / "re.npz",
            "--save", 32)
    assert r.returncode == 0, r.stderr
    z1 = snaps[1]
    o2 = _oracle(g)
    o2.set_state(ic.to_conserved(z1["rho"], z1["u"], z1["v"], z1["p"]))
    times, levels = o2.run(t_end, nout=1, save=(32,))
    re = np.load(tmp_path / "re.npz")
    assert re["U_32"].tobytes() == levels[32].tobytes() and re["t"].tobytes() == times.tobytes()
