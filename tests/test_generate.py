"""The generator's per-file logic on the CPU, with the GPU trajectory replaced by a stand-in: index
parsing (data/generate.py:36-45), atomic output and restart by skipping, and failure logs that let the
batch go on (data/generate.py:79-84)."""
import importlib

import numpy as np
import pytest

gen = importlib.import_module("neural-pde-surrogate_b200.generate")
fv = importlib.import_module("neural-pde-surrogate_b200")


def test_parse_indices():
    assert gen.parse_indices("0-3,10") == [0, 1, 2, 3, 10]
    assert gen.parse_indices("7") == [7]
    assert gen.parse_indices("5-5,2-3") == [5, 2, 3]


def _fake_ok(family, index, n, save, solver=None):
    t = 0.005 * np.arange(3)
    levels = {m: np.full((3, 4, m, m), float(index), np.float32) for m in save}
    return t, levels, 123, {"family": family, "index": index, "blasts": np.ones((2, 4))}


def _fake_nonphysical(family, index, n, save, solver=None):
    raise fv.FVError(3, "Non-physical state in cell (4, 5): rho = -0.01, p = 0.2")


def test_output_is_written_once_and_skipped_on_restart(tmp_path, monkeypatch):
    monkeypatch.setattr(gen, "trajectory", _fake_ok)
    assert gen.generate_one("blast", 12, 32, [16, 8], tmp_path) == "done"
    f = tmp_path / "blast" / "000012.npz"
    z = np.load(f)
    assert z["U_16"].shape == (3, 4, 16, 16) and z["U_8"].shape == (3, 4, 8, 8) and z["t"].shape == (3,)
    assert int(z["attr_steps"]) == 123 and int(z["attr_index"]) == 12 and str(z["attr_family"]) == "blast"
    assert z["param_blasts"].shape == (2, 4) and "param_family" not in z.files
    assert sorted(p.name for p in (tmp_path / "blast").iterdir()) == ["000012.npz"]  # no temporary left
    assert gen.generate_one("blast", 12, 32, [16, 8], tmp_path) == "skipped"
    assert gen.generate_one("blast", 12, 32, [16, 8], tmp_path, force=True) == "done"


def test_a_failed_trajectory_is_logged_and_the_batch_goes_on(tmp_path, monkeypatch):
    monkeypatch.setattr(gen, "trajectory", _fake_nonphysical)
    assert gen.generate_one("riemann", 4, 64, [16], tmp_path) == "failed"
    log = tmp_path / "riemann" / "000004.failed.txt"
    assert "Non-physical state in cell (4, 5)" in log.read_text() and "riemann 4 at 64x64" in log.read_text()
    assert not (tmp_path / "riemann" / "000004.npz").exists()
    # a restart retries it; success removes the earlier log
    monkeypatch.setattr(gen, "trajectory", _fake_ok)
    assert gen.generate_one("riemann", 4, 64, [16], tmp_path) == "done"
    assert not log.exists() and (tmp_path / "riemann" / "000004.npz").exists()


def test_other_errors_are_not_swallowed(tmp_path, monkeypatch):
    def broken(*a, **k):
        raise ValueError("save size 24 does not divide nx = 64")
    monkeypatch.setattr(gen, "trajectory", broken)
    with pytest.raises(ValueError, match="does not divide"):
        gen.generate_one("blast", 0, 64, [24], tmp_path)
    assert not list((tmp_path / "blast").iterdir())
