"""Dataset splits and packing (data/splits.py, data/pack.py semantics) on synthetic raw files in the
generator's format; no GPU needed."""
import importlib
import json

import numpy as np
import pytest

ds = importlib.import_module("neural-pde-surrogate_b200.dataset")


def test_split_rule():
    assert [ds.split_for("riemann", i) for i in range(10)] == ["train"] * 8 + ["val", "test"]
    assert ds.split_for("blast", 1238) == "val" and ds.split_for("blast", 99) == "test"
    assert ds.split_for("kh", 3) == "ood"
    with pytest.raises(ValueError):
        ds.split_for("orszag", 0)


def _write_raw(root, family, index, frames, n=8, rng=None, bad_rho=False, spacing=0.005):
    rng = rng or np.random.default_rng(index)
    t = 0.1 * (family == "kh") + spacing * np.arange(frames)
    rho = 1.0 + 0.1 * rng.random((n, n))
    U0 = np.stack([rho, 0.1 * rho, -0.2 * rho, 2.5 + 0.5 * rho ** 2])
    # a conserving "evolution": periodic shifts of the initial fields
    U = np.stack([np.roll(U0, k, axis=2) for k in range(frames)]).astype(np.float32)
    if bad_rho:
        U[frames // 2, 0, 0, 0] = -1.0
    half = U.reshape(frames, 4, n // 2, 2, n // 2, 2).mean(axis=(3, 5)).astype(np.float32)
    d = root / family
    d.mkdir(parents=True, exist_ok=True)
    np.savez(d / f"{index:06d}.npz", t=t, **{f"U_{n}": U, f"U_{n // 2}": half}, attr_family=np.asarray(family),
             attr_index=np.asarray(index), attr_solver_nx=np.asarray(64), attr_steps=np.asarray(100))


def test_pack_splits_stats_and_checks(tmp_path):
    raw, out = tmp_path / "raw", tmp_path / "packed"
    for i in range(20):
        _write_raw(raw, "riemann", i, 6)
    for i in range(10):
        _write_raw(raw, "blast", i, 5)
    for i in range(3):
        _write_raw(raw, "kh", i, 6)
    _write_raw(raw, "blast", 57, 5, spacing=0.004)  # wrong frame spacing: skipped
    assert ds.pack(raw, out, sizes=(8, 4), log=lambda *a: None)
    man = json.loads((out / "manifest.json").read_text())
    assert len(man["trajectories"]) == 33 and len(man["skipped"]) == 1
    U, t, meta = ds.load(out, "train", 8)
    assert U.shape == (24, 5, 4, 8, 8) and U.dtype == np.float32 and t.shape == (24, 5)
    assert meta["checks_passed"] and meta["frames"] == 5
    assert [(f, i) for f, i in zip(meta["family"], meta["index"])][:2] == [("blast", 0), ("blast", 1)]
    Uv, _, mv = ds.load(out, "val", 4)
    assert Uv.shape == (3, 5, 4, 4, 4) and mv["index"] == [8, 8, 18]
    Uo, to, _ = ds.load(out, "ood", 8)
    assert Uo.shape == (3, 6, 4, 8, 8) and abs(to[0, 0] - 0.1) < 1e-12
    st = json.loads((out / "stats_8.json").read_text())
    flat = np.asarray(U, np.float64).transpose(0, 1, 3, 4, 2).reshape(-1, 4)
    assert np.allclose(st["mean"], flat.mean(axis=0), rtol=1e-12) and np.allclose(st["std"], flat.std(axis=0), rtol=1e-9)
    assert abs(st["log_rho_mean"] - np.log(flat[:, 0]).mean()) < 1e-12
    dU = np.diff(np.asarray(U, np.float64), axis=1).transpose(0, 1, 3, 4, 2).reshape(-1, 4)
    assert np.allclose(st["delta_std"], dU.std(axis=0), rtol=1e-9, atol=1e-12)


def test_pack_flags_nonpositive_density(tmp_path):
    raw, out = tmp_path / "raw", tmp_path / "packed"
    _write_raw(raw, "riemann", 0, 4)
    _write_raw(raw, "riemann", 1, 4, bad_rho=True)
    assert not ds.pack(raw, out, sizes=(8,), log=lambda *a: None)
    assert not json.loads((out / "train_8.json").read_text())["checks_passed"]
