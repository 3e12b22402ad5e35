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


@pytest.fixture(scope="module")
def packed(tmp_path_factory):
    root = tmp_path_factory.mktemp("pairs")
    raw, out = root / "raw", root / "packed"
    for i in range(20):
        _write_raw(raw, "riemann", i, 7)
    for i in range(10):
        _write_raw(raw, "blast", i, 6)
    assert ds.pack(raw, out, sizes=(8,), log=lambda *a: None)
    return out


def test_pairs_cover_every_start_frame_and_line_up(packed):
    """The checks of the reference's tests/test_data.py:21-28 on the packs written here."""
    d = ds.PairDataset(packed, "train", 8, horizon=1)
    F = d.n_frames
    assert (d.n_traj, F) == (24, 6) and len(d) == d.n_traj * (F - 1)
    assert d.pairs[:, 1].max() == F - 2 and d.pairs[:, 1].min() == 0
    assert d.pairs[F - 1].tolist() == [1, 0]  # trajectory-major order
    x0, y0 = d.get([(0, 2)])
    x1, _ = d.get([(0, 3)])
    assert np.array_equal(y0[0, 0], x1[0])  # the target of (k, t) is the input of (k, t + 1)
    assert list(d.family[:2]) == ["blast", "blast"] and d.index[0] == 0


def test_normalisation_uses_the_train_statistics(packed):
    d = ds.PairDataset(packed, "train", 8)
    raw = d.trajectory(3, normalised=False)
    assert np.allclose(d.norm.decode(d.norm.encode(raw)), raw, rtol=1e-5, atol=1e-5)
    z = np.concatenate([d.trajectory(k) for k in range(d.n_traj)])
    assert np.abs(z.mean(axis=(0, 2, 3))).max() < 1e-4 and np.abs(z.std(axis=(0, 2, 3)) - 1).max() < 1e-3
    st = json.loads((packed / "stats_8.json").read_text())
    assert np.array_equal(d.norm.delta_std, np.asarray(st["delta_std"], np.float32))
    # the variable axis can be any axis: channels-last states normalise the same way
    cl = raw.transpose(0, 2, 3, 1)
    assert np.allclose(d.norm.encode(cl, axis=-1).transpose(0, 3, 1, 2), d.norm.encode(raw), atol=1e-6)
    # val and test are normalised with the train statistics, not their own
    v = ds.PairDataset(packed, "val", 8)
    assert np.array_equal(v.norm.mean, d.norm.mean) and np.array_equal(v.norm.std, d.norm.std)


def test_batches_shapes_and_reproducibility(packed):
    d = ds.PairDataset(packed, "train", 8)
    x, y = next(d.batches(8, rng=np.random.default_rng(1)))
    assert x.shape == (8, 4, 8, 8) and y.shape == (8, 1, 4, 8, 8)
    assert x.dtype == np.float32 and y.dtype == np.float32
    xa, _ = next(d.batches(8, rng=np.random.default_rng(1)))
    assert np.array_equal(x, xa)
    assert sum(1 for _ in d.batches(7, rng=np.random.default_rng(0))) == len(d) // 7
    assert sum(len(b[0]) for b in d.batches(7, drop_last=False, shuffle=False)) == len(d)
    xs, _ = next(d.batches(3, shuffle=False))
    assert np.array_equal(xs, d.get(d.pairs[:3])[0])


def test_multistep_targets_and_disk_mode(packed):
    d3 = ds.PairDataset(packed, "train", 8, horizon=3)
    x, y = d3.get([(2, 1)])
    traj = d3.trajectory(2)
    assert np.array_equal(y[0], traj[2:5]) and np.array_equal(x[0], traj[1])
    assert d3.pairs[:, 1].max() == d3.n_frames - 4
    mem = ds.PairDataset(packed, "train", 8, horizon=1)
    disk = ds.PairDataset(packed, "train", 8, horizon=1, in_memory=False)
    sel = mem.pairs[[0, 7, 50 % len(mem)]]
    for a, b in zip(disk.get(sel), mem.get(sel)):
        assert np.array_equal(a, b)
    for h in (0, mem.n_frames):
        with pytest.raises(ValueError, match="horizon must be between 1 and 5"):
            ds.PairDataset(packed, "train", 8, horizon=h)


def test_states_are_channels_last_fp64(packed):
    d = ds.PairDataset(packed, "val", 8, in_memory=False)
    S = d.states(device="cpu")
    assert tuple(S.shape) == (d.n_traj, d.n_frames, 8, 8, 4) and str(S.dtype) == "torch.float64"
    U, _, _ = ds.load(packed, "val", 8)
    assert np.array_equal(S.numpy(), np.asarray(U, np.float64).transpose(0, 1, 3, 4, 2))
