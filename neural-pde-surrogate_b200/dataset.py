"""Dataset splits and packing for the generator's trajectories (the learned part's data pipeline).

  python neural-pde-surrogate_b200/dataset.py --raw DIR --out PACKED [--sizes 128,64]

Step 1, splits (data/splits.py:29-35, :71-127): every raw trajectory DIR/<family>/<index>.npz written by
generate.py is checked (frame count, frame spacing 0.005, shapes of every stored resolution) and
assigned to a split by (family, index) alone, so that adding indices never moves a trajectory:
training families (riemann, blast) go to train when index % 10 is 0-7, to val on 8 and to test on 9;
held-out families (kh) go to ood.  The result is PACKED/manifest.json.

Step 2, packing (data/pack.py:54-112): one array per (split, resolution), every trajectory cut to
the split's shortest frame count (the families differ in length: riemann runs to t = 0.25, blast to 0.2),
    PACKED/<split>_<n>_U.npy   (N, F, 4, n, n) float32   conserved (rho, rho*u, rho*v, E)
    PACKED/<split>_<n>_t.npy   (N, F)          float64   frame times
    PACKED/<split>_<n>.json    family and index of every row, checks
as plain .npy files (numpy.load(..., mmap_mode="r") reads any (trajectory, frame) without loading
the rest; HDF5 is not available to this build).  While copying, every trajectory is checked for
positivity of rho and p and for conservation of mass and energy over its frames (relative drift
< 1e-5).  Normalisation statistics come from the train split only: per-field mean and std of U, of
log rho, and of one-frame increments, PACKED/stats_<n>.json.

Step 3, loading (surrogate/data.py): PairDataset serves (frame t, frames t+1 .. t+horizon) pairs of a
packed split, normalised by Normaliser with the train statistics, from host memory or memory-mapped;
PairDataset.states() puts a whole split in HBM for train_correction.py --packed.
"""
import argparse
import json
from collections import Counter
from pathlib import Path

import numpy as np

TRAINING_FAMILIES = ("riemann", "blast")
HELD_OUT_FAMILIES = ("kh",)
SPLITS = ("train", "val", "test", "ood")
DT_FRAME = 0.005
GAMMA = 1.4
VARS = ["rho", "rho_u", "rho_v", "E"]


def split_for(family, index):
    """The split of trajectory (family, index): data/splits.py:29-35."""
    if family in HELD_OUT_FAMILIES:
        return "ood"
    if family not in TRAINING_FAMILIES:
        raise ValueError(f"family '{family}' is neither a training nor a held-out family")
    r = int(index) % 10
    return "train" if r < 8 else ("val" if r == 8 else "test")


def _attr(z, name, default=None):
    key = f"attr_{name}"
    return z[key].item() if key in z.files else default


def inspect(path, expected_frames=None):
    """(entry, problems) of one raw trajectory file."""
    problems = []
    with np.load(path) as z:
        t = z["t"]
        sizes = sorted((int(k[2:]) for k in z.files if k.startswith("U_")), reverse=True)
        for n in sizes:
            shape = z[f"U_{n}"].shape
            if shape != (len(t), 4, n, n):
                problems.append(f"U_{n} has shape {shape}")
        entry = {"family": str(_attr(z, "family", path.parent.name)), "index": int(_attr(z, "index", int(path.stem))),
                 "path": str(path), "sizes": sizes, "frames": int(len(t)), "t_start": float(t[0]),
                 "solver_n": int(_attr(z, "solver_nx", -1)), "steps": int(_attr(z, "steps", -1))}
    if expected_frames is not None and len(t) != expected_frames:
        problems.append(f"{len(t)} frames, expected {expected_frames}")
    if len(t) > 1 and not np.allclose(np.diff(t), DT_FRAME, rtol=0, atol=1e-9):
        problems.append(f"frame spacing {np.diff(t).min():.6f}..{np.diff(t).max():.6f}, expected {DT_FRAME}")
    return entry, problems


def build_manifest(raw, out, expected_frames=None, log=print):
    files = sorted(Path(raw).glob("*/*.npz"))
    if not files:
        raise SystemExit(f"No trajectory files found under {raw}")
    entries, bad = [], []
    for path in files:
        entry, problems = inspect(path, expected_frames)
        if problems:
            bad.append((str(path), problems))
            continue
        entry["split"] = split_for(entry["family"], entry["index"])
        entries.append(entry)
    counts = Counter((e["family"], e["split"]) for e in entries)
    for fam in sorted({e["family"] for e in entries}):
        log(f"{fam:<10}" + "".join(f"{counts[(fam, s)]:>8}" for s in SPLITS))
    for path, problems in bad:
        log(f"SKIPPED {path}: {'; '.join(problems)}")
    out = Path(out)
    out.mkdir(parents=True, exist_ok=True)
    manifest = {"split_rule": "training families: index % 10 -> 0-7 train, 8 val, 9 test; held-out: ood",
                "trajectories": entries, "skipped": bad}
    (out / "manifest.json").write_text(json.dumps(manifest, indent=1))
    return manifest


class RunningStats:
    """Per-channel mean and std accumulated in float64 over many arrays (channel axis 1)."""

    def __init__(self, channels):
        self.n, self.s, self.ss = 0, np.zeros(channels), np.zeros(channels)

    def add(self, x, axis):
        x = x.astype(np.float64)
        self.n += x.size // x.shape[1]
        self.s += x.sum(axis=axis)
        self.ss += (x ** 2).sum(axis=axis)

    def result(self):
        mean = self.s / self.n
        return mean, np.sqrt(np.maximum(self.ss / self.n - mean ** 2, 0.0))


def pressure(U):
    """(frames, 4, n, n) conserved -> (frames, n, n) pressure."""
    rho, mx, my, E = U[:, 0], U[:, 1], U[:, 2], U[:, 3]
    return (GAMMA - 1) * (E - 0.5 * (mx ** 2 + my ** 2) / rho)


def pack_split(split, n, entries, out, stats=None, log=print):
    """Writes <split>_<n>_{U,t}.npy and <split>_<n>.json; returns whether every check passed."""
    out = Path(out)
    N = len(entries)
    F = min(e["frames"] for e in entries)  # families differ in length (riemann 51, blast 41): the shortest
    U = np.lib.format.open_memmap(out / f"{split}_{n}_U.npy", mode="w+", dtype=np.float32, shape=(N, F, 4, n, n))
    T = np.zeros((N, F))
    worst_drift, min_rho, min_p = 0.0, np.inf, np.inf
    for k, e in enumerate(entries):
        with np.load(e["path"]) as z:
            u = z[f"U_{n}"][:F]
            T[k] = z["t"][:F]
        U[k] = u
        min_rho = min(min_rho, float(u[:, 0].min()))
        min_p = min(min_p, float(pressure(u.astype(np.float64)).min()))
        totals = u.astype(np.float64).mean(axis=(2, 3))
        for q in (0, 3):  # mass and energy are never near zero
            worst_drift = max(worst_drift, float(np.abs(totals[:, q] - totals[0, q]).max() / abs(totals[0, q])))
        if stats is not None:
            stats["U"].add(u, axis=(0, 2, 3))
            with np.errstate(invalid="ignore", divide="ignore"):  # a non-positive rho fails the check above
                stats["log_rho"].add(np.log(u[:, :1].astype(np.float64)), axis=(0, 2, 3))
            stats["dU"].add(np.diff(u.astype(np.float64), axis=0), axis=(0, 2, 3))
    U.flush()
    del U
    np.save(out / f"{split}_{n}_t.npy", T)
    ok = bool(min_rho > 0 and min_p > 0 and worst_drift < 1e-5)
    meta = {"split": split, "n": n, "frames": F, "dt": DT_FRAME, "variables": VARS,
            "family": [e["family"] for e in entries], "index": [e["index"] for e in entries],
            "min_rho": min_rho, "min_p": min_p, "max_drift": worst_drift, "checks_passed": ok}
    (out / f"{split}_{n}.json").write_text(json.dumps(meta, indent=1))
    log(f"  {split}_{n}: {N:5d} trajectories  min rho {min_rho:.3g}  min p {min_p:.3g}  "
        f"max mass/energy drift {worst_drift:.1e}")
    return ok


def pack(raw, out, sizes=(128, 64), expected_frames=None, log=print):
    """Both steps; returns whether every check passed."""
    manifest = build_manifest(raw, out, expected_frames, log)["trajectories"]
    ok = True
    for n in sizes:
        stats = {"U": RunningStats(4), "log_rho": RunningStats(1), "dU": RunningStats(4)}
        for split in SPLITS:
            entries = sorted((e for e in manifest if e["split"] == split and n in e["sizes"]),
                             key=lambda e: (e["family"], e["index"]))
            if entries:
                ok &= pack_split(split, n, entries, out, stats if split == "train" else None, log)
        if stats["U"].n == 0:
            continue
        mean, std = stats["U"].result()
        lmean, lstd = stats["log_rho"].result()
        dmean, dstd = stats["dU"].result()
        result = {"source": "train split only", "n": n, "variables": VARS, "mean": mean.tolist(), "std": std.tolist(),
                  "log_rho_mean": float(lmean[0]), "log_rho_std": float(lstd[0]), "delta_mean": dmean.tolist(),
                  "delta_std": dstd.tolist()}
        (Path(out) / f"stats_{n}.json").write_text(json.dumps(result, indent=1))
    log("ALL CHECKS PASSED" if ok else "SOME CHECKS FAILED: see the lines above")
    return ok


def load(packed, split, n, mmap=True):
    """(U (N, F, 4, n, n) float32, t (N, F), meta dict) of one packed split."""
    packed = Path(packed)
    U = np.load(packed / f"{split}_{n}_U.npy", mmap_mode="r" if mmap else None)
    return U, np.load(packed / f"{split}_{n}_t.npy"), json.loads((packed / f"{split}_{n}.json").read_text())


# ---------------------------------------------------------------- loading for training (surrogate/data.py)


class Normaliser:
    """Per-variable affine map with the train split's statistics (PACKED/stats_<n>.json):
    encode(U) = (U - mean) / std, decode(Z) = Z * std + mean, float32 statistics, the 4 variables on
    axis `axis` (-3 for (..., 4, n, n)); the semantics of surrogate/data.py:19-40."""

    def __init__(self, stats_path):
        s = json.loads(Path(stats_path).read_text())
        self.mean = np.asarray(s["mean"], np.float32)
        self.std = np.asarray(s["std"], np.float32)
        self.delta_std = np.asarray(s["delta_std"], np.float32)

    def _on(self, v, ndim, axis):
        return np.expand_dims(v, [d for d in range(ndim) if d != axis % ndim])

    def encode(self, U, axis=-3):
        return (U - self._on(self.mean, U.ndim, axis)) / self._on(self.std, U.ndim, axis)

    def decode(self, Z, axis=-3):
        return Z * self._on(self.std, Z.ndim, axis) + self._on(self.mean, Z.ndim, axis)


class PairDataset:
    """Every (trajectory, start frame) pair of one packed split at one resolution, with `horizon` target
    frames: the interface of surrogate/data.py:43-101 (same names, pair order, normalisation and
    errors) over the .npy packs written by pack().

    x of pair (k, t) is frame t of trajectory k, y its frames t+1 .. t+horizon; a pair never runs past
    its trajectory's last frame.  in_memory=True reads the split into host memory once; False keeps it
    memory-mapped and reads only the frames each batch touches.  states() hands the whole split to the
    GPU in the layout the coarse solver and the correction network use."""

    def __init__(self, packed_dir, split, n, horizon=1, in_memory=True):
        packed_dir = Path(packed_dir)
        self.split, self.n, self.horizon, self.in_memory = split, n, horizon, in_memory
        self.path = packed_dir / f"{split}_{n}_U.npy"
        self.norm = Normaliser(packed_dir / f"stats_{n}.json")
        meta = json.loads((packed_dir / f"{split}_{n}.json").read_text())
        self.family = np.asarray(meta["family"])
        self.index = np.asarray(meta["index"])
        self.U = np.load(self.path, mmap_mode=None if in_memory else "r")
        self.n_traj, self.n_frames = self.U.shape[:2]
        if not 1 <= horizon < self.n_frames:
            raise ValueError(f"horizon must be between 1 and {self.n_frames - 1}")
        # trajectory-major: pair k * (F - horizon) + t is (k, t)
        k, t = np.divmod(np.arange(self.n_traj * (self.n_frames - horizon)), self.n_frames - horizon)
        self.pairs = np.stack([k, t], axis=1)

    def __len__(self):
        return len(self.pairs)

    def _windows(self, pairs):
        """Raw frames t .. t+horizon of each (k, t): (B, 1 + horizon, 4, n, n), one gather."""
        pairs = np.asarray(pairs).reshape(-1, 2)
        span = np.arange(self.horizon + 1)
        return self.U[pairs[:, :1], pairs[:, 1:] + span]

    def get(self, pairs):
        """Normalised float32 (x (B, 4, n, n), y (B, horizon, 4, n, n)) of (trajectory, start) pairs."""
        w = self.norm.encode(self._windows(pairs).astype(np.float32))
        return w[:, 0], w[:, 1:]

    def batches(self, batch_size, rng=None, shuffle=True, drop_last=True):
        """One pass over the pairs (shuffled by `rng` when shuffle), batch_size pairs at a time."""
        order = np.arange(len(self.pairs))
        if shuffle:
            (rng if rng is not None else np.random.default_rng()).shuffle(order)
        end = len(order) - len(order) % batch_size if drop_last else len(order)
        for s in range(0, end, batch_size):
            yield self.get(self.pairs[order[s:s + batch_size]])

    def trajectory(self, k, normalised=True):
        """All frames of trajectory k, (F, 4, n, n) float32, normalised unless asked otherwise."""
        U = np.asarray(self.U[k], np.float32)
        return self.norm.encode(U) if normalised else U

    def states(self, device="cuda"):
        """The whole split as an (N, F, n, n, 4) float64 torch tensor on `device`: conserved states per
        cell, channels last, unnormalised -- what the trainer samples its batches from on the device
        (a 64^2 split of 512 trajectories x 41 frames is 2.7 GB in FP64)."""
        import torch
        out = torch.empty((self.n_traj, self.n_frames, self.n, self.n, 4), dtype=torch.float64, device=device)
        for k in range(self.n_traj):  # one trajectory at a time: host memory stays one trajectory wide
            out[k].copy_(torch.from_numpy(np.ascontiguousarray(self.U[k].transpose(0, 2, 3, 1))))
        return out


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--raw", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--sizes", default="128,64")
    ap.add_argument("--frames", type=int, default=None, help="expected frame count (default: not checked)")
    a = ap.parse_args()
    ok = pack(a.raw, a.out, [int(s) for s in a.sizes.split(",")], a.frames)
    raise SystemExit(0 if ok else 1)


if __name__ == "__main__":
    main()
