"""The learned part's data pipeline and evaluation on the GPU.

* generate.py -> dataset.py -> train_correction.py --packed: trajectories written by the generator,
  split and packed (data/splits.py, data/pack.py semantics), loaded back into HBM, must be the very
  tensor the in-process data path builds from the same trajectories, and training on either must
  give the same loss history (same seed); the loss must fall.
* The rollout metrics (surrogate/rollout.py:54-62: RMSE over std, conservation drift over the total
  absolute amount, bad cells) computed on the GPU must match a CPU restatement of the reference's
  formulas on a real hybrid rollout, with non-physical cells planted in it.
"""
import importlib
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
PKG = "neural-pde-surrogate_b200"
fv = importlib.import_module(PKG)
gen = importlib.import_module(f"{PKG}.generate")
dsm = importlib.import_module(f"{PKG}.dataset")
tc = importlib.import_module(f"{PKG}.train_correction")
pa = importlib.import_module(f"{PKG}.pareto")


def test_packed_pipeline_trains_like_the_in_process_data(cuda_ok, tmp_path):
    import torch
    raw, packed = tmp_path / "raw", tmp_path / "packed"
    solver = fv.Solver(fv.make_grid(128, 128, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic"), "hllc", "vanleer", 0.5)
    for fam in ("riemann", "blast"):
        for idx in range(10):  # index % 10: 0-7 train, 8 val, 9 test
            assert gen.generate_one(fam, idx, 128, [64], raw, solver=solver) == "done"
    assert dsm.pack(raw, packed, sizes=(64,))
    U_packed = dsm.PairDataset(packed, "train", 64).states()
    # the pack orders trajectories by (family, index): blast 0-7, then riemann 0-7
    U_direct = tc.build_dataset(16, 128, 64, index0=0, families=("blast", "riemann"))
    assert U_packed.shape == U_direct.shape == (16, 41, 64, 64, 4)
    assert torch.equal(U_packed, U_direct)
    base = dict(out=None, coarse=64, steps=300, batch=8, unroll=1, lr=1e-3, warmup=30, eval_every=100, seed=0)
    _, hist_p = tc.train(dict(base, packed=str(packed)))
    _, hist_d = tc.train(dict(base, packed=None, n_traj=16, n_val=2, fine=128, families=("blast", "riemann")))
    train_p, train_d = [r[1] for r in hist_p], [r[1] for r in hist_d]
    assert train_p == train_d, (train_p, train_d)
    assert train_p[-1] < 0.8 * train_p[0], train_p


def _metrics_cpu(pred, true, std):
    """surrogate/rollout.py:54-62 restated in numpy, in the reference's (T, 4, n, n) layout."""
    gamma = 1.4
    rmse = np.sqrt(np.mean((pred - true) ** 2, axis=(-2, -1))) / std
    totals_p, totals_t = pred.sum(axis=(-2, -1)), true.sum(axis=(-2, -1))
    drift = (totals_p - totals_t[0]) / np.abs(true[0]).sum(axis=(-2, -1))
    with np.errstate(invalid="ignore", divide="ignore"):
        p = (gamma - 1) * (pred[:, 3] - 0.5 * (pred[:, 1] ** 2 + pred[:, 2] ** 2) / pred[:, 0])
        bad = ((pred[:, 0] <= 0) | ~(p > 0)).sum(axis=(-2, -1))
    return rmse, drift, bad


def test_rollout_metrics_match_the_reference_formulas(cuda_ok):
    import torch
    corr = importlib.import_module(f"{PKG}.correction")
    model = Path(tc.__file__).parent / "checkpoints" / "correction_64.npz"
    items = [("riemann", 200000), ("blast", 200000)]
    truth, first = pa.truth_frames(items, 256, 64, 8, [64], log=print)
    net, stats, dscale = corr.load_checkpoint(str(model), 2, 64, 64)
    cs = corr.CoarseSolver(2, 64, 64)
    x = first[64].clone()
    Uc, Un = torch.empty_like(x), torch.empty_like(x)
    fb = torch.zeros(2, dtype=torch.int32, device="cuda")
    frames = [x.clone()]
    for _ in range(8):
        corr.hybrid_step(net, cs, x, pa.DT_FRAME, stats, dscale, Uc, Un, fb, "scale")
        x.copy_(Un)
        frames.append(x.clone())
    pred = torch.stack(frames, dim=1)  # (B, T, n, n, 4)
    pred[0, 3, 5, 7, 0] = -0.5          # planted: a negative density,
    pred[0, 4, 9, 2, 3] = 0.0           # an energy below the kinetic energy (negative pressure),
    pred[1, 6, 1, 1, 3] = float("nan")  # and a NaN pressure
    std = torch.tensor([0.5, 0.3, 0.3, 1.7], dtype=torch.float64, device="cuda")
    for b in range(2):
        got = pa.rollout_metrics(pred[b], truth[b], std)
        P = pred[b].permute(0, 3, 1, 2).cpu().numpy()
        T = truth[b].permute(0, 3, 1, 2).cpu().numpy()
        rmse, drift, bad = _metrics_cpu(P, T, std.cpu().numpy())
        g_rmse, g_drift = got["rmse"].cpu().numpy(), got["drift"].cpu().numpy()
        ok = np.isfinite(rmse)
        assert (np.isfinite(g_rmse) == ok).all()
        np.testing.assert_allclose(g_rmse[ok], rmse[ok], rtol=1e-12, atol=0)
        okd = np.isfinite(drift)
        assert (np.isfinite(g_drift) == okd).all()
        # the totals agree to roundoff, so the drift is a difference of two nearly equal sums of 4096
        # terms whose last bits depend on the summation order (numpy pairwise, torch tree): ~1e-13
        np.testing.assert_allclose(g_drift[okd], drift[okd], rtol=1e-9, atol=1e-12)
        assert (got["bad_cells"].cpu().numpy() == bad).all()
    assert int(pa.rollout_metrics(pred[0], truth[0], std)["bad_cells"].sum()) == 2
    assert int(pa.rollout_metrics(pred[1], truth[1], std)["bad_cells"].sum()) == 1
    # the hybrid's own frames (before planting) conserve the totals to roundoff
    clean = torch.stack(frames, dim=1)
    d = pa.rollout_metrics(clean[0], clean[0, :1].expand_as(clean[0]), std)["drift"]
    assert float(d[:, 0].abs().max()) < 1e-13 and float(d[:, 3].abs().max()) < 1e-13
