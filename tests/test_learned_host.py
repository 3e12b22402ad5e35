"""Host-side logic of the learned part, on the CPU: the shipped checkpoint's format, the Pareto
evaluation's helpers (held-out set, block average, L1 density error, drift, per-family means) and the
trainer's normalisation statistics."""
import importlib
from pathlib import Path

import numpy as np
import torch

corr = importlib.import_module("neural-pde-surrogate_b200.correction")
pa = importlib.import_module("neural-pde-surrogate_b200.pareto")
tc = importlib.import_module("neural-pde-surrogate_b200.train_correction")
CKPT = Path(corr.__file__).parent / "checkpoints" / "correction_64.npz"


def test_shipped_checkpoint_format():
    z = np.load(CKPT)
    assert set(z.files) == {"params", "stats", "dscale", "gain"}
    assert z["params"].dtype == np.float32 and z["params"].shape == (corr.param_count(),) == (39332,)
    assert np.isfinite(z["params"]).all()
    assert z["stats"].shape == (8,) and (z["stats"][4:] > 0).all()  # mean(4), 1/std(4)
    assert z["dscale"].shape == (4,) and (z["dscale"] > 0).all()
    assert float(z["gain"]) == 0.75


def test_held_out_set_is_disjoint_from_training_indices():
    items = pa.test_set(3, 2, 1)
    assert items == [("riemann", 200000), ("riemann", 200001), ("riemann", 200002), ("blast", 200000),
                     ("blast", 200001), ("kh", 200000)]
    # training uses [0, n) and validation [100000, 100000 + n) of each family
    assert all(i >= 200000 for _, i in items)


def test_block_average_l1_and_drift():
    g = torch.Generator().manual_seed(0)
    U = torch.rand((2, 8, 8, 4), generator=g, dtype=torch.float64) + 0.5
    A = pa.block_avg(U, 4)
    assert A.shape == (2, 2, 2, 4)
    assert torch.allclose(A[1, 0, 1], U[1, 0:4, 4:8].mean(dim=(0, 1)))
    assert torch.allclose(A.sum(dim=(1, 2)) * 16, U.sum(dim=(1, 2)))  # totals are kept
    T = U.clone()
    T[0, 3, 5, 0] += 0.64
    l1 = pa.l1_density(U, T)
    assert torch.allclose(l1, torch.tensor([0.64 / 64, 0.0], dtype=torch.float64))
    d = pa.drift(T, U)
    assert d.shape == (2, 4) and float(d[1].abs().max()) == 0.0 and float(d[0, 0]) > 0


def test_per_family_final_errors():
    L1 = torch.tensor([[0.1, 0.2], [0.3, 0.4], [0.5, 0.8]])
    out = pa.by_family(L1, ["riemann", "blast", "riemann"])
    assert out == {"blast": 0.4, "riemann": round((0.2 + 0.8) / 2, 5)}
    assert pa.by_family(L1, None) == {}


def test_training_statistics():
    g = torch.Generator().manual_seed(1)
    U = torch.rand((3, 5, 4, 4, 4), generator=g, dtype=torch.float64) + 0.2
    st = tc.field_stats(U)
    flat = U.reshape(-1, 4)
    assert torch.allclose(st[:4], flat.mean(dim=0)) and torch.allclose(st[4:], 1.0 / flat.std(dim=0))
    w = tc.correction_weights(U[0, 0])
    assert torch.equal(w[..., 0], U[0, 0, ..., 0]) and torch.equal(w[..., 2], U[0, 0, ..., 0])
    assert torch.equal(w[..., 3], U[0, 0, ..., 3])
    assert abs(corr.cosine_lr(0, 100, 1e-3, 10)) < 1e-12 and abs(corr.cosine_lr(100, 100, 1e-3, 10) - 1e-5) < 1e-15
