"""Host-side logic of the learned part, on the CPU: the shipped checkpoint's format, the Pareto
evaluation's helpers (held-out set, block average, L1 density error, drift, per-family means), the
trainer's normalisation statistics and the structure of its pushforward step."""
import importlib
from pathlib import Path

import numpy as np
import pytest
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


class _FakeNet:
    def __init__(self, log):
        self.log = log

    def loss_grad(self, Un, y, Uc, stats, dscale, theta, loss_part):
        self.log.append(("loss_grad", Un.clone(), y.clone(), None if theta is None else theta.clone()))
        loss_part.fill_(2.0)

    def backward(self):
        self.log.append(("backward",))

    def adamw(self, lr):
        self.log.append(("adamw", lr))


class _FakeCorr:
    """hybrid_step stand-in: the next state is the input + 1; per-call coarse statuses from a list."""

    def __init__(self, log, statuses):
        self.log, self.statuses = log, list(statuses)

    def hybrid_step(self, net, coarse, U, dt, stats, dscale, Uc, Un, fb, mode="scale"):
        self.log.append(("hybrid", U.clone(), mode))
        Un.copy_(U + 1.0)
        return 1, self.statuses.pop(0)


def _cpu_trainer(B, unroll, statuses):
    tr = object.__new__(tc.Trainer)  # no CUDA buffers: every array of the step is a CPU tensor here
    log = []
    shape = (B, 2, 2, 4)
    x0 = torch.arange(B * 16, dtype=torch.float64).reshape(shape)
    y0 = -x0
    tr.torch, tr.corr, tr.net, tr.coarse = torch, _FakeCorr(log, statuses), _FakeNet(log), None
    tr.B, tr.unroll, tr.mode, tr.noise, tr.coarse_failures = B, unroll, "scale", 0.0, 0
    tr.stats, tr.dscale = torch.ones(8, dtype=torch.float64), torch.ones(4, dtype=torch.float64)
    tr.x, tr.Uc, tr.Un = (torch.empty(shape, dtype=torch.float64) for _ in range(3))
    tr.fb = torch.zeros(B, dtype=torch.int32)
    tr.loss_part = torch.zeros(B, dtype=torch.float64)
    tr.ok = torch.ones(B, dtype=torch.float64)
    tr._pairs = lambda U, k: (x0, y0)
    tr.train_U = None
    return tr, log, x0, y0


def test_pushforward_step_trains_only_the_last_step():
    """train.py:107-111's pushforward: unroll-1 self-fed hybrid steps give the trained step its input,
    and one backward runs through that last step alone. Its gradient is therefore the gradient of a
    one-step loss on a fixed input (tests/test_train.py:35-57 checks this equality in the reference),
    not backpropagation through the chain, which would need a backward pass per unrolled step."""
    B, unroll = 3, 4
    ok = np.zeros(B, np.int32)
    tr, log, x0, y0 = _cpu_trainer(B, unroll, [ok] * unroll)
    loss = tr.step(1e-3)
    hyb = [e for e in log if e[0] == "hybrid"]
    assert [e[2] for e in hyb] == ["scale"] * (unroll - 1) + ["keep"]  # self-fed rule, then the full correction
    for k, e in enumerate(hyb):
        assert torch.equal(e[1], x0 + k)  # each step starts from the previous step's output
    assert [e[0] for e in log[unroll:]] == ["loss_grad", "backward", "adamw"]  # after the whole unroll, once
    _, Un, y, theta = log[unroll]
    assert torch.equal(Un, x0 + unroll) and torch.equal(y, y0) and theta is None
    assert float(loss) == 2.0 * B / (B * 16)
    assert tr.coarse_failures == 0


def test_one_step_training_is_the_unroll_one_case():
    """With k = 1 the pushforward loss is the one-step loss (tests/test_train.py:37-39)."""
    tr, log, x0, _ = _cpu_trainer(2, 4, [np.zeros(2, np.int32)])
    tr.step(1e-3, unroll=1)
    assert [e[0] for e in log] == ["hybrid", "loss_grad", "backward", "adamw"]
    assert log[0][2] == "keep" and torch.equal(log[0][1], x0)


def test_a_sample_whose_coarse_solve_stopped_gets_no_gradient():
    B, unroll = 4, 3
    st = [np.array([0, 0, 0, 0]), np.array([0, 3, 0, 0]), np.array([0, 0, 0, 3])]  # sample 1 self-fed, 3 trained
    tr, log, _, _ = _cpu_trainer(B, unroll, st)
    tr.step(1e-3)
    theta = [e for e in log if e[0] == "loss_grad"][0][3]
    assert theta.tolist() == [1.0, 0.0, 1.0, 0.0]
    assert tr.coarse_failures == 2


def test_update_k_uses_optax_schedule_count_k_minus_one():
    cfg = {"steps": 1000, "lr": 1e-3, "warmup": 500}
    assert tc.update_lr(1, cfg) == 0.0  # optax: schedule(0) = init_value
    warm = min(500, 1000 // 2)
    assert tc.update_lr(warm + 1, cfg) == pytest.approx(1e-3)  # the peak, at count = warmup
    assert tc.update_lr(2, cfg) == pytest.approx(1e-3 / warm)
    assert tc.update_lr(1000, cfg) == pytest.approx(corr.cosine_lr(999, 1000, 1e-3, warm))
    assert tc.update_lr(1000, cfg) > 1e-5  # the end value is reached only at count = steps
    cfg_short = {"steps": 100, "lr": 2e-3, "warmup": 500}  # warm-up capped at half the steps
    assert tc.update_lr(51, cfg_short) == pytest.approx(2e-3)


def test_equal_error_picks_the_coarsest_plain_grid_as_accurate_as_the_hybrid():
    hyb = {"L1_per_frame": [0.02, 0.04, 0.06, 0.10], "ms_per_traj": 0.5}
    plains = [{"n": 64, "L1_per_frame": [0.03, 0.05, 0.08, 0.105], "ms_per_traj": 0.3},
              {"n": 128, "L1_per_frame": [0.02, 0.035, 0.05, 0.066], "ms_per_traj": 1.75},
              {"n": 256, "L1_per_frame": [0.01, 0.018, 0.027, 0.036], "ms_per_traj": 11.5}]
    per = pa.equal_error(hyb, plains, [1, 2, 4])
    assert per[1]["plain_n"] == 128 and per[1]["plain_L1"] == 0.02  # ties count as as-accurate
    assert per[2]["plain_n"] == 128 and per[2]["speedup"] == 1.75 / 0.5
    assert per[4]["plain_n"] == 128 and per[4]["hybrid_ms"] == 0.5
    worse = {"L1_per_frame": [0.001] * 4, "ms_per_traj": 0.5}
    assert pa.equal_error(worse, plains, [3]) == {3: {"hybrid_L1": 0.001, "plain_n": None}}
    cheap = {"L1_per_frame": [0.5] * 4, "ms_per_traj": 0.5}  # even plain 64^2 is better: speedup < 1
    assert pa.equal_error(cheap, plains, [4])[4]["plain_n"] == 64
    assert pa.equal_error(cheap, plains, [4])[4]["speedup"] == 0.3 / 0.5
