"""The learned part end to end on the GPU: solver-generated data, pushforward training with the
tensor-core kernels and AdamW, and what the trained network gains over the coarse solver without
it on held-out trajectories (a small configuration of the full training run)."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
tc = importlib.import_module("neural-pde-surrogate_b200.train_correction")


@pytest.fixture(autouse=True)
def _gpu(cuda_ok):
    pass


def test_training_improves_on_the_coarse_solver():
    """One-step training (600 steps, 16 trajectories): on held-out trajectories the hybrid step must be
    closer to the block-averaged fine solution than the coarse solver alone, in both positivity modes."""
    cfg = dict(out=None, n_traj=16, n_val=4, fine=256, coarse=64, steps=600, batch=16, unroll=1, lr=1e-3, warmup=40,
               eval_every=300, seed=0)
    tr, hist = tc.train(cfg, log=print)
    step, train_loss, val_h, val_c, ratio = hist[-1][:5]
    assert np.isfinite(train_loss) and np.isfinite(val_h)
    # untrained, the zero-initialised projection adds nothing: the hybrid equals the coarse solver;
    # trained, its normalised one-step error must be well below the coarse solver's
    assert ratio < 0.5, hist
    h, c = tr.evaluate(tr.val_U, batches=2, k=1, mode="strict")
    assert h < c, (h, c)


def test_untrained_hybrid_equals_coarse_step():
    import torch
    corr = importlib.import_module("neural-pde-surrogate_b200.correction")
    U = tc.build_dataset(2, 64, 64, index0=5)  # fine == coarse: the data are solver states themselves
    B, H, W = 2, 64, 64
    coarse = corr.CoarseSolver(B, H, W)
    net = corr.CorrectionNet(B, H, W)
    x = U[:, 0].contiguous()
    Uc = torch.empty_like(x)
    Un = torch.empty_like(x)
    fb = torch.zeros(B, dtype=torch.int32, device="cuda")
    stats = tc.field_stats(U)
    dscale = torch.ones(4, dtype=torch.float64, device="cuda")
    corr.hybrid_step(net, coarse, x, tc.DT_FRAME, stats, dscale, Uc, Un, fb)
    torch.cuda.synchronize()
    assert torch.equal(Un, Uc)  # zero-initialised last layer -> zero correction
    # and the coarse step of the hybrid is the solver itself: the data's next frame, up to the float32
    # rounding of the stored frames
    assert float(((Uc - U[:, 1]).abs() / U[:, 1].abs().clamp_min(1e-3)).max()) < 1e-3


def test_shipped_model_beats_the_plain_coarse_solver_in_rollouts():
    """The committed checkpoint, rolled out 10 frames on held-out Riemann and blast trajectories (not
    used in training), stays closer to the fine solution (512^2, block-averaged) than the plain 64^2
    solver, frame by frame, and conserves the totals to roundoff."""
    from pathlib import Path
    pa = importlib.import_module("neural-pde-surrogate_b200.pareto")
    model = Path(tc.__file__).parent / "checkpoints" / "correction_64.npz"
    items = [("riemann", 200000 + k) for k in range(3)] + [("blast", 200000 + k) for k in range(3)]
    truth, first = pa.truth_frames(items, 512, 64, 10, [64], log=print)
    z = np.load(model)
    assert float(z["gain"]) == 0.75  # the setting the checkpoint was evaluated with
    import torch
    corr = importlib.import_module("neural-pde-surrogate_b200.correction")
    _, stats, dscale = corr.load_checkpoint(str(model), 2, 64, 64)
    assert torch.equal(dscale.cpu(), torch.from_numpy(z["dscale"]) * 0.75)
    assert torch.equal(stats.cpu(), torch.from_numpy(z["stats"]))
    hyb = pa.run_hybrid(str(model), first[64], 64, 10, truth, "scale", float(z["gain"]))
    plain = pa.run_plain(first[64], 64, 64, 10, truth)
    print(hyb["L1_per_frame"], plain["L1_per_frame"])
    assert all(h < p for h, p in zip(hyb["L1_per_frame"], plain["L1_per_frame"]))
    assert hyb["drift_mass"] < 1e-13 and hyb["drift_energy"] < 1e-13 and hyb["failed"] == 0
