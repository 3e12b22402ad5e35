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
