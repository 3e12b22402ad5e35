"""The correction oracle's gradients against central finite differences (CPU, FP64), and the host
logic of the correction module (learning-rate schedule, parameter count)."""
import math

import numpy as np
import torch

from torch_correction import corr, correction_loss, unflatten


def test_parameter_count_is_about_40k():
    assert corr.param_count() == 39332


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    B, H, W = 2, 8, 8
    params = rng.normal(0, 0.2, corr.param_count())
    Uc = torch.tensor(rng.uniform(0.5, 1.5, (B, H, W, 4)))
    Y = Uc + torch.tensor(rng.normal(0, 0.01, (B, H, W, 4)))
    stats = torch.tensor([1.0, 0.0, 0.0, 2.0, 1 / 0.5, 1 / 0.3, 1 / 0.3, 1 / 0.7])
    dscale = torch.tensor([0.01, 0.02, 0.02, 0.03])
    p = torch.tensor(params, requires_grad=True)

    def loss_of(pvec):
        layers = []
        off = 0
        for ci, co, _, _ in corr.LAYERS:
            Wt = pvec[off:off + co * ci * 9].reshape(co, ci, 3, 3)
            off += co * ci * 9
            b = pvec[off:off + co]
            off += co
            layers.append((Wt, b))
        return correction_loss(layers, Uc, Y, stats, dscale)[0]

    loss = loss_of(p)
    loss.backward()
    g = p.grad.numpy()
    idx = list(rng.choice(len(params), 12, replace=False)) + [len(params) - 1, len(params) - 5, 0]
    for i in idx:
        h = 1e-6
        pp, pm = params.copy(), params.copy()
        pp[i] += h
        pm[i] -= h
        fd = (loss_of(torch.tensor(pp)).item() - loss_of(torch.tensor(pm)).item()) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-9, (i, fd, g[i])


def test_projection_conserves_totals_in_oracle():
    rng = np.random.default_rng(1)
    Uc = torch.tensor(rng.uniform(0.5, 1.5, (3, 8, 8, 4)))
    layers = unflatten(rng.normal(0, 0.3, corr.param_count()))
    stats = torch.tensor([1.0, 0.0, 0.0, 2.0, 2.0, 3.0, 3.0, 1.5])
    _, Un = correction_loss(layers, Uc, Uc, stats, torch.tensor([0.1, 0.1, 0.1, 0.1]))
    assert torch.allclose(Un.sum(dim=(1, 2)), Uc.sum(dim=(1, 2)), rtol=0, atol=1e-12)


def test_cosine_schedule():
    lr, total, warm = 1e-3, 1000, 100
    assert corr.cosine_lr(0, total, lr, warm) == 0.0
    assert math.isclose(corr.cosine_lr(warm, total, lr, warm), lr)
    assert math.isclose(corr.cosine_lr(total, total, lr, warm), 0.01 * lr)
    vals = [corr.cosine_lr(s, total, lr, warm) for s in range(warm, total + 1, 50)]
    assert all(a >= b for a, b in zip(vals, vals[1:]))
