"""CPU oracle of the learned correction (test infrastructure): torch autograd on the same maths as
the tensor-core kernels -- periodic 3x3 convolutions (the reference's PeriodicConv,
surrogate/models.py:16-29: wrap pad + VALID cross-correlation), tanh-GELU (jax.nn.gelu default,
models.py:43-44), the FP64 zero-mean projection and the normalised MSE loss.  The reference's own
models are JAX (absent here), so its gradients are restated with torch; the oracle is itself
checked against finite differences (tests/test_correction_oracle.py)."""
import importlib

import numpy as np
import torch
import torch.nn.functional as F

corr = importlib.import_module("neural-pde-surrogate_b200.correction")
LAYERS = corr.LAYERS


def unflatten(params, dtype=torch.float64):
    p = torch.as_tensor(np.asarray(params), dtype=dtype)
    out, off = [], 0
    for ci, co, _, _ in LAYERS:
        W = p[off:off + co * ci * 9].reshape(co, ci, 3, 3)
        off += co * ci * 9
        b = p[off:off + co]
        off += co
        out.append((W, b))
    return out


def conv_periodic(h, W, b):
    """h: (B, C, H, W) NCHW.  wrap-pad by 1 then VALID 3x3 cross-correlation."""
    return F.conv2d(F.pad(h, (1, 1, 1, 1), mode="circular"), W, b)


def net_forward(layers, x):
    """x: (B, H, W, 4) normalised input -> (B, H, W, 4) network output."""
    h = x.permute(0, 3, 1, 2)
    for k, (W, b) in enumerate(layers):
        h = conv_periodic(h, W, b)
        if k < len(layers) - 1:
            h = F.gelu(h, approximate="tanh")
    return h.permute(0, 2, 3, 1)


def correction_loss(layers, Uc, Y, stats, dscale):
    """Loss of one hybrid step after the coarse solve Uc (B, H, W, 4) FP64: out = net(normalise(Uc)),
    D = out * dscale * (rho, rho, rho, E) of Uc, projected to zero mean per sample and field,
    Unext = Uc + D, loss = mean of ((Unext - Y) / std)^2."""
    mean, inv_std = stats[:4], stats[4:]
    x = (Uc - mean) * inv_std
    out = net_forward(layers, x)
    w = torch.stack([Uc[..., 0], Uc[..., 0], Uc[..., 0], Uc[..., 3]], dim=-1)
    D = out * dscale * w
    D = D - D.mean(dim=(1, 2), keepdim=True)
    Un = Uc + D
    return (((Un - Y) * inv_std) ** 2).mean(), Un
