"""Tensor-core convolutions and the correction step on the GPU against the torch CPU oracle.

Inputs and weights are BF16 (exact in FP32), products are accumulated in FP32, outputs rounded to
BF16: each kernel is compared with torch FP32 on the same BF16 inputs, to 1e-2 of the output's
scale for BF16 outputs and 1e-4 for FP32 outputs (accumulation order differs)."""
import ctypes as C
import importlib

import numpy as np
import pytest
import torch
import torch.nn.functional as F

from torch_correction import conv_periodic, correction_loss, unflatten

pytestmark = pytest.mark.gpu
fv = importlib.import_module("neural-pde-surrogate_b200")
corr = importlib.import_module("neural-pde-surrogate_b200.correction")
L = fv.lib()


@pytest.fixture(autouse=True)
def _gpu(cuda_ok):
    pass


def P(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def bf(x):
    return torch.as_tensor(x, dtype=torch.float32).to(torch.bfloat16)


def rel(a, b):
    a, b = a.float().cpu(), b.float().cpu()
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))


def pack(Wc, co, ci, cop, cip):
    Wf = torch.empty(9 * cip * cop, dtype=torch.bfloat16, device="cuda")
    Wb = torch.empty_like(Wf)
    assert L.fvnet_pack_weights(co, ci, cop, cip, P(Wc), P(Wf), P(Wb), None) == 0
    return Wf, Wb


SHAPES = [(2, 8, 64), (1, 4, 128), (1, 16, 32), (3, 4, 64)]


@pytest.mark.parametrize("B,H,W", SHAPES)
@pytest.mark.parametrize("ci,co,cip,cop", [(4, 32, 16, 32), (32, 32, 32, 32)])
def test_conv_hidden_forward(B, H, W, ci, co, cip, cop):
    g = torch.Generator().manual_seed(B * 100 + H + W + ci)
    X = torch.zeros((B, H, W, cip))
    X[..., :ci] = torch.randn((B, H, W, ci), generator=g)
    Xb = bf(X).cuda()
    Wc = torch.randn((co, ci, 3, 3), generator=g) * 0.2
    b = torch.randn(cop, generator=g) * 0.1
    Wf, _ = pack(Wc.cuda().contiguous(), co, ci, cop, cip)
    Z = torch.empty((B, H, W, cop), dtype=torch.bfloat16, device="cuda")
    A = torch.empty_like(Z)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.fvnet_conv3x3(0, cip, cop, B, H, W, P(Xb), P(Wf), P(b.cuda()), None, P(Z), P(A), None, P(err), None)
    assert rc == 0, L.fv_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    x = Xb.float().cpu()[..., :ci].permute(0, 3, 1, 2)
    w = bf(Wc).float()
    z = conv_periodic(x, w, b[:co]).permute(0, 2, 3, 1)
    assert rel(Z[..., :co], z) < 1e-2
    assert rel(A[..., :co], F.gelu(z, approximate="tanh")) < 1e-2


@pytest.mark.parametrize("B,H,W", SHAPES)
def test_conv_output_forward(B, H, W):
    g = torch.Generator().manual_seed(7 + W)
    X = bf(torch.randn((B, H, W, 32), generator=g)).cuda()
    Wc = torch.randn((4, 32, 3, 3), generator=g) * 0.1
    b = torch.zeros(16)
    b[:4] = torch.randn(4, generator=g)
    Wf, _ = pack(Wc.cuda().contiguous(), 4, 32, 16, 32)
    out4 = torch.empty((B, H, W, 4), dtype=torch.float32, device="cuda")
    rc = L.fvnet_conv3x3(1, 32, 16, B, H, W, P(X), P(Wf), P(b.cuda()), None, None, None, P(out4), None, None)
    assert rc == 0, L.fv_last_error()
    torch.cuda.synchronize()
    ref = conv_periodic(X.float().cpu().permute(0, 3, 1, 2), bf(Wc).float(), b[:4]).permute(0, 2, 3, 1)
    assert rel(out4, ref) < 1e-4


@pytest.mark.parametrize("B,H,W", SHAPES)
@pytest.mark.parametrize("ci,co,cip,cop", [(32, 32, 32, 32), (32, 4, 32, 16)])
def test_conv_backward_data(B, H, W, ci, co, cip, cop):
    """d/dX of conv(X) contracted with dZ, times gelu'(Zprev) (the hidden layer below)."""
    g = torch.Generator().manual_seed(11 + W + co)
    dZ = torch.zeros((B, H, W, cop))
    dZ[..., :co] = torch.randn((B, H, W, co), generator=g)
    dZb = bf(dZ).cuda()
    Zp = bf(torch.randn((B, H, W, cip), generator=g)).cuda()
    Wc = torch.randn((co, ci, 3, 3), generator=g) * 0.2
    _, Wb = pack(Wc.cuda().contiguous(), co, ci, cop, cip)
    out = torch.empty((B, H, W, cip), dtype=torch.bfloat16, device="cuda")
    rc = L.fvnet_conv3x3(2, cop, cip, B, H, W, P(dZb), P(Wb), None, P(Zp), None, P(out), None, None, None)
    assert rc == 0, L.fv_last_error()
    torch.cuda.synchronize()
    x = torch.zeros((B, ci, H, W), requires_grad=True)
    y = conv_periodic(x, bf(Wc).float(), None)
    y.backward(dZb.float().cpu()[..., :co].permute(0, 3, 1, 2))
    zp = Zp.float().cpu().requires_grad_(True)
    gelu_grad = torch.autograd.grad(F.gelu(zp, approximate="tanh").sum(), zp)[0]
    ref = x.grad.permute(0, 2, 3, 1) * gelu_grad
    assert rel(out, ref) < 1e-2


# (3, 296, 32): 888 rows over 296 CTAs, 3 consecutive rows per CTA with image boundaries inside a CTA's
# range -- the row ring of the weight-gradient kernel reuses two of the three input rows
@pytest.mark.parametrize("B,H,W", [(2, 8, 64), (1, 4, 128), (1, 16, 32), (5, 8, 64), (3, 296, 32)])
@pytest.mark.parametrize("ci,co,cip,cop", [(4, 32, 16, 32), (32, 32, 32, 32), (32, 4, 32, 16)])
def test_conv_weight_gradient(B, H, W, ci, co, cip, cop):
    g = torch.Generator().manual_seed(23 + W + ci + co)
    X = torch.zeros((B, H, W, cip))
    X[..., :ci] = torch.randn((B, H, W, ci), generator=g)
    dZ = torch.zeros((B, H, W, cop))
    dZ[..., :co] = torch.randn((B, H, W, co), generator=g)
    Xb, dZb = bf(X).cuda(), bf(dZ).cuda()
    parts = L.fvnet_wgrad_parts(B, H)
    partial = torch.empty(parts * 9 * cip * cop, dtype=torch.float32, device="cuda")
    dW = torch.empty(co * ci * 9, dtype=torch.float32, device="cuda")
    db = torch.empty(co, dtype=torch.float32, device="cuda")
    dbp = torch.empty(parts * cop, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.fvnet_conv3x3_wgrad(cip, cop, ci, co, B, H, W, P(Xb), P(dZb), P(partial), P(dW), P(db), P(dbp), P(err), None)
    assert rc == 0, L.fv_last_error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    w = torch.zeros((co, ci, 3, 3), requires_grad=True)
    bb = torch.zeros(co, requires_grad=True)
    y = conv_periodic(Xb.float().cpu()[..., :ci].permute(0, 3, 1, 2), w, bb)
    y.backward(dZb.float().cpu()[..., :co].permute(0, 3, 1, 2))
    assert rel(dW.reshape(co, ci, 3, 3), w.grad) < 1e-4
    assert rel(db, bb.grad) < 1e-4


def _stats():
    return torch.tensor([1.0, 0.1, -0.1, 2.0, 2.0, 3.0, 3.0, 0.7], dtype=torch.float64)


def _physical(rng, shape):
    """Conserved states with rho, p in (0.5, 1.5) and |u|, |v| < 0.5."""
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    rho = rng.uniform(0.5, 1.5, shape)
    u, v = rng.uniform(-0.5, 0.5, shape), rng.uniform(-0.5, 0.5, shape)
    p = rng.uniform(0.5, 1.5, shape)
    return torch.tensor(ic.to_conserved(rho, u, v, p), dtype=torch.float64)


def test_full_network_gradient_vs_autograd():
    """Forward + backward of the whole correction loss on the GPU vs torch FP64 autograd on the same
    parameters: bf16 activations keep the agreement at the 1e-2 level of the gradient's norm."""
    B, H, W = 2, 8, 64
    rng = np.random.default_rng(4)
    params = rng.normal(0, 0.15, corr.param_count()).astype(np.float32)
    net = corr.CorrectionNet(B, H, W, params=params)
    Uc = _physical(rng, (B, H, W))
    Y = Uc + torch.tensor(rng.normal(0, 0.02, (B, H, W, 4)))
    stats = _stats()
    dscale = torch.tensor([0.02, 0.03, 0.03, 0.05], dtype=torch.float64)
    Un = torch.empty_like(Uc).cuda()
    fb = torch.zeros(B, dtype=torch.int32, device="cuda")
    lp = torch.zeros(B, dtype=torch.float64, device="cuda")
    Uc_d = Uc.cuda()
    net.correct(Uc_d, stats.cuda(), dscale.cuda(), Un, fb, mode="keep")
    net.loss_grad(Un, Y.cuda(), Uc_d, stats.cuda(), dscale.cuda(), None, lp)
    net.backward()
    torch.cuda.synchronize()
    net.check_device_error()
    p = torch.tensor(params.astype(np.float64), requires_grad=True)
    layers, off = [], 0
    for ci, co, _, _ in corr.LAYERS:
        layers.append((p[off:off + co * ci * 9].reshape(co, ci, 3, 3), p[off + co * ci * 9:off + co * ci * 9 + co]))
        off += co * ci * 9 + co
    loss, Un_ref = correction_loss(layers, Uc, Y, stats, dscale)
    loss.backward()
    assert (net.theta.cpu() == 1).all()  # KEEP: the full correction, whether or not it is physical
    assert abs(lp.sum().item() / (B * H * W * 4) - loss.item()) / loss.item() < 1e-2
    D_ref = (Un_ref.detach() - Uc).abs().max()
    assert float((Un.cpu() - Un_ref.detach()).abs().max()) < 5e-2 * float(D_ref)
    g_gpu, g_ref = net.grads.double().cpu(), p.grad
    assert float((g_gpu - g_ref).norm() / g_ref.norm()) < 5e-2


def test_projection_conserves_totals_and_falls_back():
    B, H, W = 3, 4, 64
    rng = np.random.default_rng(5)
    net = corr.CorrectionNet(B, H, W, params=rng.normal(0, 0.2, corr.param_count()).astype(np.float32))
    Uc = _physical(rng, (B, H, W))
    stats = _stats().cuda()
    Un = torch.empty_like(Uc).cuda()
    fb = torch.zeros(B, dtype=torch.int32, device="cuda")
    def totals_kept(U):  # to FP64 roundoff of the summed magnitudes
        tot_c, tot_n = Uc.sum(dim=(1, 2)), U.cpu().sum(dim=(1, 2))
        scale = U.cpu().abs().sum(dim=(1, 2)) + Uc.abs().sum(dim=(1, 2))
        return float(((tot_n - tot_c).abs() / scale).max()) < 1e-14

    def physical(U):
        r = U[..., 0]
        p = 0.4 * (U[..., 3] - 0.5 * (U[..., 1] ** 2 + U[..., 2] ** 2) / r)
        return bool((r > 0).all() and (p > 0).all())

    small = torch.tensor([1e-3] * 4, dtype=torch.float64, device="cuda")
    huge = torch.tensor([1e3] * 4, dtype=torch.float64, device="cuda")
    for mode in ("strict", "scale", "keep"):
        net.correct(Uc.cuda(), stats, small, Un, fb, mode=mode)
        torch.cuda.synchronize()
        assert (fb.cpu() == 0).all() and totals_kept(Un) and float((Un.cpu() - Uc).abs().max()) > 0
    # a huge correction makes some cells non-physical:
    net.correct(Uc.cuda(), stats, huge, Un, fb, mode="strict")  # -> the plain coarse step
    torch.cuda.synchronize()
    assert int(fb.sum()) == B
    assert torch.equal(Un.cpu(), Uc) and (net.theta.cpu() == 0).all()
    net.correct(Uc.cuda(), stats, huge, Un, fb, mode="scale")  # -> the largest physical fraction
    torch.cuda.synchronize()
    th = net.theta.cpu()
    assert int(fb.sum()) == B and (th > 0).all() and (th < 1).all()
    assert physical(Un.cpu()) and totals_kept(Un)
    net.correct(Uc.cuda(), stats, huge, Un, fb, mode="keep")  # -> full correction, flagged
    torch.cuda.synchronize()
    assert int(fb.sum()) == B and not physical(Un.cpu()) and totals_kept(Un)


def test_adamw_matches_optax_semantics():
    n = 39332
    rng = np.random.default_rng(6)
    p0 = rng.normal(0, 0.1, n).astype(np.float32)
    net = corr.CorrectionNet(1, 4, 64, params=p0)
    p, m, v = p0.astype(np.float64), np.zeros(n), np.zeros(n)
    for step in range(1, 4):
        g = rng.normal(0, 0.05 * step, n).astype(np.float32)
        net.grads.copy_(torch.tensor(g))
        lr = 1e-3 * step
        net.adamw(lr)
        norm = np.sqrt(np.sum(g.astype(np.float64) ** 2))
        gs = g * min(1.0, 1.0 / norm)
        m = 0.9 * m + 0.1 * gs
        v = 0.999 * v + 0.001 * gs * gs
        upd = (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8) + 1e-4 * p
        p = p - lr * upd
        assert abs(net.norm.item() - norm) / norm < 1e-6
    assert np.abs(net.params.cpu().numpy() - p).max() < 1e-5


def test_network_is_translation_equivariant():
    """Periodic convolutions commute with periodic shifts: tests/test_models.py:46-50 checks
    roll(model(x)) == model(roll(x)) to 1e-5 for a (7, -13) shift. Every output pixel here accumulates its
    taps and channels in the same order wherever it sits, so the rolled output is equal bit for bit."""
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    B, n = 2, 64
    rng = np.random.default_rng(11)
    net = corr.CorrectionNet(B, n, n, params=rng.normal(0, 0.1, corr.param_count()).astype(np.float32))
    U = torch.stack([torch.from_numpy(ic.to_conserved(*ic.sample("blast", k, n)[:4])) for k in range(B)]).cuda()
    stats = torch.tensor([1.0, 0.0, 0.0, 2.5, 1.0, 1.0, 1.0, 0.3], dtype=torch.float64, device="cuda")
    out = net.forward(U, stats).clone()
    assert out.abs().max() > 0
    for shift in [(7, -13), (5, 0), (0, 9), (13, 50)]:
        rolled = net.forward(torch.roll(U, shift, dims=(1, 2)).contiguous(), stats).clone()
        torch.cuda.synchronize()
        net.check_device_error()
        assert torch.equal(rolled, torch.roll(out, shift, dims=(1, 2))), shift


def test_scale_mode_bounds_the_signal_speed():
    """'scale' with a signal-speed bound: a correction that would raise max(|u|+a) + max(|v|+a) above
    the ratio times the coarse state's is halved until it does not (or dropped), and stays physical,
    conservative and no larger than the positivity-only fraction."""
    B, H, W = 3, 4, 64
    rng = np.random.default_rng(9)
    net = corr.CorrectionNet(B, H, W, params=rng.normal(0, 0.2, corr.param_count()).astype(np.float32))
    Uc = _physical(rng, (B, H, W))
    stats = _stats().cuda()
    Un = torch.empty_like(Uc).cuda()
    fb = torch.zeros(B, dtype=torch.int32, device="cuda")
    big = torch.tensor([1.0, 30.0, 30.0, 1.0], dtype=torch.float64, device="cuda")  # mostly momentum

    def speed(U):
        r = U[..., 0]
        u, v = U[..., 1] / r, U[..., 2] / r
        a = torch.sqrt(1.4 * 0.4 * (U[..., 3] - 0.5 * r * (u * u + v * v)) / r)
        return (u.abs() + a).amax(dim=(1, 2)) + (v.abs() + a).amax(dim=(1, 2))

    net.correct(Uc.cuda(), stats, big, Un, fb, mode="scale", max_speed_ratio=0.0)  # positivity only
    torch.cuda.synchronize()
    th_free = net.theta.cpu().clone()
    s_free = speed(Un.cpu())
    for ratio in (1.2, 2.0):
        net.correct(Uc.cuda(), stats, big, Un, fb, mode="scale", max_speed_ratio=ratio)
        torch.cuda.synchronize()
        th = net.theta.cpu()
        assert (th <= th_free).all()
        assert (speed(Un.cpu()) <= ratio * speed(Uc) * (1 + 1e-12)).all()
        for b in range(B):  # the bound acted only where the free fraction broke it
            if s_free[b] <= ratio * speed(Uc)[b]:
                assert th[b] == th_free[b]
            else:
                assert th[b] < th_free[b]
    assert bool((s_free > 1.2 * speed(Uc)).any())  # the case exercises the bound
    with pytest.raises(Exception):
        net.correct(Uc.cuda(), stats, big, Un, fb, mode="scale", max_speed_ratio=0.5)  # below 1: rejected
