"""Learned correction of a coarse-grid FP64 solve: a small periodic CNN on the sm_100a tensor cores.

The reference's learned models replace the solver (surrogate/models.py); a coarse solver plus a
learned correction is its listed next step (README.md:20).  This module builds that from the
reference's parts:

* ``CorrectionNet``: 3x3 periodic convolutions (PeriodicConv, models.py:16-29) 4 -> 32 -> 32 -> 32 ->
  32 -> 32 -> 4 with tanh-GELU after every hidden layer (jax.nn.gelu default, models.py:43-44) and a
  zero-initialised last layer (models.py:67-69), so an untrained network adds nothing: 39,332
  parameters.  Weights are kept in FP32 (master copy) and packed to BF16 for the tensor cores;
  activations are BF16, accumulation FP32.
* ``hybrid_step``: coarse FP64 solver over one frame interval (CFL sub-steps landing on the frame
  time, main2d.cpp:237-242), then the network's correction -- relative to the coarse cell: density
  and momentum in units of its density, energy in units of its energy -- projected to zero mean per
  conserved field in FP64 (totals of mass, momentum, energy unchanged) and added.  A step that would
  go non-physical falls back to the plain coarse step ('strict'), or keeps the largest fraction of
  the correction that stays physical ('scale', the default; fraction 0 is the plain coarse step),
  halved while the corrected state's signal speed exceeds MAX_SPEED_RATIO times the coarse state's.
* AdamW with clipping by global norm 1.0 and weight decay 1e-4 (train.py:209-211), warm-up + cosine
  decay to 0.01 * lr (optax.warmup_cosine_decay_schedule, train.py:207-208).

All tensors are CUDA torch tensors used as plain device buffers; every computation is a kernel of
libfv (include/fvnet.h).
"""
import ctypes as C
import math

import numpy as np

from ._lib import check, device_ptr, lib

CORR_MODES = {"strict": 0, "keep": 1, "scale": 2}  # FVNET_CORR_* of include/fvnet.h
# The 'scale' rule's bound on the corrected state's signal speed, relative to the coarse state's: the
# next coarse step of a hybrid rollout then takes at most 1.1 times the CFL sub-steps of the plain
# coarse state.  Without it, a correction that thins a cell out to a tenth of its density can raise
# the sound and flow speeds many-fold, and a batched coarse solve waits for that one trajectory.  On
# the bench's 128-trajectory batch (64^2, 100 frames) the bound took the slowest trajectory from 354
# to 35 sub-steps per frame and the time per trajectory from 6.5 to 1.45 ms, with the L1 errors
# unchanged to three digits (ratios 1.25, 1.5, 2 and 3 gave 1.9, 2.8, 2.8 and 2.9 ms).
MAX_SPEED_RATIO = 1.1

# (c_in, c_out, c_in padded, c_out padded) of the six convolutions
LAYERS = [(4, 32, 16, 32), (32, 32, 32, 32), (32, 32, 32, 32), (32, 32, 32, 32), (32, 32, 32, 32), (32, 4, 32, 16)]


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def param_count():
    return sum(co * ci * 9 + co for ci, co, _, _ in LAYERS)


def cosine_lr(step, total, lr, warmup):
    """optax.warmup_cosine_decay_schedule(0, lr, warmup, total, end_value=0.01*lr) at `step`."""
    end = 0.01 * lr
    if warmup > 0 and step < warmup:
        return lr * step / warmup
    frac = min(max((step - warmup) / max(total - warmup, 1), 0.0), 1.0)
    return end + (lr - end) * 0.5 * (1.0 + math.cos(math.pi * frac))


class CorrectionNet:
    """Parameters, packed weights and activation buffers of the correction CNN for a batch shape
    (B, H, W).  `params` is one flat FP32 tensor: per layer W (c_out, c_in, 3, 3) then b (c_out)."""

    def __init__(self, B, H, W, seed=0, device="cuda", params=None):
        import torch
        self.torch = torch
        self.B, self.H, self.W = B, H, W
        self.device = device
        n = param_count()
        if params is None:
            g = np.random.default_rng(seed)
            chunks = []
            for k, (ci, co, _, _) in enumerate(LAYERS):
                lim = 1.0 / math.sqrt(ci * 9)  # equinox Conv2d default: U(-1/sqrt(fan_in), 1/sqrt(fan_in))
                if k == len(LAYERS) - 1:
                    chunks += [np.zeros(co * ci * 9), np.zeros(co)]  # zero-initialised projection
                else:
                    chunks += [g.uniform(-lim, lim, co * ci * 9), g.uniform(-lim, lim, co)]
            params = np.concatenate(chunks).astype(np.float32)
        self.params = torch.as_tensor(np.asarray(params, np.float32), device=device).contiguous()
        if self.params.numel() != n:
            raise ValueError(f"params: expected {n} values, got {self.params.numel()}")
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        # views per layer
        self.Wv, self.bv, self.dWv, self.dbv = [], [], [], []
        off = 0
        for ci, co, _, _ in LAYERS:
            self.Wv.append(self.params[off:off + co * ci * 9])
            self.dWv.append(self.grads[off:off + co * ci * 9])
            off += co * ci * 9
            self.bv.append(self.params[off:off + co])
            self.dbv.append(self.grads[off:off + co])
            off += co
        bf16 = torch.bfloat16
        self.Wf = [torch.empty(9 * cip * cop, dtype=bf16, device=device) for _, _, cip, cop in LAYERS]
        self.Wb = [torch.empty(9 * cip * cop, dtype=bf16, device=device) for _, _, cip, cop in LAYERS]
        self.bias_pad = [torch.zeros(cop, dtype=torch.float32, device=device) for _, _, _, cop in LAYERS]
        npix = B * H * W
        self.X16 = torch.zeros((B, H, W, 16), dtype=bf16, device=device)
        self.Z = [torch.empty((B, H, W, 32), dtype=bf16, device=device) for _ in range(5)]
        self.A = [torch.empty((B, H, W, 32), dtype=bf16, device=device) for _ in range(5)]
        self.out4 = torch.empty((B, H, W, 4), dtype=torch.float32, device=device)
        self.dout16 = torch.zeros((B, H, W, 16), dtype=bf16, device=device)
        self.dZ = [torch.empty((B, H, W, 32), dtype=bf16, device=device) for _ in range(2)]
        parts = lib().fvnet_wgrad_parts(B, H)
        self.partial = torch.empty(parts * 9 * 32 * 32, dtype=torch.float32, device=device)
        self.db_part = torch.empty(parts * 32, dtype=torch.float32, device=device)
        self.norm_part = torch.empty(lib().fvnet_norm_partials(), dtype=torch.float64, device=device)
        self.norm = torch.zeros(1, dtype=torch.float64, device=device)
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.theta = torch.ones(B, dtype=torch.float64, device=device)
        self.npix = npix
        self.pack()

    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def pack(self):
        """FP32 master weights -> BF16 tensor-core packs (forward and backward-data)."""
        for k, (ci, co, cip, cop) in enumerate(LAYERS):
            check(lib().fvnet_pack_weights(co, ci, cop, cip, _p(self.Wv[k]), _p(self.Wf[k]), _p(self.Wb[k]),
                                           self.stream()))
            self.bias_pad[k][:co].copy_(self.bv[k])

    def check_device_error(self):
        if int(self.err.item()):
            raise RuntimeError("a bounded device-side wait of the convolution kernels gave up")

    # ---- forward / backward ---------------------------------------------------------------------
    def forward(self, U, stats):
        """U: (B, H, W, 4) float64 CUDA state -> self.out4 (B, H, W, 4) float32 network output."""
        L, st = lib(), self.stream()
        B, H, W = self.B, self.H, self.W
        Up = device_ptr(U, (B, H, W, 4), what="U")
        check(L.fvnet_prep_input(Up, self.npix, device_ptr(stats, numel=8, what="stats"), _p(self.X16), st))
        x = self.X16
        for k in range(5):
            cip, cop = LAYERS[k][2], LAYERS[k][3]
            check(L.fvnet_conv3x3(0, cip, cop, B, H, W, _p(x), _p(self.Wf[k]), _p(self.bias_pad[k]), None,
                                  _p(self.Z[k]), _p(self.A[k]), None, _p(self.err), st))
            x = self.A[k]
        check(L.fvnet_conv3x3(1, 32, 16, B, H, W, _p(x), _p(self.Wf[5]), _p(self.bias_pad[5]), None, None, None,
                              _p(self.out4), _p(self.err), st))
        return self.out4

    def backward(self, dout16=None):
        """Gradients of all parameters into self.grads from d loss / d out (B, H, W, 16) BF16."""
        L, st = lib(), self.stream()
        B, H, W = self.B, self.H, self.W
        if dout16 is not None:
            device_ptr(dout16, (B, H, W, 16), dtype="torch.bfloat16", what="dout16")
        dz = self.dout16 if dout16 is None else dout16
        for k in range(5, -1, -1):
            ci, co, cip, cop = LAYERS[k]
            xin = self.X16 if k == 0 else self.A[k - 1]
            check(L.fvnet_conv3x3_wgrad(cip, cop, ci, co, B, H, W, _p(xin), _p(dz), _p(self.partial), _p(self.dWv[k]),
                                        _p(self.dbv[k]), _p(self.db_part), _p(self.err), st))
            if k == 0:
                break
            dprev = self.dZ[k % 2]
            check(L.fvnet_conv3x3(2, cop, cip, B, H, W, _p(dz), _p(self.Wb[k]), None, _p(self.Z[k - 1]), None,
                                  _p(dprev), None, _p(self.err), st))
            dz = dprev
        return self.grads

    def adamw(self, lr, weight_decay=1e-4, max_norm=1.0, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        check(lib().fvnet_adamw(_p(self.params), _p(self.grads), _p(self.m), _p(self.v), self.params.numel(),
                                _p(self.norm_part), lr, b1, b2, eps, weight_decay, max_norm, self.step_count,
                                _p(self.norm), self.stream()))
        self.pack()

    # ---- correction step ------------------------------------------------------------------------
    def correct(self, Uc, stats, dscale, Unext, fallback, mode="scale", max_speed_ratio=MAX_SPEED_RATIO):
        """Unext = Uc + zero-mean(out * dscale), with the positivity rule `mode` (include/fvnet.h):
        'strict' -> samples that would be non-physical take the plain coarse step; 'scale' -> the
        largest fraction theta of the correction that keeps rho and p positive (self.theta), halved
        until the signal speed is at most max_speed_ratio times the coarse state's (<= 0: no bound);
        'keep' -> always the full correction (the trained step of a training iteration)."""
        self.forward(Uc, stats)
        shape = (self.B, self.H, self.W, 4)
        check(lib().fvnet_apply_correction(device_ptr(Uc, shape, what="Uc"), _p(self.out4), self.B, self.H * self.W,
                                           device_ptr(dscale, numel=4, what="dscale"),
                                           device_ptr(Unext, shape, what="Unext"),
                                           device_ptr(fallback, (self.B,), dtype="torch.int32", what="fallback"),
                                           _p(self.theta), CORR_MODES[mode], float(max_speed_ratio), self.stream()))
        return Unext

    def loss_grad(self, Unext, Y, Uc, stats, dscale, theta, loss_part):
        """Uc: the coarse state the correction was added to; theta: per-sample fraction of the
        correction applied (gradient scale), or None (1)."""
        shape = (self.B, self.H, self.W, 4)
        th = None if theta is None else device_ptr(theta, (self.B,), what="theta")
        check(lib().fvnet_loss_grad(device_ptr(Unext, shape, what="Unext"), device_ptr(Y, shape, what="Y"),
                                    device_ptr(Uc, shape, what="Uc"), self.B, self.H * self.W,
                                    device_ptr(stats, numel=8, what="stats"), device_ptr(dscale, numel=4, what="dscale"),
                                    th, device_ptr(loss_part, (self.B,), what="loss_part"), _p(self.dout16),
                                    self.stream()))
        return loss_part


class CoarseSolver:
    """The coarse FP64 step of the hybrid: B grids of H x W (periodic unit box) advanced together by
    one frame interval with their own CFL sub-steps (an fv_ensemble)."""

    def __init__(self, B, H, W, flux="hllc", limiter="vanleer", cfl=0.5, stream=None):
        from . import make_grid
        from .ensemble import Ensemble
        self.grid = make_grid(W, H, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic")
        self.ens = Ensemble([self.grid] * B, flux, limiter, cfl, stream=stream)
        self.B = B

    def advance(self, U, dt_frame, out):
        """out = U advanced by dt_frame (each sample from t = 0 to t = dt_frame)."""
        self.ens.set_all(U)
        _, steps, status = self.ens.advance_to(dt_frame, raise_on_nonphysical=False)
        self.ens.get_all(out)
        return steps, status


def load_checkpoint(path, B, H, W, gain=None, device="cuda"):
    """A trained correction for B grids of H x W: (net, stats, dscale) ready for hybrid_step.
    dscale includes the correction gain -- the checkpoint's evaluated setting (its `gain` entry,
    1 if absent) unless `gain` is given."""
    import torch
    z = np.load(path)
    g = float(z["gain"]) if gain is None and "gain" in z.files else (1.0 if gain is None else float(gain))
    net = CorrectionNet(B, H, W, device=device, params=z["params"])
    stats = torch.from_numpy(z["stats"]).to(device)
    dscale = torch.from_numpy(z["dscale"]).to(device) * g
    return net, stats, dscale


def hybrid_step(net, coarse, U, dt_frame, stats, dscale, Uc, Unext, fallback, mode="scale"):
    """One hybrid step: Uc = coarse(U, dt_frame); Unext = Uc + projected correction under the
    positivity rule `mode` ('strict': fall back to the plain coarse step; 'scale': largest physical
    fraction of the correction; 'keep': full correction).  Returns the coarse solve's (steps, status):
    status[b] != 0 means sample b's coarse step stopped at a non-physical state before dt_frame, so
    its Uc and Unext are not states at the new time -- callers must not use them as such."""
    steps, status = coarse.advance(U, dt_frame, Uc)
    net.correct(Uc, stats, dscale, Unext, fallback, mode)
    return steps, status
