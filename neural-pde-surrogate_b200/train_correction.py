"""Train the coarse-grid correction on solver-generated data (the learned part, on the GPU).

  python neural-pde-surrogate_b200/train_correction.py --out runs/corr --n-traj 512 --fine 512 \
         --coarse 64 --steps 20000 --batch 64 --unroll 4 --lr 1e-3

Data: n_traj trajectories (half four-quadrant Riemann, half blast + bubble initial conditions,
indices [index0, index0 + n_traj/2) of each family) solved by the FP64 GPU solver at fine^2 and
block-averaged to coarse^2 every 0.005 in time (generate.trajectory); or, with --packed DIR, the
train and val splits that generate.py and dataset.py wrote to DIR.  Normalisation statistics are
taken from these training frames only (data/pack.py:54-112 does the same).

Model step (correction.hybrid_step): the coarse FP64 solver advances one frame interval, the CNN
adds a zero-mean (conservative) correction.  Loss: pushforward with `unroll` steps
(surrogate/train.py:107-111): unroll-1 hybrid steps without gradient, then one trained step to the
true frame t+unroll, MSE in normalised units.  Optimiser: clip by global norm 1.0 + AdamW (weight
decay 1e-4) with warm-up + cosine decay to 0.01*lr (train.py:207-211).  Writes log.csv, config.json,
best.npz / last.npz (parameters) like the reference's run folder (train.py:197-255).
"""
import argparse
import csv
import importlib
import json
import sys
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

PKG = "neural-pde-surrogate_b200"
DT_FRAME = 0.005


def build_dataset(n_traj, fine, coarse, index0=0, families=("riemann", "blast"), frames=None, log=print):
    """(N, F, coarse, coarse, 4) float64 CUDA tensor of block-averaged conserved states; F is the
    shortest trajectory's frame count (every trajectory is truncated to it)."""
    import torch
    fv = importlib.import_module(PKG)
    gen = importlib.import_module(f"{PKG}.generate")
    solver = fv.Solver(fv.make_grid(fine, fine, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic"), "hllc", "vanleer", 0.5)
    out, t0, cells = [], time.time(), 0
    per = max(1, n_traj // len(families))
    for fam in families:
        for k in range(per):
            t, levels, steps, _ = gen.trajectory(fam, index0 + k, fine, [coarse], solver=solver)
            out.append(levels[coarse])
            cells += steps * fine * fine
    nf = min(a.shape[0] for a in out) if frames is None else frames
    data = np.stack([a[:nf] for a in out])  # (N, F, 4, c, c) float32
    U = torch.from_numpy(np.ascontiguousarray(data.transpose(0, 1, 3, 4, 2))).to("cuda", torch.float64)
    log(f"dataset: {len(out)} trajectories at {fine}^2 -> {coarse}^2, {nf} frames, {time.time() - t0:.1f} s "
        f"({cells / max(time.time() - t0, 1e-9) / 1e9:.2f} G cell-updates/s incl. transfers)")
    return U


def field_stats(U):
    """[mean(4), 1/std(4)] over every cell of every frame (FP64)."""
    import torch
    flat = U.reshape(-1, 4)
    mean = flat.mean(dim=0)
    std = flat.std(dim=0).clamp_min(1e-12)
    return torch.cat([mean, 1.0 / std]).contiguous()


def correction_weights(U):
    """(rho, rho, rho, E) of each cell: the units of the network's corrections."""
    import torch
    return torch.stack([U[..., 0], U[..., 0], U[..., 0], U[..., 3]], dim=-1)


def residual_scale(U, coarse_solver, B, rng, pairs=4):
    """Per-field std of (next frame - coarse step of this frame) in the correction's units: the size of
    what the network must add, so that its raw output is O(1) (the reference scales its output by
    delta_std, models.py:65)."""
    import torch
    N, F = U.shape[:2]
    acc = []
    Uc = torch.empty((B,) + tuple(U.shape[2:]), dtype=torch.float64, device="cuda")
    for _ in range(pairs):
        i = torch.as_tensor(rng.integers(N, size=B), device="cuda")
        t = torch.as_tensor(rng.integers(F - 1, size=B), device="cuda")
        x = U[i, t].contiguous()
        coarse_solver.advance(x, DT_FRAME, Uc)
        acc.append(((U[i, t + 1] - Uc) / correction_weights(Uc)).reshape(-1, 4))
    return torch.cat(acc).std(dim=0).clamp_min(1e-12).contiguous()


class Trainer:
    def __init__(self, train, val, batch, unroll, seed=0, log=print, init=None):
        import torch
        self.torch = torch
        corr = importlib.import_module(f"{PKG}.correction")
        self.corr = corr
        self.train_U, self.val_U = train, val
        self.B, self.unroll = batch, unroll
        H, W = train.shape[2:4]
        self.rng = np.random.default_rng(seed)
        self.coarse = corr.CoarseSolver(batch, H, W)
        if init is None:
            self.net = corr.CorrectionNet(batch, H, W, seed=seed)
            self.stats = field_stats(train)
            self.dscale = residual_scale(train, self.coarse, batch, self.rng)
        else:  # fine-tuning (train.py --init): the checkpoint's parameters and its normalisation
            z = np.load(init)
            self.net = corr.CorrectionNet(batch, H, W, params=z["params"])
            self.stats = torch.from_numpy(z["stats"]).cuda()
            self.dscale = torch.from_numpy(z["dscale"]).cuda()
        shape = (batch, H, W, 4)
        self.x = torch.empty(shape, dtype=torch.float64, device="cuda")
        self.Uc = torch.empty_like(self.x)
        self.Un = torch.empty_like(self.x)
        self.fb = torch.zeros(batch, dtype=torch.int32, device="cuda")
        self.loss_part = torch.zeros(batch, dtype=torch.float64, device="cuda")
        self.ok = torch.ones(batch, dtype=torch.float64, device="cuda")
        self.coarse_failures = 0
        self.mode = "scale"  # positivity rule of the self-fed and evaluation steps
        self.noise = 0.0     # relative input noise of the trained step (set by train())
        log(f"stats mean {self.stats[:4].tolist()} std {(1 / self.stats[4:]).tolist()}; "
            f"residual scale {self.dscale.tolist()}")

    def _pairs(self, U, k):
        N, F = U.shape[:2]
        i = self.torch.as_tensor(self.rng.integers(N, size=self.B), device="cuda")
        t = self.torch.as_tensor(self.rng.integers(F - k, size=self.B), device="cuda")
        return U[i, t].contiguous(), U[i, t + k].contiguous()

    def step(self, lr, unroll=None):
        """One pushforward training step; returns the loss tensor (not synchronised)."""
        unroll = unroll or self.unroll
        x, y = self._pairs(self.train_U, unroll)
        self.x.copy_(x)
        ok = np.ones(self.B, bool)  # samples whose coarse steps all reached the frame time
        for _ in range(unroll - 1):  # self-fed steps, no gradient
            _, status = self.corr.hybrid_step(self.net, self.coarse, self.x, DT_FRAME, self.stats, self.dscale, self.Uc,
                                              self.Un, self.fb, mode=self.mode)
            ok &= status == 0
            self.x.copy_(self.Un)
        if self.noise > 0.0:
            self.perturb(self.x, self.noise)
        # the trained step keeps its full correction even where it is non-physical: the loss then pulls
        # it toward the (physical) target instead of the sample dropping out of the gradient
        _, status = self.corr.hybrid_step(self.net, self.coarse, self.x, DT_FRAME, self.stats, self.dscale, self.Uc,
                                          self.Un, self.fb, mode="keep")
        ok &= status == 0
        # a sample whose coarse solve stopped early (a self-fed state the solver cannot advance) has no
        # state at the target time: it gets no gradient (theta 0)
        self.coarse_failures += int((~ok).sum())
        self.ok.copy_(self.torch.from_numpy(ok.astype(np.float64)))
        self.net.loss_grad(self.Un, y, self.Uc, self.stats, self.dscale, None if ok.all() else self.ok, self.loss_part)
        self.net.backward()
        self.net.adamw(lr)
        return self.loss_part.sum() / (self.B * self.Un[0].numel())

    def perturb(self, x, sigma):
        """Noise injection (in place): the input frame of a training pair gets relative noise of size
        sigma in rho and p and velocity noise of sigma times the local sound speed, in primitive
        variables so that the state stays physical; the target stays the clean next frame, so the
        network also learns to pull perturbed states back (a stand-in for its own rollout errors)."""
        torch = self.torch
        rho = x[..., 0]
        u, v = x[..., 1] / rho, x[..., 2] / rho
        p = (1.4 - 1.0) * (x[..., 3] - 0.5 * rho * (u * u + v * v))
        c = torch.sqrt(1.4 * p / rho)
        g = torch.randn_like(x)
        rho = rho * torch.exp(sigma * g[..., 0])
        p = p * torch.exp(sigma * g[..., 3])
        u = u + sigma * c * g[..., 1]
        v = v + sigma * c * g[..., 2]
        x[..., 0] = rho
        x[..., 1] = rho * u
        x[..., 2] = rho * v
        x[..., 3] = p / (1.4 - 1.0) + 0.5 * rho * (u * u + v * v)

    def evaluate(self, U, batches=4, k=1, mode=None):
        """Mean normalised MSE after k steps of (hybrid, coarse-only) on pairs drawn from U."""
        h, c = 0.0, 0.0
        inv = self.stats[4:]
        self.fallback_count = 0
        self.eval_failures = 0
        for _ in range(batches):
            x, y = self._pairs(U, k)
            xh = x.clone()
            xc = x.clone()
            ok = np.ones(self.B, bool)
            for _ in range(k):
                _, status = self.corr.hybrid_step(self.net, self.coarse, xh, DT_FRAME, self.stats, self.dscale, self.Uc,
                                                  self.Un, self.fb, mode=mode or self.mode)
                ok &= status == 0
                self.fallback_count += int(self.fb.sum())
                xh.copy_(self.Un)
                self.coarse.advance(xc, DT_FRAME, self.Uc)
                xc.copy_(self.Uc)
            self.eval_failures += int((~ok).sum())
            keep = self.torch.from_numpy(ok).cuda()
            if keep.any():  # samples whose hybrid coarse solve stopped early are counted, not scored
                h += float((((xh[keep] - y[keep]) * inv) ** 2).mean())
                c += float((((xc[keep] - y[keep]) * inv) ** 2).mean())
        return h / batches, c / batches


def update_lr(step, cfg):
    """Learning rate of the step-th update (1-based).  optax evaluates its schedule at the number of
    updates already applied, so update k uses schedule(k - 1): the first update has the warm-up's
    initial value 0 (train.py:209-211, optax.warmup_cosine_decay_schedule)."""
    corr = importlib.import_module(f"{PKG}.correction")
    return corr.cosine_lr(step - 1, cfg["steps"], cfg["lr"], min(cfg["warmup"], cfg["steps"] // 2))


def train(cfg, log=print):
    """cfg: dict (see main()).  Returns (trainer, history rows)."""
    import torch
    out = Path(cfg["out"]) if cfg.get("out") else None
    if out:
        out.mkdir(parents=True, exist_ok=True)
    t0 = time.time()
    if cfg.get("packed"):  # the generate.py -> dataset.py pipeline's packs: train and val splits
        dsm = importlib.import_module(f"{PKG}.dataset")
        train_U = dsm.PairDataset(cfg["packed"], "train", cfg["coarse"]).states()
        val_U = dsm.PairDataset(cfg["packed"], "val", cfg["coarse"]).states()
        log(f"dataset: packed {cfg['packed']}: train {tuple(train_U.shape[:2])}, val {tuple(val_U.shape[:2])} "
            f"(trajectories, frames) at {cfg['coarse']}^2")
    else:
        fams = tuple(cfg.get("families") or ("riemann", "blast"))
        train_U = build_dataset(cfg["n_traj"], cfg["fine"], cfg["coarse"], index0=0, families=fams, log=log)
        val_U = build_dataset(cfg["n_val"], cfg["fine"], cfg["coarse"], index0=100000, families=fams, log=log)
    tr = Trainer(train_U, val_U, cfg["batch"], cfg["unroll"], seed=cfg["seed"], log=log, init=cfg.get("init"))
    tr.noise = float(cfg.get("noise", 0.0))
    corr = tr.corr
    hist = []
    writer = None
    if out:
        (out / "config.json").write_text(json.dumps({**cfg, "params": corr.param_count(),
                                                      "stats": tr.stats.tolist(), "dscale": tr.dscale.tolist()},
                                                     indent=2))
        logf = open(out / "log.csv", "w", newline="")
        writer = csv.writer(logf)
        writer.writerow(["step", "train_loss", "val_hybrid", "val_coarse", "val_ratio", "lr", "elapsed_s",
                         "val_ratio_k"])
    best = np.inf
    running = []
    t_train = time.time()
    onestep_until = int(cfg.get("onestep_frac", 0.0) * cfg["steps"])
    for step in range(1, cfg["steps"] + 1):
        lr = update_lr(step, cfg)
        # curriculum: one-step training first, so that the self-fed steps of the pushforward start from
        # a model whose own rollouts are close to the data (the reference fine-tunes with --init); then
        # pushforward steps alternate with one-step steps, which keep the one-step map anchored
        pushforward = step > onestep_until and (step % 2 == 0 or not cfg.get("mix_onestep", True))
        running.append(tr.step(lr, unroll=None if pushforward else 1))
        if step % cfg["eval_every"] == 0 or step == cfg["steps"]:
            tl = float(torch.stack(running).mean())
            running = []
            vh, vc = tr.evaluate(val_U)
            # model selection on k-step rollouts (k = select_k) when asked: what a pushforward model is for
            k = int(cfg.get("select_k", 1))
            kh, kc = tr.evaluate(val_U, batches=2, k=k) if k > 1 else (vh, vc)
            row = [step, tl, vh, vc, vh / vc, lr, time.time() - t0, kh / kc]
            hist.append(row)
            log(f"{step:>6} train {tl:.3e} val hybrid {vh:.3e} coarse {vc:.3e} ratio {vh / vc:.3f} "
                f"{k}-step ratio {kh / kc:.3f} lr {lr:.2e} |g| {float(tr.net.norm):.2e} partial corrections "
                f"{tr.fallback_count}/{2 * k * tr.B} coarse failures: eval {tr.eval_failures}/{2 * tr.B} train "
                f"{tr.coarse_failures} {(time.time() - t_train) / step * 1e3:.2f} ms/step")
            if writer:
                writer.writerow(row)
                logf.flush()
            if out and kh / kc < best:
                best = kh / kc
                np.savez(out / "best.npz", params=tr.net.params.cpu().numpy(), stats=tr.stats.cpu().numpy(),
                         dscale=tr.dscale.cpu().numpy())
    tr.net.check_device_error()
    if out:
        np.savez(out / "last.npz", params=tr.net.params.cpu().numpy(), stats=tr.stats.cpu().numpy(),
                 dscale=tr.dscale.cpu().numpy())
        logf.close()
    return tr, hist


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default="runs/correction")
    ap.add_argument("--packed", default=None,
                    help="train on this packed directory (dataset.py output: its train and val splits at "
                         "--coarse) instead of solving --n-traj / --n-val trajectories at --fine")
    ap.add_argument("--n-traj", type=int, default=512)
    ap.add_argument("--n-val", type=int, default=32)
    ap.add_argument("--fine", type=int, default=512)
    ap.add_argument("--coarse", type=int, default=64)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--unroll", type=int, default=4)
    ap.add_argument("--onestep-frac", type=float, default=0.5,
                    help="fraction of the steps trained one-step before the pushforward unroll starts")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--warmup", type=int, default=500)
    ap.add_argument("--eval-every", type=int, default=500)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--init", default=None, help="start from this checkpoint (params, stats, dscale)")
    ap.add_argument("--noise", type=float, default=0.0,
                    help="relative noise injected into the trained step's input (0 = none)")
    ap.add_argument("--select-k", type=int, default=1,
                    help="keep as best.npz the model with the lowest k-step validation ratio (hybrid / coarse)")
    a = ap.parse_args()
    cfg = {k.replace("-", "_"): v for k, v in vars(a).items()}
    train(cfg)


if __name__ == "__main__":
    main()
