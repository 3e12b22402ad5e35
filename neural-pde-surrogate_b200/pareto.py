"""Accuracy against cost: hybrid coarse solver + learned correction vs the plain GPU solver.

  python neural-pde-surrogate_b200/pareto.py --model runs/correction/best.npz [--truth 1024]
         [--frames 100] [--riemann 8] [--blast 8] [--kh 4] [--plain 64,128,256,512] [--out FILE]

Held-out initial conditions: Riemann and blast members with indices >= 200000 (training uses
0..n, validation 100000..) and Kelvin-Helmholtz members (ic.kh: tanh band, shear +-0.5, p = 2.5,
seeded sin(4 pi x) perturbation, recording from t_start ~ U(0, 1)).  The truth is a plain FP64 solve
at truth^2 from which frames are kept every 0.005 after t_start.  Every method starts from the truth's
first frame block-averaged to its own resolution (experiments/solver_baseline.py:80-147 starts the
coarse solver from the true frame 0 the same way) and runs `frames` frame intervals; its density is
block-averaged to the hybrid's coarse grid and compared there with the truth, also block-averaged
(L1 = sum |rho - rho_true| dA, convergence_sine2d.py:23-25).  Reported per method: L1 at the last
frame and its mean over frames, conservation drift of the totals (rollout.py:54-62), fallback count
(hybrid), and GPU time per trajectory (CUDA events around the batched solves; every method advances
all test trajectories together: an fv_ensemble per resolution, the hybrid batched the same way).
"""
import argparse
import importlib
import json
import sys
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
PKG = "neural-pde-surrogate_b200"
DT_FRAME = 0.005


def test_set(n_riemann, n_blast, n_kh):
    return ([("riemann", 200000 + k) for k in range(n_riemann)] + [("blast", 200000 + k) for k in range(n_blast)] +
            [("kh", 200000 + k) for k in range(n_kh)])


def block_avg(U, f):
    """(B, H, W, 4) -> (B, H/f, W/f, 4) mean over f x f blocks (evaluation only)."""
    B, H, W, C = U.shape
    return U.reshape(B, H // f, f, W // f, f, C).mean(dim=(2, 4))


def truth_frames(items, n, coarse, frames, sizes, log=print):
    """Fine solves.  Returns (coarse frames (B, F+1, c, c, 4) float64 CUDA, {m: first frame at m^2})."""
    import torch
    fv = importlib.import_module(PKG)
    ic = importlib.import_module(f"{PKG}.ic")
    s = fv.Solver(fv.make_grid(n, n, 0, 1, 0, 1, "periodic", "periodic"), "hllc", "vanleer", 0.5)
    out, first = [], {m: [] for m in sizes}
    U = torch.empty((1, n, n, 4), dtype=torch.float64, device="cuda")  # frames stay on the device
    t0 = time.time()
    for fam, idx in items:
        rho, u, v, p, _, params = ic.sample(fam, idx, n)
        t_start = float(params.get("t_start", 0.0))
        s.set_primitive(rho, u, v, p)
        s.advance_to(t_start)
        s.get_state(out=U[0])
        for m in sizes:
            first[m].append(block_avg(U, n // m)[0])
        traj = [block_avg(U, n // coarse)[0]]
        for k in range(1, frames + 1):
            s.advance_to(t_start + DT_FRAME * k)
            s.get_state(out=U[0])
            traj.append(block_avg(U, n // coarse)[0])
        out.append(torch.stack(traj))
    log(f"truth: {len(items)} trajectories at {n}^2, {frames} frames, {time.time() - t0:.1f} s")
    return torch.stack(out), {m: torch.stack(v).contiguous() for m, v in first.items()}


def initial_frames(items, n, sizes):
    """{m: (B, m, m, 4)} first frames of trajectories that start at t = 0 (Riemann, blast): their
    n^2 initial conditions block-averaged to each size m (no fine solve needed)."""
    import torch
    ic = importlib.import_module(f"{PKG}.ic")
    out = {m: [] for m in sizes}
    for fam, idx in items:
        rho, u, v, p, _, params = ic.sample(fam, idx, n)
        if float(params.get("t_start", 0.0)) != 0.0:
            raise ValueError(f"{fam} {idx} starts at t > 0: its first frame needs a fine solve")
        U = torch.from_numpy(ic.to_conserved(rho, u, v, p)).cuda()[None]
        for m in sizes:
            out[m].append(block_avg(U, n // m)[0])
    return {m: torch.stack(v).contiguous() for m, v in out.items()}


def l1_density(U, T):
    """sum |rho - rho_true| dA per sample on the unit box, U and T (B, c, c, 4)."""
    c = U.shape[1]
    return (U[..., 0] - T[..., 0]).abs().sum(dim=(1, 2)) / (c * c)


def by_family(L1, families):
    """{family: mean L1 at the last frame} for per-sample L1 (B, frames)."""
    if not families:
        return {}
    out = {}
    for fam in sorted(set(families)):
        idx = [k for k, f in enumerate(families) if f == fam]
        out[fam] = round(float(L1[idx, -1].mean()), 5)
    return out


def drift(U, U0):
    """(total - total0) / sum |U0| per sample and field (rollout.py:54-62)."""
    return (U.sum(dim=(1, 2)) - U0.sum(dim=(1, 2))) / U0.abs().sum(dim=(1, 2))


GAMMA = 1.4


def rollout_metrics(pred, true, std):
    """The reference's rollout metrics (surrogate/rollout.py:54-62) on the GPU, in this build's layout:
    pred, true (T, n, n, 4) conserved FP64 tensors, std (4,) per-field scales.  Returns
      rmse       (T, 4)  root mean square error over the grid, divided by std,
      drift      (T, 4)  total of pred minus the total of true[0], over the total ABSOLUTE amount of
                         true[0] (the reference's normalisation: net momentum can be ~0),
      bad_cells  (T,)    cells with rho <= 0 or not p > 0 (a NaN pressure counts as bad)."""
    rmse = ((pred - true) ** 2).mean(dim=(-3, -2)).sqrt() / std
    drift = (pred.sum(dim=(-3, -2)) - true[0].sum(dim=(-3, -2))) / true[0].abs().sum(dim=(-3, -2))
    rho = pred[..., 0]
    p = (GAMMA - 1) * (pred[..., 3] - 0.5 * (pred[..., 1] ** 2 + pred[..., 2] ** 2) / rho)
    bad = ((rho <= 0) | ~(p > 0)).sum(dim=(-2, -1))
    return {"rmse": rmse, "drift": drift, "bad_cells": bad}


def run_plain(first, n, coarse, frames, truth, families=None):
    """All test trajectories at n^2 in one fv_ensemble; errors on the coarse grid.  The batch `first`
    may hold more trajectories than `truth`: all are advanced and timed, the errors and drifts are
    those of the first truth.shape[0]."""
    import torch
    fv = importlib.import_module(PKG)
    Ensemble = importlib.import_module(f"{PKG}.ensemble").Ensemble
    B = first.shape[0]
    g = fv.make_grid(n, n, 0, 1, 0, 1, "periodic", "periodic")
    ens = Ensemble([g] * B, "hllc", "vanleer")
    U = torch.empty_like(first)
    ens.set_all(first)
    ens.advance_to(1e-9, raise_on_nonphysical=False)  # first-launch costs out of the timed region
    ens.set_all(first)
    torch.cuda.synchronize()
    l1, ms = [], 0.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    status = np.zeros(B, np.int32)
    prev, substeps = np.zeros(B, np.int64), []
    for k in range(1, frames + 1):
        e0.record()
        _, steps, st = ens.advance_to(DT_FRAME * k, raise_on_nonphysical=False)
        e1.record()
        substeps.append((int((steps - prev).max()), float((steps - prev).mean())))
        prev = steps
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        status |= st
        ens.get_all(U)
        l1.append(l1_density(block_avg(U[:truth.shape[0]], n // coarse), truth[:, k]))
    L1 = torch.stack(l1, dim=1)
    return {"method": "plain", "n": n, "L1_final": float(L1[:, -1].mean()), "L1_mean": float(L1.mean()),
            "L1_final_by_family": by_family(L1, families),
            "L1_per_frame": [round(float(v), 5) for v in L1.mean(dim=0)],
            "ms_per_traj": ms / B, "drift_mass": float(drift(U, first)[:, 0].abs().max()),
            "drift_energy": float(drift(U, first)[:, 3].abs().max()), "failed": int((status != 0).sum()),
            "substeps_max_per_frame": max(m for m, _ in substeps),
            "substeps_mean_per_frame": float(np.mean([a for _, a in substeps])),
            "substeps_of_slowest_per_frame_mean": float(np.mean([m for m, _ in substeps]))}


def run_hybrid(model, first, coarse, frames, truth, mode="scale", gain=1.0, families=None):
    """mode: positivity rule of the correction ('strict': a step that would go non-physical is the plain
    coarse step; 'scale': the largest physical fraction of the correction).  gain: a fixed factor on
    every correction (1 = as trained).  As in run_plain, errors are those of the first
    truth.shape[0] trajectories of the (timed) batch."""
    import torch
    corr = importlib.import_module(f"{PKG}.correction")
    z = np.load(model)
    B = first.shape[0]
    net = corr.CorrectionNet(B, coarse, coarse, params=z["params"])
    stats = torch.from_numpy(z["stats"]).cuda()
    dscale = torch.from_numpy(z["dscale"]).cuda() * gain
    cs = corr.CoarseSolver(B, coarse, coarse)
    x = first.clone()
    Uc, Un = torch.empty_like(x), torch.empty_like(x)
    Uc_prev, Uc2 = first.clone(), torch.empty_like(x)
    fb = torch.zeros(B, dtype=torch.int32, device="cuda")
    corr.hybrid_step(net, cs, x.clone(), 1e-9, stats, dscale, Uc, Un, fb, mode)  # warm-up (kernel loading)
    torch.cuda.synchronize()
    l1, ms, fallbacks, theta, retried, failed = [], 0.0, 0, [], 0, 0
    substeps = []  # per frame: the coarse CFL sub-steps of the slowest and of the mean trajectory
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in range(1, frames + 1):
        e0.record()
        steps, status = corr.hybrid_step(net, cs, x, DT_FRAME, stats, dscale, Uc, Un, fb, mode)
        substeps.append((int(np.max(steps)), float(np.mean(steps))))
        bad = np.nonzero(status)[0]
        if len(bad):
            # the coarse solver cannot advance these corrected states: drop the previous frame's
            # correction (restart from its uncorrected coarse state) and take a plain coarse step
            retried += len(bad)
            idx = torch.as_tensor(bad, device="cuda")
            x2 = x.clone()
            x2[idx] = Uc_prev[idx]
            _, st2 = cs.advance(x2, DT_FRAME, Uc2)
            Uc[idx] = Uc2[idx]
            Un[idx] = Uc2[idx]
            failed += int((st2[bad] != 0).sum())
        Uc_prev.copy_(Uc)
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        fallbacks += int(fb.sum())
        theta.append(float(net.theta.mean()))
        x.copy_(Un)
        l1.append(l1_density(x[:truth.shape[0]], truth[:, k]))
    L1 = torch.stack(l1, dim=1)
    return {"method": f"hybrid-{mode}" + (f"-g{gain:g}" if gain != 1.0 else ""), "n": coarse, "gain": gain,
            "L1_final_by_family": by_family(L1, families), "L1_final": float(L1[:, -1].mean()), "L1_mean": float(L1.mean()),
            "L1_per_frame": [round(float(v), 5) for v in L1.mean(dim=0)], "mean_theta": float(np.mean(theta)),
            "ms_per_traj": ms / B, "drift_mass": float(drift(x, first)[:, 0].abs().max()),
            "drift_energy": float(drift(x, first)[:, 3].abs().max()), "fallback_steps": fallbacks,
            "coarse_retries": retried, "failed": failed,
            "substeps_max_per_frame": max(m for m, _ in substeps),
            "substeps_mean_per_frame": float(np.mean([a for _, a in substeps])),
            "substeps_of_slowest_per_frame_mean": float(np.mean([m for m, _ in substeps]))}


def equal_error(hyb, plains, horizons):
    """The equal-error comparison at each horizon h (frames): the coarsest plain resolution whose L1
    density error at frame h is at most the hybrid's, and the ratio of their GPU times per trajectory
    (> 1: the hybrid is cheaper).  plain_n is None where no plain resolution is as accurate."""
    per = {}
    for h in horizons:
        e = hyb["L1_per_frame"][h - 1]
        as_good = [r for r in plains if r["L1_per_frame"][h - 1] <= e]
        if as_good:
            best = min(as_good, key=lambda r: r["n"])
            per[h] = {"hybrid_L1": e, "plain_n": best["n"], "plain_L1": best["L1_per_frame"][h - 1],
                      "plain_ms": best["ms_per_traj"], "hybrid_ms": hyb["ms_per_traj"],
                      "speedup": best["ms_per_traj"] / hyb["ms_per_traj"]}
        else:
            per[h] = {"hybrid_L1": e, "plain_n": None}
    return per


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--model", required=True)
    ap.add_argument("--coarse", type=int, default=64)
    ap.add_argument("--truth", type=int, default=1024)
    ap.add_argument("--frames", type=int, default=100)
    ap.add_argument("--riemann", type=int, default=8)
    ap.add_argument("--blast", type=int, default=8)
    ap.add_argument("--kh", type=int, default=4)
    ap.add_argument("--plain", default="64,128,256,512")
    ap.add_argument("--out", default=None)
    ap.add_argument("--gains", default="1", help="comma-separated correction gains to evaluate (scale mode)")
    a = ap.parse_args()
    plain = [int(x) for x in a.plain.split(",")]
    items = test_set(a.riemann, a.blast, a.kh)
    truth, first = truth_frames(items, a.truth, a.coarse, a.frames, sorted(set(plain + [a.coarse])))
    gains = [float(g) for g in a.gains.split(",")]
    fams = [f for f, _ in items]
    # untimed warm-up of the whole hybrid pipeline (module loading, graph capture, clocks): the first
    # timed method must not pay one-time costs the others do not
    run_hybrid(a.model, first[a.coarse], a.coarse, min(2, a.frames), truth, "scale", 1.0, fams)
    hybrids = [run_hybrid(a.model, first[a.coarse], a.coarse, a.frames, truth, "scale", g, fams) for g in gains]
    hybrids.append(run_hybrid(a.model, first[a.coarse], a.coarse, a.frames, truth, "strict", families=fams))
    plains = [run_plain(first[n], n, a.coarse, a.frames, truth, fams) for n in plain]
    rows = hybrids + plains
    summary = {"test_set": {"riemann": a.riemann, "blast": a.blast, "kh": a.kh}, "truth": a.truth, "frames": a.frames,
               "rows": rows, "equal_error": {}}
    # equal error at several horizons: the coarsest plain resolution whose L1 at frame h is at most the
    # hybrid's, and the cost ratio (frame costs are near constant, so whole-run times compare)
    horizons = sorted({h for h in (5, 10, 20, a.frames) if h <= a.frames})
    summary["horizons"] = horizons
    for hyb in hybrids:
        summary["equal_error"][hyb["method"]] = equal_error(hyb, plains, horizons)
    print(f"{'method':18s} {'n':>5s} {'L1 final':>10s} {'L1 mean':>10s} {'ms/traj':>9s} {'drift m':>9s} {'drift E':>9s}"
          f" {'partial':>8s} {'retries':>7s}  L1 final by family")
    for r in rows:
        print(f"{r['method']:18s} {r['n']:5d} {r['L1_final']:10.3e} {r['L1_mean']:10.3e} {r['ms_per_traj']:9.2f} "
              f"{r['drift_mass']:9.1e} {r['drift_energy']:9.1e} {r.get('fallback_steps', r.get('failed', 0)):8d} "
              f"{r.get('coarse_retries', 0):7d}  {r['L1_final_by_family']}")
    for m, per in summary["equal_error"].items():
        cells = []
        for h, r in per.items():
            cells.append(f"{h}: " + (f"plain {r['plain_n']} x{r['speedup']:.2f}" if r["plain_n"] else "none"))
        print(f"equal error {m:18s} " + "; ".join(cells))
    print(json.dumps(summary))
    if a.out:
        Path(a.out).write_text(json.dumps(summary, indent=2))


if __name__ == "__main__":
    main()
