"""Benchmark of the FP64 finite-volume solver step on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 512]
                  [--build parity|tolerance] [--no-extras] [--mode trajectory|stage|correction]

Workload (one bench step): the blast + density-bubble problem at 512^2, FP64, periodic, run in
trajectory mode to t = 0.2 with 20 frames (+ frame 0) block-averaged to 128^2 and 64^2 float32,
once for each of the four flux x limiter combinations (HLLC/Rusanov x minmod/van Leer) -- four
trajectories per step, each from a fresh seeded initial condition.

Metric: FP64 cell-updates/s (nx * ny * solver steps / time), whole job.
 * value -- initial states already resident in HBM; frames written to device buffers.
 * e2e   -- the same through the C-ABI with host buffers: fv_set_primitive from host arrays and
            fv_run_trajectory into host frame buffers, copies inside the timed region.
Multi-GPU (torchrun): every rank runs its own trajectories (independent initial conditions, no
data-path collective), timing is the max over ranks: weak scaling.

On one GPU the line also carries three measured sub-objects (skipped with --no-extras):
 * tolerance -- the same workload with the tolerance build (libfv_tol.so), in a child process;
 * ensemble  -- the batched-ensemble workload: 256 trajectories of sizes {64,128,256,512}^2 to
                t = 0.25 in one fv_ensemble, against a loop of single-grid runs of the same members;
 * hybrid    -- coarse 64^2 solver + learned correction against the plain solver at 64^2-256^2, on a
                bounded sample of held-out initial conditions, L1 density error against a 1024^2 solve.

--impl reference times the reference's own CPU solver (oracle/_ref, its headers compiled with
OpenMP) on the host cores, on a bounded sample of the same workload per step.

--mode stage runs one 512^2 case and prints the stage kernels' mean launch times (the program the
stage-kernel ncu captures run); --mode correction times the correction network's convolutions.
"""
import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
PKG = "neural-pde-surrogate_b200"
METRIC = "FP64 cell-updates/s"
UNIT = "cell-updates/s"
COMBOS = [("hllc", "minmod"), ("hllc", "vanleer"), ("rusanov", "minmod"), ("rusanov", "vanleer")]
NOUT, T_END, SAVE = 20, 0.2, (128, 64)
STAGE_BYTES = {1: 64, 2: 96}  # algorithmic bytes per cell per stage launch (FP64 AoS, 32 B/state)


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


PROFILE_SUMMARIES = ("fv_stepper_kernel_blast512.md", "fv_stage_kernels_blast512.md")


def profiled(key):
    """A figure of the committed ncu summaries of the stepper and stage kernels ("key: value" line),
    or None."""
    for name in PROFILE_SUMMARIES:
        f = ROOT / "profiles" / name
        if not f.exists():
            continue
        for line in f.read_text().splitlines():
            if line.startswith(key + ":"):
                return float(line.split(":")[1])
    return None


def profiled_traffic():
    """Per-launch DRAM bytes of the stage-2 kernel from the committed ncu summary, or None."""
    return profiled("traffic_bytes_per_launch_stage2")


def fp64_roofline(n, ms, per="stage1"):
    """What binds the stage kernels instead of HBM: the FP64 flop rate of the HLLC + van Leer kernels,
    from their executed flops per cell (ncu count, committed summary) and their live mean device time
    `ms` -- per stage-1 launch (per="stage1", the per-stage kernels) or per step (per="step", the
    persistent stepper) -- against the measured FP64 peak.  None without the summary's figures."""
    key, kernel, pipe = {"stage1": ("fp64_flops_per_cell_stage1", "stage_kernel<stage 1> hllc+vanleer",
                                    "fp64_pipe_active_stage1"),
                         "step": ("fp64_flops_per_cell_step", "stepper_kernel hllc+vanleer (both stages)",
                                  "fp64_pipe_active_stepper")}[per]
    flops, peak = profiled(key), profiled("fp64_peak_tflops")
    if flops is None or peak is None or not ms > 0:
        return None
    achieved = flops * n * n / (ms / 1e3) / 1e12
    return {"kernel": kernel, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "flops_per_cell": flops, "peak_source": "measured (fv_fp64_peak, DFMA loop)",
            "pipe_active_ncu": profiled(pipe)}


def roofline_of(n, stage_ms, step_prof, peak, peak_kind):
    """The roofline object of the dominant kernel, from the live CUDA-event times of the timed region.
    fv_advance_to runs on the persistent stepper (one launch per batch of steps): its algorithmic
    bytes are 160 per cell-update (stage 1 reads U and writes U1, stage 2 reads U and U1 and writes U;
    32 B per FP64 state), divided by its mean device time per step.  With the per-stage kernels
    (FV_STEPPER=0) it is the larger stage launch and its own bytes (64 or 96 per cell)."""
    hv = COMBOS.index(("hllc", "vanleer"))
    launches = sum(x[2] for x in step_prof)
    if launches:
        steps = sum(x[1] for x in step_prof)
        ms = sum(x[0] * x[1] for x in step_prof) / max(steps, 1)
        achieved = 160.0 * n * n / (ms / 1e3) / 1e9
        traffic = profiled("traffic_bytes_per_step_stepper")
        return {"bound": "hbm", "kernel": "stepper_kernel (persistent; both RK stages, all steps of a launch)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_unit": "DRAM bytes per step (ncu)", "peak_source": peak_kind,
                "algorithmic_bytes_per_cell_update": 160, "mean_ms_per_step": ms,
                "steps_per_launch": steps / launches,
                "fp64_pipe_active_ncu": profiled("fp64_pipe_active_stepper"),
                "fp64": fp64_roofline(n, step_prof[hv][0], per="step")}
    timed_steps = sum(x[2] for x in stage_ms)
    ms1 = sum(x[0] * x[2] for x in stage_ms) / max(timed_steps, 1)
    ms2 = sum(x[1] * x[2] for x in stage_ms) / max(timed_steps, 1)
    stage = 2 if ms2 >= ms1 else 1
    dur = ms2 if stage == 2 else ms1
    achieved = STAGE_BYTES[stage] * n * n / (dur / 1e3) / 1e9 if dur > 0 else 0.0
    return {"bound": "hbm", "kernel": f"stage_kernel<stage {stage}>", "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "traffic": profiled_traffic(),
            "peak_source": peak_kind, "algorithmic_bytes_per_cell": STAGE_BYTES[stage],
            "mean_launch_ms": {"stage1": ms1, "stage2": ms2},
            "fp64_pipe_active_ncu": profiled("fp64_pipe_active_stage2"),
            "fp64": fp64_roofline(n, stage_ms[hv][0])}


def smi_id(local):
    """nvidia-smi's id of CUDA device `local`: nvidia-smi ignores CUDA_VISIBLE_DEVICES, so a masked
    process maps its ordinal through the mask (an index or a UUID, both accepted by --id)."""
    ids = [x.strip() for x in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if x.strip()]
    return ids[local] if local < len(ids) else str(local)


class Clocks:
    """Samples nvidia-smi during the timed region."""

    def __init__(self, local):
        self.index = smi_id(local)
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) == 7:
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:]))
                except ValueError:
                    pass
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, r in rows for k, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def make_ics(ic, n, count, seed0):
    out = []
    for k in range(count):
        rho, u, v, p, _, _ = ic.sample("blast", seed0 + k, n)
        out.append((rho, u, v, p))
    return out


def reduce_over_ranks(ms, cells, launches, device):
    """Whole-job figures of one timed region under torchrun: the slowest rank's time (MAX), and the
    cell-updates and kernel launches of all ranks (SUM).  Every rank calls it at the same point."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([cells, launches], device=device, dtype=torch.float64)
    dist.all_reduce(c)
    return float(t.item()), float(c[0].item()), int(c[1].item())


def bench_config(n, world, build="parity"):
    """The workload both arms report: the same keys and values for ours and the reference.  A run of
    the tolerance build says so (the default parity build is bit-identical to the reference)."""
    cfg = {"workload": f"blast+bubble {n}^2 FP64 periodic, t=0.2, 20 frames -> 128^2/64^2 f32, "
                       f"4 flux x limiter combos per step", "grid": n, "frames": NOUT,
           "combos": [f"{a}+{b}" for a, b in COMBOS], "parallelism": f"replicas x{world}",
           "l2": "GPU arm: 256 MB buffer written before every step (state 8.4 MB is L2-resident within a step)"}
    if build != "parity":
        cfg["build"] = "tolerance: FMA contraction, within 1e-12 relative per step and 1e-9 per run of the parity build"
    return cfg


def run_ours(args):
    import torch
    rank, world, local = env_rank()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    fv = importlib.import_module(PKG)
    from importlib import import_module
    ic = import_module(f"{PKG}.ic")
    solver_mod = import_module(f"{PKG}.solver")
    n = args.n
    nsteps = args.warmup + args.steps
    ics = make_ics(ic, n, nsteps, seed0=1000 * rank)
    stream = torch.cuda.Stream()
    grid = fv.make_grid(n, n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic")
    solvers = [fv.Solver(grid, f, l, 0.5, stream=stream.cuda_stream) for f, l in COMBOS]
    # device-resident inputs and outputs for `value`
    dev_U = [torch.from_numpy(ic.to_conserved(*x)).to(f"cuda:{local}") for x in ics]
    dev_out = {m: torch.empty((NOUT + 1, 4, m, m), dtype=torch.float32, device=f"cuda:{local}") for m in SAVE}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")  # > L2 (126 MB)
    # pinned host inputs for `e2e`; frames come back into pageable numpy arrays
    host_prim = [[torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in x] for x in ics]
    torch.cuda.synchronize()

    def device_step(k):
        """One bench step with resident inputs; returns cell-updates."""
        cells = 0
        with torch.cuda.stream(stream):  # the solvers' stream: device buffers need no cross-stream ordering
            flush.zero_()
            for s in solvers:
                s.set_state(dev_U[k])
                for fr in range(NOUT + 1):
                    if fr:
                        _, nst = s.advance_to(0.0 + (T_END - 0.0) * fr / NOUT)
                    for m in SAVE:
                        s.block_average(n // m, out=dev_out[m][fr])
                cells += n * n * s.time()[1]
        return cells

    def e2e_step(k):
        cells = 0
        with torch.cuda.stream(stream):
            flush.zero_()
        for s in solvers:
            s.set_primitive(*host_prim[k])
            _, _, steps = s.run_trajectory(T_END, 0.0, NOUT, SAVE)
            cells += n * n * steps
        return cells

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, profile=False):
        for k in range(args.warmup):
            fn(k)
        barrier()
        if profile:
            for s in solvers:
                solver_mod.profile(s, True)
        l0 = sum(solver_mod.launch_count(s) for s in solvers)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        cells = 0
        for k in range(args.warmup, nsteps):
            cells += fn(k)
        ev1.record(stream)
        barrier()
        ms = ev0.elapsed_time(ev1)
        launches = sum(solver_mod.launch_count(s) for s in solvers) - l0
        if world > 1:
            ms, cells, launches = reduce_over_ranks(ms, cells, launches, f"cuda:{local}")
        return ms, cells, launches

    with Clocks(local) as clk:
        ms, cells, launches = timed(device_step, profile=True)
        stage_ms = [solver_mod.profile_read(s) for s in solvers]
        step_prof = [solver_mod.profile_steps(s) for s in solvers]
        e2e_ms, e2e_cells, _ = timed(e2e_step)
    clocks = clk.summary()

    value = cells / (ms / 1e3)
    e2e = e2e_cells / (e2e_ms / 1e3)
    peak, peak_kind = measured_peaks()
    roofline = roofline_of(n, stage_ms, step_prof, peak, peak_kind)
    h2d = 4 * n * n * 8 * len(COMBOS)
    d2h = (NOUT + 1) * sum(4 * m * m * 4 for m in SAVE) * len(COMBOS)
    if rank != 0:
        _finish(world)
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded blast + bubble initial conditions)",
        "config": bench_config(n, world, args.build),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roofline,
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n, ics[0], budget_s=args.cpu_budget)
    if world == 1 and not args.no_extras:
        del solvers, dev_U, dev_out, flush
        torch.cuda.empty_cache()
        line["tolerance"] = _guarded(tolerance_leg, args)
        line["ensemble"] = _guarded(ensemble_leg, peak)
        line["hybrid"] = _guarded(hybrid_leg)
    print(json.dumps(line), flush=True)
    _finish(world)


def _guarded(fn, *a):
    """A sub-object's figures, or the error that stopped it (the main line is printed either way)."""
    try:
        return fn(*a)
    except Exception as e:  # noqa: BLE001 -- reported in the line, never silently dropped
        return {"error": f"{type(e).__name__}: {e}"[:500]}


def tolerance_leg(args):
    """The same workload and step count with the tolerance build, run in a child process (a process
    loads one of the two libraries)."""
    cmd = [sys.executable, str(ROOT / "bench.py"), "--build", "tolerance", "--steps", str(args.steps), "--warmup",
           str(args.warmup), "--n", str(args.n), "--no-cpu-baseline", "--no-extras"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(r.stderr.strip().splitlines()[-1] if r.stderr.strip() else f"exit {r.returncode}")
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    return {"value": d["value"], "unit": d["unit"], "ms_per_step": d["ms_per_step"], "e2e": d["e2e"]["value"],
            "gpu_launches": d["gpu_launches"],
            "roofline": {k: d["roofline"].get(k) for k in ("kernel", "achieved", "frac", "mean_ms_per_step",
                                                           "mean_launch_ms")},
            "fp64": d["roofline"].get("fp64"), "clocks": d.get("clocks"),
            "build": "libfv_tol.so: FMA contraction, Newton-Raphson division, face states without the "
                     "conserved/primitive round trip; within 1e-12 relative per step and 1e-9 per run of the "
                     "reference (tests/test_gpu_tolerance.py)"}


def ensemble_leg(peak, count=256, t_end=0.25, flux="hllc", limiter="vanleer"):
    """The batched-ensemble workload: `count` periodic trajectories (alternately four-quadrant Riemann
    and blast + bubble, sizes drawn from {64, 128, 256, 512}^2, ic.ensemble_spec) each to t_end with
    its own CFL dt, in one fv_ensemble; and the same members one after another through single-grid
    handles.  Initial states are resident in HBM for both arms; CUDA events on the solvers' stream."""
    import torch
    fv = importlib.import_module(PKG)
    ic = importlib.import_module(f"{PKG}.ic")
    Ensemble = importlib.import_module(f"{PKG}.ensemble").Ensemble
    spec = ic.ensemble_spec(count)
    dev_U = [torch.from_numpy(ic.to_conserved(*ic.sample(fam, idx, n)[:4])).cuda() for fam, idx, n in spec]
    grids = [fv.make_grid(n, n, 0, 1, 0, 1, "periodic", "periodic") for _, _, n in spec]
    stream = torch.cuda.Stream()
    ens = Ensemble(grids, flux, limiter, stream=stream.cuda_stream)
    sizes = sorted({n for _, _, n in spec})
    handles = {n: fv.Solver(fv.make_grid(n, n, 0, 1, 0, 1, "periodic", "periodic"), flux, limiter, 0.5,
                            stream=stream.cuda_stream) for n in sizes}
    for k, U in enumerate(dev_U):  # warm-up: kernel loading, autotuning, graph capture
        ens.set_state(k, U)
    ens.advance_to(1e-4)
    for n, s in handles.items():
        s.set_state(dev_U[[x[2] for x in spec].index(n)])
        s.advance_to(1e-4)
    for k, U in enumerate(dev_U):
        ens.set_state(k, U)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ens.launch_count()
    e0.record(stream)
    t, steps, status = ens.advance_to(t_end)
    e1.record(stream)
    torch.cuda.synchronize()
    ens_ms = e0.elapsed_time(e1)
    launches = ens.launch_count() - l0
    cells = float(sum(g.nx * g.ny * int(st) for g, st in zip(grids, steps)))
    loop_steps = []
    e0.record(stream)
    for k, (_, _, n) in enumerate(spec):
        s = handles[n]
        s.set_state(dev_U[k])
        loop_steps.append(s.advance_to(t_end)[1])
    e1.record(stream)
    torch.cuda.synchronize()
    loop_ms = e0.elapsed_time(e1)
    if [int(x) for x in steps] != [int(x) for x in loop_steps]:
        raise RuntimeError("ensemble and single-grid step counts differ")
    value = cells / (ens_ms / 1e3)
    achieved = 160.0 * value / 1e9
    return {"workload": f"{count} trajectories (Riemann/blast alternating), sizes {sizes}^2 periodic, "
                        f"{flux}+{limiter}, CFL 0.5, each to t={t_end} with its own dt",
            "value": value, "unit": UNIT, "ms": ens_ms, "cell_updates": cells, "gpu_launches": launches,
            "all_status_ok": bool((status == 0).all()),
            "per_instance_loop": {"value": cells / (loop_ms / 1e3), "ms": loop_ms},
            "speedup_vs_loop": loop_ms / ens_ms,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "algorithmic_bytes_per_cell_update": 160,
                         "note": "members' states (0.7 GB per array) stream from HBM"}}


def hybrid_leg(n_riemann=6, n_blast=6, n_kh=4, batch=128, frames=100, truth_n=1024, coarse=64, plain=(64, 128, 256),
               gain=0.75):
    """Hybrid (coarse 64^2 FP64 solve + the shipped correction, scale mode at its evaluated gain)
    against the plain solver at each resolution in `plain`, all started from the truth's first frame
    and rolled out `frames` frame intervals of 0.005; L1 density error against a truth_n^2 FP64 solve,
    compared on the 64^2 grid (pareto.py).  Every method advances and is timed on a batch of `batch`
    held-out trajectories: the evaluated ones and more Riemann/blast initial conditions (indices
    300000+, first frames block-averaged from their initial states); errors are those of the
    evaluated ones.  The equal-error comparison at each horizon: the coarsest plain resolution at least as
    accurate as the hybrid, and their GPU times per trajectory."""
    import torch
    pareto = importlib.import_module(f"{PKG}.pareto")
    items = pareto.test_set(n_riemann, n_blast, n_kh)
    fams = [f for f, _ in items]
    model = ROOT / PKG / "checkpoints" / "correction_64.npz"
    sizes = sorted(set(plain) | {coarse})
    t0 = time.perf_counter()
    truth, first = pareto.truth_frames(items, truth_n, coarse, frames, sizes, log=lambda *a: None)
    truth_s = time.perf_counter() - t0
    extra = [("riemann" if k % 2 == 0 else "blast", 300000 + k // 2) for k in range(batch - len(items))]
    if extra:
        more = pareto.initial_frames(extra, max(sizes), sizes)
        first = {m: torch.cat([first[m], more[m]]).contiguous() for m in sizes}
    pareto.run_hybrid(model, first[coarse], coarse, 2, truth, "scale", gain, fams)  # warm-up
    hyb = pareto.run_hybrid(model, first[coarse], coarse, frames, truth, "scale", gain, fams)
    plains = [pareto.run_plain(first[n], n, coarse, frames, truth, fams) for n in plain]
    horizons = sorted({h for h in (5, 10, 20, 40, frames) if h <= frames})
    eq = pareto.equal_error(hyb, plains, horizons)
    keep = ("L1_final", "L1_mean", "L1_final_by_family", "ms_per_traj", "drift_mass", "drift_energy",
            "substeps_mean_per_frame", "substeps_of_slowest_per_frame_mean", "substeps_max_per_frame")
    wins = {h: bool(r["plain_n"] and r["plain_n"] > coarse and r["speedup"] > 1.0) for h, r in eq.items()}
    return {"sample": f"errors: {n_riemann} Riemann + {n_blast} blast + {n_kh} Kelvin-Helmholtz held-out initial "
                      f"conditions (indices 200000+), {frames} frames of 0.005; times: per trajectory of a "
                      f"batch of {len(items) + len(extra)} advanced together (those and {len(extra)} more "
                      f"Riemann/blast, indices 300000+)",
            "truth": f"{truth_n}^2 FP64 plain solve, HLLC + van Leer ({truth_s:.0f} s, outside every timed figure)",
            "hybrid": {"method": f"{coarse}^2 + correction_64.npz, scale mode (signal speed at most "
                                 f"{importlib.import_module(f'{PKG}.correction').MAX_SPEED_RATIO:g}x the coarse "
                                 f"state's), gain {gain}",
                       **{k: hyb[k] for k in keep}, "fallback_steps": hyb["fallback_steps"],
                       "coarse_retries": hyb["coarse_retries"], "failed": hyb["failed"]},
            "plain": {str(r["n"]): {k: r[k] for k in keep} for r in plains},
            "equal_error": {str(h): r for h, r in eq.items()},
            "hybrid_cheaper_at_equal_error": {str(h): w for h, w in wins.items()}}


def _finish(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _cpu_solver(n):
    """The reference CPU solver (oracle/_ref) when built, else the C restatement of it."""
    from oracle import build_oracle
    from oracle import oracle as orc
    build_oracle.build_oracle()
    if orc.ref_available():
        return orc.RefSolver, "reference"
    return orc.OracleSolver, "port"


def cpu_baseline(n, prim, budget_s=12.0, flux="hllc", limiter="vanleer"):
    """Times the reference CPU solver on the host cores on a bounded sample of the workload."""
    ic = importlib.import_module(f"{PKG}.ic")
    cls, kind = _cpu_solver(n)
    s = cls(n, n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic", flux, limiter, 0.5)
    s.set_state(ic.to_conserved(*prim))
    t0 = time.perf_counter()
    steps = 0
    while True:
        dt = s.compute_dt()
        s.step(dt)
        steps += 1
        if time.perf_counter() - t0 > budget_s and steps >= 3:
            break
    secs = time.perf_counter() - t0
    return {"value": n * n * steps / secs, "unit": UNIT, "cores": s.max_threads(), "kind": kind,
            "sample": f"{steps} SSP-RK2 steps of the {n}^2 blast problem, {flux}+{limiter}, from t=0 "
                      f"({secs:.1f} s on {s.max_threads()} OpenMP threads)"}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return  # the CPU reference runs once, on rank 0
    ic = importlib.import_module(f"{PKG}.ic")
    n = args.n
    cls, kind = _cpu_solver(n)
    per_combo = args.ref_solver_steps
    ics = make_ics(ic, n, args.warmup + args.steps, seed0=0)
    solvers = [cls(n, n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic", f, l, 0.5) for f, l in COMBOS]

    def step(k):
        cells = 0
        U0 = ic.to_conserved(*ics[k])
        for s in solvers:
            s.set_state(U0)
            s.t, s.steps = 0.0, 0
            for _ in range(per_combo):  # the driver loop, bounded: first solver steps of the trajectory
                dt = min(s.compute_dt(), T_END - s.t)
                s.step(dt)
                s.t += dt
                cells += n * n
        return cells

    for k in range(args.warmup):
        step(k)
    t0 = time.perf_counter()
    cells = 0
    for k in range(args.warmup, args.warmup + args.steps):
        cells += step(k)
    secs = time.perf_counter() - t0
    value = cells / secs
    cores = solvers[0].max_threads()
    sample = (f"per step: the first {per_combo} solver steps of each of the 4 flux x limiter trajectories "
              f"of the {n}^2 blast problem")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded blast + bubble initial conditions)",
        "config": bench_config(n, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_stage_case(args):
    """One solver case on the GPU with the stage kernels' mean launch times (the counterpart of the
    reference driver's --profile table, solver2d.hpp:29-52): the program ncu captures of the stage
    kernels run.  compute_dt + step per step, as the reference's loop."""
    fv = importlib.import_module(PKG)
    ic = importlib.import_module(f"{PKG}.ic")
    solver = importlib.import_module(f"{PKG}.solver")
    rho, u, v, p, _, _ = ic.sample(args.family, args.index, args.n)
    s = fv.Solver(fv.make_grid(args.n, args.n, 0, 1, 0, 1, "periodic", "periodic"), args.flux, args.limiter, 0.5)
    s.set_primitive(rho, u, v, p)
    solver.profile(s, True)
    for _ in range(args.steps):  # the reference's loop shape: compute_dt + step (per-stage kernels)
        s.step(dt=s.compute_dt())
    s.synchronize()
    ms1, ms2, k = solver.profile_read(s)
    solver.profile(s, True)
    s.advance_to(_horizon(s, args.steps))  # the device loop (fv_advance_to): the persistent stepper
    ms_step, k2, launches = solver.profile_steps(s)
    cells = args.n * args.n
    print(json.dumps({"mode": "stage", "case": f"{args.family}[{args.index}] {args.n}^2 {args.flux}+{args.limiter}",
                      "steps": k, "stage1_us": ms1 * 1e3, "stage2_us": ms2 * 1e3,
                      "per_stage_cell_updates_per_s": cells / ((ms1 + ms2) / 1e3),
                      "stepper_steps": k2, "stepper_launches": launches, "stepper_us_per_step": ms_step * 1e3,
                      "stepper_cell_updates_per_s": cells / (ms_step / 1e3) if ms_step > 0 else None,
                      "stepper_tile": solver.stepper_tile(s), "stepper_launch": solver.stepper_launch(s),
                      "build": os.environ.get("FV_BUILD", "parity")}),
          flush=True)


def _horizon(s, steps):
    """A target time about `steps` CFL steps ahead of the solver's current state."""
    t, _ = s.time()
    return t + steps * s.compute_dt()


def run_correction_case(args):
    """Forward and backward of the correction network on a batch of coarse states (the training
    configuration: batch 64 at 64^2), timed with CUDA events; achieved BF16 tensor throughput."""
    import torch
    corr = importlib.import_module(f"{PKG}.correction")
    ic = importlib.import_module(f"{PKG}.ic")
    B, n = args.batch, args.n
    rng = np.random.default_rng(0)
    net = corr.CorrectionNet(B, n, n, params=rng.normal(0, 0.05, corr.param_count()).astype(np.float32))
    U = torch.stack([torch.from_numpy(ic.to_conserved(*ic.sample("riemann", k, n)[:4])) for k in range(B)]).cuda()
    stats = torch.tensor([1.0, 0.0, 0.0, 2.5, 1.0, 1.0, 1.0, 0.3], dtype=torch.float64, device="cuda")
    net.forward(U, stats)
    net.dout16.copy_(torch.randn_like(net.dout16, dtype=torch.float32).to(torch.bfloat16) * 1e-3)
    net.backward()
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    for _ in range(args.steps):
        net.forward(U, stats)
    e[1].record()
    for _ in range(args.steps):
        net.backward()
    e[2].record()
    torch.cuda.synchronize()
    net.check_device_error()
    fwd, bwd = e[0].elapsed_time(e[1]) / args.steps, e[1].elapsed_time(e[2]) / args.steps
    macs = sum(B * n * n * co * ci * 9 for ci, co, _, _ in corr.LAYERS)
    print(json.dumps({"mode": "correction", "batch": B, "n": n, "forward_us": fwd * 1e3, "backward_us": bwd * 1e3,
                      "forward_tflops": 2 * macs / (fwd * 1e-3) / 1e12,
                      "backward_tflops": 4 * macs / (bwd * 1e-3) / 1e12}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU work for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-solver-steps", type=int, default=20)
    ap.add_argument("--build", choices=["parity", "tolerance"], default="parity",
                    help="solver library: the bit-exact parity build, or the FMA-contracted tolerance build")
    ap.add_argument("--no-extras", action="store_true", help="skip the tolerance, ensemble and hybrid sub-objects")
    ap.add_argument("--mode", choices=["trajectory", "stage", "correction"], default="trajectory")
    ap.add_argument("--family", default="blast", help="--mode stage: initial-condition family")
    ap.add_argument("--index", type=int, default=0, help="--mode stage: initial-condition index")
    ap.add_argument("--flux", default="hllc", help="--mode stage")
    ap.add_argument("--limiter", default="vanleer", help="--mode stage")
    ap.add_argument("--batch", type=int, default=64, help="--mode correction")
    args = ap.parse_args()
    os.environ["FV_BUILD"] = args.build  # read when the solver library is first loaded
    if args.mode == "stage":
        run_stage_case(args)
    elif args.mode == "correction":
        if args.n == 512:
            args.n = 64
        run_correction_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
