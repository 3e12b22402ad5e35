"""Benchmark of the FP64 finite-volume solver step on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 512]

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

--impl reference times the reference's own CPU solver (oracle/_ref, its headers compiled with
OpenMP) on the host cores, on a bounded sample of the same workload per step.
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


def profiled(key):
    """A figure of the committed ncu summary of the stage kernels ("key: value" line), or None."""
    f = ROOT / "profiles" / "fv_stage_kernels_blast512.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(key + ":"):
            return float(line.split(":")[1])
    return None


def profiled_traffic():
    """Per-launch DRAM bytes of the stage-2 kernel from the committed ncu summary, or None."""
    return profiled("traffic_bytes_per_launch_stage2")


def fp64_roofline(n, stage1_ms):
    """What binds the stage kernels instead of HBM: FP64 flop rate of the HLLC + van Leer stage-1
    kernel, from its executed flops per cell (ncu count, committed summary) and its live mean launch
    time `stage1_ms`, against the measured FP64 peak.  None without the summary's figures."""
    flops, peak = profiled("fp64_flops_per_cell_stage1"), profiled("fp64_peak_tflops")
    if flops is None or peak is None or not stage1_ms > 0:
        return None
    achieved = flops * n * n / (stage1_ms / 1e3) / 1e12
    return {"kernel": "stage_kernel<stage 1> hllc+vanleer", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "flops_per_cell": flops, "peak_source": "measured (fv_fp64_peak, DFMA loop)",
            "pipe_active_ncu": profiled("fp64_pipe_active_stage1")}


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
        e2e_ms, e2e_cells, _ = timed(e2e_step)
    clocks = clk.summary()

    value = cells / (ms / 1e3)
    e2e = e2e_cells / (e2e_ms / 1e3)
    # roofline of the dominant kernel (the larger of the two stage kernels, averaged over combos)
    timed_steps = sum(x[2] for x in stage_ms)
    ms1 = sum(x[0] * x[2] for x in stage_ms) / max(timed_steps, 1)
    ms2 = sum(x[1] * x[2] for x in stage_ms) / max(timed_steps, 1)
    stage = 2 if ms2 >= ms1 else 1
    dur = ms2 if stage == 2 else ms1
    peak, peak_kind = measured_peaks()
    achieved = STAGE_BYTES[stage] * n * n / (dur / 1e3) / 1e9 if dur > 0 else 0.0
    traffic = profiled_traffic()
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
        "roofline": {"bound": "hbm", "kernel": f"stage_kernel<stage {stage}>", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": peak_kind, "algorithmic_bytes_per_cell": STAGE_BYTES[stage],
                     "mean_launch_ms": {"stage1": ms1, "stage2": ms2},
                     # what binds instead: the FP64 pipe (ncu share of active cycles, committed summary)
                     "fp64_pipe_active_ncu": profiled("fp64_pipe_active_stage2"),
                     "fp64": fp64_roofline(n, stage_ms[COMBOS.index(("hllc", "vanleer"))][0])},
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n, ics[0], budget_s=args.cpu_budget)
    print(json.dumps(line), flush=True)
    _finish(world)


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
    args = ap.parse_args()
    os.environ["FV_BUILD"] = args.build  # read when the solver library is first loaded
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
