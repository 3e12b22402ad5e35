"""Dataset generation with the GPU solver: (family, index) -> one trajectory, block-averaged.

The reference generator (data/generate.py:60-105) samples an initial condition, writes it as HDF5,
runs `euler2d --init ic.h5 --nout 50 --tstart T --traj traj.h5 --save 128,64` as a subprocess and
reads the HDF5 trajectory back.  Here the same steps are one in-process call through the C-ABI
(fv_set_primitive + fv_run_trajectory): no subprocess, no files, the frames stay in memory.

  python neural-pde-surrogate_b200/generate.py --family blast --indices 0-7 --n 512 --save 128,64 --out DIR
  torchrun --nproc-per-node 8 neural-pde-surrogate_b200/generate.py ...   (one GPU per rank)

Under torchrun every rank takes a cost-balanced share of the indices (shard.balanced_split) and runs
it on its own GPU; only the per-rank counts are gathered at the end (gloo, no data-path collective).

Output per trajectory: DIR/<family>/<index:06d>.npz with `t` (frames,) and `U_<m>` (frames, 4, m, m)
float32 conserved variables per save size, plus the run attributes the reference stores
(trajectory.hpp:74-89) and provenance (generate.py:87-97).  The file appears atomically
(os.replace), so an interrupted batch can simply be restarted: existing files are skipped.  A
trajectory that stops at a non-physical state leaves DIR/<family>/<index:06d>.failed.txt with the
solver's report instead, and the batch carries on.
"""
import argparse
import datetime
import importlib
import os
import platform
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

DT_FRAME = 0.005  # frame spacing shared by every family (the reference: 0.25 / 50)


def parse_indices(text):
    """'0-7' -> [0..7], '3' -> [3], '0-3,10' -> [0, 1, 2, 3, 10] (data/generate.py:36-45)."""
    out = []
    for part in text.split(","):
        if "-" in part:
            a, b = part.split("-")
            out.extend(range(int(a), int(b) + 1))
        else:
            out.append(int(part))
    return out


def trajectory(family, index, n, save, flux="hllc", limiter="vanleer", cfl=0.5, solver=None, dt_frame=DT_FRAME):
    """Runs one trajectory on the GPU.  Returns (t, {m: (frames, 4, m, m) float32}, steps, params).
    Frames are every dt_frame from t_start (0, or the family's spin-up time) to the family's t_end."""
    fv = importlib.import_module("neural-pde-surrogate_b200")
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    rho, u, v, p, t_end, params = ic.sample(family, index, n)
    t_start = float(params.get("t_start", 0.0))
    nout = int(round((t_end - t_start) / dt_frame))
    s = solver or fv.Solver(fv.make_grid(n, n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic"), flux, limiter, cfl)
    s.set_primitive(rho, u, v, p)
    t, levels, steps = s.run_trajectory(t_end, t_start, nout, save)
    return t, levels, steps, params


def generate_one(family, index, n, save, out_dir, force=False, solver=None):
    """One file; returns 'done', 'skipped' (the file exists) or 'failed' (details in
    <index>.failed.txt) -- data/generate.py:60-105 without the subprocess."""
    final = Path(out_dir) / family / f"{index:06d}.npz"
    if final.exists() and not force:
        return "skipped"
    final.parent.mkdir(parents=True, exist_ok=True)
    failed = final.with_suffix(".failed.txt")
    FVError = importlib.import_module("neural-pde-surrogate_b200").FVError
    t0 = time.time()
    try:
        t, levels, steps, params = trajectory(family, index, n, save, solver=solver)
    except FVError as e:
        # a non-physical state (or a rejected initial condition): logged beside the output, and the
        # batch goes on with the next index (data/generate.py:79-84); a restart retries it
        failed.write_text(f"{family} {index} at {n}x{n}, save {list(save)}: failed after "
                          f"{time.time() - t0:.1f} s\n{e}\n")
        return "failed"
    attrs = {"family": family, "index": index, "steps": steps, "solver_nx": n, "solver_ny": n, "gamma": 1.4, "cfl": 0.5,
             "scheme": "hllc", "limiter": "vanleer", "bc_x": "periodic", "bc_y": "periodic", "t_start": float(t[0]),
             "t_end": float(t[-1]), "frames": len(t), "variables": "rho, rho*u, rho*v, E",
             "generated_at": datetime.datetime.now().isoformat(timespec="seconds"), "host": platform.node(),
             "runtime_s": time.time() - t0}
    with tempfile.NamedTemporaryFile(dir=final.parent, suffix=".npz", delete=False) as tmp:
        np.savez(tmp, t=t, **{f"U_{m}": a for m, a in levels.items()},
                 **{f"param_{k}": np.asarray(v) for k, v in params.items() if k not in ("family", "index")},
                 **{f"attr_{k}": np.asarray(v) for k, v in attrs.items()})
    os.replace(tmp.name, final)  # the file appears only once complete
    if failed.exists():
        failed.unlink()  # an earlier attempt's log
    return "done"


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--family", required=True)
    ap.add_argument("--indices", required=True)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--save", default="128,64")
    ap.add_argument("--out", required=True)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    import torch
    shard = importlib.import_module("neural-pde-surrogate_b200.shard")
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("gloo", timeout=datetime.timedelta(minutes=30))
    fv = importlib.import_module("neural-pde-surrogate_b200")
    save = [int(s) for s in a.save.split(",")]
    solver = fv.Solver(fv.make_grid(a.n, a.n, 0.0, 1.0, 0.0, 1.0, "periodic", "periodic"), "hllc", "vanleer", 0.5)
    indices = parse_indices(a.indices)
    costs = []
    for i in indices:
        _, _, _, _, t_end, params = ic.sample(a.family, i, 8)
        costs.append(shard.trajectory_cost(a.n, t_end - float(params.get("t_start", 0.0))))
    t0 = time.time()
    status = shard.run_sharded(indices, lambda i: generate_one(a.family, i, a.n, save, a.out, a.force, solver),
                               costs=costs)
    if status is not None:
        print(f"Finished in {time.time() - t0:.1f} s: {status.count('done')} done, {status.count('skipped')} skipped, "
              f"{status.count('failed')} failed on {world} GPU(s)")
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
