"""Batched-ensemble throughput against a per-instance launch loop.

  python neural-pde-surrogate_b200/ensemble_bench.py [--count 256] [--t-end 0.25] [--check 8]

Workload: `count` FP64 trajectories, half four-quadrant Riemann and half blast + bubble initial
conditions (the seeded families of ic.py), grid sizes drawn uniformly from {64^2, 128^2, 256^2,
512^2}, periodic, HLLC + van Leer, CFL 0.5, each to t_end with its own CFL dt.
 * ensemble -- one fv_ensemble: persistent stage launches over all running members, graph batches.
 * loop     -- the same trajectories one after another, each through a single-grid handle
              (fv_advance_to), the way one driver process per trajectory would run them.
Both use device-resident initial states; time is measured with CUDA events around each arm.  A few
members (--check) are compared bit for bit between the arms.  Prints one JSON line.
"""
import argparse
import importlib
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--t-end", type=float, default=0.25)
    ap.add_argument("--sizes", default="64,128,256,512")
    ap.add_argument("--check", type=int, default=8)
    ap.add_argument("--seed", type=int, default=2026)
    a = ap.parse_args()
    import torch
    fv = importlib.import_module("neural-pde-surrogate_b200")
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    Ensemble = importlib.import_module("neural-pde-surrogate_b200.ensemble").Ensemble
    sizes = [int(s) for s in a.sizes.split(",")]
    rng = np.random.default_rng(a.seed)
    spec = []
    for k in range(a.count):
        n = sizes[int(rng.integers(len(sizes)))]
        fam = "riemann" if k % 2 == 0 else "blast"
        spec.append((fam, k // 2, n))
    dev_U = []
    for fam, idx, n in spec:
        rho, u, v, p, _, _ = ic.sample(fam, idx, n)
        dev_U.append(torch.from_numpy(ic.to_conserved(rho, u, v, p)).cuda())
    grids = [fv.make_grid(n, n, 0, 1, 0, 1, "periodic", "periodic") for _, _, n in spec]
    stream = torch.cuda.Stream()

    # warm-up both arms (autotuning, graph capture, first-launch costs) on a short horizon
    ens = Ensemble(grids, "hllc", "vanleer", stream=stream.cuda_stream)
    for k, U in enumerate(dev_U):
        ens.set_state(k, U)
    ens.advance_to(1e-4)
    handles = {n: fv.Solver(fv.make_grid(n, n, 0, 1, 0, 1, "periodic", "periodic"), "hllc", "vanleer", 0.5,
                            stream=stream.cuda_stream) for n in sizes}
    for n, s in handles.items():
        s.set_state(dev_U[[x[2] for x in spec].index(n)] if n in [x[2] for x in spec] else
                    torch.zeros((n, n, 4), dtype=torch.float64, device="cuda") + 1.0)
        s.advance_to(1e-4)
    torch.cuda.synchronize()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # ensemble arm
    for k, U in enumerate(dev_U):
        ens.set_state(k, U)
    torch.cuda.synchronize()
    e0.record(stream)
    t, steps, status = ens.advance_to(a.t_end)
    e1.record(stream)
    torch.cuda.synchronize()
    ens_ms = e0.elapsed_time(e1)
    cells = float(sum(g.nx * g.ny * int(st) for g, st in zip(grids, steps)))
    launches = ens.launch_count()

    # per-instance loop arm
    loop_steps = []
    checked = 0
    e0.record(stream)
    for k, (fam, idx, n) in enumerate(spec):
        s = handles[n]
        s.set_state(dev_U[k])
        _, st = s.advance_to(a.t_end)
        loop_steps.append(st)
        if checked < a.check and k % max(1, a.count // max(a.check, 1)) == 0:
            assert s.get_state().tobytes() == ens.get_state(k).tobytes(), f"member {k} differs"
            checked += 1
    e1.record(stream)
    torch.cuda.synchronize()
    loop_ms = e0.elapsed_time(e1)
    assert list(loop_steps) == [int(x) for x in steps], "step counts differ"
    print(json.dumps({
        "metric": "FP64 cell-updates/s", "unit": "cell-updates/s",
        "workload": f"{a.count} trajectories (riemann/blast), sizes {sizes}, HLLC+vL, t_end={a.t_end}",
        "ensemble": {"value": cells / (ens_ms / 1e3), "ms": ens_ms, "launches": launches},
        "per_instance_loop": {"value": cells / (loop_ms / 1e3), "ms": loop_ms,
                              "note": "includes bit-exact checks of a few members (host copies)"},
        "speedup": loop_ms / ens_ms, "cell_updates": cells, "members_checked_bitexact": checked,
        "all_status_ok": bool((status == 0).all())}), flush=True)


if __name__ == "__main__":
    main()
