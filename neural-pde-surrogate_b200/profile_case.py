"""Runs one solver case on the GPU and prints per-kernel timings -- the counterpart of the reference
driver's `--profile yes` phase table (solver2d.hpp:29-52, main2d.cpp:261), and the program the ncu
summaries under profiles/ are captured from.

  python neural-pde-surrogate_b200/profile_case.py [--family blast] [--index 0] [--n 512]
         [--flux hllc] [--limiter vanleer] [--steps 200]
"""
import argparse
import importlib
import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--family", default="blast")
    ap.add_argument("--index", type=int, default=0)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--flux", default="hllc")
    ap.add_argument("--limiter", default="vanleer")
    ap.add_argument("--steps", type=int, default=200)
    a = ap.parse_args()
    fv = importlib.import_module("neural-pde-surrogate_b200")
    ic = importlib.import_module("neural-pde-surrogate_b200.ic")
    solver = importlib.import_module("neural-pde-surrogate_b200.solver")
    rho, u, v, p, _, _ = ic.sample(a.family, a.index, a.n)
    s = fv.Solver(fv.make_grid(a.n, a.n, 0, 1, 0, 1, "periodic", "periodic"), a.flux, a.limiter, 0.5)
    s.set_primitive(rho, u, v, p)
    solver.profile(s, True)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        s.step(dt=s.compute_dt())
    s.synchronize()
    wall = time.perf_counter() - t0
    ms1, ms2, n = solver.profile_read(s)
    cells = a.n * a.n
    print(f"{a.family}[{a.index}] {a.n}^2 {a.flux}+{a.limiter}: {n} steps, stage1 {ms1 * 1e3:.1f} us, "
          f"stage2 {ms2 * 1e3:.1f} us per launch -> {cells / ((ms1 + ms2) / 1e3) / 1e9:.2f} G cell-updates/s "
          f"of kernel time; wall {wall:.3f} s (host-synchronous compute_dt each step)")


if __name__ == "__main__":
    main()
