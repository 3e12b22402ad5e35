"""Thread-count independence of the CPU solvers (tests/compare_runs.py:11-22 checks that serial and
parallel runs of the reference are bit-identical; solver2d.hpp:56 states it).  The compiled reference
and the C restatement are each run with 1 and with 3 OpenMP threads, in separate processes (the thread
count is fixed when OpenMP starts), and all four final states must have the same bits."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

SCRIPT = r"""
import hashlib, importlib, sys
sys.path.insert(0, sys.argv[1])
from oracle import oracle as orc
ic = importlib.import_module("neural-pde-surrogate_b200.ic")
out = []
for cls in (orc.OracleSolver, orc.RefSolver):
    for fam, idx, lim in (("riemann", 2, "vanleer"), ("blast", 5, "minmod")):
        s = cls(48, 40, 0.0, 1.0, 0.0, 1.0, "periodic", "transmissive", "hllc", lim, 0.5)
        s.set_state(ic.to_conserved(*[a[:40, :48] for a in ic.sample(fam, idx, 48)[:4]]))
        s.advance_to(0.03)
        out.append(f"{s.max_threads()} {s.steps} {hashlib.sha256(s.get_state().tobytes()).hexdigest()}")
print("\n".join(out))
"""


def _run(threads):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([sys.executable, "-c", SCRIPT, str(ROOT)], capture_output=True, text=True, env=env,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    return [ln.split() for ln in r.stdout.strip().splitlines()]


def test_serial_and_parallel_runs_are_bit_identical(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.fail("the compiled reference (oracle/_ref) is missing")
    one, three = _run(1), _run(3)
    assert all(r[0] == "1" for r in one) and all(r[0] == "3" for r in three)
    assert [r[1:] for r in one] == [r[1:] for r in three]  # same step counts, same bits
    assert all(int(r[1]) > 5 for r in one)  # the runs did step
    assert [r[1:] for r in one[:2]] == [r[1:] for r in one[2:]]  # the restatement equals the reference
