"""GPU run of the reference's own test_solver2d.cpp, built unmodified against libfv through the C++
drop-in Solver header (oracle/_ref/test_solver2d_fv, made by oracle/build_oracle.py).  The program's
ten checks (free stream, x/y transpose symmetry, conservation, the Sod plateaus; test_solver2d.cpp:37-108)
must all pass with every step running on the GPU.
"""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
EXE = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "test_solver2d_fv"


def test_reference_solver_test_passes_on_the_gpu(cuda_ok):
    if not EXE.exists():
        pytest.fail(f"{EXE} not built (the reference tree was absent when oracle/build_oracle.py ran)")
    r = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count(" PASS  (") == 10 and " FAIL  (" not in r.stdout  # the program's ten checks
    assert "ALL PASSED (0 failures)" in r.stdout
