"""Build recipe for the CPU oracle (TEST INFRASTRUCTURE ONLY).

  python oracle/build_oracle.py [--reference DIR]     # builds what it can

DIR (or the environment variable FV_REFERENCE_SRC) is the reference's solver/src folder; the default
is the read-only copy of the reference project this repository was built beside.

1. oracle/libfvoracle.so  -- the plain-C restatement (oracle/fv_oracle.c), always built.
2. oracle/_ref/libfvref.so -- oracle/ref_harness.cpp compiled against the reference's own solver
   headers where they lie (REF_SRC below, read-only), plus the reference's three C++ unit-test
   programs (test_riemann2d, test_grid2d, test_solver2d) built from their sources into oracle/_ref/.
   Skipped when the reference tree is absent (the prebuilt files travel with the repo snapshot).
3. oracle/_ref/test_solver2d_fv -- the reference's test_solver2d.cpp, unmodified, built against the
   GPU library (libfv.so) through the drop-in Solver header neural-pde-surrogate_b200/host/fv_solver2d.hpp.

Both are built WITHOUT floating-point contraction (-ffp-contract=off) and without -march, which is
what makes them bit-identical to each other and to the GPU parity build (nvcc --fmad=false).
"""
import os
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_SRC = Path(os.environ.get("FV_REFERENCE_SRC", "/root/reference/solver/src"))
REF_OUT = HERE / "_ref"

CFLAGS = ["-O3", "-fopenmp", "-ffp-contract=off", "-fPIC"]


def _run(cmd):
    subprocess.run(cmd, check=True)


def build_oracle(force=False):
    out = HERE / "libfvoracle.so"
    src = HERE / "fv_oracle.c"
    if force or not out.exists() or out.stat().st_mtime < src.stat().st_mtime:
        _run(["gcc", "-std=c11", *CFLAGS, "-shared", str(src), "-o", str(out), "-lm"])
    return out


def build_ref(force=False):
    """Returns the path of libfvref.so, or None when the reference sources are not present."""
    out = REF_OUT / "libfvref.so"
    if not REF_SRC.is_dir():
        return out if out.exists() else None
    REF_OUT.mkdir(exist_ok=True)
    harness = HERE / "ref_harness.cpp"
    if force or not out.exists() or out.stat().st_mtime < harness.stat().st_mtime:
        _run(["g++", "-std=gnu++17", *CFLAGS, "-shared", f"-I{REF_SRC}", str(harness), "-o", str(out)])
    for t in ("test_riemann2d", "test_grid2d", "test_solver2d"):
        exe = REF_OUT / t
        if force or not exe.exists():
            _run(["g++", "-std=gnu++17", "-O3", "-fopenmp", "-ffp-contract=off", f"-I{REF_SRC}",
                  str(REF_SRC / f"{t}.cpp"), "-o", str(exe)])
    return out


ADAPTER = HERE.parent / "neural-pde-surrogate_b200" / "host" / "fv_solver2d.hpp"
LIBFV_DIR = HERE.parent / "neural-pde-surrogate_b200"


def build_ref_on_fv(force=False):
    """The reference's own test_solver2d.cpp, unmodified, built against the GPU library through the
    drop-in Solver header: oracle/_ref/test_solver2d_fv.  Its `#include "solver2d.hpp"` looks in the
    including file's folder first, so the source is compiled through a symlink in a temporary folder
    beside a symlink named solver2d.hpp to the drop-in header (nothing of the reference is copied).
    Returns the program's path, or None when the reference sources or libfv.so are absent."""
    exe = REF_OUT / "test_solver2d_fv"
    if not REF_SRC.is_dir() or not (LIBFV_DIR / "libfv.so").exists():
        return exe if exe.exists() else None
    deps = [ADAPTER, LIBFV_DIR / "libfv.so", HERE.parent / "include" / "fv.h"]
    if force or not exe.exists() or any(f.stat().st_mtime > exe.stat().st_mtime for f in deps):
        REF_OUT.mkdir(exist_ok=True)
        with tempfile.TemporaryDirectory() as tmp:  # the symlinks live only while compiling
            d = Path(tmp)
            (d / "test_solver2d.cpp").symlink_to(REF_SRC / "test_solver2d.cpp")
            (d / "solver2d.hpp").symlink_to(ADAPTER)
            _run(["g++", "-std=gnu++17", "-O2", "-ffp-contract=off", f"-I{d}", f"-I{REF_SRC}",
                  f"-I{HERE.parent / 'include'}", str(d / "test_solver2d.cpp"), "-o", str(exe), f"-L{LIBFV_DIR}",
                  "-lfv", "-Wl,-rpath,$ORIGIN/../../neural-pde-surrogate_b200"])
    return exe


def build(force=False):
    build_oracle(force)
    build_ref(force)
    build_ref_on_fv(force)


if __name__ == "__main__":
    if "--reference" in sys.argv:
        REF_SRC = Path(sys.argv[sys.argv.index("--reference") + 1])
    build(force="--force" in sys.argv)
    print("oracle built:", HERE / "libfvoracle.so", "| reference:", REF_OUT / "libfvref.so")
