"""Build recipe for the native libraries of this package (in-tree, so the .so files travel with the
repository snapshot).  Cross-compiles for sm_100a with nvcc; no GPU needed to build.

  python neural-pde-surrogate_b200/build.py [--force] [-v]

libfv.so -- the finite-volume solver (csrc/fv_api.cu + csrc/fv_kernels.cuh), C-ABI in include/fv.h.
            Built with --fmad=false: no FMA contraction, which keeps every result bit-identical to
            the reference CPU solver (its build uses none either).
host/euler2d -- the reference's euler2d driver (main2d.cpp) over libfv.so's C-ABI, built with g++
            -ffp-contract=off (its host-side to_primitive for snapshots must round like the reference).
"""
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
NVCC = "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", f"-I{ROOT / 'include'}"]

LIBS = {
    "libfv.so": {
        "sources": ["fv_api.cu", "fv_peak.cu", "fv_noalloc.cu", "fv_ensemble.cu", "fvnet_conv.cu", "fvnet_ops.cu",
                    "fv_selftest.cu"],
        "deps": ["fv_api.cu", "fv_peak.cu", "fv_noalloc.cu", "fv_selftest.cu", "fv_ensemble.cu", "fv_kernels.cuh", "fv_physics.cuh", "fv_stepper.cuh",
                 "fvnet_conv.cu", "fvnet_ops.cu", "tc_sm100.cuh"],
        "flags": ["--fmad=false"],
        "headers": ["fv.h", "fvnet.h"],
    },
}
# The tolerance build: the same sources with FMA contraction, for the stated tolerances (1e-12 relative
# per step, 1e-9 per run) instead of bit-exactness; loaded only when FV_BUILD=tolerance.
LIBS["libfv_tol.so"] = {**LIBS["libfv.so"], "flags": ["--fmad=true", "-DFV_TOLERANCE_BUILD=1"]}


def _stale(out, deps, headers):
    if not out.exists():
        return True
    t = out.stat().st_mtime
    files = [CSRC / d for d in deps] + [ROOT / "include" / h for h in headers] + [Path(__file__)]
    return any(f.stat().st_mtime > t for f in files)


def build(force=False, verbose=False):
    built = []
    for name, spec in LIBS.items():
        out = PKG / name
        if not force and not _stale(out, spec["deps"], spec["headers"]):
            continue
        cmd = [NVCC, *ARCH, *COMMON, *spec["flags"], "-shared", "-o", str(out),
               *[str(CSRC / s) for s in spec["sources"]], *spec.get("libs", [])]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        built.append(name)
    exe, src = PKG / "host" / "euler2d", [PKG / "host" / "euler2d.cpp", PKG / "host" / "npz_io.hpp"]
    if force or not exe.exists() or any(f.stat().st_mtime > exe.stat().st_mtime
                                        for f in src + [PKG / "libfv.so", ROOT / "include" / "fv.h"]):
        cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", f"-I{ROOT / 'include'}", "-o", str(exe), str(src[0]),
               f"-L{PKG}", "-lfv", "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        built.append("host/euler2d")
    return built


if __name__ == "__main__":
    print("built:", build(force="--force" in sys.argv, verbose="-v" in sys.argv))
