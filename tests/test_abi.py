"""C-ABI checks that need no GPU: every library loads and exports every symbol its header in
include/ declares; argument validation fails cleanly (no compute calls are made here)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "neural-pde-surrogate_b200"

# (header, shared library that implements it): the parity build and the tolerance build
LIBS = [(h, lib) for lib in ("libfv.so", "libfv_tol.so") for h in ("fv.h", "fvnet.h")]


def declared(header):
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w ]*?[\s\*]+(\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module", autouse=True)
def built():
    import importlib
    importlib.import_module("neural-pde-surrogate_b200.build").build()


@pytest.mark.parametrize("header,lib", LIBS)
def test_library_exports_every_declared_symbol(header, lib):
    path = PKG / lib
    assert path.exists(), f"{lib} not built"
    C.CDLL(str(path))
    names = declared(header)
    assert len(names) >= 5
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, f"{lib} does not export {missing}"


def test_fv_argument_validation_without_gpu(fvpkg):
    L = fvpkg.lib()
    h = C.c_void_p()
    assert L.fv_create(0, 8, 0.0, 1.0, 0.0, 1.0, 1, 1, 1, 3, 0.5, None, C.byref(h)) == 1
    assert b"positive" in L.fv_last_error()
    assert L.fv_create(8, 8, 0.0, 1.0, 0.0, 1.0, 1, 1, 7, 3, 0.5, None, C.byref(h)) == 1
    assert L.fv_create(8, 8, 0.0, 1.0, 0.0, 1.0, 1, 1, 1, 3, -0.5, None, C.byref(h)) == 1
    assert L.fv_create(8, 8, 0.0, 1.0, 0.0, 1.0, 1, 1, 1, 3, 0.5, None, None) == 1
    assert L.fv_step(None, 0.1) == 1
    assert L.fv_version().startswith(b"fv-b200")


def test_python_mirror_rejects_unknown_names(fvpkg):
    g = fvpkg.make_grid(8, 8, 0, 1, 0, 1, "periodic", "periodic")
    with pytest.raises(ValueError, match="Unknown scheme"):
        fvpkg.Solver(g, "roe", "vanleer")
    with pytest.raises(ValueError, match="Unknown limiter"):
        fvpkg.Solver(g, "hllc", "superbee")


def test_no_cpu_fallback(fvpkg):
    """On a machine without a GPU the product path raises; it never computes on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    g = fvpkg.make_grid(8, 8, 0, 1, 0, 1, "periodic", "periodic")
    with pytest.raises(fvpkg.FVError, match="no CUDA device"):
        fvpkg.Solver(g, "hllc", "vanleer")


def test_ensemble_and_network_argument_validation_without_gpu(fvpkg):
    """Bad arguments are rejected before any CUDA call; valid ones on a machine without a GPU give
    FV_ERR_CUDA, never a crash or a CPU computation."""
    import torch
    L = fvpkg.lib()
    e = C.c_void_p()
    ints = lambda *v: (C.c_int * len(v))(*v)
    dbl = lambda *v: (C.c_double * len(v))(*v)
    P = lambda a: C.cast(a, C.c_void_p)
    nx, ny, bc = ints(64, 32), ints(64, 32), ints(1, 0)
    assert L.fv_ensemble_create(0, P(nx), P(ny), None, P(bc), P(bc), 1, 3, 0.5, None, C.byref(e)) == 1
    assert L.fv_ensemble_create(2, P(ints(64, 0)), P(ny), None, P(bc), P(bc), 1, 3, 0.5, None, C.byref(e)) == 1
    assert b"positive" in L.fv_last_error()
    assert L.fv_ensemble_create(2, P(nx), P(ny), None, P(ints(1, 9)), P(bc), 1, 3, 0.5, None, C.byref(e)) == 1
    assert b"bc" in L.fv_last_error()
    bounds = dbl(0, 1, 0, 1, 0, 1, 0.5, 0.5)  # the second member's y extent is empty
    assert L.fv_ensemble_create(2, P(nx), P(ny), P(bounds), P(bc), P(bc), 1, 3, 0.5, None, C.byref(e)) == 1
    assert b"empty domain" in L.fv_last_error()
    assert L.fv_ensemble_create(2, P(nx), P(ny), None, P(bc), P(bc), 5, 3, 0.5, None, C.byref(e)) == 1
    assert L.fv_ensemble_create(2, P(nx), P(ny), None, P(bc), P(bc), 1, 3, 0.0, None, C.byref(e)) == 1
    if not torch.cuda.is_available():
        assert L.fv_ensemble_create(2, P(nx), P(ny), None, P(bc), P(bc), 1, 3, 0.5, None, C.byref(e)) == 2
        assert b"no CUDA device" in L.fv_last_error()
    # the convolution kernels: unsupported shapes and missing buffers are rejected up front
    dummy = C.c_void_p(16)  # never dereferenced: every call below fails its checks first
    assert L.fvnet_conv3x3(0, 16, 32, 2, 8, 48, dummy, dummy, dummy, None, dummy, dummy, None, None, None) == 1
    assert b"bad shape" in L.fv_last_error()
    assert L.fvnet_conv3x3(0, 16, 32, 2, 8, 64, None, dummy, dummy, None, dummy, dummy, None, None, None) == 1
    assert L.fvnet_conv3x3(0, 16, 32, 2, 8, 64, dummy, dummy, None, None, dummy, dummy, None, None, None) == 1
    assert b"hidden needs" in L.fv_last_error()
    assert L.fvnet_conv3x3(1, 32, 16, 2, 8, 64, dummy, dummy, dummy, None, None, None, None, None, None) == 1
    assert b"output needs" in L.fv_last_error()
    assert L.fvnet_conv3x3(9, 32, 32, 2, 8, 64, dummy, dummy, dummy, None, dummy, dummy, None, None, None) == 1
    assert b"unsupported" in L.fv_last_error()


@pytest.mark.parametrize("build,marker", [(None, b"bit-exact build"), ("parity", b"bit-exact build"),
                                          ("tolerance", b"tolerance build"), ("fast", None)])
def test_fv_build_selects_the_library(build, marker):
    """FV_BUILD picks the solver library when it is first loaded; unset means the bit-exact build."""
    import os
    import sys
    env = {k: v for k, v in os.environ.items() if k != "FV_BUILD"}
    if build:
        env["FV_BUILD"] = build
    code = ("import importlib, sys; sys.path.insert(0, sys.argv[1]); "
            "print(importlib.import_module('neural-pde-surrogate_b200').lib().fv_version().decode())")
    r = subprocess.run([sys.executable, "-c", code, str(ROOT)], capture_output=True, text=True, env=env, timeout=120)
    if marker is None:
        assert r.returncode != 0 and "use one of parity, tolerance" in r.stderr
    else:
        assert r.returncode == 0, r.stderr
        assert marker.decode() in r.stdout


class _FakeCudaTensor:
    """Enough of a CUDA tensor's surface for the pointer checks (no device needed)."""

    def __init__(self, shape, dtype="torch.float64", contiguous=True):
        import math
        self.shape, self.dtype, self._contig, self.is_cuda = tuple(shape), dtype, contiguous, True
        self._numel = math.prod(shape)

    def is_contiguous(self):
        return self._contig

    def numel(self):
        return self._numel

    def data_ptr(self):
        return 4096


def test_pointer_checks_reject_what_a_kernel_would_overrun():
    import numpy as np
    from importlib import import_module
    L = import_module("neural-pde-surrogate_b200._lib")
    assert L.device_ptr(_FakeCudaTensor((2, 8, 8, 4)), (2, 8, 8, 4)).value == 4096
    assert L.device_ptr(_FakeCudaTensor((3,), "torch.int32"), (3,), dtype="torch.int32").value == 4096
    assert L.device_ptr(_FakeCudaTensor((2, 4)), numel=8).value == 4096
    with pytest.raises(ValueError, match="expected shape"):
        L.device_ptr(_FakeCudaTensor((2, 8, 8, 3)), (2, 8, 8, 4))
    with pytest.raises(TypeError, match="dtype torch.float64"):
        L.device_ptr(_FakeCudaTensor((2, 8, 8, 4), "torch.float32"), (2, 8, 8, 4))
    with pytest.raises(ValueError, match="contiguous"):
        L.device_ptr(_FakeCudaTensor((2, 8, 8, 4), contiguous=False), (2, 8, 8, 4))
    with pytest.raises(ValueError, match="expected 12 elements"):
        L.device_ptr(_FakeCudaTensor((2, 4)), numel=12)
    with pytest.raises(TypeError, match="CUDA tensor"):
        L.device_ptr(np.zeros(4), numel=4)
    import torch
    with pytest.raises(TypeError, match="CUDA tensor"):
        L.device_ptr(torch.zeros(4, dtype=torch.float64), numel=4)  # a CPU tensor
    out = np.empty((4, 2, 2), np.float32)
    assert L.host_out_ptr(out, (4, 2, 2), np.float32).value == out.ctypes.data
    with pytest.raises(ValueError, match="float32 array of shape"):
        L.host_out_ptr(np.empty((4, 2, 2), np.float64), (4, 2, 2), np.float32)
    with pytest.raises(ValueError, match="float64 array of shape"):
        L.host_out_ptr(np.empty((3, 3, 4)), (3, 4, 4), np.float64)
    with pytest.raises(ValueError, match="C-contiguous"):
        L.host_out_ptr(np.empty((4, 4, 4))[:, ::2], (4, 2, 4), np.float64)
    with pytest.raises(TypeError, match="numpy array"):
        L.host_out_ptr([0.0] * 4, (4,), np.float64)


def test_host_helpers_check_shapes_before_calling_the_library(fvpkg):
    import numpy as np
    with pytest.raises(ValueError, match="same shape"):
        fvpkg.riemann_flux("hllc", np.ones((3, 4)), np.ones((2, 4)))
    with pytest.raises(ValueError, match=r"\(ny, nx, 4\)"):
        fvpkg.fill_ghosts(np.ones((4, 4, 3)), "periodic", "periodic")


def test_division_check_entry_point_without_gpu(fvpkg):
    import numpy as np
    import torch
    L = fvpkg.lib()
    assert L.fv_eval_division(-1, None, None, None) == 1 and b"bad arguments" in L.fv_last_error()
    assert L.fv_eval_division(3, None, None, None) == 1
    assert L.fv_eval_division(0, None, None, None) == 0  # nothing to do
    with pytest.raises(ValueError, match="same shape"):
        fvpkg.eval_division(np.ones(3), np.ones(4))
    if not torch.cuda.is_available():
        with pytest.raises(fvpkg.FVError):  # computed on the GPU or not at all
            fvpkg.eval_division(np.ones(3), np.full(3, 3.0))
