"""ctypes loader for libfv.so (include/fv.h).  No CPU fallback: if the library or a GPU is missing,
calls raise instead of computing anything elsewhere."""
import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent

FV_OK, FV_ERR_ARG, FV_ERR_CUDA, FV_ERR_NONPHYSICAL, FV_ERR_TIMEOUT, FV_ERR_STATE = range(6)


class FVError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class NonPhysicalError(FVError):
    """The state failed compute_dt's check !(rho > 0) || !(p > 0) (solver2d.hpp:75); where the
    reference prints 'Non-physical state in cell (i, j): rho = ..., p = ...' and exits(1)."""

    def __init__(self, i, j, rho, p):
        super().__init__(FV_ERR_NONPHYSICAL, f"Non-physical state in cell ({i}, {j}): rho = {rho:g}, p = {p:g}")
        self.i, self.j, self.rho, self.p = i, j, rho, p


class BadCell(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("rho", C.c_double), ("p", C.c_double)]


_D, _I, _P = C.c_double, C.c_int, C.c_void_p
_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)
_LLP = C.POINTER(C.c_longlong)
_BP = C.POINTER(BadCell)

_PROTOS = {
    "fv_create": [_I, _I, _D, _D, _D, _D, _I, _I, _I, _I, _D, _P, C.POINTER(_P)],
    "fv_destroy": [_P],
    "fv_set_state": [_P, _P],
    "fv_get_state": [_P, _P],
    "fv_set_state_device": [_P, _P],
    "fv_get_state_device": [_P, _P],
    "fv_set_primitive": [_P, _P, _P, _P, _P],
    "fv_set_time": [_P, _D],
    "fv_get_time": [_P, _DP, _LLP],
    "fv_compute_dt": [_P, _DP, _BP],
    "fv_step": [_P, _D],
    "fv_advance_to": [_P, _D, _DP, _LLP, _BP],
    "fv_block_average": [_P, _I, _P],
    "fv_block_average_device": [_P, _I, _P],
    "fv_run_trajectory": [_P, _D, _D, _I, _P, _I, _P, _P, _LLP, _BP],
    "fv_synchronize": [_P],
    "fv_get_stream": [_P, C.POINTER(C.c_void_p)],
    "fv_ensemble_get_stream": [_P, C.POINTER(C.c_void_p)],
    "fv_riemann_flux": [_I, _I, _I, _P, _P, _P],
    "fv_eval_division": [_I, _P, _P, _P],
    "fv_eval_division_kind": [_I, _I, _P, _P, _P],
    "fv_division_sweep": [_I, C.c_longlong, C.c_ulonglong, _LLP, _LLP],
    "fv_fill_ghosts": [_I, _I, _I, _I, _P, _P],
    "fv_profile": [_P, _I],
    "fv_profile_read": [_P, _DP, _DP, _LLP],
    "fv_profile_steps": [_P, _DP, _LLP, _LLP],
    "fv_stepper_tile": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)],
    "fv_stepper_launch": [_P, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)],
    "fv_stepper_dependencies": [_I, _I, _I, _I, _I, _I, _P, _I, _P, _I, C.POINTER(_I)],
    "fv_launch_count": [_P, _LLP],
    "fv_fp64_peak": [_DP],
    "fv_wait_selftest": [],
    "fv_stepper_wait_selftest": [],
    "fv_ensemble_create": [_I, _P, _P, _P, _P, _P, _I, _I, _D, _P, C.POINTER(_P)],
    "fv_ensemble_destroy": [_P],
    "fv_ensemble_set_state": [_P, _I, _P],
    "fv_ensemble_set_state_device": [_P, _I, _P],
    "fv_ensemble_get_state": [_P, _I, _P],
    "fv_ensemble_state_device": [_P, _I, C.POINTER(_P)],
    "fv_ensemble_advance_to": [_P, _P, _P, _P, _P],
    "fv_ensemble_launch_count": [_P, _LLP],
    "fv_ensemble_set_all_device": [_P, _P],
    "fv_ensemble_get_all_device": [_P, _P],
    # correction network (include/fvnet.h)
    "fvnet_conv3x3": [_I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "fvnet_conv3x3_wgrad": [_I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P],
    "fvnet_wgrad_parts": [_I, _I],
    "fvnet_pack_weights": [_I, _I, _I, _I, _P, _P, _P, _P],
    "fvnet_prep_input": [_P, C.c_longlong, _P, _P, _P],
    "fvnet_apply_correction": [_P, _P, _I, _I, _P, _P, _P, _P, _I, _D, _P],
    "fvnet_loss_grad": [_P, _P, _P, _I, _I, _P, _P, _P, _P, _P, _P],
    "fvnet_adamw": [_P, _P, _P, _P, C.c_longlong, _P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                    C.c_float, _I, _P, _P],
    "fvnet_norm_partials": [],
    "fv_autotune": [_P, _I, C.POINTER(_I)],
    "fv_set_tile": [_P, _I],
    "fv_get_tile": [_P, C.POINTER(_I)],
    "fv_tile_variant": [_I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_I)],
}

_lib = None


def device_ptr(t, shape=None, numel=None, dtype="torch.float64", what="tensor"):
    """Raw pointer of a CUDA tensor that a libfv call reads or writes whole.  The call trusts the
    pointer for its full extent, so a wrong device, dtype, layout or size would make the kernel touch
    memory outside the tensor: this checks all four and raises instead (not an assert, which
    `python -O` would drop)."""
    if not (hasattr(t, "data_ptr") and getattr(t, "is_cuda", False)):
        raise TypeError(f"{what}: expected a CUDA tensor, got {type(t).__name__}")
    if str(t.dtype) != dtype:
        raise TypeError(f"{what}: expected dtype {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{what}: must be contiguous")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{what}: expected shape {tuple(shape)}, got {tuple(t.shape)}")
    if numel is not None and t.numel() != numel:
        raise ValueError(f"{what}: expected {numel} elements, got {t.numel()}")
    return C.c_void_p(t.data_ptr())


def host_out_ptr(a, shape, dtype, what="out"):
    """Raw pointer of a caller's numpy array that a libfv call writes whole: the same checks as
    device_ptr, for host memory."""
    import numpy as np
    if not isinstance(a, np.ndarray):
        raise TypeError(f"{what}: expected a numpy array, got {type(a).__name__}")
    if a.dtype != np.dtype(dtype) or a.shape != tuple(shape):
        raise ValueError(f"{what}: expected a {np.dtype(dtype)} array of shape {tuple(shape)}, "
                         f"got {a.dtype} {a.shape}")
    if not (a.flags.c_contiguous and a.flags.writeable):
        raise ValueError(f"{what}: must be C-contiguous and writeable")
    return C.c_void_p(a.ctypes.data)


class StreamOrder:
    """Orders a library handle's CUDA stream against torch's current stream.  The library queues the
    *_device copies on its own non-blocking stream, which nothing orders against torch's work: a
    tensor written by torch must be complete before the library reads it (before()), and torch must
    not read what the library writes until it is done (after())."""

    def __init__(self, getter, handle):
        p = C.c_void_p()
        check(getter(handle, C.byref(p)))
        self.ptr = p.value or 0
        self._ext = None

    def _streams(self):
        import torch
        if self._ext is None:
            self._ext = torch.cuda.ExternalStream(self.ptr) if self.ptr else torch.cuda.default_stream()
        return torch.cuda.current_stream(), self._ext

    def before(self):
        cur, ext = self._streams()
        if ext != cur:
            ext.wait_stream(cur)

    def after(self):
        cur, ext = self._streams()
        if ext != cur:
            cur.wait_stream(ext)


BUILDS = {"parity": "libfv.so", "tolerance": "libfv_tol.so"}


def lib():
    """The loaded solver library (raises if it has not been built): libfv.so, the bit-exact parity
    build, unless the environment sets FV_BUILD=tolerance (libfv_tol.so, FMA contraction)."""
    global _lib
    if _lib is None:
        build = os.environ.get("FV_BUILD", "parity")
        if build not in BUILDS:
            raise ValueError(f"FV_BUILD={build!r}: use one of {', '.join(BUILDS)}")
        path = PKG / BUILDS[build]
        if not path.exists():
            raise ImportError(f"{path} is missing: build it with `python {PKG / 'build.py'}` (nvcc, sm_100a)")
        L = C.CDLL(str(path))
        for name, args in _PROTOS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.fv_last_error.restype = C.c_char_p
        L.fv_last_error.argtypes = []
        L.fv_version.restype = C.c_char_p
        _lib = L
    return _lib


def check(rc, bad=None):
    """Raise the Python error for a non-zero status of a libfv call."""
    if rc == FV_OK:
        return
    if rc == FV_ERR_NONPHYSICAL and bad is not None:
        raise NonPhysicalError(bad.i, bad.j, bad.rho, bad.p)
    raise FVError(rc, lib().fv_last_error().decode() or f"libfv error {rc}")
