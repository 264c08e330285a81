"""ctypes binding of the C ABI in include/otmap_b200.h (libotmap_b200.so).

This is the only route from Python to the solver: there is no CPU fallback. If the
library is missing, or no CUDA device is present, calls raise.
"""

from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB

OK = 0
ERR_BAD_ARG = -1
ERR_CUDA = -2
ERR_NO_DEVICE = -3
ERR_TIMEOUT = -4
ERR_NOT_INIT = -5

CONVERGED, MAX_ITER, SMALL_STEP, NONFINITE = 0, 1, 2, 3
OPT_POISSON = 1
POISSON_AUTO, POISSON_DENSE, POISSON_FFT, POISSON_TENSOR = 0, 1, 2, 3
OPT_LOOP = 2
LOOP_GRAPH, LOOP_HOST = 0, 1
OPT_PRECISION = 4
PRECISION_FP64, PRECISION_SPLIT = 0, 1
OPT_AUTOTUNE, AUTOTUNE_OFF, AUTOTUNE_ON, INFO_STRIP_ROWS = 5, 0, 1, 6
OPT_WAIT_TEST = 3
RIO_PER_VERTEX, RIO_PER_FACE = 0, 1
INV_DENSEST, INV_FIRST = 0, 1
OUTCOMES = {CONVERGED: "converged", MAX_ITER: "max_iter", SMALL_STEP: "small_step", NONFINITE: "nonfinite"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class SolverOptionsC(C.Structure):
    _fields_ = [("beta", C.c_int), ("max_iter", C.c_int), ("threshold", C.c_double), ("max_ratio", C.c_double)]


class SolveStatsC(C.Structure):
    _fields_ = [("iterations", C.c_int), ("outcome", C.c_int), ("residual", C.c_double), ("linf", C.c_double),
                ("initial_residual", C.c_double)]


class AdjointOptionsC(C.Structure):
    _fields_ = [("mode", C.c_int), ("tol", C.c_double), ("max_iter", C.c_int), ("restart", C.c_int)]


class AdjointStatsC(C.Structure):
    _fields_ = [("iterations", C.c_int), ("relative_residual", C.c_double)]


ADJOINT_ONE_STEP, ADJOINT_KRYLOV = 0, 1


class BarycenterStatsC(C.Structure):
    _fields_ = [("iterations", C.c_int * 8), ("outcome", C.c_int * 8), ("residual", C.c_double * 8),
                ("inverse_missing", C.c_long), ("expected_mean", C.c_double), ("raster_mean", C.c_double),
                ("adjoint_solves", C.c_int * 8), ("adjoint_residual", C.c_double * 8)]


class OtmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"otmap_b200 error {code}: {msg}")
        self.code = code


_lib = None

# every entry point declared in include/otmap_b200.h, with its ctypes signature
SIGNATURES = {
    "otm_last_error": (C.c_char_p, []),
    "otm_abi_version": (C.c_int, []),
    "otm_default_options": (None, [C.POINTER(SolverOptionsC)]),
    "otm_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "otm_destroy": (C.c_int, [C.c_void_p]),
    "otm_init": (C.c_int, [C.c_void_p, C.c_int]),
    "otm_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(SolverOptionsC), C.c_void_p, C.c_void_p,
                            C.POINTER(SolveStatsC)]),
    "otm_solve_batch": (C.c_int, [C.c_void_p, C.c_int, _ip, C.POINTER(C.c_void_p), C.POINTER(SolverOptionsC),
                                  C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(SolveStatsC)]),
    "otm_map_create": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "otm_map_destroy": (C.c_int, [C.c_void_p]),
    "otm_map_init_inverse": (C.c_int, [C.c_void_p]),
    "otm_map_inverse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p,
                                  C.POINTER(C.c_long)]),
    "otm_map_inverse_mode": (C.c_int, [C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_long)]),
    "otm_rasterize": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "otm_rasterize_faces": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "otm_rasterize_mode": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                     C.c_void_p]),
    "otm_rasterize_mesh": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "otm_transport_cost": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.POINTER(C.c_double)]),
    "otm_grid_transport_cost": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.POINTER(C.c_double)]),
    "otm_mesh_blend": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p), _dp, C.c_void_p]),
    "otm_barycenter": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p), _dp, C.c_double, C.c_int,
                                 C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_double)]),
    "otm_sample_image": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_void_p, C.c_ulonglong, C.c_int, C.c_int, C.c_void_p]),
    "otm_grid_faces": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p]),
    "otm_write_off": (C.c_int, [C.c_char_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "otm_read_off": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p,
                               C.c_void_p, C.c_void_p]),
    "otm_prune_empty_faces": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                        C.POINTER(C.c_int), C.c_void_p, C.POINTER(C.c_int), C.c_void_p,
                                        C.c_void_p]),
    "otm_solve_noalloc": (C.c_int, [C.c_int, C.c_void_p, C.POINTER(SolverOptionsC), C.c_void_p, C.c_void_p,
                                    C.POINTER(SolveStatsC), C.c_void_p]),
    "otm_set_option": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "otm_default_adjoint_options": (None, [C.POINTER(AdjointOptionsC)]),
    "otm_adjoint": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(AdjointOptionsC),
                              C.c_void_p, C.POINTER(AdjointStatsC)]),
    "otm_barycenter_loss": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p), _dp, C.c_int, C.c_void_p,
                                      C.POINTER(SolverOptionsC), C.POINTER(AdjointOptionsC), C.c_void_p,
                                      C.POINTER(C.c_double), C.POINTER(C.c_void_p), C.POINTER(BarycenterStatsC)]),
    "otm_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "otm_get_option": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "otm_launch_count": (C.c_long, [C.c_void_p]),
    "otm_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "otm_profile_entry": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                                    C.POINTER(C.c_long)]),
}


def lib():
    """Loads libotmap_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"otmap_b200 CUDA library not built: {LIB_PATH} (run python -m otmap_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code):
    if code < 0:
        raise OtmError(code, lib().otm_last_error().decode(errors="replace"))
    return code


def ptr(a):
    """Address of a numpy array or torch tensor (host or device), or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return C.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    raise TypeError(f"unsupported buffer type {type(a)}")


def default_options():
    o = SolverOptionsC()
    lib().otm_default_options(C.byref(o))
    return o


class Context:
    """otm_context: one GPU, one stream."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().otm_create(int(device), C.byref(h)))
        self._h = h
        self.device = device
        self._owners = weakref.WeakSet()

    def track(self, owner):
        """Registers an object holding device maps of this context (it has a release()
        method): close() releases them before it frees the context."""
        self._owners.add(owner)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            for o in list(getattr(self, "_owners", ())):
                o.release()
            lib().otm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self, n: int):
        check(lib().otm_init(self._h, int(n)))

    def set_poisson(self, mode: int):
        check(lib().otm_set_option(self._h, OPT_POISSON, int(mode)))

    def set_loop(self, mode: int):
        check(lib().otm_set_option(self._h, OPT_LOOP, int(mode)))

    def set_precision(self, mode: int):
        """PRECISION_FP64 (default) or PRECISION_SPLIT (FP32 residuals, directions and
        transforms; FP64 potential, sums and line search)."""
        check(lib().otm_set_option(self._h, OPT_PRECISION, int(mode)))

    def set_autotune(self, on: bool):
        """AUTOTUNE_ON: the sweeps' strip height of a batch configuration is timed on its
        first call (16, 32, 64 rows) and the fastest kept; AUTOTUNE_OFF (default): a fixed rule."""
        check(lib().otm_set_option(self._h, OPT_AUTOTUNE, AUTOTUNE_ON if on else AUTOTUNE_OFF))

    def get_option(self, key: int) -> int:
        v = C.c_int(0)
        check(lib().otm_get_option(self._h, int(key), C.byref(v)))
        return v.value

    def strip_rows(self) -> int:
        """Strip height of the sweeps in the last solve call."""
        return self.get_option(INFO_STRIP_ROWS)

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().otm_stream(self._h, C.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        return int(lib().otm_launch_count(self._h))

    def profile(self, enable):
        check(lib().otm_profile(self._h, int(enable)))

    def profile_totals(self):
        """{kernel name: (total ms, launches)} of the profiled launches."""
        out = {}
        k = 0
        while True:
            name = C.c_char_p()
            ms = C.c_double()
            cnt = C.c_long()
            if not lib().otm_profile_entry(self._h, k, C.byref(name), C.byref(ms), C.byref(cnt)):
                break
            out[name.value.decode()] = (ms.value, cnt.value)
            k += 1
        return out


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(int(os.environ.get("OTMAP_DEVICE", "0")))
    return _default_ctx
