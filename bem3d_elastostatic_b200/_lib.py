"""ctypes binding of libbem3d_b200.so (the C ABI in include/bem3d_b200.h).

The library is built in-tree by ``bem3d_elastostatic_b200.build``.  There is no CPU
fallback: if the shared library is missing or cannot be loaded, every entry point
raises ``LibraryNotAvailable``.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

LIB_PATH = _build.LIB

BEM_OK = 0
BEM_ERR_ARG = -1
BEM_ERR_CUDA = -2
BEM_ERR_OOM = -3
BEM_ERR_TIMEOUT = -4
BEM_ERR_STATE = -5
BEM_ERR_MESH = -6
BEM_ERR_NOCONV = -7
BEM_ERR_TOO_LARGE = -8
NOALLOC_MAX_N = 4096

BEM_PREC_FP64 = 0
BEM_PREC_FP32_IR = 1
BEM_PREC_BF16_IR = 2
BEM_PREC_FP64_IR = 3
BEM_PROF_COUNT = 0
BEM_PROF_PHASES = 1
BEM_PROF_TRAILING = 2
BEM_ASM_FP64 = 0
BEM_ASM_FP32_FAR = 1
BEM_IP_KELVIN_CONSISTENT = 1
BEM_PIVOT_PARTIAL = 0
BEM_PIVOT_WINDOW = 1
BEM_OPT_PIVOTING = 1
BEM_OPT_WAIT_LIMIT_MS = 2
BEM_OPT_WITHHOLD_BLOCK = 3
BEM_OPT_RESIDUAL = 4
BEM_OPT_PANEL_WIDTH = 5

# every symbol the header declares, for the export check
EXPORTS = [
    "bem_ctx_create", "bem_ctx_destroy", "bem_last_error", "bem_sync", "bem_get_stream",
    "bem_set_option", "bem_set_mesh",
    "bem_set_material", "bem_set_bc", "bem_set_pins", "bem_precompute_geometry",
    "bem_get_geometry", "bem_ghmat8", "bem_set_system", "bem_get_rows", "bem_get_hg", "bem_solve", "bem_dgesv",
    "bem_reorganize", "bem_boundary_stresses", "bem_solve_transposed", "bem_adjoint_gradient", "bem_internal_points", "bem_device_state",
    "bem_internal_points_device", "bem_profile_begin", "bem_profile_end",
    "bem_dgesv_noalloc", "bem_batch_create", "bem_batch_destroy", "bem_batch_last_error",
    "bem_batch_add", "bem_batch_assemble", "bem_batch_solve", "bem_batch_get_solution",
    "bem_batch_get_system", "bem_batch_launches",
]


class LibraryNotAvailable(RuntimeError):
    pass


class BemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("restarts", C.c_int), ("rel_residual", C.c_double),
                ("factor_seconds", C.c_double), ("refine_seconds", C.c_double),
                ("gflops", C.c_double), ("pivoting", C.c_int), ("fallbacks", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchInfo(C.Structure):
    _fields_ = [("systems", C.c_int), ("sweeps", C.c_int), ("converged", C.c_int),
                ("singular", C.c_int), ("max_backward_error", C.c_double),
                ("solve_seconds", C.c_double), ("lu_threads", C.c_int),
                ("lu_ms_256", C.c_float), ("lu_ms_512", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Profile(C.Structure):
    _fields_ = [("kernel_launches", C.c_longlong), ("lu_panel_ms", C.c_double),
                ("lu_swap_ms", C.c_double), ("lu_panel_update_ms", C.c_double),
                ("lu_trsm_ms", C.c_double), ("lu_trailing_ms", C.c_double),
                ("lu_trailing_launches", C.c_longlong), ("lu_trailing_flops", C.c_double),
                ("lu_trailing_bytes", C.c_double), ("ip_points", C.c_longlong),
                ("ip_near_points", C.c_longlong), ("ip_far_evals", C.c_double),
                ("ip_near_evals", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p
_lib = None


def load(build_if_needed: bool = True):
    """Load the CUDA library (building it first when the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_needed and _build.needs_build():
        try:
            _build.build()
        except Exception as exc:  # no nvcc where the library must already exist
            if not os.path.exists(LIB_PATH):
                raise LibraryNotAvailable(f"cannot build {LIB_PATH}: {exc}") from exc
    if not os.path.exists(LIB_PATH):
        raise LibraryNotAvailable(f"{LIB_PATH} is missing; run python -m bem3d_elastostatic_b200.build")
    try:
        L = C.CDLL(LIB_PATH)
    except OSError as exc:
        raise LibraryNotAvailable(str(exc)) from exc
    ctxp = C.POINTER(C.c_void_p)
    L.bem_ctx_create.argtypes = [ctxp, C.c_int]
    L.bem_ctx_destroy.argtypes = [_vp]
    L.bem_last_error.argtypes = [_vp]
    L.bem_last_error.restype = C.c_char_p
    L.bem_sync.argtypes = [_vp]
    L.bem_get_stream.argtypes = [_vp, C.POINTER(C.c_void_p)]
    L.bem_set_option.argtypes = [_vp, C.c_int, C.c_int64]
    L.bem_set_mesh.argtypes = [_vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp]
    L.bem_set_material.argtypes = [_vp, C.c_double, C.c_double]
    L.bem_set_bc.argtypes = [_vp, _vp, _vp]
    L.bem_set_pins.argtypes = [_vp, C.c_int, _vp]
    L.bem_precompute_geometry.argtypes = [_vp]
    L.bem_get_geometry.argtypes = [_vp] + [_vp] * 8
    L.bem_ghmat8.argtypes = [_vp, C.c_int, _vp, C.c_int64, _vp]
    L.bem_set_system.argtypes = [_vp, C.c_int, _vp, C.c_int64, _vp]
    L.bem_get_rows.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int64, _vp]
    L.bem_get_hg.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int64, _vp, C.c_int64]
    L.bem_solve.argtypes = [_vp, C.c_int, C.c_double, C.c_int, _vp, _ip, C.POINTER(SolveInfo)]
    L.bem_dgesv.argtypes = [_vp, C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _ip]
    L.bem_dgesv_noalloc.argtypes = [C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, C.c_int, _ip, _vp]
    L.bem_reorganize.argtypes = [_vp, _vp, _vp]
    L.bem_boundary_stresses.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.bem_solve_transposed.argtypes = [_vp, _vp]
    L.bem_adjoint_gradient.argtypes = [_vp, _vp, _vp, _vp]
    L.bem_internal_points.argtypes = [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int]
    L.bem_device_state.argtypes = [_vp, C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
    L.bem_internal_points_device.argtypes = [_vp, C.c_int] + [_vp] * 7 + [C.c_int]
    L.bem_batch_create.argtypes = [ctxp, C.c_int]
    L.bem_batch_destroy.argtypes = [_vp]
    L.bem_batch_last_error.argtypes = [_vp]
    L.bem_batch_last_error.restype = C.c_char_p
    L.bem_batch_add.argtypes = [_vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, C.c_double, C.c_double,
                                _vp, C.c_int, _vp, C.c_int, _vp]
    L.bem_batch_assemble.argtypes = [_vp]
    L.bem_batch_solve.argtypes = [_vp, C.c_int, C.c_double, C.c_int, C.POINTER(BatchInfo)]
    L.bem_batch_get_solution.argtypes = [_vp, C.c_int, _vp]
    L.bem_batch_get_system.argtypes = [_vp, C.c_int, _vp, _vp]
    L.bem_batch_launches.argtypes = [_vp]
    L.bem_batch_launches.restype = C.c_longlong
    L.bem_profile_begin.argtypes = [_vp, C.c_int]
    L.bem_profile_end.argtypes = [_vp, C.POINTER(Profile)]
    _lib = L
    return L


def ptr(a) -> int:
    """Address of a numpy array (host) or an int device address."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    return a.ctypes.data


class Context:
    """Owns one bem_ctx (one CUDA stream on one device)."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        rc = self.L.bem_ctx_create(C.byref(h), device)
        if rc != 0:
            raise BemError(rc, f"bem_ctx_create(device={device}) failed")
        self.h = h
        self.device = device

    def check(self, rc: int, what: str) -> int:
        if rc < 0:
            msg = self.L.bem_last_error(self.h)
            raise BemError(rc, f"{what}: {msg.decode() if msg else ''}")
        return rc

    def stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        s = C.c_void_p()
        self.check(self.L.bem_get_stream(self.h, C.byref(s)), "get_stream")
        return int(s.value or 0)

    def sync(self):
        self.check(self.L.bem_sync(self.h), "sync")

    def set_option(self, option: int, value: int):
        """bem_set_option: BEM_OPT_PIVOTING, BEM_OPT_WAIT_LIMIT_MS, BEM_OPT_WITHHOLD_BLOCK,
        BEM_OPT_RESIDUAL, BEM_OPT_PANEL_WIDTH."""
        self.check(self.L.bem_set_option(self.h, int(option), int(value)), "set_option")

    def profile_begin(self, timing=True):
        """timing: True / BEM_PROF_PHASES (every LU phase), BEM_PROF_TRAILING (the
        trailing updates only), False / BEM_PROF_COUNT (launch counts only)."""
        mode = BEM_PROF_PHASES if timing is True else (BEM_PROF_COUNT if timing is False else int(timing))
        self.check(self.L.bem_profile_begin(self.h, mode), "profile_begin")

    def profile_end(self) -> dict:
        p = Profile()
        self.check(self.L.bem_profile_end(self.h, C.byref(p)), "profile_end")
        return p.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.L.bem_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
