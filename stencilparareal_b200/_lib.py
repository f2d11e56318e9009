"""ctypes binding of ``libstencilparareal.so`` (the C ABI declared in include/sp_abi.h).

The library is the product: every computation goes through it.  There is no
CPU fallback -- importing this module raises if the shared library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# STENCILPARAREAL_LIB selects another build of the library (the bounds-checked
# libstencilparareal_checked.so next to this file)
LIB_PATH = os.environ.get("STENCILPARAREAL_LIB") or os.path.join(_HERE, "libstencilparareal.so")

SP_OK = 0
SP_ERR_INVALID = -1
SP_ERR_CUDA = -2
SP_ERR_NOMEM = -3
SP_ERR_UNSUPPORTED = -4
SP_ERR_TIMEOUT = -5
SP_ERR_NONFINITE = -6
SP_ERR_STATE = -7

SP_F64 = 0
SP_F32 = 1
SP_COARSE_EULER = 0
SP_COARSE_RK4 = 1
SP_TOL_NONE = 0
SP_TOL_DEFECT = 1
SP_TOL_REFERENCE = 2
SP_MAX_ITERS = 64
SP_NOALLOC_SCRATCH_BYTES = 16 << 20


class SpParams(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int),
                ("dx", C.c_double), ("nu0", C.c_double), ("nufreq", C.c_double),
                ("cx", C.c_double), ("cy", C.c_double), ("cz", C.c_double), ("upwind", C.c_int)]


class SpLayout(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("lx", C.c_int), ("elem_size", C.c_int),
                ("px", C.c_longlong), ("py", C.c_longlong), ("pz", C.c_longlong), ("plane", C.c_longlong),
                ("origin", C.c_longlong), ("total", C.c_longlong)]


class SpPararealCfg(C.Structure):
    _fields_ = [("endTime", C.c_double), ("timeSlices", C.c_int), ("timeStepsFine", C.c_int),
                ("timeStepsCoarse", C.c_int), ("kmax", C.c_int), ("async_", C.c_int),
                ("coarse_scheme", C.c_int), ("coarse_precision", C.c_int), ("tol_kind", C.c_int),
                ("tol", C.c_double), ("skip_converged", C.c_int), ("coarse_delta", C.c_int),
                ("first_slice", C.c_int), ("slice_count", C.c_int)]


class SpPararealReport(C.Structure):
    _fields_ = [("iterations", C.c_int), ("tsFine", C.c_int), ("tsCoarse", C.c_int),
                ("dtFine", C.c_double), ("dtCoarse", C.c_double), ("timeSliceSize", C.c_double),
                ("defect", C.c_double * SP_MAX_ITERS), ("err_l2", C.c_double * SP_MAX_ITERS),
                ("err_max", C.c_double * SP_MAX_ITERS), ("seconds", C.c_double),
                ("seconds_fine", C.c_double), ("seconds_coarse", C.c_double),
                ("fine_cell_updates", C.c_longlong)]


class SpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"stencilparareal error {code}: {msg}")
        self.code = code


_lib = None

# name -> (restype, argtypes)
_vp, _i, _d, _ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
_SIGS = {
    "sp_field_layout": (_i, [_i, _i, _i, _i, C.POINTER(SpLayout)]),
    "sp_convection_create": (_i, [C.POINTER(SpParams), _i, C.POINTER(_vp)]),
    "sp_convection_destroy": (_i, [_vp]),
    "sp_convection_set_stream": (_i, [_vp, _vp]),
    "sp_convection_synchronize": (_i, [_vp]),
    "sp_do_rk4": (_i, [_vp, _vp, _vp, _d, _d, _i]),
    "sp_do_euler": (_i, [_vp, _vp, _vp, _d, _d, _i]),
    "sp_do_rk4_timestep": (_i, [_vp, _vp, _vp, _d, _d]),
    "sp_do_euler_timestep": (_i, [_vp, _vp, _vp, _d, _d]),
    "sp_do_rk4_f32": (_i, [_vp, _vp, _vp, _d, _d, _i]),
    "sp_do_euler_f32": (_i, [_vp, _vp, _vp, _d, _d, _i]),
    "sp_periodicity_apply": (_i, [_vp, _vp, _i]),
    "sp_field_import": (_i, [_vp, _vp, _vp, _i, _i]),
    "sp_field_export": (_i, [_vp, _vp, _vp, _i, _i]),
    "sp_do_rk4_host": (_i, [_vp, _vp, _vp, _d, _d, _i]),
    "sp_field_errors": (_i, [_vp, _vp, _vp, C.POINTER(_d), C.POINTER(_d)]),
    "sp_parareal_create": (_i, [_vp, C.POINTER(SpPararealCfg), C.POINTER(_vp)]),
    "sp_parareal_destroy": (_i, [_vp]),
    "sp_parareal_do_parallel": (_i, [_vp, _vp, _vp, _vp, C.POINTER(SpPararealReport)]),
    "sp_parareal_do_serial": (_i, [_vp, _vp, _vp]),
    "sp_parareal_set_host_loop": (_i, [_vp, _i]),
    "sp_adjoint_rk4": (_i, [_vp, _vp, _vp, _vp, _d, _d, _i, _i, C.POINTER(_d), _vp, C.POINTER(_d)]),
    "sp_last_error": (C.c_char_p, []),
    "sp_abi_version": (_i, []),
    "sp_launch_count": (_ll, []),
    "sp_tuned_config": (_i, [_vp, _i, _i, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "sp_autotune": (_i, [_vp, _i, _i]),
    "sp_set_tune": (_i, [_vp, _i, _i, _i, _i, _i]),
    "sp_kernel_times": (_i, [_vp, _vp, C.c_double, _i, _i, C.POINTER(C.c_float), C.POINTER(_i)]),
    "sp_selftest_wait_timeout": (_i, [_vp, C.c_double]),
    "sp_store_violations": (_i, [C.POINTER(_i), C.POINTER(C.c_longlong)]),
    "sp_do_rk4_noalloc": (_i, [C.POINTER(SpParams), _vp, _vp, _d, _d, _i, _vp]),
    "sp_parareal_window_begin": (_i, [_vp, _vp]),
    "sp_parareal_window_fine": (_i, [_vp, _i]),
    "sp_parareal_window_coarse": (_i, [_vp, _i, _vp, _vp, C.POINTER(_d)]),
    "sp_parareal_batch_create": (_i, [C.POINTER(_vp), _i, C.POINTER(_vp)]),
    "sp_parareal_batch_destroy": (_i, [_vp]),
    "sp_parareal_batch_set_host_loop": (_i, [_vp, _i]),
    "sp_parareal_batch_run": (_i, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                                   C.POINTER(SpPararealReport), C.POINTER(_d)]),
}


def lib():
    """Loads the shared library (raises ImportError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m stencilparareal_b200.build` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return lib().sp_last_error().decode(errors="replace")


def check(rc: int) -> None:
    if rc != SP_OK:
        raise SpError(rc, last_error())


def exported_symbols():
    return list(_SIGS)
