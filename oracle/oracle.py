"""ctypes wrapper of the CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``.  The oracle is a CPU restatement
of the reference's FP64 OpenMP path (andyspiros/StencilParareal,
src/Convection/Convection.cpp, ConvectionFunctions.h,
src/Communication/Periodicity.cpp, src/Parareal/Parareal.h); see
``sp_oracle.h`` for the function-by-function citations.

Arrays are numpy arrays of shape ``(nk, nj, ni)`` in C order, i.e. i fastest,
the same dense layout the product library uses for host import/export.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

COARSE_EULER_F64 = 0
COARSE_RK4_F64 = 1
COARSE_RK4_F32 = 2
COARSE_EULER_F32 = 3


class OrcParams(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int),
                ("dx", C.c_double), ("nu0", C.c_double), ("nufreq", C.c_double),
                ("cx", C.c_double), ("cy", C.c_double), ("cz", C.c_double),
                ("upwind", C.c_int)]


class OrcPararealCfg(C.Structure):
    _fields_ = [("endTime", C.c_double), ("timeSlices", C.c_int),
                ("timeStepsFine", C.c_int), ("timeStepsCoarse", C.c_int),
                ("kmax", C.c_int), ("async_", C.c_int), ("coarse", C.c_int), ("coarse_delta", C.c_int)]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        d, i, P = C.c_double, C.c_int, C.POINTER
        dp, fp = P(C.c_double), P(C.c_float)
        L.orc_set_threads.argtypes = [i]
        L.orc_get_threads.restype = i
        for name, ptr in (("orc_rk4", dp), ("orc_euler", dp), ("orc_rk4_f32", fp), ("orc_euler_f32", fp)):
            fn = getattr(L, name)
            fn.argtypes = [P(OrcParams), ptr, ptr, d, d, i]
            fn.restype = i
        for name in ("orc_rhs4", "orc_rhs2"):
            fn = getattr(L, name)
            fn.argtypes = [P(OrcParams), dp, dp, d]
            fn.restype = i
        L.orc_periodicity_jik.argtypes = [i, i, i, dp]
        L.orc_periodicity_jik.restype = i
        L.orc_parareal_derived.argtypes = [P(OrcPararealCfg), P(C.c_int), dp]
        L.orc_parareal_derived.restype = i
        L.orc_parareal.argtypes = [P(OrcParams), P(OrcPararealCfg), dp, dp, dp, dp, dp]
        L.orc_parareal.restype = i
        L.orc_parareal_ex.argtypes = [P(OrcParams), P(OrcPararealCfg), dp, dp, dp, dp, dp, dp, dp]
        L.orc_parareal_ex.restype = i
        L.orc_rk4_session_create.argtypes = [P(OrcParams), dp]
        L.orc_rk4_session_create.restype = C.c_void_p
        L.orc_rk4_session_run.argtypes = [C.c_void_p, d, d, i]
        L.orc_rk4_session_run.restype = i
        L.orc_rk4_session_result.argtypes = [C.c_void_p, dp]
        L.orc_rk4_session_result.restype = i
        L.orc_rk4_session_destroy.argtypes = [C.c_void_p]
        L.orc_rk4_session_destroy.restype = None
        L.orc_adjoint_rk4.argtypes = [P(OrcParams), dp, dp, d, d, i, dp, dp, dp]
        L.orc_adjoint_rk4.restype = i
        L.orc_exactq.argtypes = [d] * 9
        L.orc_exactq.restype = d
        L.orc_fillq.argtypes = [P(OrcParams), d, dp]
        L.orc_fillq.restype = i
        L.orc_error_maxrel.argtypes = [dp, dp, C.c_long]
        L.orc_error_maxrel.restype = d
        L.orc_error_l2rel.argtypes = [dp, dp, C.c_long]
        L.orc_error_l2rel.restype = d
        _lib = L
    return _lib


def params(n, dx=None, nu0=1.0, nufreq=0.0, cx=1.0, cy=1.0, cz=1.0, upwind=True) -> OrcParams:
    ni, nj, nk = (n, n, n) if np.isscalar(n) else tuple(n)
    if dx is None:
        dx = 1.0 / ni
    return OrcParams(ni, nj, nk, dx, nu0, nufreq, cx, cy, cz, 1 if upwind else 0)


def _ptr(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


def _check(rc, what):
    if rc != 0:
        raise ValueError(f"oracle {what} failed with status {rc}")


def _shape(p):
    return (p.nk, p.nj, p.ni)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def _prop(name, p, q, t0, dt, n, dtype):
    q = np.ascontiguousarray(q, dtype=dtype)
    assert q.shape == _shape(p), (q.shape, _shape(p))
    out = q.copy()
    ct = C.c_double if dtype == np.float64 else C.c_float
    _check(getattr(lib(), name)(C.byref(p), _ptr(q, ct), _ptr(out, ct), t0, dt, int(n)), name)
    return out


def rk4(p, q, t0, dt, n):
    """Convection::DoRK4 (Convection.cpp:292-303), FP64."""
    return _prop("orc_rk4", p, q, t0, dt, n, np.float64)


def euler(p, q, t0, dt, n):
    """Convection::DoEuler (Convection.cpp:305-316), FP64."""
    return _prop("orc_euler", p, q, t0, dt, n, np.float64)


def rk4_f32(p, q, t0, dt, n):
    return _prop("orc_rk4_f32", p, q, t0, dt, n, np.float32)


def euler_f32(p, q, t0, dt, n):
    return _prop("orc_euler_f32", p, q, t0, dt, n, np.float32)


def rhs4(p, q, t=0.0):
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.empty_like(q)
    _check(lib().orc_rhs4(C.byref(p), _ptr(q), _ptr(out), t), "rhs4")
    return out


def rhs2(p, q, t=0.0):
    q = np.ascontiguousarray(q, dtype=np.float64)
    out = np.empty_like(q)
    _check(lib().orc_rhs2(C.byref(p), _ptr(q), _ptr(out), t), "rhs2")
    return out


def periodicity_jik(field):
    """Periodicity::Apply on a halo-padded JIK array of shape (nj+4, ni+4, nk+4)."""
    f = np.ascontiguousarray(field, dtype=np.float64).copy()
    nj, ni, nk = (s - 4 for s in f.shape)
    _check(lib().orc_periodicity_jik(ni, nj, nk, _ptr(f)), "periodicity")
    return f


def parareal_cfg(endTime, timeSlices, timeStepsFine, timeStepsCoarse, kmax, async_=False,
                 coarse=COARSE_EULER_F64, delta=False) -> OrcPararealCfg:
    return OrcPararealCfg(endTime, timeSlices, timeStepsFine, timeStepsCoarse, kmax,
                          1 if async_ else 0, coarse, 1 if delta else 0)


def parareal_derived(cfg):
    out = (C.c_int * 4)()
    dout = (C.c_double * 3)()
    _check(lib().orc_parareal_derived(C.byref(cfg), out, dout), "derived")
    return dict(tsFineTotal=out[0], tsCoarseTotal=out[1], tsFine=out[2], tsCoarse=out[3],
                dtFine=dout[0], dtCoarse=dout[1], timeSliceSize=dout[2])


def parareal(p, cfg, q0):
    """Parareal::DoSerial + DoParallel (Parareal.h:110-171,250-253), serially.

    Returns (q_parareal, q_serial, err_max[kmax], err_l2[kmax])."""
    q0 = np.ascontiguousarray(q0, dtype=np.float64)
    q = np.empty_like(q0)
    qs = np.empty_like(q0)
    k = max(cfg.kmax, 1)
    em = np.zeros(k)
    el = np.zeros(k)
    _check(lib().orc_parareal(C.byref(p), C.byref(cfg), _ptr(q0), _ptr(q), _ptr(qs), _ptr(em), _ptr(el)),
           "parareal")
    return q, qs, em[:cfg.kmax], el[:cfg.kmax]


def parareal_iters(p, cfg, q0):
    """orc_parareal_ex: Parareal with the per-iteration defect and last-slice fields.

    Returns (q_serial, err_max[kmax], err_l2[kmax], defect[kmax], q_iters[kmax, nk, nj, ni])."""
    q0 = np.ascontiguousarray(q0, dtype=np.float64)
    k = max(cfg.kmax, 1)
    q = np.empty_like(q0)
    qs = np.empty_like(q0)
    em, el, de = np.zeros(k), np.zeros(k), np.zeros(k)
    qi = np.empty((k,) + q0.shape)
    _check(lib().orc_parareal_ex(C.byref(p), C.byref(cfg), _ptr(q0), _ptr(q), _ptr(qs), _ptr(em), _ptr(el),
                                 _ptr(de), _ptr(qi)), "parareal_ex")
    n = cfg.kmax
    return qs, em[:n], el[:n], de[:n], qi[:n]


class RK4Session:
    """A propagator whose fields are allocated and loaded once (orc_rk4_session):
    run() performs DoRK4(in, out, t0, dt, n) on the held fields, timing only the
    steps, as the reference's drivers time DoRK4 on fields they allocated
    up front (src/Parareal/main.cpp:187-189,218-222)."""

    def __init__(self, p, q):
        self._p = p
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.shape == _shape(p), (q.shape, _shape(p))
        self._h = lib().orc_rk4_session_create(C.byref(p), _ptr(q))
        if not self._h:
            raise ValueError("oracle session create failed")

    def run(self, t0, dt, n):
        _check(lib().orc_rk4_session_run(self._h, t0, dt, int(n)), "session run")

    def result(self):
        out = np.empty(_shape(self._p))
        _check(lib().orc_rk4_session_result(self._h, _ptr(out)), "session result")
        return out

    def close(self):
        if self._h:
            lib().orc_rk4_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def adjoint_rk4(p, q0, q_target, t0, dt, n):
    """Discrete adjoint of n RK4 steps for J = 0.5||q_n - q_target||^2.

    Returns (J, dJ/dq0, [dJ/dnu0, dJ/dcx, dJ/dcy, dJ/dcz])."""
    q0 = np.ascontiguousarray(q0, dtype=np.float64)
    qt = np.ascontiguousarray(q_target, dtype=np.float64)
    g = np.empty_like(q0)
    gp = np.zeros(4)
    J = C.c_double(0.0)
    _check(lib().orc_adjoint_rk4(C.byref(p), _ptr(q0), _ptr(qt), t0, dt, int(n), C.byref(J), _ptr(g),
                                 _ptr(gp)), "adjoint")
    return J.value, g, gp


def exactq(nu0, nufreq, cx, cy, cz, x, y, z, t):
    return lib().orc_exactq(nu0, nufreq, cx, cy, cz, x, y, z, t)


def fillq(p, t):
    out = np.empty(_shape(p))
    _check(lib().orc_fillq(C.byref(p), t, _ptr(out)), "fillq")
    return out


def error_maxrel(f, r):
    f = np.ascontiguousarray(f, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    return lib().orc_error_maxrel(_ptr(f), _ptr(r), f.size)


def error_l2rel(f, r):
    f = np.ascontiguousarray(f, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    return lib().orc_error_l2rel(_ptr(f), _ptr(r), f.size)
