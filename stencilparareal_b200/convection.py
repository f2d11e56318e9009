"""Python mirror of the reference's propagator interface.

``Convection`` follows class Convection of andyspiros/StencilParareal
(src/Convection/Convection.h:22-108): same constructor arguments
``(isize, jsize, ksize, dx, nu0, nufreq, cx, cy, cz)`` and the same methods
``DoRK4``, ``DoEuler``, ``DoRK4Timestep``, ``DoEulerTimestep`` with the same
argument order and meaning.  ``ConvectionField`` plays the role of the
reference's ConvectionField (Convection.h:13-20): a device field with a 2-cell
halo.  All work runs in ``libstencilparareal.so`` on the GPU; PyTorch only
provides the device memory.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L


def layout(ni: int, nj: int, nk: int, precision: int = L.SP_F64) -> L.SpLayout:
    out = L.SpLayout()
    L.check(L.lib().sp_field_layout(ni, nj, nk, precision, C.byref(out)))
    return out


class ConvectionField:
    """A field in the library's HBM layout (interior + periodic halo of 2)."""

    def __init__(self, ni: int, nj: int, nk: int, precision: int = L.SP_F64, device="cuda:0", name: str = ""):
        self.ni, self.nj, self.nk = ni, nj, nk
        self.precision = precision
        self.name = name
        self.layout = layout(ni, nj, nk, precision)
        dtype = torch.float64 if precision == L.SP_F64 else torch.float32
        self.data = torch.zeros(self.layout.total, dtype=dtype, device=device)

    @property
    def ptr(self) -> int:
        return self.data.data_ptr()

    @property
    def dtype(self):
        return self.data.dtype

    def interior(self) -> torch.Tensor:
        """View of the interior cells, shape (nk, nj, ni) (i fastest)."""
        lay = self.layout
        return torch.as_strided(self.data, (self.nk, self.nj, self.ni), (lay.plane, lay.px, 1), lay.origin)

    def element_offset(self, i: int, j: int, k: int) -> int:
        lay = self.layout
        return lay.origin + k * lay.plane + j * lay.px + i


class Convection:
    """class Convection (Convection.h:22-108) on one B200."""

    def __init__(self, isize: int, jsize: int, ksize: int, dx: float, nu0: float, nufreq: float,
                 cx: float, cy: float, cz: float, upwind: bool = True, device: int = 0):
        self.params = L.SpParams(isize, jsize, ksize, dx, nu0, nufreq, cx, cy, cz, 1 if upwind else 0)
        self.device = device
        h = C.c_void_p()
        L.check(L.lib().sp_convection_create(C.byref(self.params), device, C.byref(h)))
        self._h = h
        # The library works on its own torch-created stream; every call below
        # is ordered after the work already queued on torch's current stream
        # and makes that stream wait for it (fields are torch allocations).
        self.stream = torch.cuda.Stream(device)
        L.check(L.lib().sp_convection_set_stream(self._h, C.c_void_p(self.stream.cuda_stream)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            L.lib().sp_convection_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- helpers ---------------------------------------------------------------
    def field(self, precision: int = L.SP_F64, name: str = "") -> ConvectionField:
        p = self.params
        return ConvectionField(p.ni, p.nj, p.nk, precision, device=f"cuda:{self.device}", name=name)

    def set_stream(self, stream):
        """Enqueue the library's work on this (non-default) torch.cuda.Stream."""
        self.stream = stream
        L.check(L.lib().sp_convection_set_stream(self._h, C.c_void_p(stream.cuda_stream)))

    def call(self, fn, *args):
        """Runs one C-ABI call ordered with torch's current stream; raises on error."""
        cur = torch.cuda.current_stream(self.device)
        if cur.cuda_stream != self.stream.cuda_stream:
            self.stream.wait_stream(cur)
        rc = fn(*args)
        if cur.cuda_stream != self.stream.cuda_stream:
            cur.wait_stream(self.stream)
        L.check(rc)

    def synchronize(self):
        self.call(L.lib().sp_convection_synchronize, self._h)

    def _prec_check(self, f: ConvectionField, precision: int):
        if f.precision != precision:
            raise TypeError("field precision does not match the call")
        p = self.params
        if (f.ni, f.nj, f.nk) != (p.ni, p.nj, p.nk):
            raise ValueError("field grid does not match the propagator")

    # -- the reference's interface -------------------------------------------
    def DoRK4(self, inputField: ConvectionField, outputField: ConvectionField, tStart: float, dt: float,
              timesteps: int):
        """Convection::DoRK4 (Convection.cpp:292-303)."""
        for f in (inputField, outputField):
            self._prec_check(f, f.precision)
        if inputField.precision != outputField.precision:
            raise TypeError("input and output precision differ")
        fn = L.lib().sp_do_rk4 if inputField.precision == L.SP_F64 else L.lib().sp_do_rk4_f32
        self.call(fn, self._h, C.c_void_p(inputField.ptr), C.c_void_p(outputField.ptr), tStart, dt, int(timesteps))

    def DoEuler(self, inputField: ConvectionField, outputField: ConvectionField, tStart: float, dt: float,
                timesteps: int):
        """Convection::DoEuler (Convection.cpp:305-316)."""
        if inputField.precision != outputField.precision:
            raise TypeError("input and output precision differ")
        fn = L.lib().sp_do_euler if inputField.precision == L.SP_F64 else L.lib().sp_do_euler_f32
        self.call(fn, self._h, C.c_void_p(inputField.ptr), C.c_void_p(outputField.ptr), tStart, dt, int(timesteps))

    def DoRK4Timestep(self, inputField: ConvectionField, outputField: ConvectionField, t: float, dt: float):
        """Convection::DoRK4Timestep (Convection.cpp:318-370)."""
        self.DoRK4(inputField, outputField, t, dt, 1)

    def DoEulerTimestep(self, inputField: ConvectionField, outputField: ConvectionField, t: float, dt: float):
        """Convection::DoEulerTimestep (Convection.cpp:372-392)."""
        self.DoEuler(inputField, outputField, t, dt, 1)

    # -- fields <-> dense arrays ----------------------------------------------
    def Periodicity(self, f: ConvectionField):
        """Periodicity<T>::Apply (Periodicity.h:60-66) on a field, in place."""
        self.call(L.lib().sp_periodicity_apply, self._h, C.c_void_p(f.ptr), f.precision)

    def upload(self, f: ConvectionField, dense) -> ConvectionField:
        """Fills f from a dense (nk, nj, ni) array (numpy or torch) and its halo."""
        want = np.float64 if f.precision == L.SP_F64 else np.float32
        if isinstance(dense, torch.Tensor) and dense.is_cuda:
            d = dense.to(f.dtype).contiguous()
            self.call(L.lib().sp_field_import, self._h, C.c_void_p(d.data_ptr()), C.c_void_p(f.ptr), f.precision, 0)
            self.synchronize()
        else:
            a = np.ascontiguousarray(np.asarray(dense, dtype=want))
            assert a.shape == (f.nk, f.nj, f.ni), a.shape
            self.call(L.lib().sp_field_import, self._h, C.c_void_p(a.ctypes.data), C.c_void_p(f.ptr), f.precision, 1)
            self.synchronize()
        return f

    def download(self, f: ConvectionField) -> np.ndarray:
        """Dense (nk, nj, ni) copy of the interior of f."""
        want = np.float64 if f.precision == L.SP_F64 else np.float32
        out = np.empty((f.nk, f.nj, f.ni), dtype=want)
        self.call(L.lib().sp_field_export, self._h, C.c_void_p(f.ptr), C.c_void_p(out.ctypes.data), f.precision, 1)
        return out

    def errors(self, a: ConvectionField, b: ConvectionField):
        """(max|a-b|/max|a|, ||a-b||/||b||) over the interior, computed on the GPU."""
        em, el = C.c_double(), C.c_double()
        self.call(L.lib().sp_field_errors, self._h, C.c_void_p(a.ptr), C.c_void_p(b.ptr), C.byref(em), C.byref(el))
        return em.value, el.value

    def DoRK4Host(self, q_in: np.ndarray, tStart: float, dt: float, timesteps: int) -> np.ndarray:
        """Host-buffer DoRK4: dense FP64 arrays in and out (copies inside the call)."""
        a = np.ascontiguousarray(q_in, dtype=np.float64)
        out = np.empty_like(a)
        self.call(L.lib().sp_do_rk4_host, self._h, C.c_void_p(a.ctypes.data), C.c_void_p(out.ctypes.data),
                  tStart, dt, int(timesteps))
        return out

    # -- tuning ----------------------------------------------------------------
    def set_tune(self, precision: int, batch: int, ty: int, zchunk: int, kind: int):
        """kind: 0 direct loads, 1 TMA/mbarrier pipeline (single-stage kernels);
        2 fused stage pairs for FP64 RK4 steps on 64-column tiles (ty 8 or 16); 4 the
        same on 32 x 16 tiles (ty 16); 3 the cluster-resident path for FP64 RK4
        propagations of small fields, the field split into z-slabs, 5 the same
        split into (y,z) blocks (ty and zchunk unused)."""
        L.check(L.lib().sp_set_tune(self._h, precision, batch, ty, zchunk, int(kind)))

    def autotune(self, precision: int = L.SP_F64, batch: int = 1):
        self.call(L.lib().sp_autotune, self._h, precision, batch)
        return self.tuned_configs(precision, batch)

    def tuned_config(self, precision: int = L.SP_F64, batch: int = 1, op: int = 1):
        """Launch shape of stage kernel `op` (0..3 RK4 S1..S4, 4 Euler; 9, 10 the
        fused pairs 1+2 and 3+4, whose kind is 2 when RK4 steps run fused)."""
        ty, zc, tma = C.c_int(), C.c_int(), C.c_int()
        L.check(L.lib().sp_tuned_config(self._h, precision, batch, op, C.byref(ty), C.byref(zc), C.byref(tma)))
        return {"ty": ty.value, "zchunk": zc.value, "kind": tma.value}

    def kernel_times(self, field: ConvectionField, dt: float, reps: int = 10, path: str = "tuned"):
        """Average ms of each kernel of an FP64 RK4 step (CUDA events on the
        library's stream), run on a copy of `field`: {"P12", "P34"} for the fused
        pairs, {"S1".."S4"} for the stage kernels.  path: "tuned" (what DoRK4
        runs), "stages" or "pairs"."""
        ms = (C.c_float * 4)()
        cnt = C.c_int()
        code = {"tuned": 0, "stages": 1, "pairs": 2}[path]
        self.call(L.lib().sp_kernel_times, self._h, C.c_void_p(field.ptr), dt, reps, code, ms, C.byref(cnt))
        names = ("P12", "P34") if cnt.value == 2 else ("S1", "S2", "S3", "S4")
        return {k: float(ms[i]) for i, k in enumerate(names)}

    def tuned_configs(self, precision: int = L.SP_F64, batch: int = 1):
        names = {0: "S1", 1: "S2", 2: "S3", 3: "S4", 4: "euler", 9: "P12", 10: "P34", 11: "cluster"}
        return {name: self.tuned_config(precision, batch, op) for op, name in names.items()}


def launch_count() -> int:
    return int(L.lib().sp_launch_count())
