"""Python mirror of the reference's Parareal driver and its configuration.

``RuntimeConfiguration`` keeps the getters, defaults and step rounding of
src/Parareal/RuntimeConfiguration.{h,cpp} (defaults RuntimeConfiguration.cpp:7-13,
rounding :133-151, derived values RuntimeConfiguration.h:54-111); the number of
time slices, which the reference takes from the MPI communicator size
(RuntimeConfiguration.cpp:15), is an explicit argument here.

``Parareal`` follows template class Parareal (src/Parareal/Parareal.h:38-289):
constructed from a propagator, the initial and solution fields, the start
time and a configuration; ``DoParallel`` and ``DoSerial`` keep their meaning.
All P slices run on one GPU inside ``libstencilparareal.so``: the fine runs of
all slices are batched per RK stage, the coarse sweep runs slice by slice and
the correction writes straight into the next slice's input, which replaces
the MPI ring of Parareal.h:122-162.
"""
from __future__ import annotations

import ctypes as C
import math

from . import _lib as L
from .convection import Convection, ConvectionField

MODES = ("compare", "serial", "parallel", "timing")


class RuntimeConfiguration:
    def __init__(self, timeSlices: int = 1, nu0: float = 1.0, nufreq: float = 0.0, cx: float = 1.0,
                 cy: float = 1.0, cz: float = 1.0, gridSize: int = 32, endTime: float = 0.05,
                 timeStepsFine: int = 128, timeStepsCoarse: int = 32, kmax: int = 5, mat: bool = False,
                 async_: bool = True, mode: str = "compare"):
        if timeSlices < 1:
            raise ValueError("timeSlices must be >= 1")
        self._nu0, self._nufreq = nu0, nufreq
        self._cx, self._cy, self._cz = cx, cy, cz
        self._gridSize, self._endTime = gridSize, endTime
        self._timeSlices = timeSlices
        self._kmax, self._mat, self._async = kmax, mat, async_
        m = mode.lower()
        self._mode = m if m in MODES else "compare"  # unknown modes fall back to Compare (RuntimeConfiguration.cpp:125-130)
        # RuntimeConfiguration.cpp:133-151: round totals up to a multiple of the slice count
        if timeStepsFine % timeSlices != 0:
            timeStepsFine = (timeStepsFine // timeSlices + 1) * timeSlices
        if timeStepsCoarse % timeSlices != 0:
            timeStepsCoarse = (timeStepsCoarse // timeSlices + 1) * timeSlices
        self._timeStepsFine, self._timeStepsCoarse = timeStepsFine, timeStepsCoarse

    # getters (RuntimeConfiguration.h:19-31)
    def nu0(self): return self._nu0
    def nufreq(self): return self._nufreq
    def cx(self): return self._cx
    def cy(self): return self._cy
    def cz(self): return self._cz
    def timeSlices(self): return self._timeSlices
    def timeStepsFine(self): return self._timeStepsFine
    def timeStepsCoarse(self): return self._timeStepsCoarse
    def gridSize(self): return self._gridSize
    def endTime(self): return self._endTime
    def kmax(self): return self._kmax
    def mat(self): return self._mat
    def async_(self): return self._async
    def mode(self): return self._mode

    # derived (RuntimeConfiguration.h:54-111)
    def dx(self): return 1.0 / self._gridSize
    def dtFine(self): return self._endTime / self._timeStepsFine
    def dtCoarse(self): return self._endTime / self._timeStepsCoarse
    def timeStepsFinePerTimeSlice(self): return self._timeStepsFine // self._timeSlices
    def timeStepsCoarsePerTimeSlice(self): return self._timeStepsCoarse // self._timeSlices
    def timeSliceSize(self): return self._endTime / self._timeSlices
    def cflFine(self): return self._cfl(self.dtFine())
    def cflCoarse(self): return self._cfl(self.dtCoarse())

    def _cfl(self, dt):
        c = max(self._cx, self._cy, self._cz)
        dt_dx = dt / self.dx()
        return max(1.5 * self._nu0 * dt_dx / self.dx(), c * dt_dx)


class Parareal:
    """template class Parareal (Parareal.h:38-289), all slices on one GPU.

    Extra knobs beyond the reference: ``coarse`` ('euler' = the reference's
    DoEuler, or 'rk4'), ``coarse_precision`` ('f64' or 'f32'), a stopping
    tolerance ``tol`` on the relative L2 defect (``tol_kind='defect'``) or on
    the error against a given reference field (``tol_kind='reference'``), and
    ``skip_converged`` (slices < k are exact after k iterations; their fine
    runs are skipped -- the results are bit-identical) and ``coarse_delta``:
    the correction as U = F(old) + G(new - old) instead of the reference's
    G(new) + F(old) - G(old) (equal for this linear G).  Applied to the FP64
    increment, an FP32 G no longer leaves its rounding noise (~1e-7) in the
    iterate; it is the default with ``coarse_precision='f32'``.
    """

    def __init__(self, propagator: Convection, initial: ConvectionField, solution: ConvectionField,
                 tStart: float, conf: RuntimeConfiguration, coarse: str = "euler", coarse_precision: str = "f64",
                 tol: float = 0.0, tol_kind: str = "none", skip_converged: bool = True,
                 coarse_delta: bool | None = None, first_slice: int = 0, slice_count: int = 0):
        self.prop = propagator
        self.initial = initial
        self.solution = solution
        self.tStart = tStart
        self.conf = conf
        cfg = L.SpPararealCfg()
        cfg.endTime = conf.endTime()
        cfg.timeSlices = conf.timeSlices()
        cfg.timeStepsFine = conf.timeStepsFine()
        cfg.timeStepsCoarse = conf.timeStepsCoarse()
        cfg.kmax = int(conf.kmax())
        cfg.async_ = 1 if conf.async_() else 0
        cfg.coarse_scheme = {"euler": L.SP_COARSE_EULER, "rk4": L.SP_COARSE_RK4}[coarse]
        cfg.coarse_precision = {"f64": L.SP_F64, "f32": L.SP_F32}[coarse_precision]
        cfg.tol_kind = {"none": L.SP_TOL_NONE, "defect": L.SP_TOL_DEFECT, "reference": L.SP_TOL_REFERENCE}[tol_kind]
        cfg.tol = tol
        cfg.skip_converged = 1 if skip_converged else 0
        if coarse_delta is None:  # increment form by default with an FP32 coarse propagator
            coarse_delta = coarse_precision == "f32"
        cfg.coarse_delta = 1 if coarse_delta else 0
        cfg.first_slice = int(first_slice)
        cfg.slice_count = int(slice_count)
        self.cfg = cfg
        h = C.c_void_p()
        L.check(L.lib().sp_parareal_create(propagator.handle, C.byref(cfg), C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            L.lib().sp_parareal_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def DoParallel(self, reference: ConvectionField | None = None) -> dict:
        """Parareal::DoParallel (Parareal.h:110-171); returns the run report."""
        rep = L.SpPararealReport()
        ref = C.c_void_p(reference.ptr) if reference is not None else None
        self.prop.call(L.lib().sp_parareal_do_parallel, self._h, C.c_void_p(self.initial.ptr),
                       C.c_void_p(self.solution.ptr), ref, C.byref(rep))
        k = rep.iterations
        return {"iterations": k, "tsFine": rep.tsFine, "tsCoarse": rep.tsCoarse, "dtFine": rep.dtFine,
                "dtCoarse": rep.dtCoarse, "timeSliceSize": rep.timeSliceSize,
                "defect": list(rep.defect[:k]), "err_l2": list(rep.err_l2[:k]), "err_max": list(rep.err_max[:k]),
                "seconds": rep.seconds, "seconds_fine": rep.seconds_fine, "seconds_coarse": rep.seconds_coarse,
                "fine_cell_updates": rep.fine_cell_updates}

    def set_host_loop(self, host_loop: bool):
        """Measurement switch: True runs DoParallel as one graph launch and one host
        synchronisation per iteration, False (default) all iterations in one launch
        with the stopping test on the device.  The fields are identical."""
        L.check(L.lib().sp_parareal_set_host_loop(self._h, 1 if host_loop else 0))

    def DoSerial(self):
        """Parareal::DoSerial (Parareal.h:250-253)."""
        self.prop.call(L.lib().sp_parareal_do_serial, self._h, C.c_void_p(self.initial.ptr),
                       C.c_void_p(self.solution.ptr))

    @staticmethod
    def max_speedup(tau_ratio: float, kmax: int, slices: int) -> float:
        """The reference's speedup model (src/Parareal/main.cpp:208-210)."""
        nit_np = kmax / slices
        return 1.0 / (tau_ratio * (1.0 + nit_np) + nit_np)


def slice_bounds(P: int, world: int, rank: int):
    """Contiguous slice range [lo, hi) of rank `rank` when P slices are spread over `world` GPUs."""
    base, extra = divmod(P, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def cfl_ok(conf: RuntimeConfiguration) -> bool:
    return math.isfinite(conf.cflFine())


def _report(rep) -> dict:
    k = rep.iterations
    return {"iterations": k, "tsFine": rep.tsFine, "tsCoarse": rep.tsCoarse, "dtFine": rep.dtFine,
            "dtCoarse": rep.dtCoarse, "timeSliceSize": rep.timeSliceSize, "defect": list(rep.defect[:k]),
            "err_l2": list(rep.err_l2[:k]), "err_max": list(rep.err_max[:k]),
            "fine_cell_updates": rep.fine_cell_updates}


class PararealBatch:
    """Many independent Parareal solves advanced together on one GPU.

    Each instance keeps its own grid, PDE parameters, slice count and step
    counts; one CUDA graph launch runs every iteration of all of them (the
    instances' iteration graphs are concurrent child graphs inside a
    conditional WHILE node) and an instance stops, on the device, once its
    tolerance is met, its kmax is used or it is exact (k = P).
    """

    def __init__(self, instances):
        self.instances = list(instances)
        n = len(self.instances)
        arr = (C.c_void_p * n)(*[p._h.value for p in self.instances])
        h = C.c_void_p()
        L.check(L.lib().sp_parareal_batch_create(arr, n, C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            L.lib().sp_parareal_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_host_loop(self, host_loop: bool):
        """Measurement switch, as Parareal.set_host_loop, for the whole batch."""
        L.check(L.lib().sp_parareal_batch_set_host_loop(self._h, 1 if host_loop else 0))

    def run(self, references=None):
        """Runs every instance from its `initial` into its `solution`; returns (reports, seconds)."""
        import torch
        torch.cuda.synchronize()
        n = len(self.instances)
        ini = (C.c_void_p * n)(*[p.initial.ptr for p in self.instances])
        sol = (C.c_void_p * n)(*[p.solution.ptr for p in self.instances])
        ref = None
        if references is not None:
            ref = (C.c_void_p * n)(*[(r.ptr if r is not None else None) for r in references])
        reps = (L.SpPararealReport * n)()
        secs = C.c_double(0.0)
        L.check(L.lib().sp_parareal_batch_run(self._h, ini, sol, ref, reps, C.byref(secs)))
        return [_report(r) for r in reps], secs.value


class WindowParareal(Parareal):
    """Slices [first, first+count) of a Parareal whose other slices live on other GPUs.

    The steps of one iteration follow one rank of the reference's ring
    (Parareal.h:116-165): fine(k) runs the window's batched fine sweep;
    coarse(k, u_first_new) takes the previous window's last slice result
    (the reference's MPI_Recv into qinitial), runs the coarse sweep and the
    corrections, and leaves the window's last slice result in `boundary` for
    the next window (the reference's MPI_Send).
    """

    def __init__(self, propagator, initial, solution, tStart, conf, first: int, count: int, **kw):
        super().__init__(propagator, initial, solution, tStart, conf, first_slice=first, slice_count=count, **kw)
        self.first, self.count = first, count
        self.boundary = propagator.field(name="boundary")

    def make_recv_buffer(self):
        return self.prop.field(name="inbound")

    def begin(self):
        self.prop.call(L.lib().sp_parareal_window_begin, self._h, C.c_void_p(self.initial.ptr))

    def fine(self, k: int):
        self.prop.call(L.lib().sp_parareal_window_fine, self._h, int(k))

    def coarse(self, k: int, u_first_new=None, want_defect: bool = True) -> float:
        d = C.c_double(0.0)
        inb = C.c_void_p(u_first_new.ptr) if u_first_new is not None else None
        self.prop.call(L.lib().sp_parareal_window_coarse, self._h, int(k), inb, C.c_void_p(self.boundary.ptr),
                       C.byref(d) if want_defect else None)
        return d.value


class DistributedParareal:
    """Parareal over the ranks of a torch.distributed group, one slice window per rank.

    Rank r owns slices slice_bounds(P, world, r).  Per iteration every rank
    runs its fine sweep, receives the previous rank's boundary field, runs its
    coarse sweep and sends its own boundary field to the next rank -- the
    reference's pipelined ring (Parareal.h:116-165) with windows of slices
    instead of single slices.  The window object provides begin/fine/coarse,
    a `boundary` payload and `make_recv_buffer()`; fields travel as CUDA
    tensors with NCCL and through host memory with gloo.
    """

    def __init__(self, window, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.w = window
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.gloo = dist.get_backend(group) == "gloo"

    def _payload(self, field):
        t = field.data if hasattr(field, "data") else field
        return t.cpu() if (self.gloo and t.is_cuda) else t

    def run(self, kmax: int, tol: float = 0.0):
        """Runs up to kmax iterations (stops early once the max defect over all ranks is below tol).
        Returns (iterations, per-iteration max defects)."""
        import torch
        dist, w = self.dist, self.w
        w.begin()
        recv_field = w.make_recv_buffer() if self.rank > 0 else None
        defects = []
        for k in range(kmax):
            w.fine(k)
            inbound = None
            if self.rank > 0:
                buf = self._payload(recv_field)
                # NCCL has no tags (messages between two ranks arrive in order)
                dist.recv(buf, src=self.rank - 1, group=self.group, tag=k if self.gloo else 0)
                if buf is not (recv_field.data if hasattr(recv_field, "data") else recv_field):
                    (recv_field.data if hasattr(recv_field, "data") else recv_field).copy_(buf)
                inbound = recv_field
            d = w.coarse(k, inbound)
            if self.rank < self.world - 1:
                dist.send(self._payload(w.boundary), dst=self.rank + 1, group=self.group, tag=k if self.gloo else 0)
            t = torch.tensor([d], dtype=torch.float64)
            if not self.gloo:
                t = t.cuda()
            dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
            defects.append(float(t.item()))
            if tol > 0 and defects[-1] < tol:
                return k + 1, defects
        return kmax, defects
