#!/usr/bin/env python
"""Benchmark of the fine propagator and the one-GPU Parareal driver.

Default workload (one "step"): the fine-propagator throughput configuration --
256^3 periodic grid, FP64 RK4, c=(1,0.5,0.25), nu=1e-3, dt=5e-5, 500 steps,
initial field a seeded sum of 8 Fourier modes (wavenumbers 1-4, N(0,1)
amplitudes).  Metric: cell-updates per second (one cell advanced one RK4
step), reported in GCUPS, whole job (all ranks), inputs resident in HBM.
Every field (134 MB) is larger than the 126 MB L2, so no flush is needed
between timed steps.

`e2e` repeats the same step through the host-buffer C-ABI call
sp_do_rk4_host: host->device copy of the dense initial field from pinned
memory, the 500 steps, device->host copy of the result, all inside the timed
region.

`--impl reference` times the CPU restatement of the reference's OpenMP path
(oracle/, the reference itself needs Boost and MPI and cannot be built here)
on the host cores on a bounded sample of the same workload.

At N=1 the line also carries the one-GPU Parareal (`parareal`), the batch of
uneven instances (`batch`), the adjoint (`adjoint`) and `paper`: the
reference's own published GPU experiment (128^3, 32768 RK4 steps; Parareal
with 128 slices and 3 iterations) timed on this GPU beside its published
times, the only workload of this path with published numbers.

Launch: python bench.py [--gpus N --steps K --warmup W]; N>1 under torchrun.
The headline value at N>1 is N independent replicas of the fine-propagator
step (the propagator does not shard: "weak" scaling with no collective on
its data path).  At N>1 the line also carries `parareal_pipeline`: the
one-GPU Parareal workload run as the reference's slice pipeline over all N
ranks (DistributedParareal: NCCL send/recv of one field per iteration and
rank boundary), timed on the device (max over ranks) beside the same problem
on one GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Parareal time-to-1e-8 vs serial FP64 fine on 1 B200; fine GCUPS and % HBM roofline"
UNIT = "GCUPS"
N_FINE = 256
STEPS_PER_RUN = 500
DT = 5e-5
NU = 1e-3
C = (1.0, 0.5, 0.25)
# Algorithmic HBM bytes per cell of each kernel of an RK4 step (FP64 field
# accesses x 8 B): fused pairs 1+2 (q -> y2, acc) and 3+4 (y2, q, acc -> q'),
# 56 B per cell-update, or the four single-stage kernels S1 (q -> y1),
# S2 (y1, q -> y2, acc), S3 (y2, q -> y3), S4 (y3, acc, q -> q'), 104 B.
KERNEL_BYTES = {"P12": 24, "P34": 32, "S1": 16, "S2": 32, "S3": 24, "S4": 32}
KERNEL_NAMES = {"P12": "k_rk4_pair<0,...> (RK4 stages 1+2)", "P34": "k_rk4_pair<1,...> (RK4 stages 3+4)",
                "S1": "k_stage_tma<double,0,...>", "S2": "k_stage_tma<double,1,...>",
                "S3": "k_stage_tma<double,2,...>", "S4": "k_stage_tma<double,3,...>"}
WORKLOAD = (f"fine RK4 FP64 {N_FINE}^3 x {STEPS_PER_RUN} steps, c=(1,0.5,0.25), nu=1e-3, dt=5e-5, "
            "8-mode Fourier IC seed 1")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def fourier_ic(n, seed=1):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ics import fourier_modes
    return fourier_modes(n, seed=seed)


def run_reference(args, rank, world):
    """The CPU restatement of the reference's OpenMP path on the host cores."""
    if rank != 0:
        return 0
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    n = N_FINE
    steps = 8  # bounded sample per step: 8 RK4 steps of the 256^3 workload (a few s on the host cores)
    p = O.params(n, dx=1.0 / n, nu0=NU, nufreq=0.0, cx=C[0], cy=C[1], cz=C[2])
    # the propagator and its fields are allocated and loaded once, outside the
    # timed region, as the reference's drivers construct Convection and the
    # fields before they time DoRK4 (src/Parareal/main.cpp:187-189,218-222)
    sess = O.RK4Session(p, fourier_ic(n))
    for _ in range(args.warmup):
        sess.run(0.0, DT, steps)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        sess.run(0.0, DT, steps)
        times.append(time.perf_counter() - t0)
    sess.close()
    tot = sum(times)
    val = n ** 3 * steps * args.steps / tot / 1e9
    line = {"metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "sample": f"{steps} RK4 steps of {n}^3 per step"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": O.get_threads(), "kind": "port",
                             "sample": f"{steps} RK4 steps of {n}^3 per timed step on fields allocated once, "
                                       f"{args.steps} steps"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample():
    from oracle import oracle as O
    O.build()
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    n, steps = N_FINE, 24
    p = O.params(n, dx=1.0 / n, nu0=NU, nufreq=0.0, cx=C[0], cy=C[1], cz=C[2])
    sess = O.RK4Session(p, fourier_ic(n))
    sess.run(0.0, DT, 1)  # untimed: first sweep over freshly mapped pages
    t0 = time.perf_counter()
    sess.run(0.0, DT, steps)
    dt = time.perf_counter() - t0
    sess.close()
    return {"value": n ** 3 * steps / dt / 1e9, "unit": UNIT, "cores": O.get_threads(), "kind": "port",
            "sample": f"{steps} RK4 steps of {n}^3 on fields allocated once (oracle restating the reference "
                      f"OpenMP path), {dt:.1f} s"}


def cpu_vs_gpu_times(torch, sp, device, gpu_serial_128_s=None):
    """CPU (oracle, all host cores) beside GPU times for the 32^3 serial fine run in full
    (1000 RK4 steps) and for the 128^3 serial fine propagator of the Parareal workload
    (20000 steps; CPU on 200 steps, extrapolated)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ics import gaussian_noise
    from oracle import oracle as O
    O.build()
    O.set_threads(os.cpu_count() or 1)
    out = {"cores": O.get_threads()}
    n, steps, dt = 32, 1000, 1e-4
    q0 = gaussian_noise(n, seed=0)
    p = O.params(n, nu0=0.01, cx=1.0, cy=1.0, cz=1.0)
    t0 = time.perf_counter()
    O.rk4(p, q0, 0.0, dt, steps)
    cpu = time.perf_counter() - t0
    conv = sp.Convection(n, n, n, 1.0 / n, 0.01, 0.0, 1.0, 1.0, 1.0, device=device)
    fi, fo = conv.field(), conv.field()
    conv.upload(fi, q0)
    gpu = {}
    for path, kind in (("stage_kernels", (4, 8, 1)), ("autotuned", None)):
        if kind:
            conv.set_tune(sp.SP_F64, 1, *kind)
        else:
            tuned = conv.autotune(sp.SP_F64, 1)
        conv.DoRK4(fi, fo, 0.0, dt, steps)
        conv.synchronize()
        t0 = time.perf_counter()
        conv.DoRK4(fi, fo, 0.0, dt, steps)
        conv.synchronize()
        gpu[path] = time.perf_counter() - t0
    out["serial_fine_32cube_1000_steps"] = {"what": "32^3, 1000 RK4 FP64 steps, dt=1e-4, c=(1,1,1), nu=0.01",
                                            "cpu_s": cpu, "gpu_s": gpu["autotuned"],
                                            "gpu_s_stage_kernels": gpu["stage_kernels"],
                                            "gpu_path": {3: "cluster-resident on z-slabs",
                                                         5: "cluster-resident on (y,z) blocks"}.get(
                                                tuned["cluster"]["kind"], "stage kernels / fused pairs")}
    n, sample, total = 128, 200, 20000
    p = O.params(n, nu0=0.01, cx=1.0, cy=1.0, cz=1.0)
    q0 = gaussian_noise(n, seed=0)
    t0 = time.perf_counter()
    O.rk4(p, q0, 0.0, 1e-5, sample)
    cpu = time.perf_counter() - t0
    out["serial_fine_128cube_20000_steps"] = {"what": "128^3, 20000 RK4 FP64 steps, dt=1e-5",
                                              "cpu_s_extrapolated": cpu * total / sample,
                                              "cpu_sample": f"{sample} of {total} steps in {cpu:.2f} s",
                                              "gpu_s": gpu_serial_128_s}
    return out


def parareal_summary(torch, sp, device):
    """Parareal on one GPU: 128^3, P=32, T=0.2, fine RK4 FP64 dt=1e-5, coarse RK4 FP32 (rounded to 7 steps/slice).

    Two stopping rules: "reference" stops once the last slice is within 1e-8
    relative L2 of the serial FP64 fine solution (the configuration's own
    criterion; a real run does not have that solution), "defect" stops once
    every slice end changed by less than 1e-8 relative L2 in the last
    iteration (what a user without the serial solution can run)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ics import gaussian_noise
    n, P, T = 128, 32, 0.2
    conv = sp.Convection(n, n, n, 1.0 / n, 0.01, 0.0, 1.0, 1.0, 1.0, device=device)
    conv.autotune(sp.SP_F64, 1)
    conv.autotune(sp.SP_F64, P)
    conv.autotune(sp.SP_F32, 1)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.01, gridSize=n, endTime=T, timeStepsFine=20000,
                                   timeStepsCoarse=200, kmax=8)
    q0, qs, q = conv.field(), conv.field(), conv.field()
    conv.upload(q0, gaussian_noise(n, seed=0))
    par = {rule: sp.Parareal(conv, q0, q, 0.0, conf, coarse="rk4", coarse_precision="f32", tol=1e-8,
                             tol_kind=rule, skip_converged=True) for rule in ("reference", "defect")}
    ser = sp.Parareal(conv, q0, qs, 0.0, conf)
    ser.DoSerial()  # warm (graphs)
    conv.synchronize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ser.DoSerial()
    conv.synchronize()
    t_serial = time.perf_counter() - t0
    out = {"config": "128^3, P=32, T=0.2, fine RK4 FP64 dt=1e-5 (625 steps/slice), coarse RK4 FP32 "
                     "dt=0.2/224 (200 rounded up to 224 total, 7 steps/slice), increment-form correction, "
                     "Gaussian+noise IC seed 0, c=(1,1,1), nu=0.01",
           "serial_fine_s": t_serial}
    for rule, pr in par.items():
        pr.DoParallel(reference=qs)  # warm (graph capture)
        rep = pr.DoParallel(reference=qs)
        # the same run with one graph launch and one host synchronisation per
        # iteration instead of all iterations in one launch
        pr.set_host_loop(True)
        pr.DoParallel(reference=qs)
        rep_host = pr.DoParallel(reference=qs)
        pr.set_host_loop(False)
        r = {"parareal_s": rep["seconds"], "iterations": rep["iterations"],
             "err_l2_vs_serial": rep["err_l2"][-1] if rep["err_l2"] else None,
             "defects": rep["defect"], "err_l2": rep["err_l2"],
             "speedup_vs_serial": t_serial / rep["seconds"] if rep["seconds"] else None,
             "fine_s": rep["seconds_fine"], "coarse_s": rep["seconds_coarse"],
             "fine_gcups": rep["fine_cell_updates"] / rep["seconds_fine"] / 1e9 if rep["seconds_fine"] else None,
             "loop": "all iterations in one graph launch (conditional WHILE node, stopping test on the device)",
             "host_loop_s": rep_host["seconds"], "saved_by_one_launch_s": rep_host["seconds"] - rep["seconds"]}
        if rule == "reference":
            out.update(r)  # the configuration's own criterion: the headline fields
            out["stop_rule"] = "reference: last slice within 1e-8 rel. L2 of the serial FP64 fine solution"
        else:
            r["stop_rule"] = "defect: every slice end changed by < 1e-8 rel. L2 in the last iteration"
            out["defect_rule"] = r
    out["serial_fine_gcups"] = n ** 3 * 20000 / t_serial / 1e9
    return out


def paper_summary(torch, sp, device, P=128, kmax=3):
    """The reference's published GPU experiment, timed on this one GPU: 128^3,
    T=0.1, nu0=0.1, nufreq=0, c=(1,1,1), fine RK4 FP64 with 32768 steps, coarse
    upwind Euler FP64 with 2048 steps, the analytic field exactQ at t=0, no
    asynchronous first step, kmax=3 iterations without a tolerance
    (jobs/paperJobs/04-SpeedupGPU.job:42-48, 01-Convergence.job:51-57), P=128
    slices -- there one GPU per slice, here all slices on this GPU.  Published
    by the reference's job logs: the serial fine run took 191.0-191.1 s on one sm_35
    GPU (03-ReferenceGPU/run_4.log:24) and 896.7-912.0 s on 8 CPU threads
    (02-SpeedupThreads), Parareal with 128 slices 7.28 s on 128 GPUs
    (04-SpeedupGPU/runtime.dat:6), error after 3 iterations 1.73145e-07
    (01-Convergence/result.dat:5)."""
    from stencilparareal_b200.solution import fill_q
    n, nu0, T, tsF, tsC = 128, 0.1, 0.1, 32768, 2048
    conv = sp.Convection(n, n, n, 1.0 / n, nu0, 0.0, 1.0, 1.0, 1.0, device=device)
    conv.autotune(sp.SP_F64, 1)
    conv.autotune(sp.SP_F64, P)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=nu0, gridSize=n, endTime=T, timeStepsFine=tsF,
                                   timeStepsCoarse=tsC, kmax=kmax)
    q0, qs, q = conv.field(), conv.field(), conv.field()
    conv.upload(q0, fill_q(n, n, n, nu0, 0.0, 1.0, 1.0, 1.0, 0.0))
    ser = sp.Parareal(conv, q0, qs, 0.0, conf, coarse="euler", coarse_precision="f64")
    conv.synchronize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ser.DoSerial()
    conv.synchronize()
    t_serial = time.perf_counter() - t0
    par = sp.Parareal(conv, q0, q, 0.0, conf, coarse="euler", coarse_precision="f64")
    par.DoParallel(reference=qs)  # warm (graph capture)
    rep = par.DoParallel(reference=qs)
    pub_serial, pub_par = 191.0, 7.28
    return {"config": "reference paper experiment: 128^3, T=0.1, nu0=0.1, nufreq=0, c=(1,1,1), fine RK4 FP64 32768 "
                      "steps, coarse upwind Euler FP64 2048 steps, exactQ IC, kmax=3, P=128 slices on 1 GPU",
            "serial_fine_s": t_serial, "serial_fine_gcups": n ** 3 * tsF / t_serial / 1e9,
            "published_serial_fine_gpu_s": pub_serial, "published_serial_fine_cpu8_s": [896.7, 912.0],
            "serial_speedup_vs_published_gpu": pub_serial / t_serial,
            "parareal_s": rep["seconds"], "iterations": rep["iterations"],
            "err_max_vs_serial": rep["err_max"], "published_err_max_k3": 1.73145e-07,
            "published_parareal_128_gpus_s": pub_par, "parareal_1gpu_vs_published_128_gpus": pub_par / rep["seconds"],
            "speedup_vs_serial_same_gpu": t_serial / rep["seconds"]}


def batch_summary(torch, sp, device, n_inst=48, seed=2):
    """Batched uneven instances: 48 independent Parareal solves, grids drawn from {32,48,64,96}^3, nu log-uniform in
    [1e-4, 1e-2], c uniform in [-1,1]^3, 8-24 slices; T=0.05, fine RK4 FP64 dt=1e-5, coarse RK4 FP32
    dt=1e-3 (totals rounded up to a multiple of the slice count), tolerance 1e-8 relative L2 against
    each instance's serial FP64 fine solution ("reference" rule), and the same batch stopped by the
    1e-8 defect rule."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ics import gaussian_noise
    from stencilparareal_b200.parareal import PararealBatch
    rng = np.random.default_rng(seed)
    T = 0.05
    specs = []
    for i in range(n_inst):
        n = int(rng.choice([32, 48, 64, 96]))
        nu = float(10 ** rng.uniform(-4, -2))
        c = rng.uniform(-1, 1, size=3)
        P = int(rng.integers(8, 25))
        specs.append((n, nu, tuple(float(v) for v in c), P))
    tunes = {}
    inst = {"reference": [], "defect": []}
    refs, serial_s = [], 0.0
    for i, (n, nu, c, P) in enumerate(specs):
        conv = sp.Convection(n, n, n, 1.0 / n, nu, 0.0, *c, device=device)
        if n not in tunes:
            a64 = conv.autotune(sp.SP_F64, 16)
            # the cluster-resident path or the fused stage pairs when the tuner
            # preferred them, else the stage kernels' shape
            t64 = (a64["cluster"] if a64["cluster"]["kind"] in (3, 5) else
                   a64["P12"] if a64["P12"]["kind"] in (2, 4) else a64["S2"])
            tunes[n] = (t64, conv.autotune(sp.SP_F32, 1)["S2"])
        t64, t32 = tunes[n]
        conv.set_tune(sp.SP_F64, P, t64["ty"], t64["zchunk"], t64["kind"])
        conv.set_tune(sp.SP_F32, 1, t32["ty"], t32["zchunk"], t32["kind"])
        conf = sp.RuntimeConfiguration(timeSlices=P, nu0=nu, gridSize=n, endTime=T, timeStepsFine=5000,
                                       timeStepsCoarse=50, kmax=P)
        f0, fs, fr, fd = conv.field(), conv.field(), conv.field(), conv.field()
        conv.upload(f0, gaussian_noise(n, seed=seed + i))
        ser = sp.Parareal(conv, f0, fr, 0.0, conf)
        t0 = time.perf_counter()
        ser.DoSerial()
        conv.synchronize()
        serial_s += time.perf_counter() - t0
        for rule, sol in (("reference", fs), ("defect", fd)):
            inst[rule].append(sp.Parareal(conv, f0, sol, 0.0, conf, coarse="rk4", coarse_precision="f32", tol=1e-8,
                                          tol_kind=rule))
        refs.append(fr)
    out = {"config": f"{n_inst} instances, grids {{32,48,64,96}}^3, nu log-uniform [1e-4,1e-2], c U[-1,1]^3, "
                     "P 8-24, T=0.05, fine RK4 FP64 dt=1e-5, coarse RK4 FP32 dt=1e-3 (rounded per P), "
                     "increment-form correction, stop at 1e-8 rel L2 vs serial fine; seed 2",
           "instances": n_inst, "serial_fine_sum_s": serial_s,
           "grids": {str(k): sum(1 for s_ in specs if s_[0] == k) for k in (32, 48, 64, 96)},
           "tunes": {str(k): v[0] for k, v in tunes.items()}}
    for rule in ("reference", "defect"):
        batch = PararealBatch(inst[rule])
        batch.set_host_loop(True)
        batch.run(references=refs)
        _, secs_host = batch.run(references=refs)
        batch.set_host_loop(False)
        batch.run(references=refs)   # warm (first launch)
        reps, secs = batch.run(references=refs)
        fine_cu = sum(r["fine_cell_updates"] for r in reps)
        its = [r["iterations"] for r in reps]
        errs = [r["err_l2"][-1] for r in reps]
        r = {"batch_s": secs, "speedup_vs_serial_sum": serial_s / secs if secs else None,
             "iterations_max": max(its), "iterations_mean": sum(its) / len(its),
             "err_l2_max": max(errs), "fine_gcups": fine_cu / secs / 1e9,
             "loop": "every iteration of every instance in one graph launch",
             "host_loop_s": secs_host, "saved_by_one_launch_s": secs_host - secs}
        if rule == "reference":
            out.update(r)
            out["stop_rule"] = "reference: within 1e-8 rel. L2 of each instance's serial FP64 fine solution"
        else:
            r["stop_rule"] = "defect: every slice end changed by < 1e-8 rel. L2 in the last iteration"
            out["defect_rule"] = r
        del batch
    return out


def pipeline_summary(torch, sp, dist, rank, world, device, n=128, P=32, problem="config3"):
    """The Parareal slice pipeline over the ranks of the process group (one GPU
    each), rank r holding the slice window slice_bounds(P, world, r); per
    iteration every rank runs its batched fine sweep, receives the previous
    rank's boundary field (NCCL recv into its own HBM), runs its coarse sweep
    and corrections and sends its boundary field on (the reference's MPI ring,
    Parareal.h:116-165).  Time: CUDA events on each rank's library stream, max
    over ranks.  Rank 0 also times the same problem on its GPU alone
    (DoParallel, same stopping rule) for comparison.

    problem "config3": the one-GPU Parareal workload (n^3, P slices, T=0.2, fine
    RK4 FP64 dt=1e-5, coarse RK4 FP32, increment form), stopping once the
    defect over all ranks is below 1e-8.  problem "paper": the reference's
    published GPU experiment (n^3, T=0.1, nu0=0.1, 32768 fine RK4 and 2048
    coarse upwind-Euler FP64 steps, exactQ initial field, 3 iterations, no
    tolerance; jobs/paperJobs/04-SpeedupGPU.job:42-48), whose 128-slice run
    took 7.28 s on 128 GPUs (04-SpeedupGPU/runtime.dat:6)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ics import gaussian_noise
    from stencilparareal_b200.parareal import DistributedParareal, WindowParareal, slice_bounds
    from stencilparareal_b200.solution import fill_q
    paper = problem == "paper"
    if paper:
        nu0, T, tsF, tsC, kmax, tol = 0.1, 0.1, 32768, 2048, 3, 0.0
        coarse = dict(coarse="euler", coarse_precision="f64")
    else:
        nu0, T, tsF, tsC, kmax, tol = 0.01, 0.2, 20000, 200, 8, 1e-8
        coarse = dict(coarse="rk4", coarse_precision="f32")
    conv = sp.Convection(n, n, n, 1.0 / n, nu0, 0.0, 1.0, 1.0, 1.0, device=device)
    lo, hi = slice_bounds(P, world, rank)
    conv.autotune(sp.SP_F64, 1)
    conv.autotune(sp.SP_F64, hi - lo)
    if not paper:
        conv.autotune(sp.SP_F32, 1)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=nu0, gridSize=n, endTime=T, timeStepsFine=tsF,
                                   timeStepsCoarse=tsC, kmax=kmax)
    q_init = fill_q(n, n, n, nu0, 0.0, 1.0, 1.0, 1.0, 0.0) if paper else gaussian_noise(n, seed=0)
    f0, fs, fref = conv.field(), conv.field(), conv.field()
    conv.upload(f0, q_init)
    last = rank == world - 1
    if last:  # the serial fine solution, for the error of the result
        sp.Parareal(conv, f0, fref, 0.0, conf, **coarse).DoSerial()
    w = WindowParareal(conv, f0, fs, 0.0, conf, lo, hi - lo, **coarse)
    dp = DistributedParareal(w)
    dp.run(kmax, tol)  # warm: graph capture, communicator set-up
    conv.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(conv.stream)
    its, defects = dp.run(kmax, tol)
    e1.record(conv.stream)
    conv.synchronize()
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) * 1e-3
    err_max, err_l2 = conv.errors(w.boundary, fref) if last else (0.0, 0.0)
    t = torch.tensor([secs, err_max, err_l2], dtype=torch.float64,
                     device=f"cuda:{device}" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    secs_max, err_max, err_l2 = float(t[0]), float(t[1]), float(t[2])
    one_gpu_s = None
    if rank == 0:
        # the same problem on this GPU alone, for comparison
        c1 = sp.Convection(n, n, n, 1.0 / n, nu0, 0.0, 1.0, 1.0, 1.0, device=device)
        c1.autotune(sp.SP_F64, P)
        if not paper:
            c1.autotune(sp.SP_F32, 1)
        g0, g1 = c1.field(), c1.field()
        c1.upload(g0, q_init)
        stop = {} if paper else dict(tol=tol, tol_kind="defect")
        par = sp.Parareal(c1, g0, g1, 0.0, conf, **coarse, **stop)
        par.DoParallel()
        one_gpu_s = par.DoParallel()["seconds"]
    dist.barrier()
    if paper:
        cfg = (f"reference paper experiment: {n}^3, P={P}, T=0.1, nu0=0.1, c=(1,1,1), fine RK4 FP64 32768 steps, "
               f"coarse upwind Euler FP64 2048 steps (rounded up to a multiple of P), exactQ IC, 3 iterations")
        stop_rule = "fixed 3 iterations (kmax=3, no tolerance), as the reference's job"
    else:
        cfg = (f"{n}^3, P={P}, T=0.2, fine RK4 FP64 dt=1e-5, coarse RK4 FP32 (200 rounded up to a multiple "
               f"of P), increment form, Gaussian+noise IC seed 0, c=(1,1,1), nu=0.01")
        stop_rule = "defect < 1e-8 (max over ranks)"
    out = {"config": cfg + f"; slice windows {[slice_bounds(P, world, r) for r in range(world)]}",
           "ranks": world, "exchange": f"torch.distributed {dist.get_backend()} send/recv of one FP64 field "
                                       f"per iteration and rank boundary, MAX all-reduce of the defect",
           "stop_rule": stop_rule, "iterations": its, "defects": defects,
           "seconds": secs_max, "err_l2_vs_serial": err_l2, "err_max_vs_serial": err_max,
           "one_gpu_parareal_s": one_gpu_s,
           "speedup_vs_one_gpu": one_gpu_s / secs_max if one_gpu_s else None}
    if paper and n == 128 and P == 128:
        out["published_parareal_128_gpus_s"] = 7.28
    return out


def adjoint_summary(torch, sp, device):
    """Adjoint: gradient of 0.5||q(T)-q_target||^2 through 400 RK4 FP64 steps at 128^3, checkpoint 20."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ics import gaussian_noise
    from stencilparareal_b200.adjoint import misfit_gradient
    n, steps, dt = 128, 400, 5e-5
    conv = sp.Convection(n, n, n, 1.0 / n, 0.01, 0.0, 1.0, 1.0, 1.0, device=device)
    q0 = gaussian_noise(n, seed=0)
    f0, ft, fp, fo = conv.field(), conv.field(), conv.field(), conv.field()
    conv.upload(fp, q0 + 1e-2 * np.random.default_rng(3).uniform(-1, 1, size=q0.shape))
    conv.DoRK4(fp, ft, 0.0, dt, steps)
    conv.upload(f0, q0)
    misfit_gradient(conv, f0, ft, 0.0, dt, steps, checkpoint_every=20)  # warm
    conv.synchronize()
    t0 = time.perf_counter()
    J, g, gp = misfit_gradient(conv, f0, ft, 0.0, dt, steps, checkpoint_every=20)
    t_adj = time.perf_counter() - t0
    conv.DoRK4(f0, fo, 0.0, dt, steps)
    conv.synchronize()
    t0 = time.perf_counter()
    conv.DoRK4(f0, fo, 0.0, dt, steps)
    conv.synchronize()
    t_fwd = time.perf_counter() - t0
    return {"config": "128^3, 400 RK4 FP64 steps dt=5e-5, checkpoint every 20 steps, J=0.5||q(T)-q_target||^2",
            "J": J, "grad_nu_c": gp, "gradient_s": t_adj, "forward_s": t_fwd,
            "gradient_over_forward": t_adj / t_fwd}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-parareal", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-paper", action="store_true", help="skip the reference's published experiment (128^3, "
                                                            "32768 RK4 steps; Parareal P=128, kmax=3)")
    ap.add_argument("--tune", default="auto", help="'auto' or ty,zchunk,kind for the stage kernels")
    ap.add_argument("--profile", action="store_true",
                    help="profiling run: one DoRK4 of --profile-steps steps on the 256^3 workload (or a "
                         "--profile-grid cube with the Gaussian+noise field) with the given --tune, no timing")
    ap.add_argument("--profile-grid", type=int, default=N_FINE)
    ap.add_argument("--profile-steps", type=int, default=2)
    ap.add_argument("--profile-reps", type=int, default=1,
                    help="profiling run: DoRK4 calls; the line gives the wall time of the last")
    ap.add_argument("--no-pipeline", action="store_true", help="N>1: skip the Parareal slice pipeline")
    ap.add_argument("--pipeline-only", action="store_true",
                    help="N>1: run only the Parareal slice pipeline (prints its JSON object)")
    ap.add_argument("--pipeline-grid", type=int, default=128)
    ap.add_argument("--pipeline-slices", type=int, default=32)
    ap.add_argument("--pipeline-problem", default="config3", choices=["config3", "paper"],
                    help="N>1: the slice pipeline's problem: the one-GPU Parareal workload (128^3, P=32, defect "
                         "rule) or the reference's published experiment (use --pipeline-slices 128)")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="process-group backend for N>1 (gloo: exchange through host memory)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import stencilparareal_b200 as sp
    from stencilparareal_b200 import build as spbuild
    spbuild.build()

    dist = None
    device = local % max(torch.cuda.device_count(), 1)
    torch.cuda.set_device(device)
    if world > 1:
        import datetime
        import torch.distributed as dist
        kw = {"device_id": torch.device(f"cuda:{device}")} if args.dist_backend == "nccl" else {}
        dist.init_process_group(args.dist_backend, timeout=datetime.timedelta(seconds=120), **kw)
        if args.pipeline_only:
            out = pipeline_summary(torch, sp, dist, rank, world, device, args.pipeline_grid, args.pipeline_slices,
                                   args.pipeline_problem)
            if rank == 0:
                print(json.dumps({"parareal_pipeline": out}), flush=True)
            dist.barrier()
            dist.destroy_process_group()
            return 0
    n = args.profile_grid if args.profile else N_FINE
    conv = sp.Convection(n, n, n, 1.0 / n, NU, 0.0, C[0], C[1], C[2], device=device)
    if args.tune == "auto" and not args.profile:
        tune = conv.autotune(sp.SP_F64, 1)
    else:
        ty, zc, kind = (int(x) for x in (args.tune if args.tune != "auto" else "4,8,1").split(","))
        conv.set_tune(sp.SP_F64, 1, ty, zc, kind)
        tune = conv.tuned_configs(sp.SP_F64, 1)
    if n == N_FINE:
        q0 = fourier_ic(n)
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from ics import gaussian_noise
        q0 = gaussian_noise(n, seed=0)
    fin, fout = conv.field(), conv.field()
    conv.upload(fin, q0)
    if args.profile:
        secs = None
        for _ in range(max(1, args.profile_reps)):
            t0 = time.perf_counter()
            conv.DoRK4(fin, fout, 0.0, DT, args.profile_steps)
            conv.synchronize()
            secs = time.perf_counter() - t0
        what = (WORKLOAD.replace(f"x {STEPS_PER_RUN} steps", f"x {args.profile_steps} steps") if n == N_FINE
                else f"fine RK4 FP64 {n}^3 x {args.profile_steps} steps, Gaussian+noise IC seed 0")
        print(json.dumps({"profile": what, "tune": tune, "last_call_s": secs,
                          "gcups": n ** 3 * args.profile_steps / secs / 1e9}))
        return 0
    stream = conv.stream

    def one_step():
        conv.DoRK4(fin, fout, 0.0, DT, STEPS_PER_RUN)

    for _ in range(args.warmup):
        one_step()
    conv.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = sp.launch_count()
    with ClockSampler(device) as clk:
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                one_step()
            e1.record(stream)
        conv.synchronize()
        torch.cuda.synchronize()
    launches = sp.launch_count() - l0
    ms = e0.elapsed_time(e1)
    t_local = ms / 1e3
    if dist:
        t = torch.tensor([t_local], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
        dist.barrier()
    else:
        t_max = t_local
    cells = n ** 3 * STEPS_PER_RUN * args.steps
    value = cells * world / t_max / 1e9

    # e2e: host buffers through the C ABI (pinned), copies inside the timed region
    h_in = torch.from_numpy(q0).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    lib = sp._lib.lib()
    conv.call(lib.sp_do_rk4_host, conv.handle, h_in.data_ptr(), h_out.data_ptr(), 0.0, DT, STEPS_PER_RUN)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        conv.call(lib.sp_do_rk4_host, conv.handle, h_in.data_ptr(), h_out.data_ptr(), 0.0, DT, STEPS_PER_RUN)
    t_e2e = time.perf_counter() - t0
    if dist:
        t = torch.tensor([t_e2e], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = cells * world / t_e2e / 1e9

    peak, peak_kind = peaks()
    # roofline of the dominant kernel: its algorithmic bytes per launch over its
    # median launch time, every kernel of a step timed with CUDA events on the
    # library's stream
    ktimes = conv.kernel_times(fin, DT, reps=20)
    dom = max(ktimes, key=ktimes.get)
    alg_launch = KERNEL_BYTES[dom] * n ** 3
    achieved = alg_launch / (ktimes[dom] * 1e-3) / 1e9
    step_bytes = sum(KERNEL_BYTES[k] for k in ktimes)
    traffic_all = {}
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        try:
            with open(tp) as f:
                traffic_all = json.load(f)
        except Exception:
            traffic_all = {}

    def traffic_of(k):
        """ncu DRAM bytes per launch of kernel k as tuned (the pairs' traffic
        depends on their tile and range length); None where none was measured."""
        if k in ("P12", "P34"):
            sh = tune.get(k, {})
            tile = "32x16" if sh.get("kind") == 4 else f"64x{sh.get('ty', 8)}"
            return traffic_all.get("pairs_by_shape", {}).get(f"{tile}/z{sh.get('zchunk', 0)}", {}).get(k)
        return traffic_all.get("dram_bytes_per_launch", {}).get(k)
    traffic = traffic_of(dom)
    # both paths on the same field, for comparison: the four single-stage kernels
    # move 104 B per cell-update and are bound by HBM; the fused pairs move 56 B
    # and are bound on chip
    def path_roofline(kt):
        d = max(kt, key=kt.get)
        ach = KERNEL_BYTES[d] * n ** 3 / (kt[d] * 1e-3) / 1e9
        sb = sum(KERNEL_BYTES[k] for k in kt)
        tot = sum(kt.values()) * 1e-3
        return {"bound": "hbm", "kernel": KERNEL_NAMES[d], "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "traffic": traffic_of(d), "kernel_times_ms": kt,
                "algorithmic_bytes_per_cell_update": sb, "step_achieved_gbs": sb * n ** 3 / tot / 1e9,
                "step_frac": sb * n ** 3 / tot / 1e9 / peak, "step_gcups_from_kernel_times": n ** 3 / tot / 1e9}
    roofline_single = path_roofline(conv.kernel_times(fin, DT, reps=20, path="stages"))
    roofline_pairs = path_roofline(conv.kernel_times(fin, DT, reps=20, path="pairs"))
    # the timed region's step time split over the kernels by their timed shares
    step_ms = t_local / (STEPS_PER_RUN * args.steps) * 1e3
    dom_in_step = step_ms * ktimes[dom] / sum(ktimes.values())
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "l2": "inputs larger than L2 (each 256^3 FP64 field is 134 MB)",
                       "parallelism": f"replicas x{world}" + (", Parareal slice pipeline over "
                                                              f"{args.dist_backend}" if world > 1 else ""),
                       "tune": tune},
            "roofline": {"bound": "hbm", "kernel": KERNEL_NAMES[dom], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "traffic_unit": "dram bytes per launch (ncu, profiles/traffic.json)",
                         "algorithmic_bytes_per_launch": alg_launch, "kernel_ms": ktimes[dom],
                         "kernel_times_ms": ktimes, "algorithmic_bytes_per_cell_update": step_bytes,
                         "step_achieved_gbs": step_bytes * n ** 3 * STEPS_PER_RUN * args.steps / t_local / 1e9,
                         "kernel_ms_in_step": dom_in_step,
                         "achieved_in_step": alg_launch / (dom_in_step * 1e-3) / 1e9,
                         "frac_in_step": alg_launch / (dom_in_step * 1e-3) / 1e9 / peak,
                         "in_step_note": "timed region's step time x the kernel's share of the event-timed "
                                         "kernel times (launches overlap through programmatic dependent "
                                         "launch inside the step)",
                         # the whole step against the reference scheme's own traffic: 16 FP64 field
                         # accesses per cell-update (128 B) for its low-storage stage sequence
                         "step_equiv_128B_gbs": 128 * value / world,
                         "step_equiv_128B_frac": 128 * value / world / peak},
            "roofline_single_stage": roofline_single,
            "roofline_fused_pairs": roofline_pairs,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h_in.numel() * 8),
                    "d2h_bytes_per_step": int(h_out.numel() * 8)},
            "gpu_launches": int(launches), "clocks": clk.summary()}
    if rank == 0 and world == 1:
        if not args.no_parareal:
            for key, fn in (("parareal", parareal_summary), ("batch", batch_summary), ("adjoint", adjoint_summary)):
                try:
                    line[key] = fn(torch, sp, device)
                except Exception as ex:  # reported, not hidden
                    line[key] = {"error": repr(ex)}
        if not args.no_paper:
            try:
                line["paper"] = paper_summary(torch, sp, device)
            except Exception as ex:  # reported, not hidden
                line["paper"] = {"error": repr(ex)}
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_sample()
            try:
                line["cpu_vs_gpu"] = cpu_vs_gpu_times(torch, sp, device,
                                                      line.get("parareal", {}).get("serial_fine_s"))
            except Exception as ex:  # reported, not hidden
                line["cpu_vs_gpu"] = {"error": repr(ex)}
    if dist and not args.no_pipeline:
        # every rank takes part: the Parareal slice pipeline over the process group
        line["parareal_pipeline"] = pipeline_summary(torch, sp, dist, rank, world, device, args.pipeline_grid,
                                                     args.pipeline_slices, args.pipeline_problem)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
