"""Command-line drivers with the reference's option names, on the B200 library.

    python -m stencilparareal_b200.cli convection [--nu0 X --nufreq X --cx X --cy X --cz X
                                                   --gridSize N --timeSteps N --endTime T --cfl C --order 1|4 --mat]
        src/Convection/main.cpp: analytic initial field, DoRK4 (order 4) or DoEuler
        (order 1) to endTime, "Total relative error" against the analytic solution.

    python -m stencilparareal_b200.cli parareal --timeSlices P [--nu0 X --nufreq X --cx X --cy X --cz X
        --gridSize N --endTime T --timeStepsFine N --timeStepsCoarse N --kmax K --noasync
        --mode compare|serial|parallel|timing --coarse euler|rk4 --coarsePrecision f64|f32 --mat]
        src/Parareal/main.cpp: the four run modes.  The slice count, which the
        reference takes from the MPI communicator size, is --timeSlices; all slices
        run on one GPU.  Energy comes from NVML (the reference reads Cray counters).

    python -m stencilparareal_b200.cli findstable [--nu0 X --gridSize N --endTime T --order 1|4
                                                   --nufreqs 100,10,1 --minSteps N --maxSteps N]
        jobs/finalJobs/FindStable.sbatch: the convection driver over nufreq x timeSteps
        (doubling from minSteps to maxSteps), one table row per run with the maximum
        absolute and the relative error against the analytic solution.

    --mat writes the reference's MAT-v5 files into the working directory.
"""
from __future__ import annotations

import argparse
import math
import sys
import time

import numpy as np


def _energy_j(device: int):
    """Total energy of the GPU in joules from NVML, or None."""
    try:
        import pynvml
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByIndex(device)
        return pynvml.nvmlDeviceGetTotalEnergyConsumption(h) / 1000.0
    except Exception:
        return None


def convection_config(argv):
    """parseCommandLine of src/Convection/main.cpp:78-213 (defaults, --cfl logic)."""
    ap = argparse.ArgumentParser(prog="convection")
    for name in ("nu0", "nufreq", "cx", "cy", "cz", "endTime", "cfl"):
        ap.add_argument("--" + name, type=float)
    ap.add_argument("--gridSize", type=int)
    ap.add_argument("--timeSteps", type=int)
    ap.add_argument("--order", type=int, default=4)
    ap.add_argument("--mat", action="store_true")
    a = ap.parse_args(argv)
    if a.order not in (1, 4):
        raise SystemExit(f"Order {a.order} is not supported")
    c = dict(nu0=1.0, nufreq=0.0, cx=1.0, cy=1.0, cz=1.0, gridsize=32, timesteps=512, endtime=0.05, rk=a.order == 4,
             mat=a.mat)
    for k in ("nu0", "nufreq", "cx", "cy", "cz"):
        if getattr(a, k) is not None:
            c[k] = getattr(a, k)
    c["dx"] = 1.0 / c["gridsize"]
    c["dt"] = c["endtime"] / c["timesteps"]
    if a.endTime is not None:
        c["endtime"] = a.endTime
        c["dt"] = c["endtime"] / c["timesteps"]
    if a.cfl is not None and a.gridSize is not None and a.timeSteps is not None:
        raise SystemExit("Error: setting cfl, gridSize and timeSteps not allowed")
    if a.gridSize is not None:
        c["gridsize"] = a.gridSize
        c["dx"] = 1.0 / c["gridsize"]
    if a.timeSteps is not None:
        c["timesteps"] = a.timeSteps
        c["dt"] = c["endtime"] / c["timesteps"]
    if a.cfl is not None:
        if a.gridSize is not None:
            dt = c["dx"] ** 2 * a.cfl / (1.5 * c["nu0"])
            c["timesteps"] = int(c["endtime"] / dt + 0.5)
            c["dt"] = c["endtime"] / c["timesteps"]
        else:
            dx = math.sqrt(c["dt"] * c["nu0"] / a.cfl)
            c["gridsize"] = int(1.0 / dx + 0.5)
            c["dx"] = 1.0 / c["gridsize"]
    c["cfl"] = c["dt"] * 1.5 * c["nu0"] / (c["dx"] * c["dx"])
    return c


def run_convection(argv, out=sys.stdout) -> dict:
    import stencilparareal_b200 as sp
    from .solution import compute_error, fill_q
    c = convection_config(argv)
    n = c["gridsize"]
    conv = sp.Convection(n, n, n, c["dx"], c["nu0"], c["nufreq"], c["cx"], c["cy"], c["cz"])
    q_in, q_out = conv.field(), conv.field()
    conv.upload(q_in, fill_q(n, n, n, c["nu0"], c["nufreq"], c["cx"], c["cy"], c["cz"], 0.0))
    conv.synchronize()
    t0 = time.perf_counter()
    if c["rk"]:
        conv.DoRK4(q_in, q_out, 0.0, c["dt"], c["timesteps"])
    else:
        conv.DoEuler(q_in, q_out, 0.0, c["dt"], c["timesteps"])
    conv.synchronize()
    elapsed = time.perf_counter() - t0
    q_end = conv.download(q_out)
    e_inf, x_inf, rel = compute_error(q_end, c["nu0"], c["nufreq"], c["cx"], c["cy"], c["cz"], c["endtime"])
    if c.get("mat"):
        # src/Convection/main.cpp:311-327,351-355,393-405: init.mat, the cell "q" of
        # convection_0_0_0.mat (the initial field), result_0_0_0.mat with the
        # fields q (in), q (out), error and exact under the reference's names.
        # The reference writes init.mat on every run; here only with --mat.
        from .matfile import MatFile
        q0 = conv.download(q_in)
        exact = fill_q(n, n, n, c["nu0"], c["nufreq"], c["cx"], c["cy"], c["cz"], c["endtime"])
        with MatFile("init.mat") as m:
            m.addField("qIn", q0)
        with MatFile("convection_0_0_0.mat") as m:
            m.startCell("q", c["timesteps"])
            m.addField(q0, 0)
            m.endCell()
        with MatFile("result_0_0_0.mat") as m:
            m.addField("q", q0)
            m.addField("q", q_end)
            m.addField("error", q_end - exact)
            m.addField("exact", exact)
    print(f"Grid: {n}^3, timesteps: {c['timesteps']}, dt: {c['dt']:g}, CFL: {c['cfl']:g}, "
          f"order: {4 if c['rk'] else 1}", file=out)
    print(f"Timing results:\n - total time: {elapsed * 1e3:.3f} msec\n", file=out)
    # the lines src/Convection/main.cpp:378-389 prints (one process), which
    # jobs/finalJobs/FindStable.sbatch:29-30 parses
    print(f"Errors on all processes:\n - Process 0 has exact={x_inf:g}, error={e_inf:g}", file=out)
    print(f"\n Total relative error: {rel:g}", file=out)
    return dict(c, error=rel, abs_error=e_inf, seconds=elapsed)


def parareal_config(argv):
    ap = argparse.ArgumentParser(prog="parareal")
    ap.add_argument("--timeSlices", type=int, required=True)
    for name in ("nu0", "nufreq", "cx", "cy", "cz", "endTime"):
        ap.add_argument("--" + name, type=float)
    for name in ("gridSize", "timeStepsFine", "timeStepsCoarse", "kmax"):
        ap.add_argument("--" + name, type=int)
    ap.add_argument("--mat", action="store_true")
    ap.add_argument("--noasync", action="store_true")
    ap.add_argument("--mode", default="compare")
    ap.add_argument("--coarse", default="euler", choices=["euler", "rk4"])
    ap.add_argument("--coarsePrecision", default="f64", choices=["f64", "f32"])
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    from .parareal import RuntimeConfiguration
    kw = {k: getattr(a, k) for k in ("nu0", "nufreq", "cx", "cy", "cz", "endTime", "gridSize", "timeStepsFine",
                                     "timeStepsCoarse", "kmax") if getattr(a, k) is not None}
    conf = RuntimeConfiguration(timeSlices=a.timeSlices, mat=a.mat, async_=not a.noasync, mode=a.mode, **kw)
    return conf, a


def run_parareal(argv, out=sys.stdout) -> dict:
    import stencilparareal_b200 as sp
    from .solution import error_reference, fill_q
    conf, a = parareal_config(argv)
    n, P = conf.gridSize(), conf.timeSlices()
    print("Running with:\n"
          f" - initial diffusion coefficient: {conf.nu0():g}\n"
          f" - frequence of diffusion coefficient: {conf.nufreq():g}\n"
          f" - advection velocity in x: {conf.cx():g}\n - advection velocity in y: {conf.cy():g}\n"
          f" - advection velocity in z: {conf.cz():g}\n - spatial discretization step: {conf.dx():g}\n"
          f" - endtime: {conf.endTime():g}\n - number of time slices: {P}\n"
          f" - time slice size: {conf.timeSliceSize():g}\n - CFL fine: {conf.cflFine():g}\n"
          f" - CFL coarse: {conf.cflCoarse():g}\n - timestep size fine: {conf.dtFine():g}\n"
          f" - timestep size coarse: {conf.dtCoarse():g}\n"
          f" - timesteps per slice fine propagator: {conf.timeStepsFinePerTimeSlice()}\n"
          f" - timesteps per slice coarse propagator: {conf.timeStepsCoarsePerTimeSlice()}\n"
          f" - parareal iterations: {conf.kmax()}\n"
          f" - asynchronous communications: {'Enabled' if conf.async_() else 'Disabled'}\n", file=out)
    conv = sp.Convection(n, n, n, conf.dx(), conf.nu0(), conf.nufreq(), conf.cx(), conf.cy(), conf.cz(),
                         device=a.device)
    q, qinitial, qref = conv.field(), conv.field(), conv.field()
    par = sp.Parareal(conv, qinitial, q, 0.0, conf, coarse=a.coarse, coarse_precision=a.coarsePrecision)
    q0 = fill_q(n, n, n, conf.nu0(), conf.nufreq(), conf.cx(), conf.cy(), conf.cz(), 0.0)
    res = {"mode": conf.mode()}

    def timed(fn):
        conv.synchronize()
        e0 = _energy_j(a.device)
        t0 = time.perf_counter()
        r = fn()
        conv.synchronize()
        dt = time.perf_counter() - t0
        e1 = _energy_j(a.device)
        return r, dt, (e1 - e0) if (e0 is not None and e1 is not None) else None

    if conf.mode() == "compare":
        # tau_F, tau_G and the speedup model (main.cpp:197-210)
        _, tauF, _ = timed(lambda: conv.DoRK4(qinitial, qinitial, 0.0, conf.dtFine(),
                                              4 * conf.timeStepsFinePerTimeSlice()))
        _, tauG, _ = timed(lambda: conv.DoEuler(qinitial, qinitial, 0.0, conf.dtCoarse(),
                                                4 * conf.timeStepsCoarsePerTimeSlice()))
        max_speedup = sp.Parareal.max_speedup(tauG / tauF, conf.kmax(), P)
        conv.upload(qinitial, q0)
        _, t_serial, _ = timed(par.DoSerial)
        qref.data.copy_(q.data)
        conv.upload(qinitial, q0)
        rep, t_par, _ = timed(par.DoParallel)
        err = error_reference(conv.download(q), conv.download(qref))
        print(f"\nSerial run time: {t_serial:g}\nParallel run time: {t_par:g}\nSpeedup: {t_serial / t_par:g}\n"
              f"Maximal speedup: {max_speedup:g}\nError at end: {err:g}\n", file=out)
        if conf.mat():
            from .matfile import MatFile
            with MatFile("result.mat", conv) as m:  # main.cpp:251-253
                m.addField("q", q)
                m.addField("qreference", qref)
        res.update(serial_s=t_serial, parallel_s=t_par, max_speedup=max_speedup, error=err)
    elif conf.mode() == "serial":
        conv.upload(qinitial, q0)
        _, t, energy = timed(par.DoSerial)
        print(f"\nSerial run time: {t:g}", file=out)
        if energy is not None:
            print(f"Device energy : {energy:f} J  ({energy / t:.3e} W)", file=out)
        res.update(serial_s=t, energy_j=energy)
    elif conf.mode() == "parallel":
        conv.upload(qinitial, q0)
        par.DoSerial()
        print(" -- The serial computation is done", file=out)
        qref.data.copy_(q.data)
        conv.upload(qinitial, q0)
        rep, t, energy = timed(par.DoParallel)
        print(" -- The parallel computation is done", file=out)
        err = error_reference(conv.download(q), conv.download(qref))
        print(f"\nParallel run time: {t:f} s", file=out)
        if energy is not None:
            print(f"Device energy : {energy:f} J  ({energy / t:.3e} W)", file=out)
        print(f"Error of parareal: {err:.4e}\n", file=out)
        res.update(parallel_s=t, error=err, energy_j=energy)
    else:  # timing (DoTimedParallel, Parareal.h:173-248): device times of the phases
        conv.upload(qinitial, q0)
        rep = par.DoParallel()
        print("\nTimes:", file=out)
        for label, v in (("total", rep["seconds"]), ("fine", rep["seconds_fine"]), ("coarse", rep["seconds_coarse"])):
            print(f"{v:.6e}   {label}", file=out)
        res.update(report=rep)
    return res


def findstable_config(argv):
    """Options of jobs/finalJobs/FindStable.sbatch:4-20 (nu0 0.1, 128^3, T 0.1, order 4,
    nufreq in {100, 10, 1}, timeSteps doubling from 1024 to 8192)."""
    ap = argparse.ArgumentParser(prog="findstable")
    ap.add_argument("--nu0", type=float, default=0.1)
    ap.add_argument("--gridSize", type=int, default=128)
    ap.add_argument("--endTime", type=float, default=0.1)
    ap.add_argument("--order", type=int, default=4)
    ap.add_argument("--nufreqs", default="100,10,1")
    ap.add_argument("--minSteps", type=int, default=1024)
    ap.add_argument("--maxSteps", type=int, default=8192)
    a = ap.parse_args(argv)
    if a.minSteps < 1 or a.maxSteps < a.minSteps:
        raise SystemExit("need 1 <= minSteps <= maxSteps")
    steps, s = [], a.minSteps
    while s <= a.maxSteps:
        steps.append(s)
        s *= 2
    return dict(nu0=a.nu0, gridsize=a.gridSize, endtime=a.endTime, order=a.order,
                nufreqs=[float(v) for v in a.nufreqs.split(",") if v], steps=steps)


def run_findstable(argv, out=sys.stdout) -> list:
    """One convection run per (nufreq, timeSteps); prints the sweep's table
    (FindStable.sbatch:10,29-34: "Order freq tSteps AbsErr RelErr")."""
    import io
    c = findstable_config(argv)
    print("Order freq tSteps    AbsErr          RelErr", file=out)
    rows = []
    for f in c["nufreqs"]:
        for n_steps in c["steps"]:
            r = run_convection(["--nu0", str(c["nu0"]), "--nufreq", str(f), "--gridSize", str(c["gridsize"]),
                                "--endTime", str(c["endtime"]), "--timeSteps", str(n_steps),
                                "--order", str(c["order"])], out=io.StringIO())
            row = (c["order"], f, n_steps, r["abs_error"], r["error"])
            rows.append(row)
            print("%5d %4d %6d %.7e %.7e" % (row[0], int(row[1]), row[2], row[3], row[4]), file=out)
    return rows


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] not in ("convection", "parareal", "findstable"):
        print(__doc__)
        return 2
    if argv[0] == "convection":
        run_convection(argv[1:])
    elif argv[0] == "findstable":
        run_findstable(argv[1:])
    else:
        run_parareal(argv[1:])
    return 0


if __name__ == "__main__":
    sys.exit(main())
