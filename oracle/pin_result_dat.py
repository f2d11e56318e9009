"""Pins the CPU oracle against the reference's published Parareal table.

Runs the oracle's serial restatement of Parareal::DoSerial + DoParallel at the
exact configuration of jobs/paperJobs/01-Convergence.job:51-57 (128^3,
T=0.1, nu0=0.1, c=(1,1,1), 32768 fine RK4 steps, 2048 coarse upwind-Euler
steps, --noasync, IC = exactQ at t=0) for P slices and k = 1..kmax, and
writes the max-norm relative errors next to the values of
jobs/paperJobs/01-Convergence/result.dat (tests/golden/result_dat.json).

A full F sweep at 128^3 costs about 6.9e10 cell-updates, so this is a
long-running CPU job (tens of minutes per iteration on 8 cores); its output
file tests/golden/oracle_pin_P{P}_nf{nufreq}.json is committed, and the CPU
test-suite checks the recorded numbers against result.dat.

usage: python oracle/pin_result_dat.py [P] [kmax] [nufreq] [threads]
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle import oracle as O  # noqa: E402


def main(P=8, kmax=3, nufreq=0.0, threads=0):
    P, kmax, nufreq, threads = int(P), int(kmax), float(nufreq), int(threads)
    if threads:
        O.set_threads(threads)
    with open(os.path.join(os.path.dirname(HERE), "tests", "golden", "result_dat.json")) as f:
        gold = json.load(f)
    c = gold["config"]
    n = c["gridSize"]
    p = O.params(n, nu0=c["nu0"], nufreq=nufreq, cx=c["cx"], cy=c["cy"], cz=c["cz"], upwind=True)
    cfg = O.parareal_cfg(c["endTime"], P, c["timeStepsFine"], c["timeStepsCoarse"], kmax,
                         async_=False, coarse=O.COARSE_EULER_F64)
    q0 = O.fillq(p, 0.0)
    t0 = time.time()
    q, qs, em, el = O.parareal(p, cfg, q0)
    wall = time.time() - t0
    ref = [r for r in gold["rows"] if r["P"] == P and r["nufreq"] == nufreq][0]["err_max"]
    out = {"config": dict(c, P=P, nufreq=nufreq, kmax=kmax),
           "oracle_err_max": [float(x) for x in em],
           "oracle_err_l2": [float(x) for x in el],
           "result_dat_err_max": ref[:kmax],
           "rel_diff": [float(abs(a - b) / b) for a, b in zip(em, ref)],
           "threads": O.get_threads(), "wall_s": wall,
           "serial_l2_norm": float(np.sqrt((qs ** 2).sum()))}
    path = os.path.join(os.path.dirname(HERE), "tests", "golden", f"oracle_pin_P{P}_nf{int(nufreq)}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main(*sys.argv[1:])
