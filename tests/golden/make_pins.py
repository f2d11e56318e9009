"""Generates the oracle pins of the two full-size Parareal workloads.

Run once on a CPU host (the oracle needs ~30 min of 8 cores for both):

    python tests/golden/make_pins.py [--threads N]

It writes ``tests/golden/pin_parareal_128cube_P32.npz`` (128^3, 32 slices,
T = 0.2, fine RK4 FP64 dt = 1e-5, coarse RK4 FP32 with 200 steps rounded up to
224, increment-form correction, Gaussian + noise initial field seed 0,
c = (1,1,1), nu = 0.01) and ``tests/golden/pin_parareal_96cube_P12.npz``
(the first 96^3 instance of the 48-instance batch drawn from seed 2: 12 slices,
T = 0.05, fine dt = 1e-5, coarse RK4 FP32, 50 coarse steps rounded up to 60).

A full field does not fit a small fixture, so each pin keeps, for the serial
fine solution and for the last slice's result after iterations 1 and 2, the
values at 4096 cells drawn from a fixed seed (``sample_index``, flat indices
into the (nk, nj, ni) array) and the sum and sum of squares of the whole
field, together with the oracle's per-iteration relative L2 / max-norm errors
against the serial solution and its per-iteration defect.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from ics import gaussian_noise  # noqa: E402
from oracle import oracle as O  # noqa: E402

N_SAMPLE = 4096

# name -> (n, nu0, (cx, cy, cz), P, T, timeStepsFine, timeStepsCoarse, IC seed)
CASES = {
    "pin_parareal_128cube_P32": (128, 0.01, (1.0, 1.0, 1.0), 32, 0.2, 20000, 200, 0),
    "pin_parareal_96cube_P12": (96, 0.00039535049494030775,
                                (0.6284514811885606, -0.8161681157298062, 0.200201051931308), 12, 0.05, 5000, 50, 2),
}
KMAX = 2


def sample_index(n):
    return np.sort(np.random.default_rng(12345).choice(n ** 3, size=N_SAMPLE, replace=False))


def summary(q, idx):
    return q.reshape(-1)[idx].copy(), np.array([q.sum(), (q * q).sum()])


def make(name, threads):
    n, nu0, c, P, T, tsF, tsC, seed = CASES[name]
    O.build()
    O.set_threads(threads)
    p = O.params(n, nu0=nu0, cx=c[0], cy=c[1], cz=c[2])
    cfg = O.parareal_cfg(T, P, tsF, tsC, KMAX, async_=False, coarse=O.COARSE_RK4_F32, delta=True)
    q0 = gaussian_noise(n, seed=seed)
    t0 = time.perf_counter()
    qs, em, el, de, qi = O.parareal_iters(p, cfg, q0)
    idx = sample_index(n)
    out = dict(n=n, nu0=nu0, c=np.array(c), P=P, T=T, timeStepsFine=tsF, timeStepsCoarse=tsC, seed=seed,
               kmax=KMAX, err_max=em, err_l2=el, defect=de, sample_index=idx)
    out["serial_sample"], out["serial_moments"] = summary(qs, idx)
    for k in range(KMAX):
        out[f"iter{k + 1}_sample"], out[f"iter{k + 1}_moments"] = summary(qi[k], idx)
    np.savez(os.path.join(HERE, name + ".npz"), **out)
    print(f"{name}: {time.perf_counter() - t0:.0f} s, err_l2 {el}, defect {de}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--case", choices=list(CASES), action="append")
    a = ap.parse_args()
    for name in a.case or list(CASES):
        make(name, a.threads)


if __name__ == "__main__":
    main()
