"""Generates the golden fixtures under tests/golden/ from the reference.

Run in a container where the reference tree is mounted; its path is the one
required argument:

    python tests/golden/make_golden.py <path-to-the-reference-checkout>

Two fixture files come out:

* ``result_dat.json`` -- the Parareal convergence table that the reference
  committed (jobs/paperJobs/01-Convergence/result.dat:1-6): max-norm relative
  error of the last slice against the serial fine solution after k = 1..8
  iterations, for P in {8, 32, 128} slices and nufreq in {0, 100}, with the
  run configuration of jobs/paperJobs/01-Convergence.job:51-57.
* ``exactq.npz`` -- values of the analytic solution computed by the
  reference's own Python implementation (py/Convection.py:12-36,
  Convection.getExact / getSolution) at a few grids and times.
"""
import argparse
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    rows = []
    with open(os.path.join(ref, "jobs/paperJobs/01-Convergence/result.dat")) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            rows.append({"P": int(t[0]), "nufreq": float(t[1]), "err_max": [float(x) for x in t[2:]]})
    cfg = {"gridSize": 128, "endTime": 0.1, "timeStepsFine": 32768, "timeStepsCoarse": 2048,
           "nu0": 0.1, "cx": 1.0, "cy": 1.0, "cz": 1.0, "async": False, "coarse": "euler_upwind_f64",
           "ic": "exactQ at t=0"}
    with open(os.path.join(HERE, "result_dat.json"), "w") as f:
        json.dump({"source": "jobs/paperJobs/01-Convergence/result.dat:1-6",
                   "config": cfg, "rows": rows}, f, indent=1)

    spec = importlib.util.spec_from_file_location("refconv", os.path.join(ref, "py/Convection.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for name, (nu0, nufreq, cx, cy, cz, n, t) in {
        "a": (0.1, 0.0, 1.0, 1.0, 1.0, 8, 0.0),
        "b": (0.1, 100.0, 1.0, 1.0, 1.0, 8, 0.1),
        "c": (0.01, 0.0, 1.0, 0.5, 0.25, 6, 0.05),
    }.items():
        c = mod.Convection(nu0, nufreq, cx, cy, cz)
        sol = c.getSolution(n, t)  # shape [i][j][k]
        out[name] = sol
        out[name + "_args"] = np.array([nu0, nufreq, cx, cy, cz, n, t])
    np.savez(os.path.join(HERE, "exactq.npz"), **out)


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("reference", help="root of the andyspiros/StencilParareal checkout")
    main(ap.parse_args().reference)
