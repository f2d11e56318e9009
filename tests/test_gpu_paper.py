"""GPU reproduction of the reference's published Parareal convergence table
(jobs/paperJobs/01-Convergence/result.dat:1-6) at full size: 128^3, T=0.1,
nu0=0.1, c=(1,1,1), 32768 fine RK4 / 2048 coarse upwind-Euler steps (FP64),
the analytic field exactQ at t=0 as initial condition, P in {8, 32, 128},
nufreq in {0, 100}.  The metric is the reference's "Error at end",
max|q - q_serial| / max|q| after each iteration (src/Parareal/main.cpp:98-139)."""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
KMAX = 4  # errors down to ~1e-11, far above the rounding level of either run

with open(os.path.join(GOLD, "result_dat.json")) as _f:
    TABLE = json.load(_f)


@pytest.mark.parametrize("row", range(len(TABLE["rows"])),
                         ids=[f"P{r['P']}_nufreq{int(r['nufreq'])}" for r in TABLE["rows"]])
def test_result_dat_row_on_gpu(sp, row):
    from stencilparareal_b200.solution import fill_q
    cfg, r = TABLE["config"], TABLE["rows"][row]
    n, nu0, nuf = cfg["gridSize"], cfg["nu0"], r["nufreq"]
    conv = sp.Convection(n, n, n, 1.0 / n, nu0, nuf, cfg["cx"], cfg["cy"], cfg["cz"])
    conf = sp.RuntimeConfiguration(timeSlices=r["P"], nu0=nu0, nufreq=nuf, gridSize=n, endTime=cfg["endTime"],
                                   timeStepsFine=cfg["timeStepsFine"], timeStepsCoarse=cfg["timeStepsCoarse"],
                                   kmax=KMAX, async_=cfg["async"])
    fin, fsol, fref = conv.field(), conv.field(), conv.field()
    conv.upload(fin, fill_q(n, n, n, nu0, nuf, cfg["cx"], cfg["cy"], cfg["cz"], 0.0))
    ser = sp.Parareal(conv, fin, fref, 0.0, conf, coarse="euler", coarse_precision="f64")
    ser.DoSerial()
    par = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse="euler", coarse_precision="f64")
    rep = par.DoParallel(reference=fref)
    for k in range(KMAX):
        mine, theirs = rep["err_max"][k], r["err_max"][k]
        # the table prints 6 significant digits
        assert abs(mine - theirs) <= 2e-5 * theirs, (k + 1, mine, theirs)
