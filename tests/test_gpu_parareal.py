"""GPU Parareal (all slices on one GPU) against the oracle's serial restatement
of Parareal::DoSerial + DoParallel (Parareal.h:110-171,250-253)."""
import numpy as np
import pytest

from ics import gaussian_noise, rel_l2

pytestmark = pytest.mark.gpu

COARSE = {
    ("euler", "f64"): 0, ("rk4", "f64"): 1, ("rk4", "f32"): 2, ("euler", "f32"): 3,
}


def setup(sp, orc, n, P, kmax, coarse, prec, nu0=0.05, nufreq=0.0, T=0.02, tsF=160, tsC=12, async_=False,
          skip=True, seed=0):
    conv = sp.Convection(n, n, n, 1.0 / n, nu0, nufreq, 1.0, 0.5, -0.25)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=nu0, nufreq=nufreq, gridSize=n, endTime=T,
                                   timeStepsFine=tsF, timeStepsCoarse=tsC, kmax=kmax, async_=async_)
    q0 = gaussian_noise(n, seed=seed)
    fin, fsol, fref = conv.field(), conv.field(), conv.field()
    conv.upload(fin, q0)
    par = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse=coarse, coarse_precision=prec, skip_converged=skip)
    p = orc.params(n, nu0=nu0, nufreq=nufreq, cx=1.0, cy=0.5, cz=-0.25)
    cfg = orc.parareal_cfg(T, P, tsF, tsC, kmax, async_=async_, coarse=COARSE[(coarse, prec)])
    return conv, par, fin, fsol, fref, p, cfg, q0


@pytest.mark.parametrize("coarse,prec", list(COARSE))
def test_parareal_matches_oracle(sp, orc, coarse, prec):
    n, P, kmax = 16, 4, 3
    conv, par, fin, fsol, fref, p, cfg, q0 = setup(sp, orc, n, P, kmax, coarse, prec)
    # serial fine reference on the GPU (DoSerial) and on the oracle
    ser = sp.Parareal(conv, fin, fref, 0.0, par.conf, coarse=coarse, coarse_precision=prec)
    ser.DoSerial()
    rep = par.DoParallel(reference=fref)
    qo, qs, em, el = orc.parareal(p, cfg, q0)
    assert rel_l2(conv.download(fref), qs) < 1e-12
    # FP64 coarse: rounding-level agreement.  FP32 coarse: G's FP32 rounding
    # (FMA contraction and operand order differ from the oracle's literal FP32
    # order) stays in the iterate until the slices converge, ~1e-7 relative.
    tol = 1e-11 if prec == "f64" else 1e-6
    assert rel_l2(conv.download(fsol), qo) < tol
    assert rep["iterations"] == kmax
    for k in range(kmax):
        # per-iteration errors against the serial solution agree with the oracle's
        if prec == "f64":
            assert abs(rep["err_max"][k] - em[k]) <= 1e-6 * em[k] + 1e-13, (k, rep["err_max"][k], em[k])
        else:
            assert abs(rep["err_max"][k] - em[k]) <= 0.05 * em[k] + 1e-6, (k, rep["err_max"][k], em[k])


def test_exact_after_P_iterations_and_skip_is_bitwise(sp, orc):
    n, P = 12, 4
    outs = []
    for skip in (True, False):
        conv, par, fin, fsol, fref, p, cfg, q0 = setup(sp, orc, n, P, P, "rk4", "f32", skip=skip)
        ser = sp.Parareal(conv, fin, fref, 0.0, par.conf)
        ser.DoSerial()
        rep = par.DoParallel(reference=fref)
        assert rep["err_l2"][-1] < 1e-14, rep["err_l2"]
        outs.append(conv.download(fsol))
    assert np.array_equal(outs[0], outs[1])


def test_time_dependent_nu_and_async_sequence(sp, orc):
    n, P, kmax = 12, 3, 2
    for async_ in (False, True):
        conv, par, fin, fsol, fref, p, cfg, q0 = setup(sp, orc, n, P, kmax, "euler", "f64", nufreq=100.0,
                                                       async_=async_)
        par.DoParallel()
        qo, qs, em, el = orc.parareal(p, cfg, q0)
        assert rel_l2(conv.download(fsol), qo) < 1e-11


def test_rounding_and_report(sp, orc):
    n, P = 8, 32
    conv = sp.Convection(n, n, n, 1.0 / n, 0.01, 0.0, 1.0, 1.0, 1.0)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.01, gridSize=n, endTime=0.2, timeStepsFine=20000,
                                   timeStepsCoarse=200, kmax=1)
    f0, f1 = conv.field(), conv.field()
    conv.upload(f0, gaussian_noise(n))
    par = sp.Parareal(conv, f0, f1, 0.0, conf, coarse="rk4", coarse_precision="f32")
    rep = par.DoParallel()
    assert rep["tsFine"] == 625 and rep["tsCoarse"] == 7
    assert abs(rep["dtCoarse"] - 0.2 / 224) < 1e-18
    assert rep["fine_cell_updates"] == 32 * 625 * n ** 3


def test_tolerance_stops_early(sp, orc):
    n, P = 12, 8
    conv, par, fin, fsol, fref, p, cfg, q0 = setup(sp, orc, n, P, 8, "rk4", "f64")
    ser = sp.Parareal(conv, fin, fref, 0.0, par.conf)
    ser.DoSerial()
    par2 = sp.Parareal(conv, fin, fsol, 0.0, par.conf, coarse="rk4", coarse_precision="f64", tol=1e-8,
                       tol_kind="reference")
    rep = par2.DoParallel(reference=fref)
    assert rep["iterations"] < 8
    assert rep["err_l2"][-1] < 1e-8
    assert all(e >= 1e-8 for e in rep["err_l2"][:-1])


@pytest.mark.parametrize("coarse,prec", [("rk4", "f32"), ("euler", "f64"), ("rk4", "f64"), ("euler", "f32")])
def test_increment_form_matches_oracle(sp, orc, coarse, prec):
    n, P, kmax = 16, 4, 3
    conv = sp.Convection(n, n, n, 1.0 / n, 0.05, 0.0, 1.0, 0.5, -0.25)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.05, gridSize=n, endTime=0.02, timeStepsFine=160,
                                   timeStepsCoarse=12, kmax=kmax, async_=False)
    q0 = gaussian_noise(n, seed=0)
    fin, fsol = conv.field(), conv.field()
    conv.upload(fin, q0)
    par = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse=coarse, coarse_precision=prec, coarse_delta=True)
    par.DoParallel()
    p = orc.params(n, nu0=0.05, cx=1.0, cy=0.5, cz=-0.25)
    cfg = orc.parareal_cfg(0.02, P, 160, 12, kmax, coarse=COARSE[(coarse, prec)], delta=True)
    qo, qs, em, el = orc.parareal(p, cfg, q0)
    # the FP32 rounding now acts on the increment only
    tol = 1e-11 if prec == "f64" else 1e-8
    assert rel_l2(conv.download(fsol), qo) < tol


def test_increment_form_exact_bitwise_after_P_iterations(sp, orc):
    n, P = 16, 4
    conv = sp.Convection(n, n, n, 1.0 / n, 0.05, 0.0, 1.0, 0.5, -0.25)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.05, gridSize=n, endTime=0.02, timeStepsFine=160,
                                   timeStepsCoarse=12, kmax=P)
    fin, fsol, fref = conv.field(), conv.field(), conv.field()
    conv.upload(fin, gaussian_noise(n, seed=3))
    par = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse="rk4", coarse_precision="f32", coarse_delta=True)
    par.DoSerial()  # writes fsol
    fref.data.copy_(fsol.data)
    rep = par.DoParallel(reference=fref)
    # slice r is exact after r+1 iterations: F(U) + G(0) reproduces the serial run bit for bit
    assert np.array_equal(conv.download(fsol), conv.download(fref))
    assert rep["err_l2"][-1] == 0.0


def test_fp32_coarse_increment_form_removes_noise_floor(sp, orc):
    n, P, kmax = 24, 12, 6
    p = orc.params(n, nu0=0.01)
    q0 = gaussian_noise(n, seed=0)
    errs = {}
    for delta in (False, True):
        conv = sp.Convection(n, n, n, 1.0 / n, 0.01, 0.0, 1.0, 1.0, 1.0)
        conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.01, gridSize=n, endTime=0.12, timeStepsFine=1200,
                                       timeStepsCoarse=120, kmax=kmax)
        fin, fsol, fref = conv.field(), conv.field(), conv.field()
        conv.upload(fin, q0)
        par = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse="rk4", coarse_precision="f32", coarse_delta=delta)
        par.DoSerial()
        fref.data.copy_(fsol.data)
        errs[delta] = par.DoParallel(reference=fref)["err_l2"]
    # state form: FP32 rounding of G(U) stalls the error; increment form keeps converging
    assert errs[True][-1] < 1e-3 * errs[False][-1], errs


def test_batch_of_uneven_instances_equals_individual_runs(sp, orc):
    from stencilparareal_b200.parareal import PararealBatch
    specs = [  # n, nu0, c, P, coarse, precision
        (12, 0.01, (1.0, -0.5, 0.3), 4, "rk4", "f32"),
        (16, 0.003, (-0.7, 0.9, 0.1), 6, "rk4", "f32"),
        (20, 0.05, (0.2, 0.2, -1.0), 3, "euler", "f64"),
    ]
    runs = []
    for n, nu0, c, P, coarse, prec in specs:
        conv = sp.Convection(n, n, n, 1.0 / n, nu0, 0.0, *c)
        conf = sp.RuntimeConfiguration(timeSlices=P, nu0=nu0, gridSize=n, endTime=0.01, timeStepsFine=100,
                                       timeStepsCoarse=10, kmax=3)
        q0 = gaussian_noise(n, seed=n)
        fin, fa, fb, fref = conv.field(), conv.field(), conv.field(), conv.field()
        conv.upload(fin, q0)
        alone = sp.Parareal(conv, fin, fa, 0.0, conf, coarse=coarse, coarse_precision=prec)
        alone.DoSerial()
        fref.data.copy_(fa.data)
        alone.DoParallel()
        inb = sp.Parareal(conv, fin, fb, 0.0, conf, coarse=coarse, coarse_precision=prec)
        runs.append((conv, alone, inb, fa, fb, fref, q0, (n, nu0, c, P, coarse, prec)))
    batch = PararealBatch([r[2] for r in runs])
    reps, secs = batch.run(references=[r[5] for r in runs])
    assert secs > 0
    for (conv, alone, inb, fa, fb, fref, q0, spec), rep in zip(runs, reps):
        assert rep["iterations"] == 3
        assert np.array_equal(conv.download(fa), conv.download(fb))
        n, nu0, c, P, coarse, prec = spec
        cfg = orc.parareal_cfg(0.01, P, 100, 10, 3, coarse=COARSE[(coarse, prec)], delta=(prec == "f32"))
        qo, qs, em, el = orc.parareal(orc.params(n, nu0=nu0, cx=c[0], cy=c[1], cz=c[2]), cfg, q0)
        assert rel_l2(conv.download(fb), qo) < (1e-11 if prec == "f64" else 1e-8)
        assert abs(rep["err_l2"][-1] - el[-1]) <= 1e-3 * el[-1] + 1e-12


def test_nonfinite_defect_is_reported_and_handle_recovers(sp):
    """Failure detection without a GPU fault: a fine step far beyond RK4's stability
    limit (diffusion number 4, growth ~7e5 per step: the fields overflow to Inf/NaN
    within the first slice) makes DoParallel return SP_ERR_NONFINITE instead of a result; the
    same propagator handle then runs a stable Parareal bit for bit like a fresh one."""
    n, P = 16, 4
    conv = sp.Convection(n, n, n, 1.0 / n, 1.0, 0.0, 1.0, 1.0, 1.0)
    fin, fsol = conv.field(), conv.field()
    conv.upload(fin, gaussian_noise(n, seed=31))
    bad = sp.RuntimeConfiguration(timeSlices=P, nu0=1.0, gridSize=n, endTime=4.0, timeStepsFine=256,
                                  timeStepsCoarse=8, kmax=2)
    with pytest.raises(sp.SpError) as ex:
        sp.Parareal(conv, fin, fsol, 0.0, bad, coarse="rk4", coarse_precision="f64").DoParallel()
    assert ex.value.code == sp._lib.SP_ERR_NONFINITE
    good = sp.RuntimeConfiguration(timeSlices=P, nu0=1.0, gridSize=n, endTime=0.002, timeStepsFine=64,
                                   timeStepsCoarse=8, kmax=2)
    sp.Parareal(conv, fin, fsol, 0.0, good, coarse="rk4", coarse_precision="f64").DoParallel()
    got = conv.download(fsol)
    conv2 = sp.Convection(n, n, n, 1.0 / n, 1.0, 0.0, 1.0, 1.0, 1.0)
    f2, s2 = conv2.field(), conv2.field()
    conv2.upload(f2, gaussian_noise(n, seed=31))
    sp.Parareal(conv2, f2, s2, 0.0, good, coarse="rk4", coarse_precision="f64").DoParallel()
    assert np.array_equal(got, conv2.download(s2))


@pytest.mark.parametrize("tol_kind,tol", [("none", 0.0), ("defect", 1e-6), ("reference", 1e-7)])
def test_one_launch_loop_equals_host_loop(sp, tol_kind, tol):
    """All iterations in one graph launch (conditional WHILE node, stopping test on
    the device) give the host-driven loop's fields, iteration count, defects and
    errors bit for bit."""
    n, P = 16, 6
    conv = sp.Convection(n, n, n, 1.0 / n, 0.02, 0.0, 1.0, -0.5, 0.25)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.02, gridSize=n, endTime=0.03, timeStepsFine=240,
                                   timeStepsCoarse=18, kmax=5)
    fin, fref = conv.field(), conv.field()
    conv.upload(fin, gaussian_noise(n, seed=4))
    sp.Parareal(conv, fin, fref, 0.0, conf).DoSerial()
    outs = []
    for host in (True, False):
        fsol = conv.field()
        par = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse="rk4", coarse_precision="f32", tol=tol,
                          tol_kind=tol_kind)
        par.set_host_loop(host)
        rep = par.DoParallel(reference=fref)
        first = conv.download(fsol)
        rep2 = par.DoParallel(reference=fref)  # a second run of the same graph
        assert np.array_equal(conv.download(fsol), first)
        assert rep2["iterations"] == rep["iterations"]
        outs.append((first, rep))
    (a, ra), (b, rb) = outs
    assert np.array_equal(a, b)
    assert ra["iterations"] == rb["iterations"]
    # the defect and error sums are accumulated with atomics across CTAs, so
    # their last bits depend on the order of the additions
    for key in ("defect", "err_l2", "err_max"):
        assert np.allclose(ra[key], rb[key], rtol=1e-12, atol=0), key
    assert ra["fine_cell_updates"] == rb["fine_cell_updates"]
    if tol_kind == "none":
        assert ra["iterations"] == 5
    else:
        assert ra["iterations"] < 5


def test_batch_one_launch_loop_equals_host_loop(sp):
    from stencilparareal_b200.parareal import PararealBatch
    specs = [(12, 0.01, (1.0, -0.5, 0.3), 4, 1e-9), (16, 0.003, (-0.7, 0.9, 0.1), 6, 1e-6),
             (10, 0.05, (0.2, 0.2, -1.0), 3, 0.0)]
    results = []
    for host in (True, False):
        inst, refs, convs = [], [], []
        for n, nu0, c, P, tol in specs:
            conv = sp.Convection(n, n, n, 1.0 / n, nu0, 0.0, *c)
            conf = sp.RuntimeConfiguration(timeSlices=P, nu0=nu0, gridSize=n, endTime=0.01, timeStepsFine=100,
                                           timeStepsCoarse=10, kmax=P)
            fin, fs, fr = conv.field(), conv.field(), conv.field()
            conv.upload(fin, gaussian_noise(n, seed=n + 1))
            sp.Parareal(conv, fin, fr, 0.0, conf).DoSerial()
            inst.append(sp.Parareal(conv, fin, fs, 0.0, conf, coarse="rk4", coarse_precision="f32", tol=tol,
                                    tol_kind="defect" if tol > 0 else "none"))
            refs.append(fr)
            convs.append(conv)
        batch = PararealBatch(inst)
        batch.set_host_loop(host)
        reps, secs = batch.run(references=refs)
        results.append(([c.download(p.solution) for c, p in zip(convs, inst)], reps))
    (fa, ra), (fb, rb) = results
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)
    for x, y in zip(ra, rb):
        assert x["iterations"] == y["iterations"]
        assert np.allclose(x["defect"], y["defect"], rtol=1e-12, atol=0)
        assert np.allclose(x["err_l2"], y["err_l2"], rtol=1e-12, atol=0)
        assert x["fine_cell_updates"] == y["fine_cell_updates"]
    assert ra[2]["iterations"] == 3  # no tolerance: exact after P = 3 iterations
