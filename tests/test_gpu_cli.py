"""GPU tests of the command-line drivers and of the error paths of the C ABI."""
import ctypes as C
import io

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_convection_cli_converges_at_fourth_order():
    from stencilparareal_b200.cli import run_convection
    errs = []
    for n in (16, 32):
        r = run_convection(["--gridSize", str(n), "--timeSteps", "400", "--endTime", "0.02", "--nu0", "0.1"],
                           out=io.StringIO())
        errs.append(r["error"])
    order = np.log2(errs[0] / errs[1])
    assert 3.7 < order < 4.3, (errs, order)


def test_findstable_sweep_table():
    """A reduced FindStable sweep (jobs/finalJobs/FindStable.sbatch): one row per
    (nufreq, timeSteps) with the convection driver's absolute and relative errors,
    in the table format the script prints; the convection output carries the
    lines the script parses."""
    import re
    from stencilparareal_b200.cli import run_convection, run_findstable
    out = io.StringIO()
    rows = run_findstable(["--gridSize", "24", "--endTime", "0.01", "--nufreqs", "100,1", "--minSteps", "50",
                           "--maxSteps", "200"], out=out)
    lines = out.getvalue().splitlines()
    assert lines[0].split() == ["Order", "freq", "tSteps", "AbsErr", "RelErr"]
    assert [(r[1], r[2]) for r in rows] == [(100.0, 50), (100.0, 100), (100.0, 200), (1.0, 50), (1.0, 100),
                                             (1.0, 200)]
    for line, r in zip(lines[1:], rows):
        f = line.split()
        assert (int(f[0]), int(f[1]), int(f[2])) == (4, int(r[1]), r[2])
        assert abs(float(f[3]) - r[3]) <= 1e-7 * r[3] and abs(float(f[4]) - r[4]) <= 1e-7 * r[4]
        assert 0 < r[4] < 1e-2  # stable at every step count of the sweep
    conv_out = io.StringIO()
    r = run_convection(["--gridSize", "24", "--endTime", "0.01", "--timeSteps", "50", "--nufreq", "100"],
                       out=conv_out)
    text = conv_out.getvalue()
    err = re.search(r"^ - Process .* error=(.*)$", text, re.M)
    rel = re.search(r"^ Total relative error: (.*)$", text, re.M)
    assert err and rel
    assert abs(float(err.group(1)) - r["abs_error"]) <= 1e-5 * r["abs_error"]
    assert abs(float(rel.group(1)) - r["error"]) <= 1e-5 * r["error"]


def test_parareal_cli_compare_mode_matches_oracle(orc):
    from stencilparareal_b200.cli import run_parareal
    out = io.StringIO()
    r = run_parareal(["--timeSlices", "4", "--gridSize", "16", "--endTime", "0.02", "--timeStepsFine", "400",
                      "--timeStepsCoarse", "32", "--nu0", "0.1", "--kmax", "2", "--noasync"], out=out)
    assert "Error at end" in out.getvalue()
    p = orc.params(16, nu0=0.1)
    q, qs, em, el = orc.parareal(p, orc.parareal_cfg(0.02, 4, 400, 32, 2), orc.fillq(p, 0.0))
    assert abs(r["error"] - em[-1]) <= 1e-6 * em[-1]
    for mode in ("serial", "parallel", "timing"):
        run_parareal(["--timeSlices", "4", "--gridSize", "12", "--endTime", "0.01", "--timeStepsFine", "40",
                      "--timeStepsCoarse", "8", "--kmax", "2", "--mode", mode], out=io.StringIO())


def test_error_paths_return_status(sp):
    L = sp._lib
    lib = L.lib()
    c = sp.Convection(8, 8, 8, 0.125, 0.1, 0.0, 1, 1, 1)
    f = c.field()
    assert lib.sp_do_rk4(c.handle, None, C.c_void_p(f.ptr), 0.0, 1e-3, 1) == L.SP_ERR_INVALID
    assert lib.sp_do_rk4(c.handle, C.c_void_p(f.ptr), C.c_void_p(f.ptr), 0.0, 1e-3, -1) == L.SP_ERR_INVALID
    assert lib.sp_do_rk4(None, C.c_void_p(f.ptr), C.c_void_p(f.ptr), 0.0, 1e-3, 1) == L.SP_ERR_INVALID
    assert lib.sp_set_tune(c.handle, 0, 1, 5, 8, 1) == L.SP_ERR_INVALID
    p = L.SpParams(1, 8, 8, 0.125, 0.1, 0.0, 1, 1, 1, 1)
    h = C.c_void_p()
    assert lib.sp_convection_create(C.byref(p), 0, C.byref(h)) == L.SP_ERR_INVALID
    cfg = L.SpPararealCfg()
    cfg.endTime, cfg.timeSlices, cfg.timeStepsFine, cfg.timeStepsCoarse, cfg.kmax = 0.1, 0, 10, 10, 1
    assert lib.sp_parareal_create(c.handle, C.byref(cfg), C.byref(h)) == L.SP_ERR_INVALID
    cfg.timeSlices, cfg.first_slice, cfg.slice_count = 4, 3, 2
    assert lib.sp_parareal_create(c.handle, C.byref(cfg), C.byref(h)) == L.SP_ERR_INVALID
    # a window handle refuses the whole-problem entry point
    conf = sp.RuntimeConfiguration(timeSlices=4, gridSize=8, endTime=0.01, timeStepsFine=8, timeStepsCoarse=4, kmax=1)
    from stencilparareal_b200.parareal import WindowParareal
    w = WindowParareal(c, f, c.field(), 0.0, conf, 0, 2)
    with pytest.raises(sp.SpError):
        w.DoParallel()
    with pytest.raises(sp.SpError):  # a window that does not start at slice 0 needs the received field
        w2 = WindowParareal(c, f, c.field(), 0.0, conf, 2, 2)
        w2.begin()
        w2.fine(0)
        w2.coarse(0, None)


def test_mat_output_of_both_drivers(tmp_path, monkeypatch):
    import scipy.io
    from stencilparareal_b200.cli import run_convection, run_parareal
    from stencilparareal_b200.solution import fill_q
    monkeypatch.chdir(tmp_path)
    run_convection(["--gridSize", "12", "--timeSteps", "40", "--endTime", "0.01", "--mat"], out=io.StringIO())
    r = scipy.io.loadmat("result_0_0_0.mat")
    exact = fill_q(12, 12, 12, 1.0, 0.0, 1, 1, 1, 0.01).transpose(2, 1, 0)
    np.testing.assert_array_equal(r["exact"], exact)
    np.testing.assert_allclose(r["q"] - exact, r["error"], rtol=0, atol=1e-15)
    assert np.abs(r["error"]).max() < 1e-2 * np.abs(exact).max()
    init = scipy.io.loadmat("init.mat")["qIn"]
    np.testing.assert_array_equal(init, fill_q(12, 12, 12, 1.0, 0.0, 1, 1, 1, 0.0).transpose(2, 1, 0))
    np.testing.assert_array_equal(scipy.io.loadmat("convection_0_0_0.mat")["q"][0, 0], init)
    run_parareal(["--timeSlices", "4", "--gridSize", "12", "--endTime", "0.01", "--timeStepsFine", "40",
                  "--timeStepsCoarse", "8", "--kmax", "4", "--mat"], out=io.StringIO())
    m = scipy.io.loadmat("result.mat")
    assert m["q"].shape == (12, 12, 12)
    np.testing.assert_allclose(m["q"], m["qreference"], rtol=0, atol=1e-12)


def test_bounded_wait_timeout_reports_and_recovers(sp, orc):
    """A kernel wait that can never complete gives up after its limit, the call
    returns SP_ERR_TIMEOUT, and the handle keeps working."""
    import time
    L = sp._lib
    lib = L.lib()
    n = 16
    c = sp.Convection(n, n, n, 1.0 / n, 0.01, 0.0, 1.0, 1.0, 1.0)
    t0 = time.perf_counter()
    rc = lib.sp_selftest_wait_timeout(c.handle, 50.0)
    assert rc == L.SP_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    assert lib.sp_selftest_wait_timeout(c.handle, 0.0) == L.SP_ERR_INVALID
    from ics import gaussian_noise, rel_l2
    q0 = gaussian_noise(n, seed=4)
    f, g = c.field(), c.field()
    c.upload(f, q0)
    c.DoRK4(f, g, 0.0, 1e-4, 5)
    c.synchronize()
    ref = orc.rk4(orc.params(n, nu0=0.01, cx=1.0, cy=1.0, cz=1.0), q0, 0.0, 1e-4, 5)
    assert rel_l2(c.download(g), ref) < 1e-12
