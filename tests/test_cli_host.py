"""CPU tests of the analytic-solution module and the CLI option handling."""
import numpy as np

from stencilparareal_b200 import solution as S
from stencilparareal_b200.cli import convection_config, findstable_config, parareal_config


def test_fill_q_matches_oracle(orc):
    for n, args in ((8, (0.1, 0.0, 1.0, 1.0, 1.0, 0.0)), (6, (0.01, 100.0, 1.0, 0.5, 0.25, 0.05))):
        nu0, nf, cx, cy, cz, t = args
        mine = S.fill_q(n, n, n, nu0, nf, cx, cy, cz, t)
        ref = orc.fillq(orc.params(n, nu0=nu0, nufreq=nf, cx=cx, cy=cy, cz=cz), t)
        np.testing.assert_allclose(mine, ref, rtol=0, atol=1e-15)


def test_error_measures(orc):
    a = S.fill_q(8, 8, 8, 0.1, 0.0, 1, 1, 1, 0.01)
    b = a + 1e-3 * np.sin(np.arange(a.size)).reshape(a.shape)
    assert abs(S.error_reference(a, b) - orc.error_maxrel(a, b)) < 1e-16
    e_inf, x_inf, rel = S.compute_error(b, 0.1, 0.0, 1, 1, 1, 0.01)
    assert abs(rel - e_inf / x_inf) < 1e-16 and e_inf > 0


def test_convection_options_follow_reference_rules():
    # src/Convection/main.cpp:78-213: defaults, then --cfl picks the step count or the grid
    c = convection_config([])
    assert (c["gridsize"], c["timesteps"], c["endtime"], c["rk"]) == (32, 512, 0.05, True)
    c = convection_config(["--gridSize", "64", "--cfl", "0.1", "--nu0", "0.1", "--endTime", "0.01"])
    dt = (1 / 64) ** 2 * 0.1 / (1.5 * 0.1)
    assert c["timesteps"] == int(0.01 / dt + 0.5)
    c = convection_config(["--timeSteps", "100", "--cfl", "0.2", "--nu0", "0.5"])
    assert c["gridsize"] == int(1 / np.sqrt(0.05 / 100 * 0.5 / 0.2) + 0.5)
    assert convection_config(["--order", "1"])["rk"] is False


def test_parareal_options():
    conf, a = parareal_config(["--timeSlices", "32", "--gridSize", "128", "--endTime", "0.2", "--timeStepsFine",
                               "20000", "--timeStepsCoarse", "200", "--noasync", "--mode", "Serial"])
    assert conf.timeStepsCoarsePerTimeSlice() == 7 and conf.timeStepsFinePerTimeSlice() == 625
    assert conf.mode() == "serial" and not conf.async_()


def test_matfile_roundtrip(tmp_path):
    import scipy.io
    from stencilparareal_b200.matfile import MatFile
    a = S.fill_q(6, 5, 4, 0.1, 0.0, 1, 1, 1, 0.0)  # shape (4, 5, 6)
    b = (a * 2).astype(np.float32)
    fn = str(tmp_path / "t.mat")
    with MatFile(fn) as m:
        m.addField("q", a)
        m.addField("q", a, inc=3)
        m.addField(b, 2)  # addField(field, inc): the name "q" with _inc
        m.startCell("series", 2)
        m.addField(a, 0)
        m.addField(b, 1)
        m.endCell()
    d = scipy.io.loadmat(fn)
    # MATLAB q(i, j, k) = interior cell (i, j, k): dims ni x nj x nk, i fastest
    assert d["q"].shape == (6, 5, 4)
    np.testing.assert_array_equal(d["q"], a.transpose(2, 1, 0))
    np.testing.assert_array_equal(d["q_3"], a.transpose(2, 1, 0))
    np.testing.assert_array_equal(d["q_2"], b.transpose(2, 1, 0))
    cell = d["series"]
    assert cell.shape == (1, 2)
    np.testing.assert_array_equal(cell[0, 1], b.transpose(2, 1, 0))


def test_findstable_options():
    # jobs/finalJobs/FindStable.sbatch:4-20: nu0 0.1, 128^3, T 0.1, order 4,
    # nufreq 100, 10, 1 and timeSteps 1024 doubling while <= 8192
    c = findstable_config([])
    assert (c["nu0"], c["gridsize"], c["endtime"], c["order"]) == (0.1, 128, 0.1, 4)
    assert c["nufreqs"] == [100.0, 10.0, 1.0] and c["steps"] == [1024, 2048, 4096, 8192]
    c = findstable_config(["--minSteps", "100", "--maxSteps", "450", "--nufreqs", "5"])
    assert c["steps"] == [100, 200, 400] and c["nufreqs"] == [5.0]
