"""The cluster-resident paths for small FP64 fields (sp_cluster.cu): every RK4 step
of a DoRK4 call in one launch, each field held in the shared memory of one
thread-block cluster, split into z-slabs (tune kind 3) or into (y,z) blocks
(kind 5).  They must give the four single-stage kernels' fields bit for bit
(same operations, same order) and the oracle's to 1e-12."""
import numpy as np
import pytest

from ics import fourier_modes, gaussian_noise, rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
# grids: planes per CTA NZ = 2, 3, 4 (z-slabs), blocks of 2 .. 16 rows and planes
# with 1, 2 or 4 planes per unit and 256 or 512 threads ((y,z) blocks), clusters
# of 2 .. 16 CTAs, one or two cell pairs per thread, non-cubic and
# non-power-of-two extents
SIZES = [(32, 32, 32), (24, 20, 12), (64, 32, 16), (16, 16, 8), (10, 6, 4), (30, 30, 9), (32, 32, 48),
         (8, 12, 36), (40, 40, 32), (24, 24, 24)]


def _conv(sp, n, nufreq=0.0, c=(1.0, -0.5, 0.25), nu0=0.02):
    return sp.Convection(*n, 1.0 / n[0], nu0, nufreq, *c)


def _run(sp, conv, kind, q0, t0, dt, steps, in_place=False):
    if kind in (3, 5):
        conv.set_tune(sp.SP_F64, 1, 0, 0, kind)
    else:
        conv.set_tune(sp.SP_F64, 1, 4, 8, 1)
    fin, fout = conv.field(), conv.field()
    conv.upload(fin, q0)
    if in_place:
        conv.DoRK4(fin, fin, t0, dt, steps)
        return conv.download(fin), fin
    conv.DoRK4(fin, fout, t0, dt, steps)
    return conv.download(fout), fout


@pytest.mark.parametrize("kind", [3, 5])
@pytest.mark.parametrize("n", SIZES)
def test_cluster_path_equals_stage_kernels_and_oracle(sp, orc, n, kind):
    conv = _conv(sp, n)
    assert conv.tuned_config(sp.SP_F64, 1, 11)["kind"] == 0
    q0 = gaussian_noise(*n, seed=2)
    a, _ = _run(sp, conv, 1, q0, 0.0, 1e-4, 9)
    b, fb = _run(sp, conv, kind, q0, 0.0, 1e-4, 9)
    assert conv.tuned_config(sp.SP_F64, 1, 11)["kind"] == kind
    assert np.array_equal(a, b)
    p = orc.params(n, dx=1.0 / n[0], nu0=0.02, cx=1.0, cy=-0.5, cz=0.25)
    assert rel_l2(b, orc.rk4(p, q0, 0.0, 1e-4, 9)) < TOL64
    # the result carries its periodic images (the halo equals the opposite interior)
    lay = fb.layout
    full = fb.data.cpu().numpy()
    o = lay.origin
    for k in (0, n[2] - 1):
        for j in (0, n[1] - 1):
            for i in (0, 1, n[0] - 2, n[0] - 1):
                v = full[o + k * lay.plane + j * lay.px + i]
                if i < 2:
                    assert full[o + k * lay.plane + j * lay.px + i + n[0]] == v
                if k < 2:
                    assert full[o + (k + n[2]) * lay.plane + j * lay.px + i] == v


@pytest.mark.parametrize("kind", [3, 5])
def test_cluster_path_time_dependent_nu_in_place_and_long_runs(sp, orc, kind):
    n = (32, 32, 32)
    conv = _conv(sp, n, nufreq=80.0)
    q0 = fourier_modes(*n, seed=3)
    a, _ = _run(sp, conv, 1, q0, 0.004, 1e-4, 37)
    b, _ = _run(sp, conv, kind, q0, 0.004, 1e-4, 37, in_place=True)
    assert np.array_equal(a, b)
    p = orc.params(n, nu0=0.02, nufreq=80.0, cx=1.0, cy=-0.5, cz=0.25)
    assert rel_l2(b, orc.rk4(p, q0, 0.004, 1e-4, 37)) < TOL64
    # the serial fine configuration of 32^3: 1000 steps in one launch
    conv1 = sp.Convection(32, 32, 32, 1.0 / 32, 0.01, 0.0, 1.0, 1.0, 1.0)
    q1 = gaussian_noise(32, seed=0)
    c, _ = _run(sp, conv1, kind, q1, 0.0, 1e-4, 1000)
    d, _ = _run(sp, conv1, 1, q1, 0.0, 1e-4, 1000)
    assert np.array_equal(c, d)
    assert rel_l2(c, orc.rk4(orc.params(32, nu0=0.01), q1, 0.0, 1e-4, 1000)) < TOL64


def test_blocks_with_two_units_per_thread_time_dependent_nu_in_place(sp, orc):
    """(y,z) blocks in the 512-thread form with two units per thread (40^3: 4 x 4
    blocks of 10 rows and 8 planes), with per-step weights (nu(t)) and in place."""
    n = (40, 40, 32)
    conv = _conv(sp, n, nufreq=60.0)
    q0 = gaussian_noise(*n, seed=4)
    a, _ = _run(sp, conv, 1, q0, 0.01, 1e-4, 23)
    b, _ = _run(sp, conv, 5, q0, 0.01, 1e-4, 23, in_place=True)
    assert np.array_equal(a, b)
    p = orc.params(n, dx=1.0 / n[0], nu0=0.02, nufreq=60.0, cx=1.0, cy=-0.5, cz=0.25)
    assert rel_l2(b, orc.rk4(p, q0, 0.01, 1e-4, 23)) < TOL64


def test_autotuner_considers_cluster_path_and_unsupported_grids_are_refused(sp):
    conv = sp.Convection(32, 32, 32, 1.0 / 32, 0.01, 0.0, 1.0, 1.0, 1.0)
    t = conv.autotune(sp.SP_F64, 1)
    assert t["cluster"]["kind"] in (0, 3, 5)
    odd = sp.Convection(17, 19, 23, 1.0 / 17, 0.01, 0.0, 1.0, 1.0, 1.0)
    big = sp.Convection(128, 128, 128, 1.0 / 128, 0.01, 0.0, 1.0, 1.0, 1.0)
    for kind in (3, 5):
        with pytest.raises(sp.SpError):
            odd.set_tune(sp.SP_F64, 1, 0, 0, kind)
        with pytest.raises(sp.SpError):
            big.set_tune(sp.SP_F64, 1, 0, 0, kind)
    # a prime nj has no (y,z) blocks; the z-slabs still fit
    prime = sp.Convection(16, 13, 16, 1.0 / 16, 0.01, 0.0, 1.0, 1.0, 1.0)
    prime.set_tune(sp.SP_F64, 1, 0, 0, 3)
    with pytest.raises(sp.SpError):
        prime.set_tune(sp.SP_F64, 1, 0, 0, 5)


@pytest.mark.parametrize("kind", [3, 5])
@pytest.mark.parametrize("skip,P", [(True, 6), (False, 6), (True, 16), (True, 40)])
def test_parareal_fine_sweep_on_clusters_equals_stage_kernels(sp, skip, P, kind):
    """All slices' fine runs of a Parareal iteration in one launch, one cluster per
    slice (converged slices gated off on the device).  With 40 slices the z-slab
    clusters of 2 planes per CTA (8 CTAs each) would exceed the SMs, so the batch
    runs clusters of 4 planes per CTA; the (y,z) blocks take 4 x 4 blocks for 6
    and 40 slices and 2 x 4 blocks for 16."""
    n = 16
    outs = []
    for k in (1, kind):
        conv = sp.Convection(n, n, n, 1.0 / n, 0.02, 0.0, 1.0, -0.5, 0.25)
        if k != 1:
            conv.set_tune(sp.SP_F64, P, 0, 0, k)
        else:
            conv.set_tune(sp.SP_F64, P, 4, 8, 1)
        conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.02, gridSize=n, endTime=0.03, timeStepsFine=6 * P * 7,
                                       timeStepsCoarse=3 * P, kmax=4)
        fin, fsol = conv.field(), conv.field()
        conv.upload(fin, gaussian_noise(n, seed=5))
        rep = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse="rk4", coarse_precision="f32",
                          skip_converged=skip).DoParallel()
        outs.append((conv.download(fsol), rep["iterations"]))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1] == 4
