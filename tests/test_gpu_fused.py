"""GPU tests of the fused RK4 stage pairs (stages 1+2 and 3+4 in one kernel each).

The fused kernels evaluate every value with the same operations as the
single-stage kernels, so the two paths must agree bit for bit; the oracle
(the CPU restatement of the reference) is checked at the FP64 bar.
"""
import numpy as np
import pytest
import torch

from ics import gaussian_noise, rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
SIZES = [(32, 32, 32), (17, 19, 23), (70, 9, 13), (4, 4, 4), (130, 66, 40), (64, 8, 5), (5, 130, 9)]
# (ty, zchunk, kind) of both pairs: kind 2 tiles of 64 columns, kind 4 of 32 x 16
PAIR_SHAPES = [(8, 16, 2), (16, 5, 2), (8, 1, 2), (16, 64, 2), (8, 3, 2), (16, 0, 4), (16, 7, 4), (16, 1, 4),
               (16, 64, 4), (16, 24, 4)]
SINGLE = (4, 8, 1)  # single-stage TMA kernels, 4-row tiles, z-chunk 8


def make(sp, n, nu0=0.02, nufreq=0.0, cx=1.0, cy=-0.5, cz=0.25):
    return sp.Convection(*n, 1.0 / n[0], nu0, nufreq, cx, cy, cz)


def run(sp, c, q0, tune, steps, dt=1e-4, t0=0.0, inplace=False):
    c.set_tune(sp.SP_F64, 1, *tune)
    fin = c.field()
    c.upload(fin, q0)
    fout = fin if inplace else c.field()
    c.DoRK4(fin, fout, t0, dt, steps)
    return c.download(fout), fout


def halo_images_ok(f):
    """Every face halo cell (2 deep) equals the periodic image of an interior cell."""
    lay = f.layout
    a = f.data.cpu().numpy()
    ni, nj, nk = f.ni, f.nj, f.nk
    idx = lambda i, j, k: lay.origin + k * lay.plane + j * lay.px + i
    ii = np.arange(ni)
    for k in range(-2, nk + 2):
        for j in range(-2, nj + 2):
            inside = (0 <= j < nj) + (0 <= k < nk)
            if inside < 1:
                continue  # edge of the y and z halos: not read by the stencil
            src = a[idx(ii, j % nj, k % nk)]
            if not np.array_equal(a[idx(ii, j, k)], src):
                return False
            if 0 <= j < nj and 0 <= k < nk:
                for i in (-2, -1, ni, ni + 1):
                    if a[idx(i, j, k)] != a[idx(i % ni, j, k)]:
                        return False
    return True


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("shape", PAIR_SHAPES)
def test_fused_equals_single_stage(sp, n, shape):
    c = make(sp, n)
    q0 = gaussian_noise(*n, seed=5)
    ref, _ = run(sp, c, q0, SINGLE, 7)
    got, fout = run(sp, c, q0, shape, 7)
    assert np.array_equal(got, ref)
    assert halo_images_ok(fout)


@pytest.mark.parametrize("steps", [1, 2, 51, 103])
def test_fused_step_counts_and_graphs(sp, steps):
    n = (40, 24, 28)
    c = make(sp, n)
    q0 = gaussian_noise(*n, seed=6)
    ref, _ = run(sp, c, q0, SINGLE, steps, dt=5e-5)
    got, _ = run(sp, c, q0, (8, 8, 2), steps, dt=5e-5)
    assert np.array_equal(got, ref)


def test_fused_in_place_and_time_dependent_nu(sp):
    n = (36, 20, 16)
    c = make(sp, n, nufreq=40.0)
    q0 = gaussian_noise(*n, seed=7)
    ref, _ = run(sp, c, q0, SINGLE, 9, t0=0.3, inplace=True)
    got, _ = run(sp, c, q0, (16, 8, 2), 9, t0=0.3, inplace=True)
    assert np.array_equal(got, ref)


def test_fused_matches_oracle(sp, orc):
    n = (48, 40, 36)
    c = make(sp, n, nu0=0.03, cx=-0.7, cy=0.4, cz=1.1)
    q0 = gaussian_noise(*n, seed=8)
    got, _ = run(sp, c, q0, (8, 12, 2), 13, dt=1e-4)
    p = orc.params(n, dx=1.0 / n[0], nu0=0.03, nufreq=0.0, cx=-0.7, cy=0.4, cz=1.1, upwind=True)
    ref = orc.rk4(p, q0, 0.0, 1e-4, 13)
    assert rel_l2(got, ref) < TOL64


def test_default_tune_runs_fused_pairs(sp):
    c = make(sp, (64, 64, 64))
    cfg = c.tuned_configs(sp.SP_F64, 1)
    assert cfg["P12"]["kind"] == 2 and cfg["P34"]["kind"] == 2
    assert cfg["P12"]["ty"] in (8, 16)
    # too small for 4-cell images: single-stage kernels
    c2 = make(sp, (3, 8, 8))
    assert c2.tuned_configs(sp.SP_F64, 1)["P12"]["kind"] == 0
    with pytest.raises(sp.SpError):
        c2.set_tune(sp.SP_F64, 1, 8, 8, 2)


def test_fused_batch_autotune_picks_a_valid_shape(sp):
    n = (64, 64, 64)
    c = make(sp, n)
    cfg = c.autotune(sp.SP_F64, 1)
    assert cfg["P12"]["ty"] in (8, 16) and cfg["P34"]["ty"] in (8, 16)
    q0 = gaussian_noise(*n, seed=9)
    fin, fout = c.field(), c.field()
    c.upload(fin, q0)
    c.DoRK4(fin, fout, 0.0, 1e-4, 3)
    got = c.download(fout)
    c.set_tune(sp.SP_F64, 1, *SINGLE)
    c.DoRK4(fin, fout, 0.0, 1e-4, 3)
    ref = c.download(fout)
    if cfg["P12"]["kind"] in (2, 4):
        assert np.array_equal(got, ref)
    else:  # the tuner may pick direct-load stage kernels (difference form of the update)
        assert rel_l2(got, ref) < 1e-13
    torch.cuda.synchronize()


@pytest.mark.parametrize("skip", [True, False])
def test_parareal_fine_sweep_fused_equals_single_stage(sp, skip):
    """The batched F sweep of Parareal (all slices per launch, converged slices
    skipped) gives the same fields with fused pairs as with single-stage kernels."""
    n, P = 20, 4
    outs = []
    for tune in (SINGLE, (8, 0, 2), (16, 0, 4)):
        conv = sp.Convection(n, n, n, 1.0 / n, 0.05, 0.0, 1.0, 0.5, -0.25)
        conv.set_tune(sp.SP_F64, P, *tune)
        conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.05, gridSize=n, endTime=0.02, timeStepsFine=160,
                                       timeStepsCoarse=12, kmax=3)
        fin, fsol = conv.field(), conv.field()
        conv.upload(fin, gaussian_noise(n, seed=11))
        par = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse="rk4", coarse_precision="f64", skip_converged=skip)
        par.DoParallel()
        outs.append(conv.download(fsol))
        cfg = conv.tuned_configs(sp.SP_F64, P)
        assert cfg["P12"]["kind"] == (tune[2] if tune[2] in (2, 4) else 0)
    for o in outs[1:]:
        assert np.array_equal(outs[0], o)


def test_batch_autotune_then_parareal_equals_single_stage(sp):
    """The tuner's batched-step choice (fused pairs or stage kernels, by timing
    four batched steps of each) leaves the Parareal fields bit for bit unchanged."""
    n, P = 24, 4
    outs = []
    bitwise = True
    for tune in ("auto", SINGLE):
        conv = sp.Convection(n, n, n, 1.0 / n, 0.05, 0.0, 1.0, 0.5, -0.25)
        if tune == "auto":
            cfg = conv.autotune(sp.SP_F64, P)
            assert cfg["P12"]["kind"] in (0, 2, 4) and cfg["P12"]["ty"] in (8, 16)
            # direct-load stage kernels evaluate R in the difference form: not bit for bit
            bitwise = cfg["P12"]["kind"] in (2, 4) or all(cfg[k]["kind"] == 1 for k in ("S1", "S2", "S3", "S4"))
        else:
            conv.set_tune(sp.SP_F64, P, *tune)
        conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.05, gridSize=n, endTime=0.02, timeStepsFine=120,
                                       timeStepsCoarse=12, kmax=2)
        fin, fsol = conv.field(), conv.field()
        conv.upload(fin, gaussian_noise(n, seed=13))
        par = sp.Parareal(conv, fin, fsol, 0.0, conf, coarse="rk4", coarse_precision="f64")
        par.DoParallel()
        outs.append(conv.download(fsol))
    if bitwise:
        assert np.array_equal(outs[0], outs[1])
    else:
        assert rel_l2(outs[0], outs[1]) < 1e-13


def test_kernel_times_paths_leave_field_unchanged(sp):
    n = (32, 32, 32)
    c = make(sp, n)
    f = c.field()
    c.upload(f, gaussian_noise(*n, seed=12))
    before = f.data.clone()
    kp = c.kernel_times(f, 1e-4, reps=2, path="pairs")
    ks = c.kernel_times(f, 1e-4, reps=2, path="stages")
    kt = c.kernel_times(f, 1e-4, reps=2)
    assert set(kp) == {"P12", "P34"} and set(kt) == {"P12", "P34"}
    assert set(ks) == {"S1", "S2", "S3", "S4"}
    assert all(v > 0 for v in list(kp.values()) + list(ks.values()))
    # a single-stage tune keeps valid pair shapes for timing the pairs
    c.set_tune(sp.SP_F64, 1, 4, 8, 1)
    kp2 = c.kernel_times(f, 1e-4, reps=2, path="pairs")
    assert set(kp2) == {"P12", "P34"} and all(v > 0 for v in kp2.values())
    assert torch.equal(f.data, before)


@pytest.mark.parametrize("n", [(96, 24, 20), (48, 48, 12), (33, 17, 9), (256, 16, 8)])
def test_narrow_tiles_on_grids_of_odd_tile_counts(sp, orc, n):
    """Tiles of 32 x 16 cells (sp_set_tune kind 4): grids whose width is not a multiple
    of 64 (96, 48, odd), bit for bit with the single-stage kernels and with the
    64-column tiles, across a graph chunk and in place."""
    c = make(sp, n)
    q0 = gaussian_noise(*n, seed=17)
    a, _ = run(sp, c, q0, SINGLE, 53)
    b, fb = run(sp, c, q0, (16, 0, 4), 53)
    d, _ = run(sp, c, q0, (16, 0, 4), 53, inplace=True)
    e, _ = run(sp, c, q0, (8, 0, 2), 53)
    assert np.array_equal(a, b) and np.array_equal(a, d) and np.array_equal(a, e)
    assert halo_images_ok(fb)
    p = orc.params(n, dx=1.0 / n[0], nu0=0.02, cx=1.0, cy=-0.5, cz=0.25)
    assert rel_l2(b, orc.rk4(p, q0, 0.0, 1e-4, 53)) < TOL64
