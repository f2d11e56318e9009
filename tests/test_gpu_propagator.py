"""GPU parity of the propagator against the CPU oracle (FP64 bar: 1e-12 relative L2)."""
import numpy as np
import pytest

from ics import fourier_modes, gaussian_noise, rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12   # relative L2, FP64 kernels vs the oracle's restatement of the reference
TOL32 = 2e-5    # relative L2, FP32 kernels vs the oracle computing in FP32

SIZES = [(32, 32, 32), (17, 19, 23), (16, 24, 40), (64, 8, 8), (2, 3, 5), (130, 66, 12)]
# kind: 0 direct loads, 1 TMA/mbarrier pipeline
SHAPES = [dict(kind=1, ty=8, zchunk=16), dict(kind=1, ty=4, zchunk=5), dict(kind=1, ty=16, zchunk=64),
          dict(kind=0, ty=8, zchunk=7), dict(kind=1, ty=4, zchunk=1), dict(kind=1, ty=8, zchunk=3)]


def make(sp, n, **kw):
    ni, nj, nk = n
    args = dict(nu0=0.01, nufreq=0.0, cx=1.0, cy=1.0, cz=1.0, upwind=True)
    args.update(kw)
    c = sp.Convection(ni, nj, nk, 1.0 / ni, args["nu0"], args["nufreq"], args["cx"], args["cy"], args["cz"],
                      upwind=args["upwind"])
    return c, args


def orc_params(orc, n, args):
    return orc.params(n, dx=1.0 / n[0], nu0=args["nu0"], nufreq=args["nufreq"], cx=args["cx"], cy=args["cy"],
                      cz=args["cz"], upwind=args["upwind"])


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("shape", range(len(SHAPES)))
def test_rk4_fp64_parity(sp, orc, n, shape):
    c, args = make(sp, n, cx=1.0, cy=-0.5, cz=0.25, nu0=0.02)
    s = SHAPES[shape]
    c.set_tune(sp.SP_F64, 1, s["ty"], s["zchunk"], s["kind"])
    q0 = gaussian_noise(*n, seed=0)
    dt, steps = 1e-4, 7
    fin, fout = c.field(), c.field()
    c.upload(fin, q0)
    c.DoRK4(fin, fout, 0.0, dt, steps)
    got = c.download(fout)
    ref = orc.rk4(orc_params(orc, n, args), q0, 0.0, dt, steps)
    assert rel_l2(got, ref) < TOL64
    # single step
    c.DoRK4Timestep(fin, fout, 0.0, dt)
    ref1 = orc.rk4(orc_params(orc, n, args), q0, 0.0, dt, 1)
    assert rel_l2(c.download(fout), ref1) < TOL64


@pytest.mark.parametrize("n", SIZES[:4])
@pytest.mark.parametrize("upwind", [True, False])
def test_euler_fp64_parity(sp, orc, n, upwind):
    c, args = make(sp, n, cx=0.8, cy=-0.3, cz=0.0, nu0=0.05, upwind=upwind)
    q0 = gaussian_noise(*n, seed=3)
    fin, fout = c.field(), c.field()
    c.upload(fin, q0)
    for steps in (1, 4, 5):
        c.DoEuler(fin, fout, 0.0, 1e-4, steps)
        ref = orc.euler(orc_params(orc, n, args), q0, 0.0, 1e-4, steps)
        assert rel_l2(c.download(fout), ref) < TOL64


@pytest.mark.parametrize("n", [(32, 32, 32), (17, 19, 23), (130, 66, 12)])
def test_fp32_coarse_parity(sp, orc, n):
    c, args = make(sp, n, cx=1.0, cy=0.5, cz=0.25, nu0=0.01)
    q0 = gaussian_noise(*n, seed=1).astype(np.float32)
    fin, fout = c.field(sp.SP_F32), c.field(sp.SP_F32)
    c.upload(fin, q0)
    c.DoRK4(fin, fout, 0.0, 1e-3, 7)
    ref = orc.rk4_f32(orc_params(orc, n, args), q0, 0.0, 1e-3, 7)
    assert rel_l2(c.download(fout), ref) < TOL32
    c.DoEuler(fin, fout, 0.0, 1e-4, 5)
    ref = orc.euler_f32(orc_params(orc, n, args), q0, 0.0, 1e-4, 5)
    assert rel_l2(c.download(fout), ref) < TOL32


def test_serial_fine_32cube_1000_steps(sp, orc):
    """Serial fine propagator, FP64, 32^3, c=(1,1,1), nu=0.01, Gaussian + noise, dt=1e-4, 1000 steps."""
    n = (32, 32, 32)
    c, args = make(sp, n, nu0=0.01, cx=1.0, cy=1.0, cz=1.0)
    q0 = gaussian_noise(32, seed=0)
    fin, fout = c.field(), c.field()
    c.upload(fin, q0)
    c.DoRK4(fin, fout, 0.0, 1e-4, 1000)
    ref = orc.rk4(orc_params(orc, n, args), q0, 0.0, 1e-4, 1000)
    assert rel_l2(c.download(fout), ref) < TOL64


def test_time_dependent_nu_sequence(sp, orc):
    n = (16, 16, 16)
    c, args = make(sp, n, nu0=0.05, nufreq=100.0)
    q0 = fourier_modes(16, seed=4)
    fin, fout = c.field(), c.field()
    c.upload(fin, q0)
    c.DoRK4(fin, fout, 0.013, 1e-4, 123)   # crosses graph chunks and the remainder path
    ref = orc.rk4(orc_params(orc, n, args), q0, 0.013, 1e-4, 123)
    assert rel_l2(c.download(fout), ref) < TOL64


def test_chunked_graph_path_and_inplace(sp, orc):
    n = (24, 20, 28)
    c, args = make(sp, n, nu0=0.03, cx=-1.0, cy=0.4, cz=0.9)
    q0 = fourier_modes(*n, seed=2)
    f = c.field()
    c.upload(f, q0)
    c.DoRK4(f, f, 0.0, 2e-4, 137)   # in place, 2 graph chunks of 50 + 36 direct steps
    ref = orc.rk4(orc_params(orc, n, args), q0, 0.0, 2e-4, 137)
    assert rel_l2(c.download(f), ref) < TOL64
    g = c.field()
    c.upload(g, q0)
    c.DoEuler(g, g, 0.0, 1e-4, 3)
    ref = orc.euler(orc_params(orc, n, args), q0, 0.0, 1e-4, 3)
    assert rel_l2(c.download(g), ref) < TOL64


def test_zero_steps_leave_output_untouched(sp):
    c, _ = make(sp, (8, 8, 8))
    fin, fout = c.field(), c.field()
    c.upload(fin, gaussian_noise(8))
    c.upload(fout, np.full((8, 8, 8), 3.0))
    c.DoRK4(fin, fout, 0.0, 1e-3, 0)
    assert np.all(c.download(fout) == 3.0)


def test_periodicity_matches_reference_halo(sp, orc):
    ni, nj, nk = 5, 4, 6
    c, _ = make(sp, (ni, nj, nk))
    f = c.field()
    enc = np.zeros((nk, nj, ni))
    for k in range(nk):
        for j in range(nj):
            for i in range(ni):
                enc[k, j, i] = k + 100 * j + 10000 * i
    import torch
    f.interior().copy_(torch.from_numpy(enc).cuda())
    c.Periodicity(f)
    c.synchronize()
    full = f.data.cpu().numpy()
    lay = f.layout
    jik = np.zeros((nj + 4, ni + 4, nk + 4))
    jik[2:-2, 2:-2, 2:-2] = enc.transpose(1, 2, 0)
    jik = orc.periodicity_jik(jik)
    for k in range(-2, nk + 2):
        for j in range(-2, nj + 2):
            for i in range(-2, ni + 2):
                assert full[lay.origin + k * lay.plane + j * lay.px + i] == jik[j + 2, i + 2, k + 2]


def test_import_export_roundtrip_and_host_entry(sp, orc):
    n = (20, 12, 9)
    c, args = make(sp, n)
    q0 = gaussian_noise(*n, seed=9)
    f = c.field()
    c.upload(f, q0)
    assert np.array_equal(c.download(f), q0)
    out = c.DoRK4Host(q0, 0.0, 1e-4, 11)
    ref = orc.rk4(orc_params(orc, n, args), q0, 0.0, 1e-4, 11)
    assert rel_l2(out, ref) < TOL64


def test_gpu_error_metric_matches_reference_definition(sp, orc):
    c, _ = make(sp, (16, 16, 16))
    a, b = gaussian_noise(16, seed=1), gaussian_noise(16, seed=2)
    fa, fb = c.field(), c.field()
    c.upload(fa, a)
    c.upload(fb, b)
    em, el = c.errors(fa, fb)
    assert abs(em - orc.error_maxrel(a, b)) < 1e-15
    assert abs(el - orc.error_l2rel(a, b)) < 1e-14


@pytest.mark.parametrize("n", [64, 128])
def test_fp32_coarse_has_no_drift(sp, orc, n):
    """The FP32 coarse propagator against FP64 over 28 steps of the one-GPU Parareal
    workload's coarse step (dt = 0.2/224, nu = 0.01): no worse than twice the
    oracle's own FP32 restatement (the stencil's weights, rounded to FP32, must not
    act on the O(1) field values themselves, or every field drifts)."""
    q0 = gaussian_noise(n, seed=0)
    conv = sp.Convection(n, n, n, 1.0 / n, 0.01, 0.0, 1.0, 1.0, 1.0)
    conv.autotune(sp.SP_F32, 1)
    fin, fout = conv.field(sp.SP_F32), conv.field(sp.SP_F32)
    conv.upload(fin, q0.astype(np.float32))
    dt, steps = 0.2 / 224, 28
    conv.DoRK4(fin, fout, 0.0, dt, steps)
    got = conv.download(fout).astype(np.float64)
    p = orc.params(n, nu0=0.01)
    ref64 = orc.rk4(p, q0, 0.0, dt, steps)
    ref32 = orc.rk4_f32(p, q0.astype(np.float32), 0.0, dt, steps).astype(np.float64)
    assert rel_l2(got, ref64) < max(2.0 * rel_l2(ref32, ref64), 2e-7), (rel_l2(got, ref64), rel_l2(ref32, ref64))
    # Euler in FP32 likewise
    conv.DoEuler(fin, fout, 0.0, 1e-4, steps)
    e64 = orc.euler(p, q0, 0.0, 1e-4, steps)
    e32 = orc.euler_f32(p, q0.astype(np.float32), 0.0, 1e-4, steps).astype(np.float64)
    eg = conv.download(fout).astype(np.float64)
    assert rel_l2(eg, e64) < max(2.0 * rel_l2(e32, e64), 2e-7), (rel_l2(eg, e64), rel_l2(e32, e64))
