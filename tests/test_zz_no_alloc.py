"""GPU test of sp_do_rk4_noalloc, the allocation-free form of DoRK4.

It serves callers that cannot call cudaMalloc (their process's GPU memory
belongs to another allocator or is reserved up front, or they may only touch
the buffers they are handed): the RK4 work fields live in a device array
built into the library, so the call needs no handle and allocates nothing.
The tests call it through the C ABI and check its results against the CPU
oracle and against the regular handle-based entry point sp_do_rk4, at the
FP64 tolerance of the parity tests: two calls in a row, a time-dependent
diffusivity from a non-zero start time, in-place stepping, zero steps and a
grid at the size limit of the built-in array.  This file is collected last on
purpose.
"""
import ctypes as C

import pytest
import torch

from ics import fourier_modes, gaussian_noise, rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _noalloc(sp, p, fin, fout, t0, dt, steps):
    L = sp._lib
    torch.cuda.synchronize()
    rc = L.lib().sp_do_rk4_noalloc(C.byref(p), C.c_void_p(fin.ptr), C.c_void_p(fout.ptr), t0, dt, steps, None)
    L.check(rc)
    torch.cuda.synchronize()


def _orc_params(orc, conv):
    p = conv.params
    return orc.params((p.ni, p.nj, p.nk), dx=p.dx, nu0=p.nu0, nufreq=p.nufreq, cx=p.cx, cy=p.cy, cz=p.cz,
                      upwind=bool(p.upwind))


def test_noalloc_matches_handle_entry_point_on_two_calls_in_a_row(sp, orc):
    n = (48, 40, 36)
    conv = sp.Convection(*n, 1.0 / n[0], 0.02, 0.0, 1.0, -0.5, 0.25)
    p = conv.params
    runs = [(gaussian_noise(*n, seed=0), 0.0, 17), (fourier_modes(*n, seed=1), 0.003, 9)]
    fields = [(conv.field(), conv.field(), conv.field()) for _ in runs]
    for call, ((q0, t0, steps), (fin, ref, out)) in enumerate(zip(runs, fields)):
        conv.upload(fin, q0)
        conv.DoRK4(fin, ref, t0, 1e-4, steps)
        conv.synchronize()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _noalloc(sp, p, fin, out, t0, 1e-4, steps)
        if call == 1:
            # the second call reuses the built-in array: it takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        got = conv.download(out)
        assert rel_l2(got, conv.download(ref)) < TOL64, call
        assert rel_l2(got, orc.rk4(_orc_params(orc, conv), q0, t0, 1e-4, steps)) < TOL64, call


def test_noalloc_time_dependent_nu_from_nonzero_start(sp, orc):
    """nu(t) = nu0 (1 + sin(nufreq t)/2) per step from tStart (Convection.h:81-84)."""
    n = (33, 20, 27)
    conv = sp.Convection(*n, 1.0 / n[0], 0.05, 50.0, -0.7, 0.4, 1.0)
    q0 = gaussian_noise(*n, seed=5)
    fin, ref, out = conv.field(), conv.field(), conv.field()
    conv.upload(fin, q0)
    t0, dt, steps = 0.0125, 2e-4, 23
    conv.DoRK4(fin, ref, t0, dt, steps)
    conv.synchronize()
    _noalloc(sp, conv.params, fin, out, t0, dt, steps)
    got = conv.download(out)
    assert rel_l2(got, conv.download(ref)) < TOL64
    assert rel_l2(got, orc.rk4(_orc_params(orc, conv), q0, t0, dt, steps)) < TOL64


def test_noalloc_in_place_and_zero_steps(sp, orc):
    n = (24, 24, 24)
    conv = sp.Convection(*n, 1.0 / n[0], 0.01, 0.0, 1.0, 1.0, 1.0)
    q0 = fourier_modes(*n, seed=7)
    f = conv.field()
    conv.upload(f, q0)
    # zero steps leave the output untouched (DoRK4, Convection.cpp:292-303)
    other = conv.field()
    conv.upload(other, gaussian_noise(*n, seed=8))
    before = other.data.clone()
    _noalloc(sp, conv.params, f, other, 0.0, 1e-4, 0)
    assert torch.equal(other.data, before)
    # in == out: the field is advanced in place
    _noalloc(sp, conv.params, f, f, 0.0, 1e-4, 11)
    assert rel_l2(conv.download(f), orc.rk4(_orc_params(orc, conv), q0, 0.0, 1e-4, 11)) < TOL64


def test_noalloc_grid_at_the_size_limit(sp, orc):
    """81^3 FP64, the largest cube that fits: three work fields of 96 x 85 x 85 doubles,
    16.65 MB of the 16 MiB (16.78 MB) array."""
    n = (81, 81, 81)
    lay = sp.layout(*n)
    assert 3 * lay.total * 8 <= sp._lib.SP_NOALLOC_SCRATCH_BYTES
    conv = sp.Convection(*n, 1.0 / n[0], 0.01, 0.0, 1.0, 0.5, 0.25)
    q0 = gaussian_noise(*n, seed=9)
    fin, out = conv.field(), conv.field()
    conv.upload(fin, q0)
    _noalloc(sp, conv.params, fin, out, 0.0, 1e-4, 6)
    assert rel_l2(conv.download(out), orc.rk4(_orc_params(orc, conv), q0, 0.0, 1e-4, 6)) < TOL64


def test_noalloc_rejects_grids_beyond_the_builtin_scratch(sp):
    L = sp._lib
    for n in ((256, 256, 256), (82, 82, 82)):
        lay = sp.layout(*n)
        assert 3 * lay.total * 8 > L.SP_NOALLOC_SCRATCH_BYTES
        p = L.SpParams(*n, 1.0 / n[0], 1e-3, 0.0, 1.0, 0.5, 0.25, 1)
        rc = L.lib().sp_do_rk4_noalloc(C.byref(p), C.c_void_p(0x1000), C.c_void_p(0x1000), 0.0, 1e-4, 1, None)
        assert rc == L.SP_ERR_INVALID
        assert "built-in scratch" in L.last_error()
