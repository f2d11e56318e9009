"""GPU test of sp_do_rk4_noalloc, the allocation-free form of DoRK4.

It serves callers that cannot call cudaMalloc (their process's GPU memory
belongs to another allocator or is reserved up front, or they may only touch
the buffers they are handed): the RK4 work fields live in a device array
built into the library, so the call needs no handle and allocates nothing.
The test calls it through the C ABI twice in a row and checks each result
against the regular handle-based entry point sp_do_rk4 at the FP64 tolerance
of the parity tests.  This file is collected last on purpose.
"""
import ctypes as C

import pytest
import torch

from ics import fourier_modes, gaussian_noise, rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def test_noalloc_matches_handle_entry_point_on_two_calls_in_a_row(sp):
    L = sp._lib
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
        rc = L.lib().sp_do_rk4_noalloc(C.byref(p), C.c_void_p(fin.ptr), C.c_void_p(out.ptr), t0, 1e-4, steps,
                                       None)
        L.check(rc)
        torch.cuda.synchronize()
        if call == 1:
            # the second call reuses the built-in array: it takes no device memory
            assert torch.cuda.mem_get_info()[0] == free_before
        assert rel_l2(conv.download(out), conv.download(ref)) < TOL64, call


def test_noalloc_rejects_grids_beyond_the_builtin_scratch(sp):
    L = sp._lib
    p = L.SpParams(256, 256, 256, 1.0 / 256, 1e-3, 0.0, 1.0, 0.5, 0.25, 1)
    rc = L.lib().sp_do_rk4_noalloc(C.byref(p), C.c_void_p(0x1000), C.c_void_p(0x1000), 0.0, 1e-4, 1, None)
    assert rc == L.SP_ERR_INVALID
    assert "built-in scratch" in L.last_error()
