"""CPU tests of the C ABI boundary (no GPU compute)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "sp_abi.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*|long long)\s+(sp_[a-z0-9_]+)\(", src, re.M)))


def test_library_loads_and_exports_every_declared_symbol(sp):
    lib = sp._lib.lib()
    names = header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(sp._lib.exported_symbols())
    assert lib.sp_abi_version() == 1


def test_field_layout_geometry(sp):
    for prec, es in ((sp.SP_F64, 8), (sp.SP_F32, 4)):
        for n in ((2, 2, 2), (17, 19, 23), (256, 256, 256), (48, 32, 96)):
            lay = sp.layout(*n, prec)
            assert lay.elem_size == es
            assert lay.lx * es == 16
            assert lay.px % 32 == 0 and lay.px >= n[0] + 2 * lay.lx
            assert lay.py == n[1] + 4 and lay.pz == n[2] + 4
            assert lay.plane == lay.px * lay.py
            assert lay.origin == 2 * lay.plane + 2 * lay.px + lay.lx
            assert lay.total == lay.plane * lay.pz
            # interior rows start 16-byte aligned (128-bit loads / TMA boxes)
            assert (lay.origin * es) % 16 == 0 and (lay.px * es) % 16 == 0


def test_invalid_arguments_return_status(sp):
    lib = sp._lib.lib()
    out = sp._lib.SpLayout()
    assert lib.sp_field_layout(1, 4, 4, 0, C.byref(out)) == sp._lib.SP_ERR_INVALID
    assert "2^3" in sp._lib.last_error()
    assert lib.sp_field_layout(4, 4, 4, 7, C.byref(out)) == sp._lib.SP_ERR_INVALID


def test_no_device_is_an_error_not_a_fallback(sp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = sp._lib.SpParams(8, 8, 8, 0.125, 0.1, 0.0, 1.0, 1.0, 1.0, 1)
    h = C.c_void_p()
    rc = sp._lib.lib().sp_convection_create(C.byref(p), 0, C.byref(h))
    assert rc in (sp._lib.SP_ERR_UNSUPPORTED, sp._lib.SP_ERR_CUDA)
    with pytest.raises(sp.SpError):
        sp.Convection(8, 8, 8, 0.125, 0.1, 0.0, 1, 1, 1)


def test_runtime_configuration_matches_oracle(sp, orc):
    from stencilparareal_b200.parareal import RuntimeConfiguration
    for P, f, g in ((32, 20000, 200), (8, 32768, 2048), (12, 5000, 50), (7, 100, 3)):
        conf = RuntimeConfiguration(timeSlices=P, endTime=0.2, timeStepsFine=f, timeStepsCoarse=g)
        d = orc.parareal_derived(orc.parareal_cfg(0.2, P, f, g, 1))
        assert conf.timeStepsFine() == d["tsFineTotal"] and conf.timeStepsCoarse() == d["tsCoarseTotal"]
        assert conf.timeStepsFinePerTimeSlice() == d["tsFine"]
        assert conf.timeStepsCoarsePerTimeSlice() == d["tsCoarse"]
        assert conf.dtFine() == d["dtFine"] and conf.dtCoarse() == d["dtCoarse"]
        assert conf.timeSliceSize() == d["timeSliceSize"]
    # defaults of RuntimeConfiguration.cpp:7-13
    c = RuntimeConfiguration()
    assert (c.nu0(), c.nufreq(), c.gridSize(), c.endTime(), c.kmax(), c.async_()) == (1.0, 0.0, 32, 0.05, 5, True)
    assert RuntimeConfiguration(mode="bogus").mode() == "compare"
    # cfl (RuntimeConfiguration.h:105-111)
    c = RuntimeConfiguration(timeSlices=8, nu0=0.1, gridSize=128, endTime=0.1, timeStepsFine=32768,
                             timeStepsCoarse=2048)
    assert abs(c.cflFine() - 0.0075) < 1e-12 and abs(c.cflCoarse() - 0.12) < 1e-12
