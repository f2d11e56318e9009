"""Large grids through a size-independent property: translation invariance.

A 1024^3 field made of 4 x 4 x 4 copies of a 256^3 field, stepped with the
256^3 grid's spacing, must become 4 x 4 x 4 copies of the 256^3 result: the
grid is periodic, so every cell sees the same neighbour values and the same
weights as its image in the small grid, and the fields agree bit for bit.  The
256^3 results are themselves pinned to the oracle (tests/test_gpu_pins.py), so
this carries that parity to fields of 1.1e9 cells (8.6 GB each, five of them on
the device): the 64-bit offsets, tile and plane-range counts and tensor maps of
both FP64 paths at the largest grid these tests hold."""
import pytest
import torch

from ics import fourier_modes

pytestmark = pytest.mark.gpu

SMALL, REP, STEPS = 256, 4, 3
NU, C, DT = 1e-3, (1.0, 0.5, 0.25), 5e-5


@pytest.mark.parametrize("tune", [(16, 64, 4), (4, 8, 1)], ids=["fused-pairs-32x16", "stage-kernels"])
def test_tiled_1024cube_equals_tiled_256cube(sp, tune):
    dx = 1.0 / SMALL
    small = sp.Convection(SMALL, SMALL, SMALL, dx, NU, 0.0, *C)
    small.set_tune(sp.SP_F64, 1, *tune)
    q0 = torch.from_numpy(fourier_modes(SMALL, seed=1)).cuda()
    a, b = small.field(), small.field()
    small.upload(a, q0)
    small.DoRK4(a, b, 0.0, DT, STEPS)
    ref = b.interior().clone()
    del a, b, small
    torch.cuda.empty_cache()

    n = SMALL * REP
    big = sp.Convection(n, n, n, dx, NU, 0.0, *C)
    big.set_tune(sp.SP_F64, 1, *tune)
    fin, fout = big.field(), big.field()
    big.upload(fin, q0.repeat(REP, REP, REP))
    big.DoRK4(fin, fout, 0.0, DT, STEPS)
    big.synchronize()
    got = fout.interior().view(REP, SMALL, REP, SMALL, REP, SMALL)
    for kz in range(REP):
        for ky in range(REP):
            for kx in range(REP):
                assert torch.equal(got[kz, :, ky, :, kx, :], ref), (kz, ky, kx)
