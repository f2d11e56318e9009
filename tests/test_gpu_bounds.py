"""GPU test of the bounds-checked build (libstencilparareal_checked.so, built
with -DSP_BOUNDS_CHECK=1): every global store of the stage, fused-pair and
widening kernels is tested against its output allocation and skipped, not
made, when it falls outside; sp_store_violations counts those stores.  The
stand-in for a memory sanitizer: ragged grids, every kernel kind and shape,
FP32, batched Parareal with converged-slice skipping and the adjoint must store
inside their allocations.  A run with the allocation bounds narrowed on the host
by one plane (SP_BOUNDS_SHRINK_PLANES) shows that the check counts stores --
those it skips lie inside the real allocation, so nothing is written out of
bounds either way."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "stencilparareal_b200", "libstencilparareal_checked.so")

SCRIPT = r"""
import ctypes as C, json, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np
import stencilparareal_b200 as sp
from ics import gaussian_noise
L = sp._lib

def violations():
    chk, cnt = C.c_int(), C.c_longlong()
    L.check(L.lib().sp_store_violations(C.byref(chk), C.byref(cnt)))
    return chk.value, cnt.value

out = {{"lib": L.LIB_PATH}}
full = {full}
sizes = [(17, 19, 23), (130, 66, 12), (4, 4, 4), (64, 8, 5), (5, 130, 9)] if full else [(17, 19, 23)]
for n in sizes:
    c = sp.Convection(*n, 1.0 / n[0], 0.02, 0.0, 1.0, -0.5, 0.25)
    q0 = gaussian_noise(*n, seed=1)
    tunes = ([(4, 8, 1), (16, 3, 1), (8, 5, 0), (8, 0, 2), (16, 2, 2), (16, 0, 4), (16, 3, 4)] if full
             else [(4, 8, 1), (8, 0, 2), (16, 0, 4)])
    for tune in tunes:
        c.set_tune(sp.SP_F64, 1, *tune)
        fi, fo = c.field(), c.field()
        c.upload(fi, q0)
        c.DoRK4(fi, fo, 0.0, 1e-4, 3)
        c.DoEuler(fi, fo, 0.0, 1e-4, 2)
    if full:
        gi, go = c.field(sp.SP_F32), c.field(sp.SP_F32)
        c.upload(gi, q0.astype(np.float32))
        c.DoRK4(gi, go, 0.0, 1e-3, 2)
if full:
    n, P = 20, 4
    for tune in ((4, 8, 1), (8, 0, 2), (16, 0, 4)):
        conv = sp.Convection(n, n, n, 1.0 / n, 0.05, 0.0, 1.0, 0.5, -0.25)
        conv.set_tune(sp.SP_F64, P, *tune)
        conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.05, gridSize=n, endTime=0.01, timeStepsFine=80,
                                       timeStepsCoarse=8, kmax=3)
        fin, fsol = conv.field(), conv.field()
        conv.upload(fin, gaussian_noise(n, seed=2))
        sp.Parareal(conv, fin, fsol, 0.0, conf, coarse="rk4", coarse_precision="f32").DoParallel()
    from stencilparareal_b200.adjoint import misfit_gradient
    conv = sp.Convection(12, 12, 12, 1.0 / 12, 0.05, 0.0, 0.7, -0.4, 0.3)
    f0, ft = conv.field(), conv.field()
    conv.upload(f0, gaussian_noise(12, seed=3, amp=1e-2))
    conv.upload(ft, gaussian_noise(12, seed=4, amp=1e-2))
    misfit_gradient(conv, f0, ft, 0.0, 2e-3, 6, checkpoint_every=2)
out["checked"], out["count"] = violations()
print(json.dumps(out))
"""


def run_checked(full: bool, shrink: int = 0) -> dict:
    env = dict(os.environ, STENCILPARAREAL_LIB=CHECKED)
    if shrink:
        env["SP_BOUNDS_SHRINK_PLANES"] = str(shrink)
    script = SCRIPT.format(root=ROOT, tests=os.path.join(ROOT, "tests"), full=full)
    r = subprocess.run([sys.executable, "-c", script], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module")
def checked_lib():
    if not os.path.exists(CHECKED):
        pytest.fail("libstencilparareal_checked.so is missing: run __graft_entry__.build()")
    return CHECKED


def test_every_stencil_store_inside_its_allocation(checked_lib):
    out = run_checked(full=True)
    assert out["lib"] == checked_lib and out["checked"] == 1
    assert out["count"] == 0


def test_narrowed_bounds_are_counted(checked_lib):
    # z-images of the planes z = 0, 1 land in the last padded plane of every field
    out = run_checked(full=False, shrink=1)
    assert out["checked"] == 1 and out["count"] > 0


def test_release_build_reports_unchecked(sp):
    import ctypes as C
    chk, cnt = C.c_int(-1), C.c_longlong(-1)
    assert sp._lib.lib().sp_store_violations(C.byref(chk), C.byref(cnt)) == sp._lib.SP_OK
    assert chk.value == 0 and cnt.value == 0
