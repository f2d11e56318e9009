"""The C++ facade (include/sp_convection.hpp) compiled into a Compare-mode driver
shaped like the reference's src/Parareal/main.cpp; its per-iteration errors
must equal the oracle's serial restatement of the same run."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_compare_driver_matches_oracle(sp, orc, tmp_path):
    exe = str(tmp_path / "compare_main")
    libdir = os.path.join(ROOT, "stencilparareal_b200")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "compare_main.cpp"), "-L", libdir, "-lstencilparareal",
                    "-Xlinker", "-rpath", "-Xlinker", libdir, "-o", exe], check=True)
    P, N, K = 4, 24, 3
    args = ["--gridSize", str(N), "--endTime", "0.02", "--timeStepsFine", "400", "--timeStepsCoarse", "30",
            "--nu0", "0.1", "--kmax", str(K), "--noasync"]
    out = subprocess.run([exe, str(P)] + args, check=True, capture_output=True, text=True).stdout
    errs = [float(x) for x in re.findall(r"Error after iteration \d+: (\S+)", out)]
    assert len(errs) == K
    # 30 coarse steps over 4 slices -> rounded up to 32 (RuntimeConfiguration.cpp:143-151)
    assert "timesteps per slice coarse propagator: 8" in out
    p = orc.params(N, nu0=0.1)
    cfg = orc.parareal_cfg(0.02, P, 400, 30, K, coarse=orc.COARSE_EULER_F64)
    q, qs, em, el = orc.parareal(p, cfg, orc.fillq(p, 0.0))
    for mine, ref in zip(errs, em):
        assert abs(mine - ref) <= 1e-6 * ref, (mine, ref)
