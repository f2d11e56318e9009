"""The multi-GPU slice pipeline (DistributedParareal) with world_size 2 gloo ranks.

On CPU the windows are oracle-backed (tests/oracle_window.py); the last rank's
result must equal the serial oracle Parareal on the whole slice range.  On a
GPU the two ranks share one device (gloo exchange through host memory; no
kernel waits on another process) and must reproduce the single-process GPU
Parareal bit for bit.
"""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from ics import gaussian_noise

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _cpu_rank(rank, world, port, out, spec):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    from oracle import oracle as O
    from oracle_window import OracleWindow
    from stencilparareal_b200.parareal import DistributedParareal, slice_bounds
    O.set_threads(1)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    n, P, kmax, coarse, delta = spec
    lo, hi = slice_bounds(P, world, rank)
    p = O.params(n, nu0=0.05, cx=1.0, cy=0.5, cz=-0.25)
    w = OracleWindow(p, 0.02, P, 120, 14, lo, hi - lo, gaussian_noise(n, seed=1), coarse=coarse, delta=delta)
    its, defects = DistributedParareal(w).run(kmax)
    if rank == world - 1:
        np.save(out, w.boundary.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("coarse,delta", [(0, False), (2, True), (1, False)])
def test_gloo_world2_oracle_windows_equal_serial_parareal(orc, coarse, delta):
    n, P, kmax = 8, 5, 3
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "last.npy")
        mp.start_processes(_cpu_rank, args=(2, _free_port(), out, (n, P, kmax, coarse, delta)), nprocs=2,
                           join=True, start_method="spawn")
        last = np.load(out)
    p = orc.params(n, nu0=0.05, cx=1.0, cy=0.5, cz=-0.25)
    cfg = orc.parareal_cfg(0.02, P, 120, 14, kmax, coarse=coarse, delta=delta)
    q, qs, em, el = orc.parareal(p, cfg, gaussian_noise(n, seed=1))
    assert np.array_equal(last, q)


def _gpu_rank(rank, world, port, out, spec):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    import stencilparareal_b200 as sp
    from stencilparareal_b200.parareal import DistributedParareal, WindowParareal, slice_bounds
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    n, P, kmax, coarse, prec = spec
    lo, hi = slice_bounds(P, world, rank)
    conv = sp.Convection(n, n, n, 1.0 / n, 0.05, 0.0, 1.0, 0.5, -0.25)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.05, gridSize=n, endTime=0.02, timeStepsFine=120,
                                   timeStepsCoarse=14, kmax=kmax)
    f0, fs = conv.field(), conv.field()
    conv.upload(f0, gaussian_noise(n, seed=1))
    w = WindowParareal(conv, f0, fs, 0.0, conf, lo, hi - lo, coarse=coarse, coarse_precision=prec)
    DistributedParareal(w).run(kmax)
    conv.synchronize()
    if rank == world - 1:
        np.save(out, conv.download(w.boundary))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("coarse,prec", [("rk4", "f32"), ("euler", "f64")])
def test_two_processes_one_gpu_equal_single_process(sp, orc, coarse, prec):
    n, P, kmax = 12, 5, 3
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "last.npy")
        mp.start_processes(_gpu_rank, args=(2, _free_port(), out, (n, P, kmax, coarse, prec)), nprocs=2,
                           join=True, start_method="spawn")
        last = np.load(out)
    conv = sp.Convection(n, n, n, 1.0 / n, 0.05, 0.0, 1.0, 0.5, -0.25)
    conf = sp.RuntimeConfiguration(timeSlices=P, nu0=0.05, gridSize=n, endTime=0.02, timeStepsFine=120,
                                   timeStepsCoarse=14, kmax=kmax)
    f0, fs = conv.field(), conv.field()
    q0 = gaussian_noise(n, seed=1)
    conv.upload(f0, q0)
    sp.Parareal(conv, f0, fs, 0.0, conf, coarse=coarse, coarse_precision=prec).DoParallel()
    assert np.array_equal(last, conv.download(fs))
    # and against the oracle's serial restatement of DoParallel (Parareal.h:110-171);
    # with FP32 G the windows use the increment form, as the single-process default
    kind = {("rk4", "f32"): orc.COARSE_RK4_F32, ("euler", "f64"): orc.COARSE_EULER_F64}[(coarse, prec)]
    cfg = orc.parareal_cfg(0.02, P, 120, 14, kmax, coarse=kind, delta=(prec == "f32"))
    q, qs, em, el = orc.parareal(orc.params(n, nu0=0.05, cx=1.0, cy=0.5, cz=-0.25), cfg, q0)
    diff = float(np.sqrt(((last - q) ** 2).sum() / (q ** 2).sum()))
    assert diff < (1e-11 if prec == "f64" else 1e-8), diff


@pytest.mark.gpu
@pytest.mark.parametrize("problem", ["config3", "paper"])
def test_benchmark_slice_pipeline_two_ranks_one_gpu(sp, problem):
    """bench.py's N>1 Parareal slice pipeline, launched as the benchmark is (torchrun,
    one process per rank), with the gloo backend so that both ranks can share the
    one GPU here (the exchange goes through host memory; no kernel waits on the
    other process).  On N GPUs the same code exchanges over NCCL.  Both problems:
    the one-GPU Parareal workload (defect rule) and the reference's published
    experiment (Euler coarse, exactQ, 3 fixed iterations), on a 16^3 grid."""
    import json
    import subprocess
    import sys
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--gpus", "2",
           "--pipeline-only", "--dist-backend", "gloo", "--pipeline-grid", "16", "--pipeline-slices", "6",
           "--pipeline-problem", problem]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    out = json.loads(line)["parareal_pipeline"]
    assert out["ranks"] == 2
    if problem == "config3":
        assert 1 <= out["iterations"] <= 6 and out["defects"][-1] < 1e-8
        assert out["err_l2_vs_serial"] < 1e-8
    else:
        # three iterations of 6 slices: the result approaches the serial fine run
        # (at 128^3 the reference's table has 1e-3, 1e-5, 1e-7; the upwind Euler
        # coarse propagator is less accurate on 16^3: 1.4e-4 after 3 iterations)
        assert out["iterations"] == 3
        assert 0 < out["err_max_vs_serial"] < 1e-3
        assert out["defects"][0] > out["defects"][1] > out["defects"][2]
    assert out["seconds"] > 0 and out["one_gpu_parareal_s"] > 0
