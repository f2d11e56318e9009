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
def test_two_processes_one_gpu_equal_single_process(sp, coarse, prec):
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
    conv.upload(f0, gaussian_noise(n, seed=1))
    sp.Parareal(conv, f0, fs, 0.0, conf, coarse=coarse, coarse_precision=prec).DoParallel()
    assert np.array_equal(last, conv.download(fs))
