"""Builds the sm_100a shared library ``stencilparareal_b200/libstencilparareal.so``
and, with ``checked=True``, its bounds-checked variant
``libstencilparareal_checked.so`` (``-DSP_BOUNDS_CHECK=1``: every global store of
the stencil-producing kernels is tested against its output allocation; see
sp_store_violations in include/sp_abi.h).

nvcc cross-compiles for sm_100a without a GPU.  The CUDA runtime is linked
statically so the library does not depend on which libcudart a host process
(e.g. PyTorch) loaded first.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libstencilparareal.so")
LIB_CHECKED = os.path.join(HERE, "libstencilparareal_checked.so")
SOURCES = ["sp_kernels.cu", "sp_fused.cu", "sp_cluster.cu", "sp_lib.cu", "sp_noalloc.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, checked=False):
    lib = LIB_CHECKED if checked else LIB
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(os.path.dirname(HERE), "include", "sp_abi.h"), os.path.abspath(__file__)]
    if not force and not _stale(lib, deps):
        return lib
    objs = []
    bdir = os.path.join(HERE, "_build_checked" if checked else "_build")
    os.makedirs(bdir, exist_ok=True)
    flags = NVCC_FLAGS + (["-DSP_BOUNDS_CHECK=1"] if checked else [])
    # the translation units compile in parallel (one nvcc process each)
    procs = []
    for src in SOURCES:
        obj = os.path.join(bdir, src.replace(".cu", ".o"))
        cmd = [nvcc()] + flags + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [cmd for cmd, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
