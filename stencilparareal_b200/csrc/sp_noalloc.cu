// sp_noalloc.cu -- DoRK4 for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside a host process
// whose device memory is owned by another allocator (a framework's caching
// pool, a solver that pre-reserves all of HBM), code paths that must not
// allocate after start-up (real-time loops, code between allocation-free
// checkpoints), and plugins that may only use memory handed to them.  The
// regular sp_do_rk4 needs a handle whose creation allocates the RK4 work
// fields.  sp_do_rk4_noalloc instead keeps its work fields in a file-scope
// device array that exists from the moment the library is loaded on a
// device until the process exits, so it allocates nothing: the caller passes
// only the input and output fields.
//
// The array is SP_NOALLOC_SCRATCH_BYTES (16 MiB) on every GPU that loads the
// library, enough for the three work fields of grids up to about 80^3 in
// FP64.  All calls share it: two calls whose kernels overlap on the GPU (for
// example on two streams, or from two host threads) race on it and corrupt
// each other's results.  Each call overwrites every scratch cell it later
// reads, so the contents left by the previous call do not matter; only the
// error word is cleared at the start of each call.  Every call waits for
// its stream before it returns: it reads the error word of the bounded
// in-kernel waits back to the host, as sp_convection_synchronize does for a
// handle.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/sp_abi.h"
#include "sp_internal.h"

namespace {

constexpr size_t kScratchBytes = SP_NOALLOC_SCRATCH_BYTES;

// Lives in every GPU's memory from module load until process exit.  In host
// code these names are only host-side stand-ins: the device address comes from
// cudaGetSymbolAddress (see device_setup).
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];
static __device__ __align__(256) int g_err_word[64];

constexpr int kMaxDevices = 64;

struct DeviceSetup {
    bool done = false;        // set only after a set-up that succeeded
    int major = 0, minor = 0; // compute capability of the device
    void* scratch = nullptr;  // device address of g_scratch on this device
    int* err = nullptr;       // device address of g_err_word on this device
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

// Once per device, with that device current: read its compute capability,
// look up the device addresses of the file-scope arrays and raise the
// shared-memory limit of the TMA kernels.  A set-up that fails is not
// remembered: the next call on that device tries again.
cudaError_t device_setup(int dev, DeviceSetup** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& s = g_setup[dev];
    *out = &s;
    if (s.done) return cudaSuccess;
    int major = 0, minor = 0;
    cudaError_t e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (e != cudaSuccess) return e;
    s.major = major;
    s.minor = minor;
    if (major < 10) return cudaSuccess;  // rejected by the caller; nothing to set up
    void* p = nullptr;
    void* q = nullptr;
    if ((e = cudaGetSymbolAddress(&p, g_scratch)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress(&q, g_err_word)) != cudaSuccess) return e;
    if ((e = sp::prepare_kernels()) != cudaSuccess) return e;
    s.scratch = p;
    s.err = static_cast<int*>(q);
    s.done = true;
    return cudaSuccess;
}

}  // namespace

extern "C" int sp_do_rk4_noalloc(const sp_params* p, const double* in, double* out, double tStart, double dt,
                                 int timesteps, void* stream) {
    using namespace sp;
    if (!p || !in || !out) return sp_report(SP_ERR_INVALID, "sp_do_rk4_noalloc: null argument");
    if (p->ni < 2 || p->nj < 2 || p->nk < 2 || !(p->dx > 0))
        return sp_report(SP_ERR_INVALID, "sp_do_rk4_noalloc: grid must be at least 2^3 and dx positive");
    if (timesteps < 0) return sp_report(SP_ERR_INVALID, "sp_do_rk4_noalloc: negative step count");
    const Geo g = make_geo(p->ni, p->nj, p->nk, 8);
    const size_t need = (size_t)3 * g.total * sizeof(double);
    if (need > kScratchBytes)
        return sp_report(SP_ERR_INVALID,
                         "sp_do_rk4_noalloc: a %dx%dx%d FP64 grid needs %zu bytes of work fields, more than the "
                         "%zu-byte built-in scratch (use sp_do_rk4 with a handle)",
                         p->ni, p->nj, p->nk, need, kScratchBytes);
    if (timesteps == 0) return SP_OK;  // as DoRK4: no step, output untouched
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return sp_report(SP_ERR_CUDA, "sp_do_rk4_noalloc: no usable current device");
    DeviceSetup* ds = nullptr;
    if ((e = device_setup(dev, &ds)) != cudaSuccess)
        return sp_report(SP_ERR_CUDA, "sp_do_rk4_noalloc: set-up on device %d failed: %s", dev, cudaGetErrorString(e));
    if (ds->major < 10)
        return sp_report(SP_ERR_UNSUPPORTED, "this library is built for sm_100a (found sm_%d%d)", ds->major, ds->minor);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* ya = static_cast<double*>(ds->scratch);
    double* yb = ya + g.total;
    double* acc = yb + g.total;
    const Coef coef = make_coef(p->dx, p->cx, p->cy, p->cz, p->upwind);
    Tune t;
    {
        Shape sh;
        const long long tiles = (long long)((p->ni + 63) / 64) * ((p->nj + 3) / 4);
        int zc = p->nk;
        while (zc > 8 && tiles * ((p->nk + zc - 1) / zc) < 148LL * 8) zc = (zc + 1) / 2;
        sh.zchunk = zc < 1 ? 1 : zc;
        t.set_all(sh);
    }
    if ((e = cudaMemsetAsync(ds->err, 0, sizeof(int), s)) != cudaSuccess ||
        (e = launch_periodicity(g, const_cast<double*>(in), 1, s)) != cudaSuccess)
        return sp_report(SP_ERR_CUDA, "sp_do_rk4_noalloc: %s", cudaGetErrorString(e));
    for (int i = 0; i < timesteps; ++i) {
        // DoRK4 (Convection.cpp:292-303): step 0 reads `in`, later steps run in
        // place on `out`; step i uses nu(tStart + i*dt).
        const double tt = i == 0 ? tStart : tStart + i * dt;
        const void* src = i == 0 ? static_cast<const void*>(in) : static_cast<const void*>(out);
        StageLaunch L;
        L.prec = 0;
        L.items = 1;
        L.coef = coef;
        L.nu = p->nu0 * (1. + .5 * std::sin(p->nufreq * tt));
        const double dthalf = dt * .5;
        L.op = OP_RK_S1; L.yin = src; L.yout = ya; L.acc = acc; L.c_y = dthalf; L.c_acc = dt / 6.;
        if ((e = launch_stage(g, L, t, s, ds->err)) != cudaSuccess) break;
        L.op = OP_RK_S2; L.yin = ya; L.q = src; L.yout = yb; L.c_y = dthalf; L.c_acc = dt / 3.;
        if ((e = launch_stage(g, L, t, s, ds->err)) != cudaSuccess) break;
        L.op = OP_RK_S3; L.yin = yb; L.q = src; L.yout = ya; L.c_y = dt; L.c_acc = dt / 3.;
        if ((e = launch_stage(g, L, t, s, ds->err)) != cudaSuccess) break;
        L.op = OP_RK_S4; L.yin = ya; L.q = src; L.yout = out; L.c_acc = dt / 6.;
        if ((e = launch_stage(g, L, t, s, ds->err)) != cudaSuccess) break;
    }
    if (e != cudaSuccess) return sp_report(SP_ERR_CUDA, "sp_do_rk4_noalloc: launch failed: %s", cudaGetErrorString(e));
    int word = 0;
    if ((e = cudaMemcpyAsync(&word, ds->err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return sp_report(SP_ERR_CUDA, "sp_do_rk4_noalloc: %s", cudaGetErrorString(e));
    if (word != 0) return sp_report(SP_ERR_TIMEOUT, "sp_do_rk4_noalloc: a bounded in-kernel wait gave up");
    return SP_OK;
}
