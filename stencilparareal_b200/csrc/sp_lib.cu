// sp_lib.cu -- the C ABI (include/sp_abi.h): propagator handles, the time-step
// loop (CUDA-graph chunks), the one-GPU Parareal driver, the adjoint.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <functional>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sp_abi.h"
#include "sp_internal.h"

using namespace sp;

namespace {
// Host-side NVTX range over a phase of the driver (propagation calls, the
// Parareal predictor and iterations, the adjoint); the header-only NVTX v3
// records nothing unless a profiler that collects NVTX is attached.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace

// ---------------------------------------------------------------------------
// Errors.
namespace {
thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define SP_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail(SP_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                           "sp_lib.cu", __LINE__);                                      \
    } while (0)

// computenu (Convection.h:81-84)
inline double computenu(double nu0, double nufreq, double t) { return nu0 * (1. + .5 * std::sin(nufreq * t)); }

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    // Allocates and zeroes n bytes.  The zeroing is complete on return: the
    // library's work runs on non-blocking streams, which do not order after
    // cudaMemset's legacy-stream work.
    cudaError_t alloc(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) { p = nullptr; return e; }
        bytes = n;
        e = cudaMemset(p, 0, n);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        return e;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace

int sp::sp_report(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

// ---------------------------------------------------------------------------
// Propagator handle.
struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    long long nodes = 0;
};

struct sp_convection {
    sp_params P{};
    int device = 0;
    Geo g[2];          // [0] FP64, [1] FP32
    Geo g4;            // FP64 with 4-cell halos: internal fields of the fused stage pairs
    Coef coef;
    cudaStream_t own = nullptr, user = nullptr;
    DevBuf scratch[2];  // per precision: ya, yb, acc (x batch) for DoRK4 / Euler ping-pong
    int scratch_items[2] = {0, 0};
    DevBuf wide;        // fused-pair fields (geometry g4): two step-start/accumulator fields and y2 (x batch)
    int wide_items = 0;
    DevBuf err;         // device error word
    DevBuf red;         // reduction scratch (8 doubles)
    DevBuf dense;       // staging for the host-buffer entry point
    DevBuf adj_ckpt, adj_seg, adj_work, adj_par;  // adjoint workspace, kept between calls
    DevBuf ctab;        // per-step stencil weights of the cluster-resident path (nu(t) varies)
    std::map<std::tuple<int, int>, Tune> tunes;  // (prec, items) -> tune
    std::map<std::tuple<int, const void*, double, double, int>, GraphEntry> graphs;
    cudaStream_t stream() const { return user ? user : own; }
    ~sp_convection() {
        for (auto& kv : graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (own) cudaStreamDestroy(own);
    }
    Tune tune(int prec, int items) {
        auto it = tunes.find({prec, items});
        if (it != tunes.end()) return it->second;
        // default before tuning: TMA pipeline, 4-row tiles, z-chunks that give
        // at least ~8 CTAs per SM, the same shape for every stage
        Shape sh;
        sh.ty = 4;
        const int VX = prec == 0 ? 2 : 4;
        const long long tiles = (long long)((P.ni + 32 * VX - 1) / (32 * VX)) * ((P.nj + 3) / 4) * items;
        int zc = P.nk;
        while (zc > 8 && tiles * ((P.nk + zc - 1) / zc) < 148LL * 8) zc = (zc + 1) / 2;
        sh.zchunk = std::max(1, zc);
        Tune t;
        t.set_all(sh);
        // FP64 RK4: fused stage pairs, 8-row tiles, one plane range per resident CTA
        if (prec == 0 && pair_supported(g4)) {
            Shape ps;
            ps.ty = 8;
            ps.zchunk = 0;
            t.pair[0] = t.pair[1] = ps;
            t.fused = 1;
        }
        return t;
    }
    void drop_graphs() {
        for (auto& kv : graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        graphs.clear();
    }
    int ensure_scratch(int prec, int items) {
        if (scratch_items[prec] >= items) return SP_OK;
        drop_graphs();  // captured graphs hold the old scratch addresses
        const size_t n = (size_t)3 * items * g[prec].total * g[prec].es;
        cudaError_t e = scratch[prec].alloc(n);
        if (e != cudaSuccess) return fail(SP_ERR_NOMEM, "scratch allocation of %zu bytes: %s", n, cudaGetErrorString(e));
        scratch_items[prec] = items;
        return SP_OK;
    }
    int ensure_wide(int items) {
        if (wide_items >= items) return SP_OK;
        drop_graphs();
        const size_t n = (size_t)3 * items * g4.total * g4.es;
        cudaError_t e = wide.alloc(n);
        if (e != cudaSuccess) return fail(SP_ERR_NOMEM, "fused-pair fields of %zu bytes: %s", n, cudaGetErrorString(e));
        wide_items = items;
        return SP_OK;
    }
    // fused-pair field `which` (0, 1: step start / accumulator, 2: y2) of a batch of `items`
    void* wbuf(int which, int items) const {
        return static_cast<char*>(wide.p) + (size_t)which * items * g4.total * g4.es;
    }
    void* sbuf(int prec, int which, int items) const {
        return static_cast<char*>(scratch[prec].p) + (size_t)which * items * g[prec].total * g[prec].es;
    }
};

namespace {

int check_handle(sp_convection* h) {
    if (!h) return fail(SP_ERR_INVALID, "null handle");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, "cudaSetDevice(%d): %s", h->device, cudaGetErrorString(e));
    return SP_OK;
}

// Per-item diffusivity source for a stage launch.
struct NuSrc {
    double nu = 0;
    const double* items = nullptr;
};

// One RK4 step over `items` fields: in -> out, with scratch ya/yb/acc.
cudaError_t enqueue_rk4_step3(const Geo& g, int prec, const Coef& c, double dt, NuSrc nu, const void* in, void* out,
                              void* ya, void* yb, void* yc, void* acc, int items, const int* item_lo, int item_base,
                              const Tune& t, cudaStream_t s, int* err) {
    StageLaunch L;
    L.prec = prec;
    L.items = items;
    L.item_lo = item_lo;
    L.item_base = item_base;
    L.nu = nu.nu;
    L.nu_items = nu.items;
    L.coef = c;
    const double dthalf = dt * .5;  // Convection.cpp:320
    // S1
    L.op = OP_RK_S1; L.yin = in; L.yout = ya; L.acc = acc; L.c_y = dthalf; L.c_acc = dt / 6.;
    cudaError_t e = launch_stage(g, L, t, s, err);
    if (e != cudaSuccess) return e;
    // S2
    L.op = OP_RK_S2; L.yin = ya; L.q = in; L.yout = yb; L.c_y = dthalf; L.c_acc = dt / 3.;
    if ((e = launch_stage(g, L, t, s, err)) != cudaSuccess) return e;
    // S3
    L.op = OP_RK_S3; L.yin = yb; L.q = in; L.yout = yc; L.c_y = dt; L.c_acc = dt / 3.;
    if ((e = launch_stage(g, L, t, s, err)) != cudaSuccess) return e;
    // S4
    L.op = OP_RK_S4; L.yin = yc; L.q = in; L.yout = out; L.c_acc = dt / 6.;
    return launch_stage(g, L, t, s, err);
}

cudaError_t enqueue_rk4_step(const Geo& g, int prec, const Coef& c, double dt, NuSrc nu, const void* in, void* out,
                             void* ya, void* yb, void* acc, int items, const int* item_lo, int item_base,
                             const Tune& t, cudaStream_t s, int* err) {
    return enqueue_rk4_step3(g, prec, c, dt, nu, in, out, ya, yb, ya, acc, items, item_lo, item_base, t, s, err);
}

cudaError_t enqueue_euler_step(const Geo& g, int prec, const Coef& c, double dt, NuSrc nu, const void* in, void* out,
                               int items, const int* item_lo, int item_base, const Tune& t, cudaStream_t s,
                               int* err) {
    StageLaunch L;
    L.op = OP_EULER;
    L.prec = prec;
    L.items = items;
    L.item_lo = item_lo;
    L.item_base = item_base;
    L.nu = nu.nu;
    L.nu_items = nu.items;
    L.coef = c;
    L.yin = in;
    L.yout = out;
    L.c_y = dt;
    return launch_stage(g, L, t, s, err);
}

// Graph of `n` in-place RK4 steps on a single field (constant nu).
int get_chunk_graph(sp_convection* h, int prec, void* field, double dt, double nu, int n, GraphEntry** out) {
    auto key = std::make_tuple(prec, (const void*)field, dt, nu, n);
    auto it = h->graphs.find(key);
    if (it != h->graphs.end()) { *out = &it->second; return SP_OK; }
    if (h->graphs.size() > 32) {  // bounded cache
        for (auto& kv : h->graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        h->graphs.clear();
    }
    int rc = h->ensure_scratch(prec, 1);
    if (rc) return rc;
    const Tune t = h->tune(prec, 1);
    cudaStream_t s = h->stream();
    SP_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    const long long before = launches();
    for (int i = 0; i < n && e == cudaSuccess; ++i)
        e = enqueue_rk4_step(h->g[prec], prec, h->coef, dt, NuSrc{nu, nullptr}, field, field, h->sbuf(prec, 0, 1),
                             h->sbuf(prec, 1, 1), h->sbuf(prec, 2, 1), 1, nullptr, 0, t, s, h->err.as<int>());
    const long long nodes = launches() - before;
    add_launches(-nodes);  // captured, not launched
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &graph);
    if (e != cudaSuccess) { if (graph) cudaGraphDestroy(graph); return fail(SP_ERR_CUDA, "capture: %s", cudaGetErrorString(e)); }
    if (e2 != cudaSuccess) return fail(SP_ERR_CUDA, "end capture: %s", cudaGetErrorString(e2));
    GraphEntry ge;
    e = cudaGraphInstantiate(&ge.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    ge.nodes = nodes;
    auto res = h->graphs.emplace(key, ge);
    *out = &res.first->second;
    return SP_OK;
}

// One fused RK4 step on internal fields (geometry g4): q -> (y2, acc) -> out,
// where out is `acc` (geometry g4, updated in place) or a caller field of geometry go.
cudaError_t enqueue_pair_step(sp_convection* h, const Tune& t, double dt, double nu, const void* q, void* acc,
                              void* y2, void* out, const Geo& go, int items, const int* item_lo, int item_base,
                              cudaStream_t s, int* err) {
    PairLaunch L;
    L.items = items;
    L.item_lo = item_lo;
    L.item_base = item_base;
    L.nu = nu;
    L.dt = dt;
    L.coef = h->coef;
    L.pair = 0; L.q = q; L.y2 = y2; L.acc = acc;
    cudaError_t e = launch_pair(h->g4, h->g4, L, t.pair[0], s, err);
    if (e != cudaSuccess) return e;
    L.pair = 1; L.out = out;
    return launch_pair(h->g4, go, L, t.pair[1], s, err);
}

// Graph of `n` (even) internal fused steps starting from wbuf(0) (constant nu, one field).
int get_fused_graph(sp_convection* h, double dt, double nu, int n, GraphEntry** out) {
    auto key = std::make_tuple(2, (const void*)nullptr, dt, nu, n);
    auto it = h->graphs.find(key);
    if (it != h->graphs.end()) { *out = &it->second; return SP_OK; }
    if (h->graphs.size() > 32) h->drop_graphs();
    const Tune t = h->tune(0, 1);
    cudaStream_t s = h->stream();
    SP_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    const long long before = launches();
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        void* Q = h->wbuf(i % 2, 1);
        void* A = h->wbuf((i + 1) % 2, 1);
        e = enqueue_pair_step(h, t, dt, nu, Q, A, h->wbuf(2, 1), A, h->g4, 1, nullptr, 0, s, h->err.as<int>());
    }
    const long long nodes = launches() - before;
    add_launches(-nodes);  // captured, not launched
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &graph);
    if (e != cudaSuccess) { if (graph) cudaGraphDestroy(graph); return fail(SP_ERR_CUDA, "capture: %s", cudaGetErrorString(e)); }
    if (e2 != cudaSuccess) return fail(SP_ERR_CUDA, "end capture: %s", cudaGetErrorString(e2));
    GraphEntry ge;
    e = cudaGraphInstantiate(&ge.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    ge.nodes = nodes;
    auto res = h->graphs.emplace(key, ge);
    *out = &res.first->second;
    return SP_OK;
}

bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &st);
    return st != cudaStreamCaptureStatusNone;
}

constexpr int kChunk = 50;  // RK4 steps per captured graph
// The tuner keeps the fused pairs only when they beat the four stage kernels by
// more than 2 %: the two paths give the same fields bit for bit and usually run
// within 1-2 % of each other, about the spread of repeated timings, and the
// stage kernels' speed (HBM-bound) varies less from box to box.
constexpr float kPairMargin = 0.98f;
// Each path the tuner compares first runs back to back for this long before it
// is timed.  Under its 1000 W cap a B200 lowers its clocks once a path draws
// more than the cap, and the stage kernels (twice the HBM bytes of the fused
// pairs) draw more: timed cold, they win by 1-3 %; sustained (the clocks at
// ~1.55 GHz instead of ~1.9 GHz), the pairs are ~9 % faster at 256^3.
constexpr double kSustainSeconds = 0.4;
// The pairs on 32 x 16 tiles carry less halo per cell than on 64-column tiles
// (TMA boxes of 40 x 24 against 72 x 16 cells per 512), so they move fewer DRAM
// bytes and draw less power at the same speed per clock: where the cap bites
// they keep a higher clock (256^3: 52.3 against 50.8 GCUPS on one box, equal
// where neither path reaches the cap).  Timed at sustained clocks, they are kept
// unless more than 1 % slower than the per-pair best of the isolated timings.
constexpr float kNarrowMargin = 1.01f;

// Runs fn back to back (synchronising after each) until kSustainSeconds have passed.
template <typename F>
int sustain(cudaStream_t s, F&& fn) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        int rc = fn();
        if (rc) return rc;
        if (cudaStreamSynchronize(s) != cudaSuccess) return fail(SP_ERR_CUDA, "tuning: synchronize failed");
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= kSustainSeconds)
            return SP_OK;
    }
}

// Convection::DoRK4 / DoEuler on single fields of precision prec.
int do_prop(sp_convection* h, int prec, bool rk, const void* in, void* out, double tStart, double dt, int n) {
    NvtxRange range(rk ? "Convection::DoRK4" : "Convection::DoEuler");
    int rc = check_handle(h);
    if (rc) return rc;
    if (!in || !out) return fail(SP_ERR_INVALID, "null field");
    if (n < 0) return fail(SP_ERR_INVALID, "negative step count");
    if (n == 0) return SP_OK;  // Convection.cpp:296: no step, output untouched
    if ((rc = h->ensure_scratch(prec, 1))) return rc;
    const Geo& g = h->g[prec];
    cudaStream_t s = h->stream();
    int* err = h->err.as<int>();
    const Tune t = h->tune(prec, 1);
    // Periodicity on the input, in place, as before the reference's first stencil.
    SP_CUDA(launch_periodicity(g, const_cast<void*>(in), 1, s));
    const bool const_nu = h->P.nufreq == 0.;
    if (rk && t.cluster && prec == 0 && cluster_supported(g, t.cluster) && (const_nu || !capturing(s))) {
        // small field: every step in one launch, the field held in a cluster's
        // shared memory (sp_cluster.cu); then the periodic images of `out`
        ClusterLaunch L;
        L.mode = t.cluster;
        L.in = in;
        L.out = out;
        L.nsteps = n;
        L.dt = dt;
        L.coef = h->coef;
        L.nu = computenu(h->P.nu0, h->P.nufreq, tStart);
        if (!const_nu) {
            // nu(tStart + i dt) per step (Convection.cpp:296-302), as weights
            const size_t wb = cluster_weights_bytes();
            std::vector<unsigned char> tab((size_t)n * wb);
            for (int i = 0; i < n; ++i)
                fill_cluster_weights(tab.data() + (size_t)i * wb, h->coef,
                                     computenu(h->P.nu0, h->P.nufreq, i == 0 ? tStart : tStart + i * dt));
            if (h->ctab.alloc(tab.size()) != cudaSuccess) return fail(SP_ERR_NOMEM, "weight table");
            SP_CUDA(cudaMemcpyAsync(h->ctab.p, tab.data(), tab.size(), cudaMemcpyHostToDevice, s));
            SP_CUDA(cudaStreamSynchronize(s));  // the host table goes out of scope
            L.wtab = h->ctab.p;
        }
        SP_CUDA(launch_rk4_cluster(g, L, s, err));
        SP_CUDA(launch_periodicity(g, out, 1, s));
    } else if (rk && t.fused && prec == 0 && pair_supported(h->g4)) {
        // fused stage pairs: widen the input once, alternate the step-start
        // field between wbuf(0) and wbuf(1), write the last step to `out`
        if ((rc = h->ensure_wide(1))) return rc;
        SP_CUDA(launch_widen(h->g4, h->wbuf(0, 1), g, in, 1, nullptr, 0, s));
        int i = 0;
        if (const_nu && !capturing(s) && n - 1 >= kChunk) {
            GraphEntry* ge = nullptr;
            if ((rc = get_fused_graph(h, dt, computenu(h->P.nu0, h->P.nufreq, tStart), kChunk, &ge))) return rc;
            for (; n - 1 - i >= kChunk; i += kChunk) {  // kChunk is even: every chunk starts at wbuf(0)
                SP_CUDA(cudaGraphLaunch(ge->exec, s));
                add_launches(ge->nodes);
            }
        }
        for (; i < n; ++i) {
            const double tt = tStart + i * dt;  // Convection.cpp:302
            void* Q = h->wbuf(i % 2, 1);
            void* A = h->wbuf((i + 1) % 2, 1);
            const bool last = i == n - 1;
            SP_CUDA(enqueue_pair_step(h, t, dt, computenu(h->P.nu0, h->P.nufreq, tt), Q, A, h->wbuf(2, 1),
                                      last ? out : A, last ? g : h->g4, 1, nullptr, 0, s, err));
        }
    } else if (rk) {
        SP_CUDA(enqueue_rk4_step(g, prec, h->coef, dt, NuSrc{computenu(h->P.nu0, h->P.nufreq, tStart), nullptr}, in,
                                 out, h->sbuf(prec, 0, 1), h->sbuf(prec, 1, 1), h->sbuf(prec, 2, 1), 1, nullptr, 0, t,
                                 s, err));
        int i = 0;
        int left = n - 1;
        if (const_nu && !capturing(s)) {
            const double nu = computenu(h->P.nu0, h->P.nufreq, tStart);
            if (left >= kChunk) {
                GraphEntry* ge = nullptr;
                if ((rc = get_chunk_graph(h, prec, out, dt, nu, kChunk, &ge))) return rc;
                while (left >= kChunk) {
                    SP_CUDA(cudaGraphLaunch(ge->exec, s));
                    add_launches(ge->nodes);
                    left -= kChunk;
                    i += kChunk;
                }
            }
        }
        for (; left > 0; --left) {
            const double tt = tStart + (++i) * dt;  // Convection.cpp:302
            SP_CUDA(enqueue_rk4_step(g, prec, h->coef, dt, NuSrc{computenu(h->P.nu0, h->P.nufreq, tt), nullptr}, out,
                                     out, h->sbuf(prec, 0, 1), h->sbuf(prec, 1, 1), h->sbuf(prec, 2, 1), 1, nullptr, 0,
                                     t, s, err));
        }
    } else {
        // Euler: one fused pass per step (out = in + dt R2(in)) needs distinct
        // input and output, so steps alternate between `out` and scratch.
        void* tmp = h->sbuf(prec, 0, 1);
        const void* src = in;
        for (int i = 0; i < n; ++i) {
            const double tt = i == 0 ? tStart : tStart + i * dt;
            // pick the destination so that the last step lands in `out`
            void* dst = ((n - 1 - i) % 2 == 0) ? out : tmp;
            if (dst == src) dst = (dst == out) ? tmp : out;
            SP_CUDA(enqueue_euler_step(g, prec, h->coef, dt, NuSrc{computenu(h->P.nu0, h->P.nufreq, tt), nullptr}, src,
                                       dst, 1, nullptr, 0, t, s, err));
            src = dst;
        }
        if (src != out) {
            SP_CUDA(cudaMemcpyAsync(out, src, g.total * g.es, cudaMemcpyDeviceToDevice, s));
        }
    }
    return SP_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI.
extern "C" {

const char* sp_last_error(void) { return g_err.c_str(); }
int sp_abi_version(void) { return SP_ABI_VERSION; }
long long sp_launch_count(void) { return launches(); }

int sp_field_layout(int ni, int nj, int nk, int precision, sp_layout* out) {
    if (!out || ni < 2 || nj < 2 || nk < 2 || (precision != SP_F64 && precision != SP_F32))
        return fail(SP_ERR_INVALID, "sp_field_layout: grid must be at least 2^3 and precision SP_F64/SP_F32");
    const Geo g = make_geo(ni, nj, nk, precision == SP_F64 ? 8 : 4);
    out->ni = ni; out->nj = nj; out->nk = nk; out->lx = g.lx; out->elem_size = g.es;
    out->px = g.px; out->py = g.py; out->pz = g.pz; out->plane = g.plane; out->origin = g.origin;
    out->total = g.total;
    return SP_OK;
}

int sp_convection_create(const sp_params* p, int device, sp_convection** out) {
    if (!p || !out) return fail(SP_ERR_INVALID, "null argument");
    *out = nullptr;
    if (p->ni < 2 || p->nj < 2 || p->nk < 2) return fail(SP_ERR_INVALID, "grid %dx%dx%d: every axis needs >= 2 cells", p->ni, p->nj, p->nk);
    if (!(p->dx > 0)) return fail(SP_ERR_INVALID, "dx must be positive");
    if ((long long)p->nk + 4 > 65535LL * 8) return fail(SP_ERR_INVALID, "nk too large");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SP_ERR_UNSUPPORTED, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(SP_ERR_INVALID, "device %d out of range", device);
    SP_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    SP_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(SP_ERR_UNSUPPORTED, "this library is built for sm_100a (found sm_%d%d)", prop.major, prop.minor);
    std::unique_ptr<sp_convection> h(new sp_convection());
    h->P = *p;
    h->device = device;
    h->g[0] = make_geo(p->ni, p->nj, p->nk, 8);
    h->g[1] = make_geo(p->ni, p->nj, p->nk, 4);
    h->g4 = make_geo(p->ni, p->nj, p->nk, 8, 4);
    h->coef = make_coef(p->dx, p->cx, p->cy, p->cz, p->upwind);
    SP_CUDA(cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking));
    if (h->err.alloc(64) != cudaSuccess) return fail(SP_ERR_NOMEM, "error word");
    if (h->red.alloc(64 * sizeof(double)) != cudaSuccess) return fail(SP_ERR_NOMEM, "reduction scratch");
    SP_CUDA(prepare_kernels());
    *out = h.release();
    return SP_OK;
}

int sp_convection_destroy(sp_convection* h) {
    if (!h) return SP_OK;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream());
    delete h;
    return SP_OK;
}

int sp_convection_set_stream(sp_convection* h, void* stream) {
    if (!h) return fail(SP_ERR_INVALID, "null handle");
    h->user = static_cast<cudaStream_t>(stream);
    return SP_OK;
}

int sp_convection_synchronize(sp_convection* h) {
    int rc = check_handle(h);
    if (rc) return rc;
    SP_CUDA(cudaStreamSynchronize(h->stream()));
    int word = 0;
    SP_CUDA(cudaMemcpy(&word, h->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (word != 0) {
        cudaMemsetAsync(h->err.p, 0, sizeof(int), h->stream());
        cudaStreamSynchronize(h->stream());
        return fail(SP_ERR_TIMEOUT, "a bounded in-kernel wait gave up (device error word %d)", word);
    }
    return SP_OK;
}

int sp_set_tune(sp_convection* h, int precision, int batch, int ty, int zchunk, int kind) {
    if (!h || (precision != SP_F64 && precision != SP_F32) || batch < 1) return fail(SP_ERR_INVALID, "bad tune args");
    if (kind < 0 || kind > 5)
        return fail(SP_ERR_INVALID, "kernel kind must be 0 (direct), 1 (TMA), 2 (fused pairs), 3 (cluster-resident "
                                    "on z-slabs), 4 (fused pairs on 32-column tiles) or 5 (cluster-resident on (y,z) "
                                    "blocks)");
    if (kind == 3 || kind == 5) {
        if (precision != SP_F64 || !cluster_supported(h->g[0], kind == 3 ? 1 : 2))
            return fail(SP_ERR_INVALID, kind == 3 ? "the cluster-resident path on z-slabs needs FP64, an even ni, small "
                                                    "planes and nk = C x {2,3,4} with 2 <= C <= 16"
                                                  : "the cluster-resident path on (y,z) blocks needs FP64, an even ni "
                                                    "and nj = cy x BY, nk = cz x BZ with cy, cz, BY, BZ >= 2, "
                                                    "cy x cz <= 16, whose buffers fit in shared memory");
        Tune t = h->tune(precision, batch);
        t.cluster = kind == 3 ? 1 : 2;
        h->tunes[{precision, batch}] = t;
        h->drop_graphs();
        return SP_OK;
    }
    if (zchunk < (kind == 2 || kind == 4 ? 0 : 1))
        return fail(SP_ERR_INVALID, "zchunk must be >= 1 (>= 0 for fused pairs: planes per CTA, 0 = automatic)");
    if (kind == 2 || kind == 4) {
        if (precision != SP_F64 || !pair_supported(h->g4))
            return fail(SP_ERR_INVALID, "fused stage pairs need FP64 and at least 4 cells per axis");
        if (kind == 2 && ty != 8 && ty != 16) return fail(SP_ERR_INVALID, "fused pairs: ty must be 8 or 16");
        if (kind == 4 && ty != 16) return fail(SP_ERR_INVALID, "fused pairs on 32-column tiles: ty must be 16");
        Tune t = h->tune(precision, batch);
        Shape sh;
        sh.ty = ty;
        sh.zchunk = zchunk;
        sh.tx = kind == 4 ? 32 : 64;
        t.pair[0] = t.pair[1] = sh;
        t.fused = 1;
        h->tunes[{precision, batch}] = t;
        h->drop_graphs();
        return SP_OK;
    }
    if (ty != 4 && ty != 8 && ty != 16) return fail(SP_ERR_INVALID, "ty must be 4, 8 or 16");
    Shape sh;
    sh.ty = ty;
    sh.zchunk = zchunk;
    sh.tma = kind;
    Tune t;
    t.set_all(sh);
    t.fused = 0;
    h->tunes[{precision, batch}] = t;
    h->drop_graphs();
    return SP_OK;
}

// op 0..8: single-stage kernels (tma: 0 direct, 1 TMA); op 9, 10: fused pairs
// 1+2 and 3+4 (tma: 2 when RK4 steps run fused, 4 when fused on 32-column
// tiles, else 0); op 11: the cluster-resident path (tma: 3 when FP64 RK4
// propagations use it on z-slabs, 5 on (y,z) blocks, else 0).
int sp_tuned_config(sp_convection* h, int precision, int batch, int op, int* ty, int* zchunk, int* tma) {
    if (!h) return fail(SP_ERR_INVALID, "null handle");
    const Tune tn = h->tune(precision, batch);
    Shape t;
    int kind;
    if (op == kNumOps || op == kNumOps + 1) {
        t = tn.pair[op - kNumOps];
        kind = tn.fused ? (t.tx == 32 ? 4 : 2) : 0;
    } else if (op == kNumOps + 2) {
        t = Shape{0, 0, 0};
        kind = tn.cluster == 2 ? 5 : (tn.cluster ? 3 : 0);
    } else {
        t = tn.op[op < 0 || op >= kNumOps ? OP_RK_S2 : op];
        kind = t.tma;
    }
    if (ty) *ty = t.ty;
    if (zchunk) *zchunk = t.zchunk;
    if (tma) *tma = kind;
    return SP_OK;
}

int sp_do_rk4(sp_convection* h, const double* in, double* out, double tStart, double dt, int timesteps) {
    return do_prop(h, 0, true, in, out, tStart, dt, timesteps);
}
int sp_do_euler(sp_convection* h, const double* in, double* out, double tStart, double dt, int timesteps) {
    return do_prop(h, 0, false, in, out, tStart, dt, timesteps);
}
int sp_do_rk4_timestep(sp_convection* h, const double* in, double* out, double t, double dt) {
    return do_prop(h, 0, true, in, out, t, dt, 1);
}
int sp_do_euler_timestep(sp_convection* h, const double* in, double* out, double t, double dt) {
    return do_prop(h, 0, false, in, out, t, dt, 1);
}
int sp_do_rk4_f32(sp_convection* h, const float* in, float* out, double tStart, double dt, int timesteps) {
    return do_prop(h, 1, true, in, out, tStart, dt, timesteps);
}
int sp_do_euler_f32(sp_convection* h, const float* in, float* out, double tStart, double dt, int timesteps) {
    return do_prop(h, 1, false, in, out, tStart, dt, timesteps);
}

int sp_periodicity_apply(sp_convection* h, void* field, int precision) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!field || (precision != SP_F64 && precision != SP_F32)) return fail(SP_ERR_INVALID, "bad field/precision");
    SP_CUDA(launch_periodicity(h->g[precision], field, 1, h->stream()));
    return SP_OK;
}

int sp_field_import(sp_convection* h, const void* dense, void* field, int precision, int dense_on_host) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!dense || !field || (precision != SP_F64 && precision != SP_F32)) return fail(SP_ERR_INVALID, "bad args");
    const Geo& g = h->g[precision];
    cudaStream_t s = h->stream();
    const void* src = dense;
    if (dense_on_host) {
        const size_t n = (size_t)g.ni * g.nj * g.nk * g.es;
        if (h->dense.alloc(n) != cudaSuccess) return fail(SP_ERR_NOMEM, "staging");
        SP_CUDA(cudaMemcpyAsync(h->dense.p, dense, n, cudaMemcpyHostToDevice, s));
        src = h->dense.p;
    }
    SP_CUDA(launch_dense_to_field(g, src, precision, field, s));
    return SP_OK;
}

int sp_field_export(sp_convection* h, const void* field, void* dense, int precision, int dense_on_host) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!dense || !field || (precision != SP_F64 && precision != SP_F32)) return fail(SP_ERR_INVALID, "bad args");
    const Geo& g = h->g[precision];
    cudaStream_t s = h->stream();
    if (dense_on_host) {
        const size_t n = (size_t)g.ni * g.nj * g.nk * g.es;
        if (h->dense.alloc(n) != cudaSuccess) return fail(SP_ERR_NOMEM, "staging");
        SP_CUDA(launch_field_to_dense(g, field, h->dense.p, precision, s));
        SP_CUDA(cudaMemcpyAsync(dense, h->dense.p, n, cudaMemcpyDeviceToHost, s));
        SP_CUDA(cudaStreamSynchronize(s));
    } else {
        SP_CUDA(launch_field_to_dense(g, field, dense, precision, s));
    }
    return SP_OK;
}

int sp_do_rk4_host(sp_convection* h, const double* in_host, double* out_host, double tStart, double dt,
                   int timesteps) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!in_host || !out_host) return fail(SP_ERR_INVALID, "null host buffer");
    if (timesteps < 0) return fail(SP_ERR_INVALID, "negative step count");
    if ((rc = h->ensure_scratch(0, 2))) return rc;  // fields 3 and 4 of the 2-item scratch hold in/out
    const Geo& g = h->g[0];
    double* f_in = static_cast<double*>(h->sbuf(0, 3, 1));
    double* f_out = static_cast<double*>(h->sbuf(0, 4, 1));
    if ((rc = sp_field_import(h, in_host, f_in, SP_F64, 1))) return rc;
    if (timesteps == 0) {
        SP_CUDA(cudaMemcpyAsync(f_out, f_in, g.total * g.es, cudaMemcpyDeviceToDevice, h->stream()));
    } else if ((rc = sp_do_rk4(h, f_in, f_out, tStart, dt, timesteps))) {
        return rc;
    }
    if ((rc = sp_field_export(h, f_out, out_host, SP_F64, 1))) return rc;
    return sp_convection_synchronize(h);
}

int sp_field_errors(sp_convection* h, const double* a, const double* b, double* err_max, double* err_l2) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!a || !b) return fail(SP_ERR_INVALID, "null field");
    cudaStream_t s = h->stream();
    SP_CUDA(cudaMemsetAsync(h->red.p, 0, 4 * sizeof(double), s));
    SP_CUDA(launch_errors(h->g[0], a, b, h->red.as<double>(), s));
    double r[4];
    SP_CUDA(cudaMemcpyAsync(r, h->red.p, sizeof r, cudaMemcpyDeviceToHost, s));
    SP_CUDA(cudaStreamSynchronize(s));
    if (err_max) *err_max = r[2] / r[3];
    if (err_l2) *err_l2 = std::sqrt(r[0] / r[1]);
    return SP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Error-path self-test: a kernel whose wait can never complete gives up after
// limit_ms; the call returns the status the handle then reports (SP_ERR_TIMEOUT)
// and leaves the handle usable.
extern "C" int sp_store_violations(int* checked, long long* count) {
    if (!checked || !count) return fail(SP_ERR_INVALID, "null argument");
#if defined(SP_BOUNDS_CHECK) && SP_BOUNDS_CHECK
    *checked = 1;
#else
    *checked = 0;
#endif
    SP_CUDA(cudaDeviceSynchronize());
    *count = (long long)(take_store_violations_stages() + take_store_violations_pairs());
    return SP_OK;
}

extern "C" int sp_selftest_wait_timeout(sp_convection* h, double limit_ms) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!(limit_ms > 0.) || limit_ms > 2000.) return fail(SP_ERR_INVALID, "limit_ms must be in (0, 2000]");
    SP_CUDA(launch_wait_selftest(h->err.as<int>(), (unsigned long long)(limit_ms * 1e6), h->stream()));
    return sp_convection_synchronize(h);
}

// ---------------------------------------------------------------------------
// Per-kernel durations of FP64 RK4 steps (CUDA events around every launch on
// the handle's stream), on a copy of `field`; the field is not modified.
extern "C" int sp_kernel_times(sp_convection* h, const double* field, double dt, int reps, int path, float* ms,
                               int* count) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!field || !ms || !count || reps < 1 || path < 0 || path > 2) return fail(SP_ERR_INVALID, "bad arguments");
    cudaStream_t s = h->stream();
    if (capturing(s)) return fail(SP_ERR_STATE, "cannot time kernels while the stream is capturing");
    const Tune t = h->tune(0, 1);
    const Geo& g = h->g[0];
    const double nu = computenu(h->P.nu0, h->P.nufreq, 0.0);
    int* err = h->err.as<int>();
    std::vector<float> times[4];  // per kernel, one duration per timed rep
    if (path == 2 && !pair_supported(h->g4)) return fail(SP_ERR_INVALID, "fused pairs need >= 4 cells per axis");
    const bool fused = path == 2 || (path == 0 && t.fused && pair_supported(h->g4));
    if (fused) {
        if ((rc = h->ensure_wide(1))) return rc;
    } else if ((rc = h->ensure_scratch(0, 2))) {  // fields 0, 3, 4, 5 of the 2-item scratch
        return rc;
    }
    // All launches are enqueued before one synchronisation, so that the GPU
    // never waits for the host between them; rep 0 is an untimed warm-up.  An
    // event between two kernels keeps them from overlapping, so each launch is
    // timed alone.
    const int nk = fused ? 2 : 4;
    const int nrep = reps + 1;
    std::vector<cudaEvent_t> ev((size_t)nrep * nk + 1, nullptr);
    cudaError_t e = cudaSuccess;
    for (auto& x : ev)
        if (e == cudaSuccess) e = cudaEventCreate(&x);
    if (fused) {
        if (e == cudaSuccess) e = launch_widen(h->g4, h->wbuf(0, 1), g, field, 1, nullptr, 0, s);
        PairLaunch L;
        L.nu = nu; L.dt = dt; L.coef = h->coef;
        if (e == cudaSuccess) e = cudaEventRecord(ev[0], s);
        for (int r = 0; r < nrep && e == cudaSuccess; ++r) {
            void* Q = h->wbuf(r % 2, 1);
            void* A = h->wbuf((r + 1) % 2, 1);
            L.pair = 0; L.q = Q; L.y2 = h->wbuf(2, 1); L.acc = A; L.out = A;
            e = launch_pair(h->g4, h->g4, L, t.pair[0], s, err);
            cudaEventRecord(ev[(size_t)r * 2 + 1], s);
            L.pair = 1;
            if (e == cudaSuccess) e = launch_pair(h->g4, h->g4, L, t.pair[1], s, err);
            cudaEventRecord(ev[(size_t)r * 2 + 2], s);
        }
    } else {
        void* q = h->sbuf(0, 3, 1);
        void* ya = h->sbuf(0, 4, 1);
        void* yb = h->sbuf(0, 5, 1);
        void* ac = h->sbuf(0, 0, 1);
        if (e == cudaSuccess) e = cudaMemcpyAsync(q, field, g.total * g.es, cudaMemcpyDeviceToDevice, s);
        StageLaunch L;
        L.prec = 0; L.items = 1; L.nu = nu; L.coef = h->coef;
        const double dthalf = dt * .5;
        const int op[4] = {OP_RK_S1, OP_RK_S2, OP_RK_S3, OP_RK_S4};
        const void* yin[4] = {q, ya, yb, ya};
        void* yout[4] = {ya, yb, ya, q};
        const double cy[4] = {dthalf, dthalf, dt, 0.}, ca[4] = {dt / 6., dt / 3., dt / 3., dt / 6.};
        if (e == cudaSuccess) e = cudaEventRecord(ev[0], s);
        for (int r = 0; r < nrep && e == cudaSuccess; ++r) {
            for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
                L.op = op[k]; L.yin = yin[k]; L.yout = yout[k]; L.acc = ac; L.q = k == 0 ? nullptr : q;
                L.c_y = cy[k]; L.c_acc = ca[k];
                e = launch_stage(g, L, t, s, err);
                cudaEventRecord(ev[(size_t)r * 4 + k + 1], s);
            }
        }
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(ev.back());
    for (int r = 1; r < nrep && e == cudaSuccess; ++r)
        for (int k = 0; k < nk; ++k) {
            float m = 0;
            cudaEventElapsedTime(&m, ev[(size_t)r * nk + k], ev[(size_t)r * nk + k + 1]);
            times[k].push_back(m);
        }
    *count = nk;
    for (auto& x : ev)
        if (x) cudaEventDestroy(x);
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, "kernel timing: %s", cudaGetErrorString(e));
    // the median: a rep in which the host fell behind the GPU (the GPU idling
    // inside an event interval) does not move it
    for (int k = 0; k < *count; ++k) {
        std::vector<float>& v = times[k];
        std::sort(v.begin(), v.end());
        const size_t h = v.size() / 2;
        ms[k] = v.empty() ? 0.f : (v.size() % 2 ? v[h] : 0.5f * (v[h - 1] + v[h]));
    }
    return sp_convection_synchronize(h);
}

namespace {
// Tuning data: the paths are timed on fields of varying values at a stable
// step, as they run in practice.  On all-zero fields at a vanishing step the
// kernels draw far less power and never reach the GPU's power cap, which
// decides between them on real data.
template <typename T>
__global__ void k_fill_wave(T* p, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = (T)(sin(1e-3 * (double)i) + 0.25 * sin(0.37 * (double)i));
}
cudaError_t fill_wave(void* p, size_t bytes, int es, cudaStream_t s) {
    const long long n = (long long)(bytes / es);
    if (es == 8) k_fill_wave<double><<<1184, 256, 0, s>>>(static_cast<double*>(p), n);
    else k_fill_wave<float><<<1184, 256, 0, s>>>(static_cast<float*>(p), n);
    return cudaGetLastError();
}
// A tenth of RK4's stability bound for this grid's velocity and diffusivity.
double tune_dt(const sp_convection* h) {
    const double dx = h->P.dx;
    const double adv = (std::fabs(h->P.cx) + std::fabs(h->P.cy) + std::fabs(h->P.cz)) * 1.5 / dx;
    const double dif = 1.5 * std::fabs(h->P.nu0) * 3. * 16. / 12. / (dx * dx);  // nu(t) <= 1.5 nu0
    const double lam = adv + dif;
    return lam > 0 ? 0.1 * 2.78 / lam : 1e-9;
}
}  // namespace

// ---------------------------------------------------------------------------
// Autotuner: for every stage kernel (RK4 S1..S4, Euler) times each candidate
// launch shape (kernel kind x tile rows x z-chunk) on scratch fields and keeps
// the fastest shape per stage; then the same for the fused stage pairs, and
// picks fused pairs or four stage kernels per RK4 step.
extern "C" int sp_autotune(sp_convection* h, int precision, int batch) {
    int rc = check_handle(h);
    if (rc) return rc;
    if ((precision != SP_F64 && precision != SP_F32) || batch < 1) return fail(SP_ERR_INVALID, "bad args");
    cudaStream_t s = h->stream();
    if (capturing(s)) return fail(SP_ERR_STATE, "cannot tune while the stream is capturing");
    const Geo& g = h->g[precision];
    DevBuf buf;
    const size_t fb = (size_t)batch * g.total * g.es;
    if (buf.alloc(5 * fb) != cudaSuccess) return fail(SP_ERR_NOMEM, "tuning buffers");
    char* p = buf.as<char>();
    SP_CUDA(fill_wave(p, 5 * fb, g.es, s));
    const double dtt = tune_dt(h);
    cudaEvent_t e0, e1;
    SP_CUDA(cudaEventCreate(&e0));
    SP_CUDA(cudaEventCreate(&e1));
    Tune best = h->tune(precision, batch);
    std::vector<int> zcs = {4, 8, 16, 32, 64};
    zcs.push_back(g.nk);
    float op_ms[kNumOps];
    for (auto& m : op_ms) m = 1e30f;
    for (int op : {OP_RK_S1, OP_RK_S2, OP_RK_S3, OP_RK_S4, OP_EULER}) {
        StageLaunch L;
        L.op = op;
        L.prec = precision;
        L.items = batch;
        L.coef = h->coef;
        L.nu = h->P.nu0;
        L.yin = p; L.q = p + fb; L.acc = p + 2 * fb; L.yout = p + 3 * fb;
        L.c_y = 1e-9; L.c_acc = 1e-9;
        float best_ms = 1e30f;
        for (int kind = 1; kind >= 0; --kind)
            for (int ty : {4, 8, 16})
                for (int zc : zcs) {
                    if (zc > g.nk && zc != g.nk) continue;
                    if ((long long)((g.nk + zc - 1) / zc) > 65535) continue;
                    Tune t;
                    Shape sh;
                    sh.tma = kind; sh.ty = ty; sh.zchunk = zc;
                    t.set_all(sh);
                    cudaError_t e = launch_stage(g, L, t, s, h->err.as<int>());
                    if (e != cudaSuccess) { cudaGetLastError(); continue; }
                    float ms = 1e30f;
                    for (int r = 0; r < 3; ++r) {
                        cudaEventRecord(e0, s);
                        launch_stage(g, L, t, s, h->err.as<int>());
                        cudaEventRecord(e1, s);
                        cudaEventSynchronize(e1);
                        float m = 0;
                        cudaEventElapsedTime(&m, e0, e1);
                        ms = std::min(ms, m);
                    }
                    if (ms < best_ms) { best_ms = ms; best.op[op] = sh; }
                }
        op_ms[op] = best_ms;
    }
    // fused stage pairs (FP64): best shape per pair, then fused or single-stage
    // steps by timing whole steps of both paths
    best.fused = 0;
    if (precision == SP_F64 && pair_supported(h->g4)) {
        const Geo& g4 = h->g4;
        const size_t wb = (size_t)batch * g4.total * g4.es;
        DevBuf wbuf;
        if (wbuf.alloc(3 * wb) == cudaSuccess) {
            char* w = wbuf.as<char>();
            float pair_ms[2] = {1e30f, 1e30f};
            float narrow_ms[2] = {1e30f, 1e30f};  // the best shape on 32 x 16 tiles
            Shape narrow[2];
            for (int pair = 0; pair < 2; ++pair) {
                PairLaunch L;
                L.pair = pair;
                L.items = batch;
                L.coef = h->coef;
                L.nu = h->P.nu0;
                L.dt = 1e-9;
                L.q = w; L.acc = w + wb; L.y2 = w + 2 * wb; L.out = w + wb;
                for (int ty : {8, 16, 32})  // 32: tiles of 32 x 16 cells
                    for (int zc : {0, 16, 24, 32, 48, 64}) {
                        if (zc > g.nk) continue;
                        Shape sh;
                        sh.ty = ty == 32 ? 16 : ty; sh.tx = ty == 32 ? 32 : 64; sh.zchunk = zc;
                        cudaError_t e = launch_pair(g4, g4, L, sh, s, h->err.as<int>());
                        if (e != cudaSuccess) { cudaGetLastError(); continue; }
                        float ms = 1e30f;
                        for (int r = 0; r < 3; ++r) {
                            cudaEventRecord(e0, s);
                            launch_pair(g4, g4, L, sh, s, h->err.as<int>());
                            cudaEventRecord(e1, s);
                            cudaEventSynchronize(e1);
                            float m = 0;
                            cudaEventElapsedTime(&m, e0, e1);
                            ms = std::min(ms, m);
                        }
                        if (ms < pair_ms[pair]) { pair_ms[pair] = ms; best.pair[pair] = sh; }
                        if (ty == 32 && ms < narrow_ms[pair]) { narrow_ms[pair] = ms; narrow[pair] = sh; }
                    }
            }
            // the pair shapes to compare at sustained clocks: the per-pair best and,
            // when it differs, the best on 32 x 16 tiles for both pairs
            Tune alt = best;
            alt.pair[0] = narrow[0];
            alt.pair[1] = narrow[1];
            const bool try_narrow = narrow_ms[0] < 1e29f && narrow_ms[1] < 1e29f &&
                                    !(same_shape(alt.pair[0], best.pair[0]) && same_shape(alt.pair[1], best.pair[1]));
            best.fused = (pair_ms[0] + pair_ms[1]) < (op_ms[OP_RK_S1] + op_ms[OP_RK_S2] + op_ms[OP_RK_S3] +
                                                      op_ms[OP_RK_S4]) ? 1 : 0;
            if (batch == 1) {
                // Single fields: decide by DoRK4 itself (one graph chunk of
                // steps), where consecutive kernels overlap through programmatic
                // dependent launch and four stage kernels overlap more than two
                // pairs, so that the sums of isolated kernel times mislead.
                SP_CUDA(fill_wave(p, 2 * fb, g.es, s));
                float path_ms[3] = {1e30f, 1e30f, 1e30f};  // stages, best pairs, pairs on 32 x 16 tiles
                for (int f = 0; f < (try_narrow ? 3 : 2) && rc == SP_OK; ++f) {
                    Tune tt = f == 2 ? alt : best;
                    tt.fused = f ? 1 : 0;
                    h->tunes[{precision, batch}] = tt;
                    h->drop_graphs();
                    rc = do_prop(h, precision, true, p, p + fb, 0.0, dtt, kChunk + 1);  // captures the graph
                    if (rc == SP_OK)  // at the clocks the path sustains
                        rc = sustain(s, [&]() { return do_prop(h, precision, true, p, p + fb, 0.0, dtt, kChunk + 1); });
                    for (int r = 0; r < 3 && rc == SP_OK; ++r) {
                        cudaEventRecord(e0, s);
                        rc = do_prop(h, precision, true, p, p + fb, 0.0, dtt, kChunk + 1);
                        cudaEventRecord(e1, s);
                        cudaEventSynchronize(e1);
                        float m = 0;
                        cudaEventElapsedTime(&m, e0, e1);
                        path_ms[f] = std::min(path_ms[f], m);
                    }
                }
                if (rc != SP_OK) {
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                    h->drop_graphs();
                    return rc;
                }
                if (try_narrow && path_ms[2] <= kNarrowMargin * path_ms[1]) {
                    best.pair[0] = alt.pair[0];
                    best.pair[1] = alt.pair[1];
                    path_ms[1] = path_ms[2];
                }
                best.fused = path_ms[1] < kPairMargin * path_ms[0] ? 1 : 0;
            } else {
                // Batches (the Parareal F sweep): four consecutive batched steps of
                // each path as the sweep launches them, after one untimed step.
                SP_CUDA(fill_wave(p, 4 * fb, g.es, s));
                SP_CUDA(fill_wave(w, 3 * wb, g4.es, s));
                const double nu = computenu(h->P.nu0, h->P.nufreq, 0.0);
                int* err = h->err.as<int>();
                Tune ts = best;
                ts.fused = 0;
                auto stage_steps = [&](int k) {
                    cudaError_t x = cudaSuccess;
                    for (int i = 0; i < k && x == cudaSuccess; ++i)
                        x = enqueue_rk4_step(g, precision, h->coef, dtt, NuSrc{nu, nullptr}, p, p, p + fb,
                                             p + 2 * fb, p + 3 * fb, batch, nullptr, 0, ts, s, err);
                    return x;
                };
                auto pair_steps = [&](const Tune& pt, int k) {
                    cudaError_t x = cudaSuccess;
                    for (int i = 0; i < k && x == cudaSuccess; ++i) {
                        char* Q = w + (size_t)(i % 2) * wb;
                        char* A = w + (size_t)((i + 1) % 2) * wb;
                        x = enqueue_pair_step(h, pt, dtt, nu, Q, A, w + 2 * wb, A, h->g4, batch, nullptr, 0, s, err);
                    }
                    return x;
                };
                auto path_steps = [&](int f, int k) {
                    return f == 0 ? stage_steps(k) : pair_steps(f == 2 ? alt : best, k);
                };
                float path_ms[3] = {1e30f, 1e30f, 1e30f};  // stages, best pairs, pairs on 32 x 16 tiles
                cudaError_t x = cudaSuccess;
                for (int f = 0; f < (try_narrow ? 3 : 2) && x == cudaSuccess; ++f) {
                    x = path_steps(f, 1);
                    if (x == cudaSuccess) {  // at the clocks the path sustains
                        int rs = sustain(s, [&]() {
                            cudaError_t y = path_steps(f, 4);
                            return y == cudaSuccess ? SP_OK : fail(SP_ERR_CUDA, "tuning: %s", cudaGetErrorString(y));
                        });
                        if (rs) x = cudaErrorUnknown;
                    }
                    for (int r = 0; r < 3 && x == cudaSuccess; ++r) {
                        cudaEventRecord(e0, s);
                        x = path_steps(f, 4);
                        cudaEventRecord(e1, s);
                        cudaEventSynchronize(e1);
                        float m = 0;
                        cudaEventElapsedTime(&m, e0, e1);
                        path_ms[f] = std::min(path_ms[f], m);
                    }
                }
                if (x != cudaSuccess) {
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                    return fail(SP_ERR_CUDA, "tuning batched steps: %s", cudaGetErrorString(x));
                }
                if (try_narrow && path_ms[2] <= kNarrowMargin * path_ms[1]) {
                    best.pair[0] = alt.pair[0];
                    best.pair[1] = alt.pair[1];
                    path_ms[1] = path_ms[2];
                }
                best.fused = path_ms[1] < kPairMargin * path_ms[0] ? 1 : 0;
            }
        }
    }
    // small fields: the cluster-resident paths (z-slabs, (y,z) blocks) against
    // the best of the above, timed as they are used (a DoRK4 of a graph chunk of
    // steps for one field; four batched steps for a batch)
    best.cluster = 0;
    if (precision == SP_F64 && (cluster_supported(g, 1) || cluster_supported(g, 2))) {
        int* err = h->err.as<int>();
        float path_ms[3] = {1e30f, 1e30f, 1e30f};
        SP_CUDA(fill_wave(p, 5 * fb, g.es, s));
        for (int c = 0; c < 3 && rc == SP_OK; ++c) {
            if (c && !cluster_supported(g, c)) continue;
            Tune tt = best;
            tt.cluster = c;
            h->tunes[{precision, batch}] = tt;
            h->drop_graphs();
            auto run = [&]() -> int {
                if (batch == 1) return do_prop(h, precision, true, p, p + fb, 0.0, dtt, kChunk + 1);
                const double nu = computenu(h->P.nu0, h->P.nufreq, 0.0);
                cudaError_t x = cudaSuccess;
                if (c) {
                    ClusterLaunch L;
                    L.mode = c;
                    L.in = p; L.out = p; L.items = batch; L.nsteps = 4; L.dt = dtt; L.nu = nu; L.coef = h->coef;
                    x = launch_rk4_cluster(g, L, s, err);
                } else {
                    for (int i = 0; i < 4 && x == cudaSuccess; ++i)
                        x = enqueue_rk4_step(g, precision, h->coef, dtt, NuSrc{nu, nullptr}, p, p, p + fb, p + 2 * fb,
                                             p + 3 * fb, batch, nullptr, 0, tt, s, err);
                }
                return x == cudaSuccess ? SP_OK : fail(SP_ERR_CUDA, "tuning: %s", cudaGetErrorString(x));
            };
            rc = run();  // captures the graphs / warms up
            for (int r = 0; r < 3 && rc == SP_OK; ++r) {
                cudaEventRecord(e0, s);
                rc = run();
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                float m = 0;
                cudaEventElapsedTime(&m, e0, e1);
                path_ms[c] = std::min(path_ms[c], m);
            }
            if (rc != SP_OK && c) {
                // a cluster launch can be refused (cluster shape not schedulable): keep the other paths
                cudaGetLastError();
                rc = SP_OK;
                path_ms[c] = 1e30f;
            }
        }
        for (int c = 1; c < 3; ++c)
            if (path_ms[c] < path_ms[best.cluster]) best.cluster = c;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    SP_CUDA(cudaStreamSynchronize(s));
    h->tunes[{precision, batch}] = best;
    h->drop_graphs();
    return SP_OK;
}

// ---------------------------------------------------------------------------
// Parareal.

namespace {

// Device state of an iteration loop that runs inside one graph launch: a
// conditional WHILE node repeats the iteration body; the body's last kernel
// turns the per-slice defect sums into the iteration's defect (and errors
// against the reference), records them and sets the loop condition.
struct LoopCtl {
    int k;                           // iterations done in this run
    int nonfinite;                   // 1: a defect sum was not finite (the loop stopped there)
    int stopped;                     // batch: this instance no longer iterates
    int pad;
    unsigned long long t_head, t_mid;
    unsigned long long ns_fine, ns_coarse;  // %globaltimer time of the fine / coarse sweeps
    double defect[SP_MAX_ITERS];
    double err_l2[SP_MAX_ITERS];
    double err_max[SP_MAX_ITERS];
};

struct LoopArgs {
    LoopCtl* c;
    int* item_lo;
    const double* def;   // 2P defect sums
    const double* err4;  // error sums against the reference
    int P, skip, kmax, tol_kind, has_ref;
    double tol;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Iteration k's first slice still iterating: slices < k are exact after k iterations.
__device__ __forceinline__ int loop_lo(const LoopArgs& a, int k) { return a.skip ? min(k, a.P) : 0; }

__global__ void k_loop_head(LoopArgs a) {
    a.c->t_head = global_ns();
    *a.item_lo = loop_lo(a, a.c->k);
}

__global__ void k_loop_mid(LoopCtl* c) { c->t_mid = global_ns(); }

// The host loop's per-iteration decision (sp_parareal_do_parallel), on the
// device: defect = max over iterating slices of sqrt(sum (U+ - U)^2 / sum U+^2).
// Returns whether the instance iterates again.
__device__ bool loop_decide(const LoopArgs& a) {
    LoopCtl* c = a.c;
    const unsigned long long t = global_ns();
    c->ns_fine += c->t_mid - c->t_head;
    c->ns_coarse += t - c->t_mid;
    const int k = c->k;
    double defect = 0.;
    bool finite = true;
    for (int r = loop_lo(a, k); r < a.P; ++r) {
        const double num = a.def[2 * r], den = a.def[2 * r + 1];
        if (!isfinite(num) || !isfinite(den)) finite = false;
        if (den > 0) defect = fmax(defect, sqrt(num / den));
    }
    double el2 = 0., emax = 0.;
    if (a.has_ref) {
        el2 = sqrt(a.err4[0] / a.err4[1]);
        emax = a.err4[2] / a.err4[3];
    }
    c->defect[k] = defect;
    c->err_l2[k] = el2;
    c->err_max[k] = emax;
    c->k = k + 1;
    bool cont = finite && k + 1 < a.kmax;
    if (!finite) c->nonfinite = 1;
    if (a.tol_kind == SP_TOL_DEFECT && defect < a.tol) cont = false;
    if (a.tol_kind == SP_TOL_REFERENCE && a.has_ref && el2 < a.tol) cont = false;
    return cont;
}

__global__ void k_loop_tail(LoopArgs a, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, loop_decide(a) ? 1u : 0u);
}

// Batch of instances (sp_parareal_batch_run): before each iteration every
// instance that has not stopped gets its item_lo, a stopped one item_lo = P
// (its kernels return at once).
__global__ void k_batch_head(const LoopArgs* a, int n) {
    const unsigned long long t = global_ns();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        LoopCtl* c = a[i].c;
        if (!c->stopped && c->k >= a[i].kmax) c->stopped = 1;
        *a[i].item_lo = c->stopped ? a[i].P : loop_lo(a[i], c->k);
        c->t_head = c->t_mid = t;
    }
}

// After each iteration: the decision of every running instance (an instance is
// also exact, and stops, after P iterations); the loop goes on while any runs.
__global__ void k_batch_tail(const LoopArgs* a, int n, cudaGraphConditionalHandle h) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        LoopCtl* c = a[i].c;
        if (c->stopped) continue;
        const bool cont = loop_decide(a[i]) && c->k < a[i].P;
        if (cont) atomicOr(&any, 1);
        else c->stopped = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

}  // namespace

struct sp_parareal {
    sp_convection* prop = nullptr;
    sp_parareal_cfg cfg{};
    int P = 0, tsF = 0, tsC = 0;
    int first = 0, Pglobal = 0;  // slice window [first, first + P) of Pglobal slices
    cudaGraphExec_t wfine = nullptr, wcoarse = nullptr;  // window-mode graphs
    long long wfine_nodes = 0, wcoarse_nodes = 0;
    DevBuf Z;              // one zero coarse field (window-mode injection)
    double dtF = 0, dtC = 0, slice = 0;
    int cprec = 0;         // coarse precision index
    Geo g64, gc;
    DevBuf U;              // P+1 FP64 fields: slice inputs U_0..U_{P-1}, last slice result U_P
    DevBuf F;              // P FP64 fields: fine results
    DevBuf fs;             // 3P FP64 fields: fine scratch ya, yb, acc (single-stage F sweep)
    DevBuf fw;             // 3P fields of geometry g4: step start / accumulator x2, y2 (fused F sweep)
    DevBuf Gold;           // P coarse fields (reference form of the correction)
    DevBuf D;              // P+1 coarse fields: slice increments (increment form)
    DevBuf Gt;             // 2 coarse fields (coarse result / ping-pong) + 3 coarse scratch
    DevBuf ctl;            // device control: item_lo (int) + defect sums (2P doubles) + err4
    DevBuf nutab;          // fine nu table (tsF x P) when nufreq != 0
    int* h_itemlo = nullptr;   // pinned
    double* h_def = nullptr;   // pinned, 2P + 4
    cudaGraphExec_t iter = nullptr;
    long long iter_nodes = 0;
    cudaGraphExec_t loop = nullptr;      // all iterations in one launch (conditional WHILE node)
    const double* loop_ref = nullptr;    // reference field the loop graph was captured with
    long long loop_nodes = 0;            // kernel launches of one loop iteration
    DevBuf lctl;                         // LoopCtl
    LoopCtl* h_lctl = nullptr;           // pinned copy
    int host_loop = 0;                   // 1: one graph launch and one host sync per iteration
    int coarse_res = 0;    // which Gt buffer holds the coarse result after a sweep step
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    ~sp_parareal() {
        if (iter) cudaGraphExecDestroy(iter);
        if (loop) cudaGraphExecDestroy(loop);
        if (h_lctl) cudaFreeHost(h_lctl);
        if (wfine) cudaGraphExecDestroy(wfine);
        if (wcoarse) cudaGraphExecDestroy(wcoarse);
        if (h_itemlo) cudaFreeHost(h_itemlo);
        if (h_def) cudaFreeHost(h_def);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
    double* u(int r) const { return U.as<double>() + (size_t)r * g64.total; }
    double* f(int r) const { return F.as<double>() + (size_t)r * g64.total; }
    void* gold(int r) const { return static_cast<char*>(Gold.p) + (size_t)r * gc.total * gc.es; }
    void* dlt(int r) const { return static_cast<char*>(D.p) + (size_t)r * gc.total * gc.es; }
    void* gt(int i) const { return static_cast<char*>(Gt.p) + (size_t)i * gc.total * gc.es; }
    int* itemlo() const { return static_cast<int*>(ctl.p); }
    double* def() const { return reinterpret_cast<double*>(static_cast<char*>(ctl.p) + 256); }
    double* err4() const { return def() + 2 * P; }
};

namespace {

// Coarse propagation G of one field: src (FP64 slice input, geometry g64) ->
// result in pr->gt(pr->coarse_res), n steps from t0.  Every kernel is gated by
// item_lo against `item` when gate is set.
int enqueue_coarse(sp_parareal* pr, const void* src, const Geo& gsrc, double t0, int n, bool gate, int item,
                   cudaStream_t s) {
    sp_convection* h = pr->prop;
    const int cp = pr->cprec;
    const Geo& gc = pr->gc;
    const Tune t = h->tune(cp, 1);
    int* err = h->err.as<int>();
    const int* lo = gate ? pr->itemlo() : nullptr;
    void* A = pr->gt(0);
    void* B = pr->gt(1);
    void* ya = pr->gt(2);
    void* yb = pr->gt(3);
    void* acc = pr->gt(4);
    // bring the input into coarse precision / geometry
    SP_CUDA(launch_convert(gc, A, gsrc, src, s, lo, item));
    void* cur = A;
    void* other = B;
    for (int i = 0; i < n; ++i) {
        const double tt = i == 0 ? t0 : t0 + i * pr->dtC;
        const NuSrc nu{computenu(h->P.nu0, h->P.nufreq, tt), nullptr};
        if (pr->cfg.coarse_scheme == SP_COARSE_RK4) {
            SP_CUDA(enqueue_rk4_step(gc, cp, h->coef, pr->dtC, nu, cur, cur, ya, yb, acc, 1, lo, item, t, s, err));
        } else {
            SP_CUDA(enqueue_euler_step(gc, cp, h->coef, pr->dtC, nu, cur, other, 1, lo, item, t, s, err));
            std::swap(cur, other);
        }
    }
    pr->coarse_res = (cur == A) ? 0 : 1;
    return SP_OK;
}

// Captures one Parareal iteration (Parareal.h:116-165 for every slice):
//   F sweep   : tsF RK4 steps of all slices r >= item_lo, batched per stage
//   G sweep   : for r = item_lo..P-1: G(U_r) (coarse), correction into U_{r+1}
// parts: 1 = F sweep, 2 = G sweep, 3 = both.  zero_min: in the increment form the
// G sweep zeroes the increment of its first iterating slice unless that is a slice
// below zero_min (a window's slice 0 gets its increment from the previous window).
// The F sweep's path: every step of all slices in one cluster-resident launch
// (small fields), fused stage pairs, or the four stage kernels per step.
bool cluster_sweep(const sp_parareal* pr) {
    sp_convection* h = pr->prop;
    const int mode = h->tune(0, pr->P).cluster;
    return h->P.nufreq == 0. && mode && cluster_supported(pr->g64, mode);
}
bool fused_sweep(const sp_parareal* pr) {
    sp_convection* h = pr->prop;
    return !cluster_sweep(pr) && h->P.nufreq == 0. && h->tune(0, pr->P).fused && pair_supported(h->g4);
}

// Allocates the fine-sweep scratch of the path the tune selects; must run
// before a capture of the iteration.
int prepare_iteration(sp_parareal* pr, int parts) {
    if (!(parts & 1) || cluster_sweep(pr)) return SP_OK;
    const int P = pr->P;
    const Geo& g = pr->g64;
    const Geo& g4 = pr->prop->g4;
    if ((fused_sweep(pr) ? pr->fw.alloc((size_t)3 * P * g4.total * g4.es)
                         : pr->fs.alloc((size_t)3 * P * g.total * g.es)) != cudaSuccess)
        return fail(SP_ERR_NOMEM, "fine-sweep scratch for %d slices", P);
    return SP_OK;
}

// Enqueues one Parareal iteration (Parareal.h:116-165 for every slice) on s,
// which is being captured:
//   F sweep   : tsF RK4 steps of all slices r >= item_lo, batched per stage
//   G sweep   : for r = item_lo..P-1: G(U_r) (coarse), correction into U_{r+1}
// parts: 1 = F sweep, 2 = G sweep, 3 = both.  zero_min: in the increment form the
// G sweep zeroes the increment of its first iterating slice unless that is a slice
// below zero_min (a window's slice 0 gets its increment from the previous window).
// mid (may be null): a kernel enqueued between the two sweeps.
int emit_iteration(sp_parareal* pr, cudaStream_t s, bool events, int parts, int zero_min,
                   const std::function<cudaError_t()>& mid = nullptr) {
    sp_convection* h = pr->prop;
    const int P = pr->P;
    const Geo& g = pr->g64;
    const Tune tf = h->tune(0, P);
    int* err = h->err.as<int>();
    const bool const_nu = h->P.nufreq == 0.;
    // F sweep as fused stage pairs when the tune says so and one nu serves all slices
    const bool fused = fused_sweep(pr);
    const Geo& g4 = h->g4;
    const size_t fstride = (size_t)P * g.total;
    double* ya = pr->fs.as<double>();
    double* yb = ya + fstride;
    double* acc = yb + fstride;
    int rc = SP_OK;
    cudaError_t e = events ? cudaEventRecordWithFlags(pr->ev[0], s, cudaEventRecordExternal) : cudaSuccess;
    const bool cluster = cluster_sweep(pr);
    if (cluster && (parts & 1) && e == cudaSuccess) {
        // every fine step of every iterating slice in one launch, each slice in one cluster
        ClusterLaunch L;
        L.mode = tf.cluster;
        L.in = pr->u(0);
        L.out = pr->f(0);
        L.items = P;
        L.nsteps = pr->tsF;
        L.dt = pr->dtF;
        L.nu = h->P.nu0;
        L.coef = h->coef;
        L.item_lo = pr->itemlo();
        e = launch_rk4_cluster(g, L, s, err);
        if (e == cudaSuccess) e = launch_periodicity(g, pr->f(0), P, s);
    }
    if (fused && (parts & 1)) {
        // widen the slice inputs once, alternate step start / accumulator
        // between W0 and W1, write the last step into the fine results
        const size_t w4 = (size_t)P * g4.total;
        double* W0 = pr->fw.as<double>();
        double* W1 = W0 + w4;
        double* WY = W1 + w4;
        if (e == cudaSuccess) e = launch_widen(g4, W0, g, pr->u(0), P, pr->itemlo(), 0, s);
        PairLaunch L;
        L.items = P;
        L.item_lo = pr->itemlo();
        L.nu = h->P.nu0;
        L.dt = pr->dtF;
        L.coef = h->coef;
        for (int i = 0; i < pr->tsF && e == cudaSuccess; ++i) {
            double* Q = (i % 2) ? W1 : W0;
            double* A = (i % 2) ? W0 : W1;
            const bool last = i + 1 == pr->tsF;
            L.pair = 0; L.q = Q; L.y2 = WY; L.acc = A;
            e = launch_pair(g4, g4, L, tf.pair[0], s, err);
            L.pair = 1; L.out = last ? (void*)pr->f(0) : (void*)A;
            if (e == cudaSuccess) e = launch_pair(g4, last ? g : g4, L, tf.pair[1], s, err);
        }
    }
    for (int i = 0; i < pr->tsF && e == cudaSuccess && (parts & 1) && !fused && !cluster; ++i) {
        NuSrc nu;
        if (const_nu) nu.nu = h->P.nu0;
        else nu.items = pr->nutab.as<double>() + (size_t)i * P;
        const void* in = i == 0 ? (const void*)pr->u(0) : (const void*)pr->f(0);
        e = enqueue_rk4_step(g, 0, h->coef, pr->dtF, nu, in, pr->f(0), ya, yb, acc, P, pr->itemlo(), 0, tf, s, err);
    }
    if (e == cudaSuccess && events) e = cudaEventRecordWithFlags(pr->ev[1], s, cudaEventRecordExternal);
    if (e == cudaSuccess && mid) e = mid();
    if (e == cudaSuccess && (parts & 2)) e = cudaMemsetAsync(pr->def(), 0, 2 * P * sizeof(double), s);
    const bool delta = pr->cfg.coarse_delta != 0;
    // increment form: the first slice still iterating receives an unchanged input
    if (e == cudaSuccess && delta && (parts & 2))
        e = launch_zero_item(pr->D.p, (long long)pr->gc.total * pr->gc.es, P, pr->itemlo(), s, zero_min);
    for (int r = 0; r < P && e == cudaSuccess && rc == SP_OK && (parts & 2); ++r) {
        const double tStart = pr->slice * (pr->first + r);
        if (delta) {
            rc = enqueue_coarse(pr, pr->dlt(r), pr->gc, tStart, pr->tsC, true, r, s);
            if (rc) break;
            e = launch_update_delta(g, pr->gc, pr->gt(pr->coarse_res), pr->f(r), pr->u(r + 1), pr->dlt(r + 1),
                                    pr->def() + 2 * r, pr->itemlo(), r, s);
        } else {
            rc = enqueue_coarse(pr, pr->u(r), g, tStart, pr->tsC, true, r, s);
            if (rc) break;
            e = launch_update(g, pr->gc, pr->gt(pr->coarse_res), pr->f(r), pr->gold(r), pr->u(r + 1),
                              pr->def() + 2 * r, pr->itemlo(), r, s);
        }
    }
    if (e == cudaSuccess && rc == SP_OK && events) e = cudaEventRecordWithFlags(pr->ev[2], s, cudaEventRecordExternal);
    if (rc != SP_OK) return rc;
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, "iteration capture: %s", cudaGetErrorString(e));
    return SP_OK;
}

// Captures one Parareal iteration (emit_iteration) into a new graph.
int capture_iteration(sp_parareal* pr, bool events, cudaGraph_t* out, long long* nodes_out, int parts = 3,
                      int zero_min = 0) {
    cudaStream_t s = pr->prop->stream();
    int rc = prepare_iteration(pr, parts);
    if (rc) return rc;
    SP_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const long long before = launches();
    rc = emit_iteration(pr, s, events, parts, zero_min);
    const long long nodes = launches() - before;
    add_launches(-nodes);
    cudaGraph_t graph = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &graph);
    if (rc != SP_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e2 != cudaSuccess) return fail(SP_ERR_CUDA, "iteration end capture: %s", cudaGetErrorString(e2));
    *out = graph;
    *nodes_out = nodes;
    return SP_OK;
}

int build_iteration_graph(sp_parareal* pr) {
    cudaGraph_t graph = nullptr;
    long long nodes = 0;
    int rc = capture_iteration(pr, true, &graph, &nodes);
    if (rc) return rc;
    cudaError_t e = cudaGraphInstantiate(&pr->iter, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, "iteration instantiate: %s", cudaGetErrorString(e));
    pr->iter_nodes = nodes;
    return SP_OK;
}

LoopArgs loop_args(sp_parareal* pr, const double* reference) {
    LoopArgs a;
    a.c = pr->lctl.as<LoopCtl>();
    a.item_lo = pr->itemlo();
    a.def = pr->def();
    a.err4 = pr->err4();
    a.P = pr->P;
    a.skip = pr->cfg.skip_converged ? 1 : 0;
    a.kmax = pr->cfg.kmax;
    a.tol_kind = pr->cfg.tol_kind;
    a.has_ref = reference ? 1 : 0;
    a.tol = pr->cfg.tol;
    return a;
}

// Every iteration of DoParallel (Parareal.h:116-165) in one graph: a
// conditional WHILE node whose body is k_loop_head (item_lo from the device
// iteration counter), the iteration, the errors against `reference` (if any)
// and k_loop_tail, which records the defect and decides on the device whether
// to iterate again (the host loop's test: kmax, the tolerance, non-finite
// defects).  Rebuilt when the reference field changes.
int build_loop_graph(sp_parareal* pr, const double* reference) {
    if (pr->loop && pr->loop_ref == reference) return SP_OK;
    if (pr->loop) {
        cudaGraphExecDestroy(pr->loop);
        pr->loop = nullptr;
    }
    int rc = prepare_iteration(pr, 3);
    if (rc) return rc;
    if (pr->lctl.alloc(sizeof(LoopCtl)) != cudaSuccess) return fail(SP_ERR_NOMEM, "loop control");
    if (!pr->h_lctl) SP_CUDA(cudaMallocHost(&pr->h_lctl, sizeof(LoopCtl)));
    cudaStream_t s = pr->prop->stream();
    const LoopArgs a = loop_args(pr, reference);
    cudaGraph_t g = nullptr;
    SP_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle hc;
    cudaError_t e = cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = hc;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(SP_ERR_CUDA, "loop graph: %s", cudaGetErrorString(e));
    }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(SP_ERR_CUDA, "loop capture: %s", cudaGetErrorString(e));
    }
    const long long before = launches();
    k_loop_head<<<1, 1, 0, s>>>(a);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        rc = emit_iteration(pr, s, false, 3, 0, [&]() -> cudaError_t {
            k_loop_mid<<<1, 1, 0, s>>>(a.c);
            return cudaGetLastError();
        });
    }
    if (e == cudaSuccess && rc == SP_OK && reference) {
        e = cudaMemsetAsync(pr->err4(), 0, 4 * sizeof(double), s);
        if (e == cudaSuccess) e = launch_errors(pr->g64, pr->u(pr->P), reference, pr->err4(), s);
    }
    if (e == cudaSuccess && rc == SP_OK) {
        k_loop_tail<<<1, 1, 0, s>>>(a, hc);
        e = cudaGetLastError();
    }
    const long long nodes = launches() - before + 3;  // + head, mid and tail
    add_launches(-(launches() - before));
    cudaGraph_t captured = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &captured);
    if (rc != SP_OK || e != cudaSuccess || e2 != cudaSuccess) {
        cudaGraphDestroy(g);
        if (rc != SP_OK) return rc;
        return fail(SP_ERR_CUDA, "loop capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    e = cudaGraphInstantiate(&pr->loop, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        pr->loop = nullptr;
        return fail(SP_ERR_CUDA, "loop instantiate: %s", cudaGetErrorString(e));
    }
    pr->loop_ref = reference;
    pr->loop_nodes = nodes;
    return SP_OK;
}

// The initial field into U_0 and the coarse predictor (Parareal.h:113-114):
// U_r = G^{tsC*r}(q0) from t = 0, Gold_r = G(U_r) (reference form), and the
// last slice's end value U_P = G(U_{P-1}), all enqueued on s.
int enqueue_predictor(sp_parareal* pr, const double* initial, cudaStream_t s) {
    sp_convection* h = pr->prop;
    const int P = pr->P;
    const Geo& g = pr->g64;
    int rc = SP_OK;
    // rank 0's qinitial is the initial field
    SP_CUDA(cudaMemcpyAsync(pr->u(0), initial, g.total * 8, cudaMemcpyDeviceToDevice, s));
    SP_CUDA(launch_periodicity(g, pr->u(0), 1, s));
    const size_t cb = (size_t)pr->gc.total * pr->gc.es;
    const bool delta = pr->cfg.coarse_delta != 0;
    const int F0 = pr->first;
    if (F0 > 0) {
        // a window's first slice: G^{tsC*first}(q0) from t = 0, as the reference's rank `first` computes it
        if ((rc = enqueue_coarse(pr, initial, g, 0., pr->tsC * F0, false, 0, s))) return rc;
        SP_CUDA(launch_convert(g, pr->u(0), pr->gc, pr->gt(pr->coarse_res), s));
    }
    if (h->P.nufreq == 0.) {
        // With constant nu, U_r = G^{tsC*r}(q0) from t=0 equals the chain
        // U_{r+1} = G(U_r) step for step, and Gold_r = G(U_r) = U_{r+1}.
        for (int r = 0; r < P; ++r) {
            if ((rc = enqueue_coarse(pr, pr->u(r), g, pr->slice * (F0 + r), pr->tsC, false, 0, s))) return rc;
            if (!delta)
                SP_CUDA(cudaMemcpyAsync(pr->gold(r), pr->gt(pr->coarse_res), cb, cudaMemcpyDeviceToDevice, s));
            SP_CUDA(launch_convert(g, pr->u(r + 1), pr->gc, pr->gt(pr->coarse_res), s));
        }
    } else {
        for (int r = 1; r < P; ++r) {
            if ((rc = enqueue_coarse(pr, initial, g, 0., pr->tsC * (F0 + r), false, 0, s))) return rc;
            SP_CUDA(launch_convert(g, pr->u(r), pr->gc, pr->gt(pr->coarse_res), s));
        }
        for (int r = delta ? P - 1 : 0; r < P; ++r) {
            if ((rc = enqueue_coarse(pr, pr->u(r), g, pr->slice * (F0 + r), pr->tsC, false, 0, s))) return rc;
            if (!delta)
                SP_CUDA(cudaMemcpyAsync(pr->gold(r), pr->gt(pr->coarse_res), cb, cudaMemcpyDeviceToDevice, s));
            if (r == P - 1) SP_CUDA(launch_convert(g, pr->u(P), pr->gc, pr->gt(pr->coarse_res), s));
        }
    }
    return rc;
}

}  // namespace

extern "C" {

int sp_parareal_create(sp_convection* prop, const sp_parareal_cfg* cfg, sp_parareal** out) {
    int rc = check_handle(prop);
    if (rc) return rc;
    if (!cfg || !out) return fail(SP_ERR_INVALID, "null argument");
    *out = nullptr;
    const sp_parareal_cfg& c = *cfg;
    if (c.timeSlices < 1 || c.timeStepsFine < 1 || c.timeStepsCoarse < 1 || c.kmax < 0 || !(c.endTime > 0))
        return fail(SP_ERR_INVALID, "bad Parareal configuration");
    if (c.kmax > SP_MAX_ITERS) return fail(SP_ERR_INVALID, "kmax > %d", SP_MAX_ITERS);
    if (c.coarse_scheme != SP_COARSE_EULER && c.coarse_scheme != SP_COARSE_RK4)
        return fail(SP_ERR_INVALID, "coarse_scheme");
    if (c.coarse_precision != SP_F64 && c.coarse_precision != SP_F32) return fail(SP_ERR_INVALID, "coarse_precision");
    std::unique_ptr<sp_parareal> pr(new sp_parareal());
    pr->prop = prop;
    pr->cfg = c;
    const int PG = c.timeSlices;
    if (c.first_slice < 0 || c.slice_count < 0 || c.first_slice + std::max(c.slice_count, 1) > PG ||
        (c.slice_count == 0 && c.first_slice != 0))
        return fail(SP_ERR_INVALID, "slice window [%d, +%d) outside %d slices", c.first_slice, c.slice_count, PG);
    const int P = c.slice_count > 0 ? c.slice_count : PG;
    pr->P = P;
    pr->first = c.first_slice;
    pr->Pglobal = PG;
    // RuntimeConfiguration.cpp:133-151: totals rounded up to a multiple of the slice count.
    int f = c.timeStepsFine, g = c.timeStepsCoarse;
    if (f % PG != 0) f = (f / PG + 1) * PG;
    if (g % PG != 0) g = (g / PG + 1) * PG;
    pr->tsF = f / PG;
    pr->tsC = g / PG;
    pr->dtF = c.endTime / f;  // RuntimeConfiguration.h:54-65
    pr->dtC = c.endTime / g;
    pr->slice = c.endTime / PG;
    pr->cprec = c.coarse_precision == SP_F64 ? 0 : 1;
    pr->g64 = prop->g[0];
    pr->gc = prop->g[pr->cprec];
    const size_t f64b = (size_t)pr->g64.total * 8;
    const size_t cb = (size_t)pr->gc.total * pr->gc.es;
    const bool delta = c.coarse_delta != 0;
    if (pr->U.alloc((P + 1) * f64b) != cudaSuccess || pr->F.alloc(P * f64b) != cudaSuccess ||
        (delta ? pr->D.alloc((P + 1) * cb) : pr->Gold.alloc(P * cb)) != cudaSuccess || pr->Z.alloc(cb) != cudaSuccess ||
        pr->Gt.alloc(5 * cb) != cudaSuccess || pr->ctl.alloc(256 + (2 * P + 8) * sizeof(double)) != cudaSuccess)
        return fail(SP_ERR_NOMEM, "Parareal state for %d slices", P);
    if (prop->P.nufreq != 0.) {
        // nu(t) per slice and fine step (Convection.h:81-84) with the time
        // sequence of DoRK4 (Convection.cpp:296-302) or of the split first
        // step of the asynchronous variant (Parareal.h:119-124).
        std::vector<double> tab((size_t)pr->tsF * P);
        for (int r = 0; r < P; ++r) {
            const double tStart = pr->slice * (pr->first + r);
            const double tStartFine = tStart + pr->dtF;
            for (int i = 0; i < pr->tsF; ++i) {
                double t;
                if (c.async && pr->first + r != 0)
                    t = i == 0 ? tStart : (i == 1 ? tStartFine : tStartFine + (i - 1) * pr->dtF);
                else t = i == 0 ? tStart : tStart + i * pr->dtF;
                tab[(size_t)i * P + r] = computenu(prop->P.nu0, prop->P.nufreq, t);
            }
        }
        if (pr->nutab.alloc(tab.size() * sizeof(double)) != cudaSuccess) return fail(SP_ERR_NOMEM, "nu table");
        SP_CUDA(cudaMemcpy(pr->nutab.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    SP_CUDA(cudaMallocHost(&pr->h_itemlo, sizeof(int)));
    SP_CUDA(cudaMallocHost(&pr->h_def, (2 * P + 8) * sizeof(double)));
    for (auto& e : pr->ev) SP_CUDA(cudaEventCreate(&e));
    *out = pr.release();
    return SP_OK;
}

int sp_parareal_destroy(sp_parareal* pr) {
    if (!pr) return SP_OK;
    cudaSetDevice(pr->prop->device);
    cudaStreamSynchronize(pr->prop->stream());
    delete pr;
    return SP_OK;
}

int sp_parareal_set_host_loop(sp_parareal* pr, int host_loop) {
    if (!pr) return fail(SP_ERR_INVALID, "null Parareal handle");
    pr->host_loop = host_loop ? 1 : 0;
    return SP_OK;
}

int sp_parareal_do_serial(sp_parareal* pr, const double* initial, double* solution) {
    NvtxRange range("Parareal::DoSerial");
    if (!pr) return fail(SP_ERR_INVALID, "null Parareal handle");
    // Parareal::DoSerial (Parareal.h:250-253)
    return sp_do_rk4(pr->prop, initial, solution, 0., pr->dtF, pr->tsF * pr->Pglobal);
}

int sp_parareal_do_parallel(sp_parareal* pr, const double* initial, double* solution, const double* reference,
                            sp_parareal_report* rep) {
    if (!pr) return fail(SP_ERR_INVALID, "null Parareal handle");
    sp_convection* h = pr->prop;
    int rc = check_handle(h);
    if (rc) return rc;
    if (!initial || !solution) return fail(SP_ERR_INVALID, "null field");
    if (pr->P != pr->Pglobal) return fail(SP_ERR_STATE, "a slice-window handle runs through sp_parareal_window_*");
    cudaStream_t s = h->stream();
    if (capturing(s)) return fail(SP_ERR_STATE, "DoParallel cannot run inside a stream capture");
    const int P = pr->P;
    const Geo& g = pr->g64;
    const int cp = pr->cprec;
    if ((rc = h->ensure_scratch(cp, 1))) return rc;
    if (rep) {
        std::memset(rep, 0, sizeof *rep);
        rep->tsFine = pr->tsF; rep->tsCoarse = pr->tsC;
        rep->dtFine = pr->dtF; rep->dtCoarse = pr->dtC; rep->timeSliceSize = pr->slice;
    }
    if (pr->host_loop) {
        if (!pr->iter && (rc = build_iteration_graph(pr))) return rc;
    } else if (pr->cfg.kmax > 0 && (rc = build_loop_graph(pr, reference))) {
        return rc;
    }

    NvtxRange range("Parareal::DoParallel");
    SP_CUDA(cudaEventRecord(pr->ev[3], s));
    {
        NvtxRange pred("predictor");
        if ((rc = enqueue_predictor(pr, initial, s))) return rc;
    }
    // Iterations (Parareal.h:116-165).
    int k = 0;
    double t_f = 0., t_c = 0.;
    long long fine_cu = 0;
    const long long cells = (long long)g.ni * g.nj * g.nk;
    const bool device_loop = !pr->host_loop && pr->cfg.kmax > 0;
    if (device_loop) {
        // all iterations in one graph launch; the stopping test runs on the
        // device, and the host reads the loop's record once, after the run
        NvtxRange it("iterations (one launch)");
        SP_CUDA(cudaMemsetAsync(pr->lctl.p, 0, sizeof(LoopCtl), s));
        SP_CUDA(cudaGraphLaunch(pr->loop, s));
        SP_CUDA(cudaMemcpyAsync(pr->h_lctl, pr->lctl.p, sizeof(LoopCtl), cudaMemcpyDeviceToHost, s));
    }
    for (; pr->host_loop && k < pr->cfg.kmax; ++k) {
        char label[32];
        std::snprintf(label, sizeof label, "iteration %d", k + 1);
        NvtxRange it(label);
        const int lo = pr->cfg.skip_converged ? std::min(k, P) : 0;
        *pr->h_itemlo = lo;
        SP_CUDA(cudaMemcpyAsync(pr->itemlo(), pr->h_itemlo, sizeof(int), cudaMemcpyHostToDevice, s));
        SP_CUDA(cudaGraphLaunch(pr->iter, s));
        add_launches(pr->iter_nodes);
        fine_cu += (long long)(P - lo) * pr->tsF * cells;
        if (reference) {
            SP_CUDA(cudaMemsetAsync(pr->err4(), 0, 4 * sizeof(double), s));
            SP_CUDA(launch_errors(g, pr->u(P), reference, pr->err4(), s));
        }
        SP_CUDA(cudaMemcpyAsync(pr->h_def, pr->def(), (2 * P + 4) * sizeof(double), cudaMemcpyDeviceToHost, s));
        SP_CUDA(cudaStreamSynchronize(s));
        float ms1 = 0, ms2 = 0;
        cudaEventElapsedTime(&ms1, pr->ev[0], pr->ev[1]);
        cudaEventElapsedTime(&ms2, pr->ev[1], pr->ev[2]);
        t_f += ms1 * 1e-3;
        t_c += ms2 * 1e-3;
        double defect = 0.;
        bool finite = true;
        for (int r = lo; r < P; ++r) {
            const double num = pr->h_def[2 * r], den = pr->h_def[2 * r + 1];
            if (!std::isfinite(num) || !std::isfinite(den)) finite = false;
            if (den > 0) defect = std::max(defect, std::sqrt(num / den));
        }
        double el2 = 0., emax = 0.;
        if (reference) {
            const double* e4 = pr->h_def + 2 * P;
            el2 = std::sqrt(e4[0] / e4[1]);
            emax = e4[2] / e4[3];
        }
        if (rep) {
            rep->defect[k] = defect;
            rep->err_l2[k] = el2;
            rep->err_max[k] = emax;
        }
        if (!finite) {
            if (rep) rep->iterations = k + 1;
            return fail(SP_ERR_NONFINITE, "Parareal defect is not finite at iteration %d", k + 1);
        }
        if (pr->cfg.tol_kind == SP_TOL_DEFECT && defect < pr->cfg.tol) { ++k; break; }
        if (pr->cfg.tol_kind == SP_TOL_REFERENCE && reference && el2 < pr->cfg.tol) { ++k; break; }
    }
    SP_CUDA(cudaMemcpyAsync(solution, pr->u(P), g.total * 8, cudaMemcpyDeviceToDevice, s));
    SP_CUDA(cudaEventRecord(pr->ev[4], s));
    SP_CUDA(cudaEventSynchronize(pr->ev[4]));
    float ms = 0;
    cudaEventElapsedTime(&ms, pr->ev[3], pr->ev[4]);
    if (device_loop) {
        const LoopCtl& c = *pr->h_lctl;
        k = c.k;
        add_launches((long long)k * pr->loop_nodes);
        for (int i = 0; i < k; ++i) {
            const int lo = pr->cfg.skip_converged ? std::min(i, P) : 0;
            fine_cu += (long long)(P - lo) * pr->tsF * cells;
            if (rep) {
                rep->defect[i] = c.defect[i];
                rep->err_l2[i] = c.err_l2[i];
                rep->err_max[i] = c.err_max[i];
            }
        }
        t_f = c.ns_fine * 1e-9;
        t_c = c.ns_coarse * 1e-9;
        if (c.nonfinite) {
            if (rep) rep->iterations = k;
            return fail(SP_ERR_NONFINITE, "Parareal defect is not finite at iteration %d", k);
        }
    }
    if (rep) {
        rep->iterations = k;
        rep->seconds = ms * 1e-3;
        rep->seconds_fine = t_f;
        rep->seconds_coarse = t_c;
        rep->fine_cell_updates = fine_cu;
    }
    return sp_convection_synchronize(h);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint of DoRK4 (Convection.cpp:292-370).  Per step, with h = dt, forward
// stage inputs y1 = q, y2 = q + h/2 k1, y3 = q + h/2 k2, y4 = q + h k3 and the
// step-end adjoint lam:
//   mu4 = h/6 lam,               ybar4 = R^T mu4
//   mu3 = h/3 lam + h   ybar4,   ybar3 = R^T mu3
//   mu2 = h/3 lam + h/2 ybar3,   ybar2 = R^T mu2
//   mu1 = h/6 lam + h/2 ybar2,   ybar1 = R^T mu1
//   lam_prev = lam + ybar1 + ybar2 + ybar3 + ybar4
//   dJ/dtheta += sum_s mu_s . dR/dtheta (y_s)
// R^T is the same stencil with the velocity negated (D_d is antisymmetric
// and Laplace4 symmetric on the periodic grid).  Checkpoints every `ck` steps;
// each segment's stage inputs are recomputed and stored before its backward
// sweep.
extern "C" int sp_adjoint_rk4(sp_convection* h, const double* q0, const double* q_target, const double* lambda_n,
                              double tStart, double dt, int n, int ck, double* J, double* grad_q0,
                              double* grad_par) {
    NvtxRange range("adjoint RK4");
    int rc = check_handle(h);
    if (rc) return rc;
    if (!q0 || !grad_q0 || (!q_target && !lambda_n)) return fail(SP_ERR_INVALID, "null field");
    if (n < 0) return fail(SP_ERR_INVALID, "negative step count");
    cudaStream_t s = h->stream();
    if (capturing(s)) return fail(SP_ERR_STATE, "the adjoint cannot run inside a stream capture");
    if (ck <= 0) ck = std::max(1, (int)std::ceil(std::sqrt((double)std::max(n, 1))));
    ck = std::min(ck, std::max(n, 1));
    const int nseg = n > 0 ? (n + ck - 1) / ck : 0;
    const Geo& g = h->g[0];
    const size_t fb = (size_t)g.total * 8;
    if ((rc = h->ensure_scratch(0, 1))) return rc;
    DevBuf& ckpt = h->adj_ckpt;
    DevBuf& seg = h->adj_seg;
    DevBuf& work = h->adj_work;
    DevBuf& par = h->adj_par;
    // work: qn, lam, lam_acc, mu_a, mu_b, dummy
    if (ckpt.alloc(std::max(nseg, 1) * fb) != cudaSuccess || seg.alloc((size_t)4 * ck * fb) != cudaSuccess ||
        work.alloc(6 * fb) != cudaSuccess || par.alloc(8 * sizeof(double)) != cudaSuccess)
        return fail(SP_ERR_NOMEM, "adjoint buffers (%d checkpoints, %d-step segments)", nseg, ck);
    auto CK = [&](int i) { return ckpt.as<double>() + (size_t)i * g.total; };
    auto SG = [&](int i) { return seg.as<double>() + (size_t)i * g.total; };  // [y2 | y3 | y4 | state] x ck
    auto WK = [&](int i) { return work.as<double>() + (size_t)i * g.total; };
    double* qn = WK(0);
    double* lam = WK(1);
    double* lamacc = WK(2);
    double* mua = WK(3);
    double* mub = WK(4);
    double* dummy = WK(5);
    const Tune t = h->tune(0, 1);
    int* err = h->err.as<int>();
    double* ya = static_cast<double*>(h->sbuf(0, 0, 1));
    double* yb = static_cast<double*>(h->sbuf(0, 1, 1));
    double* acc = static_cast<double*>(h->sbuf(0, 2, 1));
    const double nu0 = h->P.nu0, nuf = h->P.nufreq;
    SP_CUDA(cudaMemsetAsync(par.p, 0, 8 * sizeof(double), s));
    // forward sweep, keeping checkpoints
    SP_CUDA(cudaMemcpyAsync(nseg > 0 ? CK(0) : qn, q0, fb, cudaMemcpyDeviceToDevice, s));
    SP_CUDA(launch_periodicity(g, nseg > 0 ? CK(0) : qn, 1, s));
    for (int sg = 0; sg < nseg; ++sg) {
        const int s0 = sg * ck, s1 = std::min(n, s0 + ck);
        double* dst = (sg + 1 < nseg) ? CK(sg + 1) : qn;
        for (int st = s0; st < s1; ++st) {
            const double tt = tStart + st * dt;
            SP_CUDA(enqueue_rk4_step(g, 0, h->coef, dt, NuSrc{computenu(nu0, nuf, tt), nullptr},
                                     st == s0 ? (const void*)CK(sg) : (const void*)dst, dst, ya, yb, acc, 1, nullptr,
                                     0, t, s, err));
        }
    }
    // terminal adjoint
    if (lambda_n) {
        SP_CUDA(cudaMemcpyAsync(lam, lambda_n, fb, cudaMemcpyDeviceToDevice, s));
        SP_CUDA(launch_periodicity(g, lam, 1, s));
    } else {
        SP_CUDA(launch_misfit(g, qn, q_target, lam, par.as<double>() + 4, s));
    }
    // backward sweep
    for (int sg = nseg - 1; sg >= 0; --sg) {
        const int s0 = sg * ck, s1 = std::min(n, s0 + ck), m = s1 - s0;
        auto Y2 = [&](int i) { return SG(4 * i + 0); };
        auto Y3 = [&](int i) { return SG(4 * i + 1); };
        auto Y4 = [&](int i) { return SG(4 * i + 2); };
        auto ST = [&](int i) { return i == 0 ? CK(sg) : SG(4 * (i - 1) + 3); };  // state at step s0+i
        for (int i = 0; i < m; ++i) {
            const double tt = tStart + (s0 + i) * dt;
            double* next = (i + 1 < m) ? SG(4 * i + 3) : dummy;
            SP_CUDA(enqueue_rk4_step3(g, 0, h->coef, dt, NuSrc{computenu(nu0, nuf, tt), nullptr}, ST(i), next, Y2(i),
                                      Y3(i), Y4(i), acc, 1, nullptr, 0, t, s, err));
        }
        for (int i = m - 1; i >= 0; --i) {
            const double tt = tStart + (s0 + i) * dt;
            StageLaunch L;
            L.prec = 0;
            L.items = 1;
            L.coef = h->coef;
            L.nu = computenu(nu0, nuf, tt);
            L.dnu = 1. + .5 * std::sin(nuf * tt);
            L.par_acc = par.as<double>();
            // A4: stencil lam (mu4 = h/6 lam)
            L.op = OP_ADJ + 0; L.yin = lam; L.sigma = dt / 6.; L.ypt = Y4(i);
            L.yout = mua; L.lam_acc = lamacc; L.c_ybar = dt; L.c_lam = dt / 3.;
            SP_CUDA(launch_stage(g, L, t, s, err));
            // A3: stencil mu3
            L.op = OP_ADJ + 1; L.yin = mua; L.sigma = 1.; L.ypt = Y3(i); L.lam = lam;
            L.yout = mub; L.c_ybar = dt * .5; L.c_lam = dt / 3.;
            SP_CUDA(launch_stage(g, L, t, s, err));
            // A2: stencil mu2
            L.op = OP_ADJ + 2; L.yin = mub; L.ypt = Y2(i);
            L.yout = mua; L.c_ybar = dt * .5; L.c_lam = dt / 6.;
            SP_CUDA(launch_stage(g, L, t, s, err));
            // A1: stencil mu1 -> lam_prev (with images)
            L.op = OP_ADJ + 3; L.yin = mua; L.ypt = ST(i); L.yout = lamacc;
            SP_CUDA(launch_stage(g, L, t, s, err));
            std::swap(lam, lamacc);
        }
    }
    SP_CUDA(cudaMemcpyAsync(grad_q0, lam, fb, cudaMemcpyDeviceToDevice, s));
    double hp[8];
    SP_CUDA(cudaMemcpyAsync(hp, par.p, sizeof hp, cudaMemcpyDeviceToHost, s));
    if ((rc = sp_convection_synchronize(h))) return rc;
    if (grad_par) for (int i = 0; i < 4; ++i) grad_par[i] = hp[i];
    if (J) *J = lambda_n ? 0. : hp[4];
    return SP_OK;
}

// ---------------------------------------------------------------------------
// Many independent Parareal solves (uneven grids, parameters and slice
// counts) advanced together: each instance's iteration graph becomes a child
// graph of one parent graph, so one graph launch per iteration runs every
// instance's batched fine sweep and coarse sweep concurrently.  An instance
// that has converged (or used its kmax) gets item_lo = P, which turns its
// kernels into immediate returns.
struct sp_parareal_batch {
    std::vector<sp_parareal*> ins;
    int device = 0;
    cudaStream_t root = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long nodes = 0;
    std::vector<cudaGraph_t> children;     // each instance's captured iteration
    cudaGraphExec_t loop = nullptr;        // all iterations of all instances in one launch
    std::vector<const double*> loop_refs;  // reference fields the loop graph was built with
    long long loop_nodes = 0;
    DevBuf args;                           // LoopArgs of every instance
    int host_loop = 0;                     // 1: one graph launch and one host sync per iteration
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> done;
    ~sp_parareal_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (loop) cudaGraphExecDestroy(loop);
        for (auto c : children)
            if (c) cudaGraphDestroy(c);
        for (auto e : ev)
            if (e) cudaEventDestroy(e);
        for (auto e : done)
            if (e) cudaEventDestroy(e);
        if (root) cudaStreamDestroy(root);
    }
};

extern "C" int sp_parareal_batch_create(sp_parareal* const* ins, int n, sp_parareal_batch** out) {
    if (!ins || n < 1 || !out) return fail(SP_ERR_INVALID, "sp_parareal_batch_create: bad arguments");
    *out = nullptr;
    std::unique_ptr<sp_parareal_batch> b(new sp_parareal_batch());
    for (int i = 0; i < n; ++i) {
        if (!ins[i]) return fail(SP_ERR_INVALID, "null Parareal handle %d", i);
        if (ins[i]->P != ins[i]->Pglobal) return fail(SP_ERR_INVALID, "instance %d is a slice window", i);
        if (i && ins[i]->prop->device != ins[0]->prop->device)
            return fail(SP_ERR_INVALID, "all instances must live on one device");
        b->ins.push_back(ins[i]);
    }
    b->device = ins[0]->prop->device;
    SP_CUDA(cudaSetDevice(b->device));
    SP_CUDA(cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking));
    for (auto& e : b->ev) SP_CUDA(cudaEventCreate(&e));
    b->done.resize(n, nullptr);
    for (auto& e : b->done) SP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaGraph_t parent = nullptr;
    SP_CUDA(cudaGraphCreate(&parent, 0));
    b->children.resize(n, nullptr);
    for (int i = 0; i < n; ++i) {
        long long nodes = 0;
        int rc = capture_iteration(b->ins[i], false, &b->children[i], &nodes);
        if (rc) { cudaGraphDestroy(parent); return rc; }
        cudaGraphNode_t node;
        cudaError_t e = cudaGraphAddChildGraphNode(&node, parent, nullptr, 0, b->children[i]);
        if (e != cudaSuccess) { cudaGraphDestroy(parent); return fail(SP_ERR_CUDA, "child graph: %s", cudaGetErrorString(e)); }
        b->nodes += nodes;
    }
    cudaError_t e = cudaGraphInstantiate(&b->exec, parent, 0);
    cudaGraphDestroy(parent);
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, "batch instantiate: %s", cudaGetErrorString(e));
    *out = b.release();
    return SP_OK;
}

namespace {
// Every iteration of every instance in one graph launch: a conditional WHILE
// node whose body runs k_batch_head, the instances' iterations (child graphs,
// concurrent), the errors against the references and k_batch_tail, which
// records each instance's defect, stops the instances that are done and ends
// the loop when none is left.  Rebuilt when the reference fields change.
int build_batch_loop(sp_parareal_batch* b, const double* const* reference) {
    const int n = (int)b->ins.size();
    std::vector<const double*> refs(n, nullptr);
    for (int i = 0; i < n; ++i) refs[i] = reference ? reference[i] : nullptr;
    if (b->loop && refs == b->loop_refs) return SP_OK;
    if (b->loop) {
        cudaGraphExecDestroy(b->loop);
        b->loop = nullptr;
    }
    std::vector<LoopArgs> hargs(n);
    for (int i = 0; i < n; ++i) {
        sp_parareal* pr = b->ins[i];
        if (pr->lctl.alloc(sizeof(LoopCtl)) != cudaSuccess) return fail(SP_ERR_NOMEM, "loop control");
        if (!pr->h_lctl) SP_CUDA(cudaMallocHost(&pr->h_lctl, sizeof(LoopCtl)));
        hargs[i] = loop_args(pr, refs[i]);
    }
    if (b->args.alloc(n * sizeof(LoopArgs)) != cudaSuccess) return fail(SP_ERR_NOMEM, "loop arguments");
    SP_CUDA(cudaMemcpy(b->args.p, hargs.data(), n * sizeof(LoopArgs), cudaMemcpyHostToDevice));
    const LoopArgs* dargs = b->args.as<LoopArgs>();
    cudaStream_t s = b->root;
    cudaGraph_t g = nullptr;
    SP_CUDA(cudaGraphCreate(&g, 0));
    auto bail = [&](cudaError_t e, const char* what) {
        cudaGraphDestroy(g);
        return fail(SP_ERR_CUDA, "batch loop graph (%s): %s", what, cudaGetErrorString(e));
    };
    cudaGraphConditionalHandle hc;
    cudaError_t e = cudaGraphConditionalHandleCreate(&hc, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = hc;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t cnode;
    if (e == cudaSuccess) e = cudaGraphAddNode(&cnode, g, nullptr, 0, &np);
    if (e != cudaSuccess) return bail(e, "conditional node");
    cudaGraph_t body = np.conditional.phGraph_out[0];
    // head
    cudaGraph_t cap = nullptr;
    e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return bail(e, "head capture");
    k_batch_head<<<1, 128, 0, s>>>(dargs, n);
    e = cudaGetLastError();
    cudaError_t e2 = cudaStreamEndCapture(s, &cap);
    if (e != cudaSuccess || e2 != cudaSuccess) return bail(e != cudaSuccess ? e : e2, "head");
    cudaGraphNode_t head = nullptr;
    size_t count = 1;
    e = cudaGraphGetNodes(body, &head, &count);
    if (e != cudaSuccess || count != 1) return bail(e, "head node");
    // the instances' iterations, concurrent
    std::vector<cudaGraphNode_t> kids(n);
    for (int i = 0; i < n; ++i) {
        e = cudaGraphAddChildGraphNode(&kids[i], body, &head, 1, b->children[i]);
        if (e != cudaSuccess) return bail(e, "child node");
    }
    // errors against the references, decision
    e = cudaStreamBeginCaptureToGraph(s, body, kids.data(), nullptr, n, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return bail(e, "tail capture");
    long long extra = 2;
    const long long before = launches();
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        if (!refs[i]) continue;
        sp_parareal* pr = b->ins[i];
        e = cudaMemsetAsync(pr->err4(), 0, 4 * sizeof(double), s);
        if (e == cudaSuccess) e = launch_errors(pr->g64, pr->u(pr->P), refs[i], pr->err4(), s);
        ++extra;
    }
    if (e == cudaSuccess) {
        k_batch_tail<<<1, 128, 0, s>>>(dargs, n, hc);
        e = cudaGetLastError();
    }
    add_launches(-(launches() - before));
    e2 = cudaStreamEndCapture(s, &cap);
    if (e != cudaSuccess || e2 != cudaSuccess) return bail(e != cudaSuccess ? e : e2, "tail");
    e = cudaGraphInstantiate(&b->loop, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->loop = nullptr;
        return fail(SP_ERR_CUDA, "batch loop instantiate: %s", cudaGetErrorString(e));
    }
    b->loop_refs = refs;
    b->loop_nodes = b->nodes + extra;
    return SP_OK;
}
}  // namespace

extern "C" int sp_parareal_batch_set_host_loop(sp_parareal_batch* b, int host_loop) {
    if (!b) return fail(SP_ERR_INVALID, "null batch handle");
    b->host_loop = host_loop ? 1 : 0;
    return SP_OK;
}

extern "C" int sp_parareal_batch_destroy(sp_parareal_batch* b) {
    if (!b) return SP_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->root);
    delete b;
    return SP_OK;
}

extern "C" int sp_parareal_batch_run(sp_parareal_batch* b, const double* const* initial, double* const* solution,
                                     const double* const* reference, sp_parareal_report* reports,
                                     double* seconds) {
    NvtxRange range("PararealBatch::run");
    if (!b || !initial || !solution) return fail(SP_ERR_INVALID, "sp_parareal_batch_run: null argument");
    const int n = (int)b->ins.size();
    SP_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = b->root;
    for (int i = 0; i < n; ++i) {
        sp_parareal* pr = b->ins[i];
        if (!initial[i] || !solution[i]) return fail(SP_ERR_INVALID, "null field of instance %d", i);
        int rc = pr->prop->ensure_scratch(pr->cprec, 1);
        if (rc) return rc;
        if (reports) {
            std::memset(&reports[i], 0, sizeof reports[i]);
            reports[i].tsFine = pr->tsF; reports[i].tsCoarse = pr->tsC;
            reports[i].dtFine = pr->dtF; reports[i].dtCoarse = pr->dtC; reports[i].timeSliceSize = pr->slice;
        }
    }
    SP_CUDA(cudaEventRecord(b->ev[0], s));
    // predictors, one stream per instance handle, joined back into the root stream
    for (int i = 0; i < n; ++i) {
        sp_parareal* pr = b->ins[i];
        cudaStream_t si = pr->prop->stream();
        SP_CUDA(cudaStreamWaitEvent(si, b->ev[0], 0));
        int rc = enqueue_predictor(pr, initial[i], si);
        if (rc) return rc;
        SP_CUDA(cudaEventRecord(b->done[i], si));
        SP_CUDA(cudaStreamWaitEvent(s, b->done[i], 0));
    }
    std::vector<int> iters(n, 0);
    std::vector<char> active(n, 1);
    int kmax = 0;
    for (auto* pr : b->ins) kmax = std::max(kmax, pr->cfg.kmax);
    const bool device_loop = !b->host_loop && kmax > 0;
    if (device_loop) {
        // every iteration of every instance in one graph launch
        int rc = build_batch_loop(b, reference);
        if (rc) return rc;
        for (auto* pr : b->ins) SP_CUDA(cudaMemsetAsync(pr->lctl.p, 0, sizeof(LoopCtl), s));
        SP_CUDA(cudaGraphLaunch(b->loop, s));
        for (auto* pr : b->ins)
            SP_CUDA(cudaMemcpyAsync(pr->h_lctl, pr->lctl.p, sizeof(LoopCtl), cudaMemcpyDeviceToHost, s));
    }
    for (int k = 0; k < kmax && !device_loop; ++k) {
        int n_active = 0;
        for (int i = 0; i < n; ++i) {
            sp_parareal* pr = b->ins[i];
            if (active[i] && k >= pr->cfg.kmax) active[i] = 0;
            *pr->h_itemlo = !active[i] ? pr->P : (pr->cfg.skip_converged ? std::min(k, pr->P) : 0);
            n_active += active[i];
            SP_CUDA(cudaMemcpyAsync(pr->itemlo(), pr->h_itemlo, sizeof(int), cudaMemcpyHostToDevice, s));
        }
        if (!n_active) break;
        SP_CUDA(cudaGraphLaunch(b->exec, s));
        add_launches(b->nodes);
        for (int i = 0; i < n; ++i) {
            if (!active[i]) continue;
            sp_parareal* pr = b->ins[i];
            if (reference && reference[i]) {
                SP_CUDA(cudaMemsetAsync(pr->err4(), 0, 4 * sizeof(double), s));
                SP_CUDA(launch_errors(pr->g64, pr->u(pr->P), reference[i], pr->err4(), s));
            }
            SP_CUDA(cudaMemcpyAsync(pr->h_def, pr->def(), (2 * pr->P + 4) * sizeof(double), cudaMemcpyDeviceToHost, s));
        }
        SP_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < n; ++i) {
            if (!active[i]) continue;
            sp_parareal* pr = b->ins[i];
            const int lo = pr->cfg.skip_converged ? std::min(k, pr->P) : 0;
            double defect = 0.;
            bool finite = true;
            for (int r = lo; r < pr->P; ++r) {
                const double num = pr->h_def[2 * r], den = pr->h_def[2 * r + 1];
                if (!std::isfinite(num) || !std::isfinite(den)) finite = false;
                if (den > 0) defect = std::max(defect, std::sqrt(num / den));
            }
            double el2 = 0., emax = 0.;
            const bool has_ref = reference && reference[i];
            if (has_ref) {
                const double* e4 = pr->h_def + 2 * pr->P;
                el2 = std::sqrt(e4[0] / e4[1]);
                emax = e4[2] / e4[3];
            }
            iters[i] = k + 1;
            if (reports) {
                reports[i].defect[k] = defect;
                reports[i].err_l2[k] = el2;
                reports[i].err_max[k] = emax;
                reports[i].fine_cell_updates +=
                    (long long)(pr->P - lo) * pr->tsF * pr->g64.ni * pr->g64.nj * pr->g64.nk;
            }
            if (!finite) return fail(SP_ERR_NONFINITE, "instance %d: defect not finite at iteration %d", i, k + 1);
            if ((pr->cfg.tol_kind == SP_TOL_DEFECT && defect < pr->cfg.tol) ||
                (pr->cfg.tol_kind == SP_TOL_REFERENCE && has_ref && el2 < pr->cfg.tol) || k + 1 >= pr->P)
                active[i] = 0;
        }
    }
    for (int i = 0; i < n; ++i) {
        sp_parareal* pr = b->ins[i];
        SP_CUDA(cudaMemcpyAsync(solution[i], pr->u(pr->P), pr->g64.total * 8, cudaMemcpyDeviceToDevice, s));
    }
    SP_CUDA(cudaEventRecord(b->ev[1], s));
    SP_CUDA(cudaEventSynchronize(b->ev[1]));
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]);
    if (seconds) *seconds = ms * 1e-3;
    if (device_loop) {
        int kdone = 0, bad = -1;
        for (int i = 0; i < n; ++i) {
            sp_parareal* pr = b->ins[i];
            const LoopCtl& c = *pr->h_lctl;
            iters[i] = c.k;
            kdone = std::max(kdone, c.k);
            if (c.nonfinite && bad < 0) bad = i;
            if (!reports) continue;
            for (int k = 0; k < c.k; ++k) {
                const int lo = pr->cfg.skip_converged ? std::min(k, pr->P) : 0;
                reports[i].defect[k] = c.defect[k];
                reports[i].err_l2[k] = c.err_l2[k];
                reports[i].err_max[k] = c.err_max[k];
                reports[i].fine_cell_updates +=
                    (long long)(pr->P - lo) * pr->tsF * pr->g64.ni * pr->g64.nj * pr->g64.nk;
            }
        }
        add_launches((long long)kdone * b->loop_nodes);
        if (bad >= 0) {
            if (reports)
                for (int i = 0; i < n; ++i) reports[i].iterations = iters[i];
            return fail(SP_ERR_NONFINITE, "instance %d: defect not finite at iteration %d", bad, iters[bad]);
        }
    }
    if (reports)
        for (int i = 0; i < n; ++i) reports[i].iterations = iters[i];
    for (auto* pr : b->ins) {
        int rc = sp_convection_synchronize(pr->prop);
        if (rc) return rc;
    }
    return SP_OK;
}

// ---------------------------------------------------------------------------
// Slice-window steps (Parareal over several GPUs; the exchange between windows
// is the caller's, e.g. NCCL send/recv of the boundary field).
namespace {
int window_graphs(sp_parareal* pr) {
    if (pr->wfine) return SP_OK;
    cudaGraph_t g1 = nullptr, g2 = nullptr;
    long long n1 = 0, n2 = 0;
    int rc = capture_iteration(pr, false, &g1, &n1, 1, 0);
    if (rc) return rc;
    rc = capture_iteration(pr, false, &g2, &n2, 2, 1);
    if (rc) { cudaGraphDestroy(g1); return rc; }
    cudaError_t e = cudaGraphInstantiate(&pr->wfine, g1, 0);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&pr->wcoarse, g2, 0);
    cudaGraphDestroy(g1);
    cudaGraphDestroy(g2);
    if (e != cudaSuccess) return fail(SP_ERR_CUDA, "window graphs: %s", cudaGetErrorString(e));
    pr->wfine_nodes = n1;
    pr->wcoarse_nodes = n2;
    return SP_OK;
}

int window_itemlo(sp_parareal* pr, int k) {
    // global slices < k are exact after k iterations; local index of the first that is not
    return pr->cfg.skip_converged ? std::max(0, std::min(k - pr->first, pr->P)) : 0;
}
}  // namespace

extern "C" int sp_parareal_window_begin(sp_parareal* pr, const double* initial) {
    if (!pr || !initial) return fail(SP_ERR_INVALID, "null argument");
    int rc = check_handle(pr->prop);
    if (rc) return rc;
    cudaStream_t s = pr->prop->stream();
    if ((rc = pr->prop->ensure_scratch(pr->cprec, 1))) return rc;
    if ((rc = window_graphs(pr))) return rc;
    return enqueue_predictor(pr, initial, s);
}

extern "C" int sp_parareal_window_fine(sp_parareal* pr, int k) {
    if (!pr || k < 0) return fail(SP_ERR_INVALID, "bad argument");
    int rc = check_handle(pr->prop);
    if (rc) return rc;
    if ((rc = window_graphs(pr))) return rc;
    cudaStream_t s = pr->prop->stream();
    *pr->h_itemlo = window_itemlo(pr, k);
    SP_CUDA(cudaMemcpyAsync(pr->itemlo(), pr->h_itemlo, sizeof(int), cudaMemcpyHostToDevice, s));
    SP_CUDA(cudaGraphLaunch(pr->wfine, s));
    add_launches(pr->wfine_nodes);
    return SP_OK;
}

extern "C" int sp_parareal_window_coarse(sp_parareal* pr, int k, const double* u_first_new, double* q_last,
                                         double* defect) {
    if (!pr || k < 0) return fail(SP_ERR_INVALID, "bad argument");
    int rc = check_handle(pr->prop);
    if (rc) return rc;
    if ((rc = window_graphs(pr))) return rc;
    if ((pr->first > 0) != (u_first_new != nullptr))
        return fail(SP_ERR_INVALID, "u_first_new is required exactly when the window does not start at slice 0");
    cudaStream_t s = pr->prop->stream();
    const Geo& g = pr->g64;
    const int lo = window_itemlo(pr, k);
    // the window's first slice input: U_0 <- received value (the reference's
    // MPI_Recv into qinitial, Parareal.h:132-139); increment form: D_0 = new - old
    if (pr->cfg.coarse_delta) {
        if (u_first_new) {
            SP_CUDA(launch_update_delta(g, pr->gc, pr->Z.p, u_first_new, pr->u(0), pr->dlt(0), pr->err4(), nullptr,
                                        0, s));
        } else {
            SP_CUDA(cudaMemsetAsync(pr->dlt(0), 0, (size_t)pr->gc.total * pr->gc.es, s));
        }
    } else if (u_first_new) {
        SP_CUDA(cudaMemcpyAsync(pr->u(0), u_first_new, g.total * 8, cudaMemcpyDeviceToDevice, s));
        SP_CUDA(launch_periodicity(g, pr->u(0), 1, s));
    }
    (void)lo;
    SP_CUDA(cudaGraphLaunch(pr->wcoarse, s));
    add_launches(pr->wcoarse_nodes);
    if (q_last) SP_CUDA(cudaMemcpyAsync(q_last, pr->u(pr->P), g.total * 8, cudaMemcpyDeviceToDevice, s));
    if (defect) {
        SP_CUDA(cudaMemcpyAsync(pr->h_def, pr->def(), 2 * pr->P * sizeof(double), cudaMemcpyDeviceToHost, s));
        SP_CUDA(cudaStreamSynchronize(s));
        double d = 0.;
        for (int r = window_itemlo(pr, k); r < pr->P; ++r)
            if (pr->h_def[2 * r + 1] > 0) d = std::max(d, std::sqrt(pr->h_def[2 * r] / pr->h_def[2 * r + 1]));
        *defect = d;
    }
    return SP_OK;
}
