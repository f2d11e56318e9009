// sp_internal.h -- shared host-side declarations of the B200 propagator library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace sp {

// Geometry of one field in HBM (see sp_field_layout in include/sp_abi.h).
struct Geo {
    int ni = 0, nj = 0, nk = 0;
    int lx = 0;         // columns left of interior i = 0 (a multiple of 16 bytes, >= halo)
    int es = 0;         // element size in bytes
    int halo = 2;       // periodic image depth in y and z (and at least this much in x)
    long long px = 0, py = 0, pz = 0, plane = 0, origin = 0, total = 0;
};

// halo 2: the caller-visible layout of sp_field_layout.  halo 4: internal
// fields of the fused stage pairs.
Geo make_geo(int ni, int nj, int nk, int es, int halo = 2);

// Kernel families.
enum Op : int {
    OP_RK_S1 = 0,  // k=R(q);  y1=q+(dt/2)k                               (reads q)
    OP_RK_S2 = 1,  // k=R(y1); y2=q+(dt/2)k; a=q+(y1-q)/3+(dt/3)k         (reads y1, q)
    OP_RK_S3 = 2,  // k=R(y2); y3=q+dt k                                  (reads y2, q)
    OP_RK_S4 = 3,  // k=R(y3); out=a+(y3-q)/3+(dt/6)k                     (reads y3, a, q)
    OP_EULER = 4,  // k=R2(y); out=y+dt k
    OP_ADJ = 5,    // adjoint stage (see sp_adjoint.cu)
    OP_COUNT = 6
};

// Launch shape of one stage kernel.
struct Shape {
    int ty = 4;       // rows of a CTA tile
    int zchunk = 8;   // planes marched by one CTA
    int tma = 1;      // 1: TMA/mbarrier pipeline kernel; 0: direct-load kernel
    int tx = 64;      // fused pairs: tile columns (64, or 32 with two tile rows per warp)
};
inline bool same_shape(const Shape& a, const Shape& b) {
    return a.ty == b.ty && a.zchunk == b.zchunk && a.tma == b.tma && a.tx == b.tx;
}

// Launch shapes of all stage kernels (indexed by Op, adjoint stages included).
constexpr int kNumOps = OP_ADJ + 4;
struct Tune {
    Shape op[kNumOps];
    Shape pair[2] = {Shape{8, 0, 1}, Shape{8, 0, 1}};  // fused stage pairs 1+2 and 3+4 (ty 8 or 16)
    int fused = 0;    // 1: FP64 RK4 steps run as the two fused pairs
    int cluster = 0;  // FP64 RK4 propagations of small fields run cluster-resident (sp_cluster.cu):
                      // 1 on z-slabs, 2 on (y,z) blocks
    void set_all(const Shape& s) {
        for (auto& o : op) o = s;
    }
};

// Coefficients of the right-hand side, precomputed on the host.
struct Coef {
    // RHS4: R = cax*(8(q-1 - q+1) - (q-2 - q+2))_x + ... + nu*s4*(16 S1 - S2 - 90 q)
    double ca[3] = {0, 0, 0};  // c_d / (12 dx)
    double s4 = 0;             // 1 / (12 dx^2)
    // RHS2: R2 = sum_d u_d * dq_d + nu*s2*(S1 - 6q), dq_d per mode
    double u[3] = {0, 0, 0};
    int mode[3] = {0, 0, 0};   // 0: q - q[-1] (upwind, c>0); 1: q[+1] - q (upwind, c<=0); 2: q[-1] - q[+1] (central)
    double s2 = 0;             // 1 / dx^2
    double dx = 0;
};

Coef make_coef(double dx, double cx, double cy, double cz, int upwind);

// One stage launch over `items` fields stored back to back (item stride = geo.total).
struct StageLaunch {
    int op = OP_RK_S1;
    int prec = 0;                    // 0: FP64, 1: FP32
    const void* yin = nullptr;       // stencil input (field base of item 0)
    const void* q = nullptr;         // step-start field (S2, S3)
    void* acc = nullptr;             // accumulator (S1 writes, S2/S3 read+write, S4 reads)
    void* yout = nullptr;            // stencil output (written with periodic images)
    int items = 1;
    const int* item_lo = nullptr;    // device word: items below it are skipped (may be null)
    int item_base = 0;               // index of item 0 in the item_lo numbering
    double nu = 0;                   // diffusivity (all items) ...
    const double* nu_items = nullptr;// ... or one value per item (device)
    double c_y = 0, c_acc = 0;       // stage coefficients
    Coef coef;
    // adjoint extras
    const void* ypt = nullptr;       // forward stage value (pointwise)
    const void* lam = nullptr;       // adjoint of the step end (pointwise)
    void* lam_acc = nullptr;         // accumulated adjoint of the step start
    double* par_acc = nullptr;       // 4 partial sums (nu, cx, cy, cz) for the parameter gradient
    double c_lam = 0, c_ybar = 0;    // mu_{s-1} = c_lam*lam + c_ybar*ybar_s
    double sigma = 1;                // mu_s = sigma * (stencil input)
    double dnu = 1;                  // d nu / d nu0
    int adj_first = 0;               // 1: lam_acc = lam + ybar (first adjoint stage of a step)
};

// Many FP64 RK4 steps of small fields in one launch, each field held in the
// distributed shared memory of one thread-block cluster (sp_cluster.cu).  Reads
// the interiors of `items` fields at `in`, writes the interiors of the results
// at `out` (in == out allowed; the periodic images of `out` are left to the
// caller).  Step i uses the weights of `nu`, or wtab[i] (cluster_weights_bytes()
// each, device memory) when wtab is set.
struct ClusterLaunch {
    const void* in = nullptr;
    void* out = nullptr;
    int items = 1;
    int nsteps = 0;
    double dt = 0, nu = 0;
    Coef coef;
    const void* wtab = nullptr;
    const int* item_lo = nullptr;    // as in StageLaunch
    int item_base = 0;
    int mode = 1;                    // 1: z-slabs (k_rk4_cluster), 2: (y,z) blocks (k_rk4_cluster2d)
};
// mode 1: FP64, even ni, small planes, nk = C * {2,3,4} with 2 <= C <= 16;
// mode 2: FP64, even ni, nj = cy * BY, nk = cz * BZ with cy, cz, BY, BZ >= 2, cy * cz <= 16
bool cluster_supported(const Geo& g, int mode = 1);
cudaError_t prepare_cluster();
cudaError_t launch_rk4_cluster(const Geo& g, const ClusterLaunch& L, cudaStream_t s, int* err);
size_t cluster_weights_bytes();
void fill_cluster_weights(void* w13, const Coef& c, double nu);  // one entry of wtab (host memory)
constexpr int kClusterSmemMax = 227 * 1024;

// Launches one stage kernel; counts the launch.  err: device error word.
cudaError_t launch_stage(const Geo& g, const StageLaunch& L, const Tune& t, cudaStream_t s, int* err);

// Fused RK4 stage pairs (sp_fused.cu) on internal FP64 fields of geometry g4
// (make_geo(..., 8, 4)).  Pair 0 (stages 1+2): reads q; writes y2 (with
// images) and acc.  Pair 1 (stages 3+4): reads y2, q and acc; writes the step
// result to `out` in geometry go (g4, with out == acc allowed, or the caller's
// layout), with periodic images go.halo deep.
struct PairLaunch {
    int pair = 0;
    const void* q = nullptr;
    void* y2 = nullptr;
    void* acc = nullptr;
    void* out = nullptr;
    int items = 1;
    const int* item_lo = nullptr;    // as in StageLaunch
    int item_base = 0;
    double nu = 0, dt = 0;
    Coef coef;
};
bool pair_supported(const Geo& g);  // FP64, at least 4 interior cells per dimension
cudaError_t launch_pair(const Geo& g4, const Geo& go, const PairLaunch& L, const Shape& sh, cudaStream_t s, int* err);
// dst (geometry g4) <- interior of src (geometry gs), with g4.halo-deep images (FP64, items fields).
cudaError_t launch_widen(const Geo& g4, void* dst, const Geo& gs, const void* src, int items, const int* item_lo,
                         int item_base, cudaStream_t s);
cudaError_t prepare_pairs();
// Stores counted outside their output allocation by the bounds-checked build
// (stage kernels; pair and widening kernels) since the previous call; reset.
unsigned long long take_store_violations_stages();
unsigned long long take_store_violations_pairs();
// One CTA waiting on an mbarrier that never completes, bounded by limit_ns;
// sets *err to the timeout code (test of the bounded-wait error path).
cudaError_t launch_wait_selftest(int* err, unsigned long long limit_ns, cudaStream_t s);

// Pointwise helpers.
cudaError_t launch_periodicity(const Geo& g, void* field, int items, cudaStream_t s);
cudaError_t launch_dense_to_field(const Geo& g, const void* dense, int dense_prec, void* field, cudaStream_t s);
cudaError_t launch_field_to_dense(const Geo& g, const void* field, void* dense, int dense_prec, cudaStream_t s);
// dst (geo gd, precision of gd.es) <- src (geo gs), interior with images.
cudaError_t launch_convert(const Geo& gd, void* dst, const Geo& gs, const void* src, cudaStream_t s,
                           const int* item_lo = nullptr, int item = 0);
// Sets the dynamic shared-memory limit of every TMA stage kernel on the current device.
cudaError_t prepare_kernels();
// Parareal correction: Q = (gnew + f) - gold written to u_next (FP64, with images);
// gold <- gnew; defect sums (sum (Q-u_old)^2, sum Q^2) atomically added to def[0..1].
cudaError_t launch_update(const Geo& g64, const Geo& gc, const void* gnew, const double* f, void* gold,
                          double* u_next, double* def, const int* item_lo, int item, cudaStream_t s);
// Increment form: Q = f + gd written to u_next (images); d_next = Q - u_next(old) in
// coarse precision (images); defect sums into def[0..1].
cudaError_t launch_update_delta(const Geo& g64, const Geo& gc, const void* gd, const double* f, double* u_next,
                                void* d_next, double* def, const int* item_lo, int item, cudaStream_t s);
// Zeroes field *item_lo of an array of nitems fields of `bytes` bytes each (bytes % 16 == 0),
// unless *item_lo < min_item.
cudaError_t launch_zero_item(void* base, long long bytes, int nitems, const int* item_lo, cudaStream_t s,
                             int min_item = 0);
// err[0] += sum (a-b)^2 ; err[1] += sum b^2 ; err[2] = max |a-b| ; err[3] = max |a|   (FP64 fields)
cudaError_t launch_errors(const Geo& g, const double* a, const double* b, double* acc4, cudaStream_t s);
// Pointwise axpby on FP64 fields (interior+images): out = alpha*x + beta*y (y may be null).
cudaError_t launch_axpby(const Geo& g, double* out, double alpha, const double* x, double beta, const double* y,
                         cudaStream_t s);
// 0.5*||a-b||^2 and lam = a - b (lam may alias nothing; written with images).
cudaError_t launch_misfit(const Geo& g, const double* a, const double* b, double* lam, double* jacc, cudaStream_t s);

long long launches();
void add_launches(long long n);

// Records `fmt` as the calling thread's last error (sp_last_error) and returns code.
int sp_report(int code, const char* fmt, ...);

}  // namespace sp
