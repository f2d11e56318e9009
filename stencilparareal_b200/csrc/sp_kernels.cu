// sp_kernels.cu -- sm_100a kernels of the advection-diffusion propagator.
//
// Stage kernels.  One launch evaluates the right-hand side on every cell of
// one or more fields and fuses the Runge-Kutta (or Euler, or adjoint)
// pointwise update and the periodic halo into the same pass:
//
//   reference (Convection.cpp:318-370), per RK4 step:
//     4 x [Periodicity I/J/K kernels + RHS4 stencil] + 3 x Euler + 1 x RK
//   here, per RK4 step (q = step start, y = stage values, a = accumulator):
//     S1: k=R(q);  y1=q+dt/2 k
//     S2: k=R(y1); y2=q+dt/2 k;  a=q+(y1-q)/3+dt/3 k
//     S3: k=R(y2); y3=q+dt k
//     S4: k=R(y3); q'=a+(y3-q)/3+dt/6 k   (13 field accesses per cell-update)
//   ((y1-q)/3 = dt/6 k1 and (y3-q)/3 = dt/3 k3 recover two accumulator terms
//   from stage values, so that only S2 writes the accumulator)
//
// R is RHS4Stage (Convection.cpp:57-82): Advection4 (ConvectionFunctions.h:66-104)
// plus nu * Laplace4 (ConvectionFunctions.h:135-167), written as
//   R = sum_d c_d/(12dx) * (8(q[-1]-q[+1]) - (q[-2]-q[+2]))_d
//     + nu/(12dx^2) * (16 S1 - S2 - 90 q),  S1/S2 = sums of the +-1/+-2 neighbours,
// the same coefficients regrouped into differences (the direct-load kernel and
// the adjoint); the TMA RK stages use them combined into 13 per-offset weights
// (rhs_w13, sp_stencil.cuh), as the fused stage pairs do.  R2 is RHS2Stage
// (Convection.cpp:30-55) with the upwind Advection2 (ConvectionFunctions.h:18-42).
//
// Fields carry a 2-cell halo (layout in include/sp_abi.h).  Every kernel that
// writes a stencil input also writes the periodic images of the cells within
// two of a face, which replaces Periodicity::Apply (Periodicity.cu:146-214).
//
// Two implementations of every stage:
//  * k_stage_tma: a CTA owns a (32*VX) x TY tile of one field and marches a
//    chunk of z-planes.  One elected thread streams each plane's tile plus its
//    x/y halo with a single 3-D TMA box (cp.async.bulk.tensor) into a ring of
//    shared-memory slots completed on mbarriers; pointwise operands arrive the
//    same way.  The z-neighbours live in registers.  16-byte shared and global
//    accesses, VX = 2 (FP64) or 4 (FP32) cells per thread.
//  * k_stage_direct: one thread per column, loads straight from global memory
//    through L1; used for cross-checking and when the tuner prefers it.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <cstdio>
#include <mutex>
#include <type_traits>

#include "sp_device.cuh"
#include "sp_internal.h"
#include "sp_stencil.cuh"

namespace sp {

namespace {
std::atomic<long long> g_launches{0};
}
long long launches() { return g_launches.load(); }
void add_launches(long long n) { g_launches += n; }

Geo make_geo(int ni, int nj, int nk, int es, int halo) {
    Geo g;
    g.ni = ni; g.nj = nj; g.nk = nk; g.es = es; g.halo = halo;
    g.lx = (halo * es + 15) / 16 * 16 / es;
    const long long need = (long long)ni + 2 * g.lx;
    g.px = (need + 31) / 32 * 32;
    g.py = nj + 2 * halo;
    g.pz = nk + 2 * halo;
    g.plane = g.px * g.py;
    g.origin = halo * g.plane + halo * g.px + g.lx;
    g.total = g.plane * g.pz;
    return g;
}

Coef make_coef(double dx, double cx, double cy, double cz, int upwind) {
    Coef c;
    const double cs[3] = {cx, cy, cz};
    for (int d = 0; d < 3; ++d) {
        c.ca[d] = cs[d] / (12. * dx);
        if (upwind) {
            // Advection2, UPWINDADVECTION: -(c*dq)/dx, dq one-sided by the sign of c
            c.mode[d] = cs[d] > 0. ? 0 : 1;
            c.u[d] = -cs[d] / dx;
        } else {
            c.mode[d] = 2;
            c.u[d] = cs[d] / (2. * dx);
        }
    }
    c.s4 = 1. / (12. * dx * dx);
    c.s2 = 1. / (dx * dx);
    c.dx = dx;
    return c;
}

// Kernel arguments.
template <typename T>
struct KArgs {
    T* yout;          // stencil output (with images)
    T* aout;          // pointwise output (accumulator / adjoint accumulator)
    const T* yin;     // stencil input
    const T* pw0;     // pointwise operands (meaning per op)
    const T* pw1;
    const T* pw2;
    long long item_stride, origin, px, plane;
    int ni, nj, nk, pz;
    int tiles_x, zchunk, nzc;
    int zrev;         // TMA kernel: CTAs take items and z-chunks in descending order
    StoreBounds sb_y, sb_a;  // output allocations of yout and aout (bounds-checked builds)
    const int* item_lo;
    int item_base;
    T ca0, ca1, ca2;          // c_d/(12dx)
    T u0, u1, u2;             // RHS2 advection coefficients
    int m0, m1, m2;           // RHS2 difference modes
    double nu;                // diffusivity (when nu_items is null)
    const double* nu_items;   // per-item diffusivity
    double lap_scale;         // 1/(12dx^2) (RHS4) or 1/dx^2 (RHS2)
    T c_y, c_acc;             // stage coefficients
    T sigma;                  // adjoint: mu_s = sigma * (stencil input)
    double* par_acc;          // adjoint: 4 parameter-gradient sums
    double gs_nu, gs_c;       // adjoint: scales of the nu and c sums
    W13<T> w;                 // RHS4 weights for the launch's nu (TMA RK stages)
    int* err;
};

template <int OP>
struct OpTraits {
    static constexpr int npw = (OP == OP_RK_S2 || OP == OP_RK_S3) ? 1   // q
                             : (OP == OP_RK_S4) ? 2                        // acc, q
                             : (OP == OP_ADJ + 0) ? 1      // ADJ4: y4
                             : (OP == OP_ADJ + 1 || OP == OP_ADJ + 2) ? 3   // ADJ3/ADJ2: y, lam, lam_acc
                             : (OP == OP_ADJ + 3) ? 2      // ADJ1: y1, lam_acc
                             : 0;
    static constexpr bool writes_a = (OP == OP_RK_S2 || OP == OP_ADJ + 0 ||
                                      OP == OP_ADJ + 1 || OP == OP_ADJ + 2);
    static constexpr bool adjoint = OP >= OP_ADJ;
};

template <typename T>
__device__ __forceinline__ T diff_mode(int m, T c, T lo, T hi) {
    return m == 0 ? c - lo : (m == 1 ? hi - c : lo - hi);
}

// One cell of one stage.  p0..p2: pointwise operands; oy/oa: outputs;
// g[4]: adjoint parameter partial sums (unscaled).
template <typename T, int OP>
__device__ __forceinline__ void cell_op(const KArgs<T>& a, T nl, const Nb<T>& s, T p0, T p1, T p2, T& oy, T& oa,
                                        double* g, bool live) {
    if constexpr (OP == OP_EULER) {
        const T dqx = diff_mode(a.m0, s.c, s.xm1, s.xp1);
        const T dqy = diff_mode(a.m1, s.c, s.ym1, s.yp1);
        const T dqz = diff_mode(a.m2, s.c, s.zm1, s.zp1);
        const T adv = fmaT(a.u0, dqx, fmaT(a.u1, dqy, a.u2 * dqz));
        T lap;
        if constexpr (sizeof(T) == 4) {
            // FP32: the sum of the neighbours' differences from the centre (exact
            // and small), not the cancelling S1 - 6q (see rhs_w13)
            const T c = s.c;
            lap = ((s.xm1 - c) + (s.xp1 - c)) + ((s.ym1 - c) + (s.yp1 - c)) + ((s.zm1 - c) + (s.zp1 - c));
        } else {
            lap = ((s.xm1 + s.xp1) + (s.ym1 + s.yp1) + (s.zm1 + s.zp1)) - T(6) * s.c;
        }
        const T k = fmaT(nl, lap, adv);
        oy = fmaT(a.c_y, k, s.c);
        (void)p0; (void)p1; (void)p2; (void)oa; (void)g; (void)live;
    } else {
        const T ax = fmaT(T(8), s.xm1 - s.xp1, s.xp2 - s.xm2);
        const T ay = fmaT(T(8), s.ym1 - s.yp1, s.yp2 - s.ym2);
        const T az = fmaT(T(8), s.zm1 - s.zp1, s.zp2 - s.zm2);
        T lap;
        if constexpr (sizeof(T) == 4) {
            // FP32: 16 D1 - D2 with D1, D2 the neighbours' differences from the
            // centre (equal to -90 q + 16 S1 - S2; see rhs_w13)
            const T c = s.c;
            const T D1 = ((s.xm1 - c) + (s.xp1 - c)) + ((s.ym1 - c) + (s.yp1 - c)) + ((s.zm1 - c) + (s.zp1 - c));
            const T D2 = ((s.xm2 - c) + (s.xp2 - c)) + ((s.ym2 - c) + (s.yp2 - c)) + ((s.zm2 - c) + (s.zp2 - c));
            lap = fmaT(T(16), D1, -D2);
        } else {
            const T S1 = (s.xm1 + s.xp1) + (s.ym1 + s.yp1) + (s.zm1 + s.zp1);
            const T S2 = (s.xm2 + s.xp2) + (s.ym2 + s.yp2) + (s.zm2 + s.zp2);
            lap = fmaT(T(-90), s.c, fmaT(T(16), S1, -S2));
        }
        const T adv = fmaT(a.ca0, ax, fmaT(a.ca1, ay, a.ca2 * az));
        if constexpr (!OpTraits<OP>::adjoint) {
            const T k = fmaT(nl, lap, adv);
            if constexpr (OP == OP_RK_S1) {
                oy = fmaT(a.c_y, k, s.c);
            } else if constexpr (OP == OP_RK_S2) {
                oy = fmaT(a.c_y, k, p0);
                oa = fmaT(a.c_acc, k, add_third(s.c, p0, p0));
            } else if constexpr (OP == OP_RK_S3) {
                oy = fmaT(a.c_y, k, p0);
            } else {  // S4
                oy = fmaT(a.c_acc, k, add_third(s.c, p1, p0));
            }
            (void)g; (void)live; (void)p1; (void)oa;
        } else {
            // R^T m = -sum_d c_d D_d m + nu L m (D_d antisymmetric, L symmetric on the periodic grid)
            const T ybar = a.sigma * fmaT(nl, lap, -adv);
            if (live) {
                g[0] += (double)p0 * (double)lap;
                g[1] += (double)p0 * (double)ax;
                g[2] += (double)p0 * (double)ay;
                g[3] += (double)p0 * (double)az;
            }
            if constexpr (OP == OP_ADJ + 0) {         // stencil input is lam
                oy = fmaT(a.c_y, ybar, a.c_acc * s.c);  // mu3 = h ybar4 + h/3 lam
                oa = s.c + ybar;                       // lam_acc = lam + ybar4
            } else if constexpr (OP == OP_ADJ + 1 || OP == OP_ADJ + 2) {
                oy = fmaT(a.c_y, ybar, a.c_acc * p1);  // mu_{s-1} = c_y ybar_s + c_acc lam
                oa = p2 + ybar;
            } else {                                   // ADJ1: final lam_n
                oy = p1 + ybar;
            }
        }
    }
}

// Stores one value and its periodic images.  base = interior origin of the item.
template <typename T>
__device__ __forceinline__ void store_images1(T* base, int x, int y, int z, T v, const KArgs<T>& a) {
    T* row = base + (long long)z * a.plane + (long long)y * a.px;
    const StoreBounds& b = a.sb_y;
    gst1(b, row + x, v);
    if (x < 2) gst1(b, row + x + a.ni, v);
    if (x >= a.ni - 2) gst1(b, row + x - a.ni, v);
    if (y < 2) gst1(b, row + (long long)a.nj * a.px + x, v);
    if (y >= a.nj - 2) gst1(b, row - (long long)a.nj * a.px + x, v);
    if (z < 2) gst1(b, row + (long long)a.nk * a.plane + x, v);
    if (z >= a.nk - 2) gst1(b, row - (long long)a.nk * a.plane + x, v);
}

template <typename T, int N>
__device__ __forceinline__ void put_vec(const StoreBounds& b, T* p, int x, int ni, const Vec<T, N>& v) {
    if (x + N <= ni) {
        gst16<T>(b, p, v);
    } else {
#pragma unroll
        for (int e = 0; e < N; ++e)
            if (x + e < ni) gst1(b, p + e, v.v[e]);
    }
}

// Vector store of cells x..x+N-1 of row (y,z) plus periodic images.
template <typename T, int N>
__device__ __forceinline__ void store_images_vec(T* base, int x, int y, int z, const Vec<T, N>& v, const KArgs<T>& a,
                                                 bool images) {
    T* row = base + (long long)z * a.plane + (long long)y * a.px + x;
    const StoreBounds& b = a.sb_y;
    put_vec<T, N>(b, row, x, a.ni, v);
    if (!images) return;
#pragma unroll
    for (int e = 0; e < N; ++e) {
        const int xe = x + e;
        if (xe < a.ni) {
            if (xe < 2) gst1(b, row + e + a.ni, v.v[e]);
            if (xe >= a.ni - 2) gst1(b, row + e - a.ni, v.v[e]);
        }
    }
    if (y < 2) put_vec<T, N>(b, row + (long long)a.nj * a.px, x, a.ni, v);
    if (y >= a.nj - 2) put_vec<T, N>(b, row - (long long)a.nj * a.px, x, a.ni, v);
    if (z < 2) put_vec<T, N>(b, row + (long long)a.nk * a.plane, x, a.ni, v);
    if (z >= a.nk - 2) put_vec<T, N>(b, row - (long long)a.nk * a.plane, x, a.ni, v);
}

template <typename T>
__device__ __forceinline__ T item_nl(const KArgs<T>& a, int b) {
    const double nu = a.nu_items ? a.nu_items[b] : a.nu;
    return (T)(nu * a.lap_scale);
}

// Reduces the four adjoint parameter sums over the CTA (warp shuffles, then
// shared memory) and adds them to par_acc with one atomic per CTA and sum.
// Every thread of the CTA must call it.
__device__ __forceinline__ void reduce_par(double* g, double* par_acc, double gs_nu, double gs_c) {
    __shared__ double red[32][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
        for (int o = 16; o > 0; o >>= 1) g[i] += __shfl_xor_sync(0xffffffffu, g[i], o);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nwarp = (blockDim.x * blockDim.y + 31) / 32;
    if ((tid & 31) == 0)
#pragma unroll
        for (int i = 0; i < 4; ++i) red[tid >> 5][i] = g[i];
    __syncthreads();
    if (tid < 4) {
        double v = 0.;
        for (int w = 0; w < nwarp; ++w) v += red[w][tid];
        atomicAdd(par_acc + tid, (tid == 0 ? gs_nu : gs_c) * v);
    }
}

// ---------------------------------------------------------------------------
// Direct-load stage kernel: block (32, TYD), one thread per (x, y) column,
// marching zchunk planes; grid (ceil(ni/32), ceil(nj/TYD), nzc * items).
template <typename T, int OP, int TYD>
__global__ void __launch_bounds__(32 * TYD) k_stage_direct(const KArgs<T> a) {
    const int zc = blockIdx.z % a.nzc;
    const int b = blockIdx.z / a.nzc;
    if (a.item_lo && b + a.item_base < *a.item_lo) return;
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * TYD + threadIdx.y;
    double g[4] = {0., 0., 0., 0.};
    const bool live = x < a.ni && y < a.nj;
    if (live) {
        const long long ob = (long long)b * a.item_stride + a.origin;
        const long long col = ob + (long long)y * a.px + x;
        const T* S = a.yin + col;
        const int z0 = zc * a.zchunk;
        const int z1 = min(z0 + a.zchunk, a.nk);
        const T nl = item_nl(a, b);
        const long long pl = a.plane;
        T zm2 = __ldg(S + (z0 - 2) * pl), zm1 = __ldg(S + (z0 - 1) * pl);
        T zc0 = __ldg(S + z0 * pl), zp1 = __ldg(S + (z0 + 1) * pl);
        for (int z = z0; z < z1; ++z) {
            const T zp2 = __ldg(S + (z + 2) * pl);
            const T* P = S + z * pl;
            Nb<T> s;
            s.c = zc0; s.zm1 = zm1; s.zp1 = zp1; s.zm2 = zm2; s.zp2 = zp2;
            s.xm1 = __ldg(P - 1); s.xp1 = __ldg(P + 1); s.xm2 = __ldg(P - 2); s.xp2 = __ldg(P + 2);
            s.ym1 = __ldg(P - a.px); s.yp1 = __ldg(P + a.px);
            s.ym2 = __ldg(P - 2 * a.px); s.yp2 = __ldg(P + 2 * a.px);
            const long long off = col + z * pl;
            T p0 = 0, p1 = 0, p2 = 0;
            constexpr int NPW = OpTraits<OP>::npw;
            if constexpr (NPW > 0) p0 = a.pw0[off];
            if constexpr (NPW > 1) p1 = a.pw1[off];
            if constexpr (NPW > 2) p2 = a.pw2[off];
            T oy = 0, oa = 0;
            cell_op<T, OP>(a, nl, s, p0, p1, p2, oy, oa, g, true);
            store_images1<T>(a.yout + ob, x, y, z, oy, a);
            if constexpr (OpTraits<OP>::writes_a) gst1(a.sb_a, a.aout + off, oa);
            zm2 = zm1; zm1 = zc0; zc0 = zp1; zp1 = zp2;
        }
    }
    if constexpr (OpTraits<OP>::adjoint) reduce_par(g, a.par_acc, a.gs_nu, a.gs_c);
}

// ---------------------------------------------------------------------------
// TMA stage kernel.  Block = 32*TY threads (warp w owns tile row w), grid
// (tiles_x*tiles_y, nzc, items), taken in descending item / z-chunk order when
// zrev is set.  Shared memory: NS stencil-input slots of (TX+2LX) x (TY+4)
// elements and NP pointwise slots of npw x TX x TY elements, followed by NS+NP
// mbarriers.  Ring bookkeeping uses running slot indices and phase bits instead
// of divisions; lanes whose cells are two or more cells away from every y face
// store one 16-byte vector (plus the x images of cells next to an x face)
// except on the four planes next to the z faces.


template <typename T, int OP, int TY, int NS, int NP>
__global__ void __launch_bounds__(32 * TY)
    k_stage_tma(const __grid_constant__ CUtensorMap tm_s, const __grid_constant__ CUtensorMap tm_p0,
                const __grid_constant__ CUtensorMap tm_p1, const __grid_constant__ CUtensorMap tm_p2,
                const KArgs<T> a) {
    constexpr int VX = V16<T>::N;
    constexpr int TX = 32 * VX;
    constexpr int LX = VX;
    constexpr int W = TX + 2 * LX;
    constexpr int H = TY + 4;
    constexpr int YT = W * H;
    constexpr int PT = TX * TY;
    constexpr int NPA = OpTraits<OP>::npw;
    constexpr uint32_t YBYTES = YT * sizeof(T);
    constexpr uint32_t PBYTES = NPA * PT * sizeof(T);
    constexpr bool RK = OP <= OP_RK_S4;
    static_assert((YT * sizeof(T)) % 128 == 0 && (PT * sizeof(T)) % 128 == 0, "slot alignment");
    static_assert(NS >= 4, "ring depth");
    using V = Vec<T, VX>;

    extern __shared__ unsigned char smem_raw[];
    unsigned char* sbase =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    T* ys = reinterpret_cast<T*>(sbase);
    T* ps = ys + NS * YT;
    uint64_t* bar = reinterpret_cast<uint64_t*>(ps + NP * NPA * PT);

    // zrev: items and z-chunks in descending order, so that a launch starts on
    // the planes the previous launch (ascending) touched last, still in L2
    const int b = a.zrev ? (int)(gridDim.z - 1 - blockIdx.z) : (int)blockIdx.z;
    const int x0 = (blockIdx.x % a.tiles_x) * TX;
    const int y0 = (blockIdx.x / a.tiles_x) * TY;
    const int z0 = (a.zrev ? (int)(gridDim.y - 1 - blockIdx.y) : (int)blockIdx.y) * a.zchunk;
    const int z1 = min(z0 + a.zchunk, a.nk);
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int zb = b * a.pz + 2;  // padded plane index of interior z = 0 of item b
    const int ylast = z1 + 1;     // last stencil plane needed
    const bool leader = threadIdx.x == 0;

    pdl_trigger();  // the next kernel's CTAs may start as this grid's CTAs retire
    if (leader) {
        prefetch_tensormap(&tm_s);
#pragma unroll
        for (int i = 0; i < NS + NP; ++i) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    __syncthreads();
    pdl_wait();     // fields written by the previous kernel are read from here on
    if (a.item_lo && b + a.item_base < *a.item_lo) return;  // the same for all threads of the CTA

    // tile t (interior plane, z0-2 <= t <= z1+1) -> slot (t - z0 + 2) % NS
    auto issue_y = [&](int t) {
        const int s = (t - z0 + 2) % NS;
        mbar_arrive_expect_tx(&bar[s], YBYTES);
        tma_load_3d(ys + s * YT, &tm_s, x0, y0, zb + t, &bar[s]);
    };
    auto issue_p = [&](int t) {
        const int s = (t - z0) % NP;
        mbar_arrive_expect_tx(&bar[NS + s], PBYTES);
        T* d = ps + s * NPA * PT;
        if constexpr (NPA > 0) tma_load_3d(d, &tm_p0, x0 + LX, y0 + 2, zb + t, &bar[NS + s]);
        if constexpr (NPA > 1) tma_load_3d(d + PT, &tm_p1, x0 + LX, y0 + 2, zb + t, &bar[NS + s]);
        if constexpr (NPA > 2) tma_load_3d(d + 2 * PT, &tm_p2, x0 + LX, y0 + 2, zb + t, &bar[NS + s]);
    };
    int y_hi = z0 - 3, p_hi = z0 - 1;  // highest tiles issued (leader only)
    if (leader) {
        for (int t = z0 - 2; t < z0 - 2 + NS && t <= ylast; ++t) { issue_y(t); y_hi = t; }
        if constexpr (NPA > 0)
            for (int t = z0; t < z0 + NP && t < z1; ++t) { issue_p(t); p_hi = t; }
    }

    // running ring positions: slot and phase of stencil tile z+2 (the next
    // centre), of tile z (x/y neighbours) and of pointwise tile z.  Shared
    // memory is read by 32-bit address with constant offsets, and the z-window
    // of centres lives in five registers renamed statically (the plane loop is
    // unrolled by five), so that no plane moves values between registers.
    constexpr int ES = (int)sizeof(T);
    const uint32_t ys_base = smem_u32(ys);
    const uint32_t ps_base = smem_u32(ps);
    const uint32_t own8 = (uint32_t)(((w + 2) * W + LX + lane * VX) * ES);  // this thread's centre
    const uint32_t pw8 = (uint32_t)((w * TX + lane * VX) * ES);
    int s_c = 0;
    uint32_t ph_c = 0;
    bool bad = false;
    auto next_center = [&]() -> V {
        if (!mbar_wait_bounded(&bar[s_c], ph_c)) bad = true;
        const V v = lds16<T>(ys_base + (uint32_t)s_c * YBYTES + own8);
        if (++s_c == NS) { s_c = 0; ph_c ^= 1u; }
        return v;
    };
    auto drain = [&](int y_done, int p_done) {
        if (!leader) return;
        for (int t = y_done + 1; t <= y_hi; ++t) {
            const int u = t - z0 + 2;
            (void)mbar_wait_bounded(&bar[u % NS], (uint32_t)((u / NS) & 1));
        }
        for (int t = p_done + 1; t <= p_hi; ++t)
            (void)mbar_wait_bounded(&bar[NS + (t - z0) % NP], (uint32_t)(((t - z0) / NP) & 1));
    };

    V cw[5];  // centres of planes z-2 .. z+2 at cw[(z - z0 + 0..4) % 5]
    cw[0] = next_center();
    cw[1] = next_center();
    cw[2] = next_center();
    cw[3] = next_center();
    if (__syncthreads_or(bad)) {
        if (leader) atomicExch(a.err, DEV_WAIT_TIMEOUT);
        drain(z0 + 1, z0 - 1);
        return;
    }
    if (leader) {
        fence_proxy_async_smem();
        for (int t = z0 - 2 + NS; t <= z0 - 1 + NS && t <= ylast; ++t) { issue_y(t); y_hi = t; }
    }

    const T nl = item_nl(a, b);
    const int y = y0 + w;
    const int x = x0 + lane * VX;
    const bool live = y < a.nj && x < a.ni;
    const bool full_vec = x + VX <= a.ni;
    // rows whose cells have no y image and vectors whose cells all lie inside
    // take the plain store (plus x images where a cell is within 2 of an x face)
    const bool x_img = x < 2 || x + VX > a.ni - 2;
    const bool y_img = y < 2 || y >= a.nj - 2 || !full_vec;
    const long long ob = (long long)b * a.item_stride + a.origin;
    T* yrow_out = a.yout + ob + (long long)z0 * a.plane + (long long)y * a.px + x;
    T* arow_out = nullptr;
    if constexpr (OpTraits<OP>::writes_a) arow_out = a.aout + ob + (long long)z0 * a.plane + (long long)y * a.px + x;
    double g[4] = {0., 0., 0., 0.};
    int s_n = 2 % NS;  // slot of tile z (neighbours)
    int s_p = 0;
    uint32_t ph_p = 0;

    // one plane; K = (z - z0) % 5 names the registers of the z-window
    auto iterate = [&](auto kc, int z) -> bool {
        constexpr int K = decltype(kc)::value;
        cw[(K + 4) % 5] = next_center();
        const V& cm2 = cw[K];
        const V& cm1 = cw[(K + 1) % 5];
        const V& c0 = cw[(K + 2) % 5];
        const V& cp1 = cw[(K + 3) % 5];
        const V& cp2 = cw[(K + 4) % 5];
        [[maybe_unused]] V p0v, p1v, p2v;
        if constexpr (NPA > 0) {
            if (!mbar_wait_bounded(&bar[NS + s_p], ph_p)) bad = true;
            const uint32_t P = ps_base + (uint32_t)s_p * (uint32_t)(NPA * PT * ES) + pw8;
            p0v = lds16<T>(P);
            if constexpr (NPA > 1) p1v = lds16<T, PT * ES>(P);
            if constexpr (NPA > 2) p2v = lds16<T, 2 * PT * ES>(P);
            if (++s_p == NP) { s_p = 0; ph_p ^= 1u; }
        }
        const uint32_t C = ys_base + (uint32_t)s_n * YBYTES + own8;
        if (++s_n == NS) s_n = 0;
        T row[3 * VX];
        {
            const V r0 = lds16<T, -LX * ES>(C), r2 = lds16<T, VX * ES>(C);  // c0: this plane's centre
#pragma unroll
            for (int e = 0; e < VX; ++e) { row[e] = r0.v[e]; row[VX + e] = c0.v[e]; row[2 * VX + e] = r2.v[e]; }
        }
        const V ym2 = lds16<T, -2 * W * ES>(C), ym1 = lds16<T, -W * ES>(C);
        const V yp1 = lds16<T, W * ES>(C), yp2 = lds16<T, 2 * W * ES>(C);
        V oy, oa;
#pragma unroll
        for (int e = 0; e < VX; ++e) {
            Nb<T> s;
            s.c = row[LX + e];
            s.xm1 = row[LX + e - 1]; s.xp1 = row[LX + e + 1];
            s.xm2 = row[LX + e - 2]; s.xp2 = row[LX + e + 2];
            s.ym1 = ym1.v[e]; s.yp1 = yp1.v[e]; s.ym2 = ym2.v[e]; s.yp2 = yp2.v[e];
            s.zm1 = cm1.v[e]; s.zp1 = cp1.v[e]; s.zm2 = cm2.v[e]; s.zp2 = cp2.v[e];
            [[maybe_unused]] T q0 = 0, q1 = 0, q2 = 0;
            if constexpr (NPA > 0) q0 = p0v.v[e];
            if constexpr (NPA > 1) q1 = p1v.v[e];
            if constexpr (NPA > 2) q2 = p2v.v[e];
            T vy = 0, va = 0;
            if constexpr (RK) {
                const T k = rhs_w13(a.w, s);
                if constexpr (OP == OP_RK_S1) {
                    vy = fmaT(a.c_y, k, s.c);
                } else if constexpr (OP == OP_RK_S2) {
                    vy = fmaT(a.c_y, k, q0);
                    va = fmaT(a.c_acc, k, add_third(s.c, q0, q0));
                } else if constexpr (OP == OP_RK_S3) {
                    vy = fmaT(a.c_y, k, q0);
                } else {
                    vy = fmaT(a.c_acc, k, add_third(s.c, q1, q0));
                }
            } else {
                cell_op<T, OP>(a, nl, s, q0, q1, q2, vy, va, g, live && x + e < a.ni);
            }
            oy.v[e] = vy;
            oa.v[e] = va;
        }
        if (live) {
            if (!y_img && z >= 2 && z < a.nk - 2) {
                gst16<T>(a.sb_y, yrow_out, oy);
                if (x_img) {
#pragma unroll
                    for (int e = 0; e < VX; ++e) {
                        if (x + e < 2) gst1(a.sb_y, yrow_out + e + a.ni, oy.v[e]);
                        if (x + e >= a.ni - 2) gst1(a.sb_y, yrow_out + e - a.ni, oy.v[e]);
                    }
                }
            } else {
                store_images_vec<T, VX>(a.yout + ob, x, y, z, oy, a, true);
            }
            if constexpr (OpTraits<OP>::writes_a) {
                if (full_vec) gst16<T>(a.sb_a, arow_out, oa);
                else put_vec<T, VX>(a.sb_a, arow_out, x, a.ni, oa);
            }
        }
        yrow_out += a.plane;
        if constexpr (OpTraits<OP>::writes_a) arow_out += a.plane;
        if (__syncthreads_or(bad)) {
            if (leader) atomicExch(a.err, DEV_WAIT_TIMEOUT);
            drain(z + 2, z);
            return false;
        }
        if (leader) {
            fence_proxy_async_smem();
            if (z + NS <= ylast) { issue_y(z + NS); y_hi = z + NS; }
            if constexpr (NPA > 0)
                if (z + NP < z1) { issue_p(z + NP); p_hi = z + NP; }
        }
        return true;
    };
    for (int zz = z0; zz < z1; zz += 5) {
        if (!iterate(std::integral_constant<int, 0>{}, zz)) return;
        if (zz + 1 < z1 && !iterate(std::integral_constant<int, 1>{}, zz + 1)) return;
        if (zz + 2 < z1 && !iterate(std::integral_constant<int, 2>{}, zz + 2)) return;
        if (zz + 3 < z1 && !iterate(std::integral_constant<int, 3>{}, zz + 3)) return;
        if (zz + 4 < z1 && !iterate(std::integral_constant<int, 4>{}, zz + 4)) return;
    }
    if constexpr (OpTraits<OP>::adjoint) reduce_par(g, a.par_acc, a.gs_nu, a.gs_c);
}

// ---------------------------------------------------------------------------
// Host side of the stage launches.

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

}  // namespace

bool make_tmap(CUtensorMap* tm, const Geo& g, const void* base, int items, int bw, int bh) {
    auto enc = encode_fn();
    if (!enc || !base) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)(g.pz * items)};
    const cuuint64_t strides[2] = {(cuuint64_t)(g.px * g.es), (cuuint64_t)(g.plane * g.es)};
    const cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt = g.es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    CUresult r = enc(tm, dt, 3, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

namespace {

template <typename T>
KArgs<T> make_args(const Geo& g, const StageLaunch& L, const Shape& t, int* err) {
    KArgs<T> a{};
    a.yout = (T*)L.yout;
    a.yin = (const T*)L.yin;
    a.item_stride = g.total; a.origin = g.origin; a.px = g.px; a.plane = g.plane;
    a.ni = g.ni; a.nj = g.nj; a.nk = g.nk; a.pz = (int)g.pz;
    a.zchunk = t.zchunk;
    a.nzc = (g.nk + t.zchunk - 1) / t.zchunk;
    a.item_lo = L.item_lo;
    a.item_base = L.item_base;
    const Coef& c = L.coef;
    a.ca0 = (T)c.ca[0]; a.ca1 = (T)c.ca[1]; a.ca2 = (T)c.ca[2];
    a.u0 = (T)c.u[0]; a.u1 = (T)c.u[1]; a.u2 = (T)c.u[2];
    a.m0 = c.mode[0]; a.m1 = c.mode[1]; a.m2 = c.mode[2];
    a.nu = L.nu; a.nu_items = L.nu_items;
    a.lap_scale = (L.op == OP_EULER) ? c.s2 : c.s4;
    a.c_y = (T)L.c_y; a.c_acc = (T)L.c_acc;
    a.err = err;
    // RK4 stages alternate the sweep direction (S1, S3 descending; S2, S4 ascending),
    // so that each stage starts on the planes the previous one touched last
    a.zrev = (L.op == OP_RK_S1 || L.op == OP_RK_S3) ? 1 : 0;
    a.sb_y = out_bounds(L.yout, g, L.items);
    fill_w13<T>(a.w, c, L.nu);  // RHS4 as per-offset weights (TMA RK stages; one nu per launch)
    switch (L.op) {
        case OP_RK_S1: break;
        case OP_RK_S2: a.aout = (T*)L.acc; a.pw0 = (const T*)L.q; break;
        case OP_RK_S3: a.pw0 = (const T*)L.q; break;
        case OP_RK_S4: a.pw0 = (const T*)L.acc; a.pw1 = (const T*)L.q; break;
        case OP_EULER: break;
        case OP_ADJ + 0: a.aout = (T*)L.lam_acc; a.pw0 = (const T*)L.ypt; break;
        case OP_ADJ + 1:
        case OP_ADJ + 2:
            a.aout = (T*)L.lam_acc; a.pw0 = (const T*)L.ypt; a.pw1 = (const T*)L.lam; a.pw2 = (const T*)L.lam_acc;
            break;
        case OP_ADJ + 3: a.pw0 = (const T*)L.ypt; a.pw1 = (const T*)L.lam_acc; break;
        default: break;
    }
    a.sb_a = out_bounds(a.aout, g, L.items);
    if (L.op >= OP_ADJ) {
        a.c_y = (T)L.c_ybar;
        a.c_acc = (T)L.c_lam;
        a.sigma = (T)L.sigma;
        a.par_acc = L.par_acc;
        a.gs_nu = L.dnu * L.sigma * c.s4;   // nu-sum * dnu * sigma / (12 dx^2)
        a.gs_c = -L.sigma / (12. * c.dx);   // c-sums: -sigma * D_d m = -sigma (8d1-d2)/(12dx)
    }
    return a;
}

template <typename T, int OP>
cudaError_t launch_direct_T(const Geo& g, const KArgs<T>& a, const Shape& t, int items, cudaStream_t s) {
    const int tyd = t.ty;
    dim3 grid((g.ni + 31) / 32, (g.nj + tyd - 1) / tyd, a.nzc * items);
    if (grid.z > 65535u) return cudaErrorInvalidConfiguration;
    switch (tyd) {
        case 4: k_stage_direct<T, OP, 4><<<grid, dim3(32, 4), 0, s>>>(a); break;
        case 8: k_stage_direct<T, OP, 8><<<grid, dim3(32, 8), 0, s>>>(a); break;
        case 16: k_stage_direct<T, OP, 16><<<grid, dim3(32, 16), 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename T, int OP, int TY, int NS, int NP>
size_t tma_smem_bytes() {
    constexpr int VX = V16<T>::N, TX = 32 * VX, W = TX + 2 * VX, H = TY + 4;
    constexpr int NPA = OpTraits<OP>::npw;
    return 128 + (size_t)NS * W * H * sizeof(T) + (size_t)NP * NPA * TX * TY * sizeof(T) + (NS + NP) * 8;
}

template <typename T, int OP, int TY, int NS, int NP>
cudaError_t launch_tma_T(const Geo& g, const StageLaunch& L, KArgs<T> a, const Shape& t, cudaStream_t s) {
    constexpr int VX = V16<T>::N, TX = 32 * VX, W = TX + 2 * VX, H = TY + 4;
    CUtensorMap ts{}, t0{}, t1{}, t2{};
    if (!make_tmap(&ts, g, L.yin, L.items, W, H)) return cudaErrorInvalidValue;
    const void* pw[3] = {a.pw0, a.pw1, a.pw2};
    CUtensorMap* tp[3] = {&t0, &t1, &t2};
    for (int i = 0; i < OpTraits<OP>::npw; ++i)
        if (!make_tmap(tp[i], g, pw[i], L.items, TX, TY)) return cudaErrorInvalidValue;
    a.tiles_x = (g.ni + TX - 1) / TX;
    const int tiles_y = (g.nj + TY - 1) / TY;
    dim3 grid(a.tiles_x * tiles_y, a.nzc, L.items);
    if (grid.y > 65535u || grid.z > 65535u) return cudaErrorInvalidConfiguration;
    const size_t smem = tma_smem_bytes<T, OP, TY, NS, NP>();
    return launch_pdl(k_stage_tma<T, OP, TY, NS, NP>, grid, dim3(32 * TY), smem, s, ts, t0, t1, t2, a);
}

template <typename T, int OP, int TY, int NS, int NP>
cudaError_t set_attr_T() {
    return cudaFuncSetAttribute(k_stage_tma<T, OP, TY, NS, NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)tma_smem_bytes<T, OP, TY, NS, NP>());
}

template <typename T, int OP>
cudaError_t set_attr_op() {
    cudaError_t e = set_attr_T<T, OP, 4, 5, 3>();
    if (e == cudaSuccess) e = set_attr_T<T, OP, 8, 5, 3>();
    if (e == cudaSuccess) e = set_attr_T<T, OP, 16, 4, 2>();
    return e;
}


// Ring depths per tile height: NS stencil slots (prefetch NS-3 planes ahead),
// NP pointwise slots (prefetch NP-1 planes ahead).
template <typename T, int OP>
cudaError_t launch_tma_op(const Geo& g, const StageLaunch& L, const KArgs<T>& a, const Shape& t, cudaStream_t s) {
    switch (t.ty) {
        case 4: return launch_tma_T<T, OP, 4, 5, 3>(g, L, a, t, s);
        case 8: return launch_tma_T<T, OP, 8, 5, 3>(g, L, a, t, s);
        case 16: return launch_tma_T<T, OP, 16, 4, 2>(g, L, a, t, s);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t launch_T(const Geo& g, const StageLaunch& L, const Shape& t, cudaStream_t s, int* err) {
    KArgs<T> a = make_args<T>(g, L, t, err);
    // one diffusivity per item (batched slices with nufreq != 0): direct kernel
    const bool tma = t.tma && !L.nu_items;
#define SP_OPCASE(OPV)                                                              \
    case OPV:                                                                       \
        return tma ? launch_tma_op<T, OPV>(g, L, a, t, s)                           \
                   : launch_direct_T<T, OPV>(g, a, t, L.items, s);
    switch (L.op) {
        SP_OPCASE(OP_RK_S1)
        SP_OPCASE(OP_RK_S2)
        SP_OPCASE(OP_RK_S3)
        SP_OPCASE(OP_RK_S4)
        SP_OPCASE(OP_EULER)
        default: break;
    }
    if constexpr (sizeof(T) == 8) {
        switch (L.op) {
            SP_OPCASE(OP_ADJ + 0)
            SP_OPCASE(OP_ADJ + 1)
            SP_OPCASE(OP_ADJ + 2)
            SP_OPCASE(OP_ADJ + 3)
            default: break;
        }
    }
#undef SP_OPCASE
    return cudaErrorInvalidValue;
}

}  // namespace

unsigned long long take_store_violations_stages() {
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_store_violations, sizeof v) != cudaSuccess) return 0;
    const unsigned int zero = 0;
    cudaMemcpyToSymbol(g_store_violations, &zero, sizeof zero);
    return v;
}

cudaError_t prepare_kernels() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    chk(set_attr_op<double, OP_RK_S1>()); chk(set_attr_op<double, OP_RK_S2>());
    chk(set_attr_op<double, OP_RK_S3>()); chk(set_attr_op<double, OP_RK_S4>());
    chk(set_attr_op<double, OP_EULER>());
    chk(set_attr_op<double, OP_ADJ + 0>()); chk(set_attr_op<double, OP_ADJ + 1>());
    chk(set_attr_op<double, OP_ADJ + 2>()); chk(set_attr_op<double, OP_ADJ + 3>());
    chk(set_attr_op<float, OP_RK_S1>()); chk(set_attr_op<float, OP_RK_S2>());
    chk(set_attr_op<float, OP_RK_S3>()); chk(set_attr_op<float, OP_RK_S4>());
    chk(set_attr_op<float, OP_EULER>());
    chk(prepare_pairs());
    chk(prepare_cluster());
    return e;
}

namespace {
// Self-test of the bounded waits: one CTA waits on an mbarrier that nothing
// arrives on, gives up after limit_ns like every pipeline wait, records the
// timeout in the device error word and returns.
__global__ void k_wait_selftest(int* err, unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, limit_ns);
    if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicExch(err, DEV_WAIT_TIMEOUT);
}
}  // namespace

cudaError_t launch_wait_selftest(int* err, unsigned long long limit_ns, cudaStream_t s) {
    add_launches(1);
    k_wait_selftest<<<1, 64, 0, s>>>(err, limit_ns);
    return cudaGetLastError();
}

cudaError_t launch_stage(const Geo& g, const StageLaunch& L, const Tune& t, cudaStream_t s, int* err) {
    add_launches(1);
    if (L.op < 0 || L.op >= kNumOps) return cudaErrorInvalidValue;
    const Shape& sh = t.op[L.op];
    if (L.prec == 0) return launch_T<double>(g, L, sh, s, err);
    return launch_T<float>(g, L, sh, s, err);
}

// ---------------------------------------------------------------------------
// Pointwise kernels.

// Periodicity: the three passes of Periodicity.cu:12-144 (I, then J over all I,
// then K over all I and J), here for `items` fields.
template <typename T>
__global__ void k_period_i(T* f, Geo g, int items) {
    const long long n = (long long)g.nj * g.nk * items;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(t % g.nj);
        const int k = (int)((t / g.nj) % g.nk);
        const int b = (int)(t / ((long long)g.nj * g.nk));
        T* row = f + b * g.total + g.origin + (long long)k * g.plane + (long long)j * g.px;
        row[-2] = row[g.ni - 2];
        row[-1] = row[g.ni - 1];
        row[g.ni] = row[0];
        row[g.ni + 1] = row[1];
    }
}
template <typename T>
__global__ void k_period_j(T* f, Geo g, int items) {
    const int wi = g.ni + 4;
    const long long n = (long long)wi * g.nk * items;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % wi) - 2;
        const int k = (int)((t / wi) % g.nk);
        const int b = (int)(t / ((long long)wi * g.nk));
        T* c = f + b * g.total + g.origin + (long long)k * g.plane + i;
        c[-2 * g.px] = c[(long long)(g.nj - 2) * g.px];
        c[-1 * g.px] = c[(long long)(g.nj - 1) * g.px];
        c[(long long)g.nj * g.px] = c[0];
        c[(long long)(g.nj + 1) * g.px] = c[g.px];
    }
}
template <typename T>
__global__ void k_period_k(T* f, Geo g, int items) {
    const int wi = g.ni + 4, wj = g.nj + 4;
    const long long n = (long long)wi * wj * items;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % wi) - 2;
        const int j = (int)((t / wi) % wj) - 2;
        const int b = (int)(t / ((long long)wi * wj));
        T* c = f + b * g.total + g.origin + (long long)j * g.px + i;
        c[-2 * g.plane] = c[(long long)(g.nk - 2) * g.plane];
        c[-1 * g.plane] = c[(long long)(g.nk - 1) * g.plane];
        c[(long long)g.nk * g.plane] = c[0];
        c[(long long)(g.nk + 1) * g.plane] = c[g.plane];
    }
}

static unsigned grid_for(long long n, int block) {
    long long b = (n + block - 1) / block;
    if (b > 148LL * 64) b = 148LL * 64;
    if (b < 1) b = 1;
    return (unsigned)b;
}

cudaError_t launch_periodicity(const Geo& g, void* field, int items, cudaStream_t s) {
    add_launches(3);
    if (g.es == 8) {
        k_period_i<double><<<grid_for((long long)g.nj * g.nk * items, 256), 256, 0, s>>>((double*)field, g, items);
        k_period_j<double><<<grid_for((long long)(g.ni + 4) * g.nk * items, 256), 256, 0, s>>>((double*)field, g, items);
        k_period_k<double><<<grid_for((long long)(g.ni + 4) * (g.nj + 4) * items, 256), 256, 0, s>>>((double*)field, g, items);
    } else {
        k_period_i<float><<<grid_for((long long)g.nj * g.nk * items, 256), 256, 0, s>>>((float*)field, g, items);
        k_period_j<float><<<grid_for((long long)(g.ni + 4) * g.nk * items, 256), 256, 0, s>>>((float*)field, g, items);
        k_period_k<float><<<grid_for((long long)(g.ni + 4) * (g.nj + 4) * items, 256), 256, 0, s>>>((float*)field, g, items);
    }
    return cudaGetLastError();
}

// Writes v at interior (x,y,z) of a field (origin-relative base) plus images.
template <typename T>
__device__ __forceinline__ void put_img(T* base, const Geo& g, int x, int y, int z, T v) {
    T* row = base + (long long)z * g.plane + (long long)y * g.px;
    row[x] = v;
    if (x < 2) row[x + g.ni] = v;
    if (x >= g.ni - 2) row[x - g.ni] = v;
    if (y < 2) row[(long long)g.nj * g.px + x] = v;
    if (y >= g.nj - 2) row[-(long long)g.nj * g.px + x] = v;
    if (z < 2) row[(long long)g.nk * g.plane + x] = v;
    if (z >= g.nk - 2) row[-(long long)g.nk * g.plane + x] = v;
}

template <typename TD, typename TF>
__global__ void k_dense_to_field(const TD* d, TF* f, Geo g) {
    const long long n = (long long)g.ni * g.nj * g.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % g.ni);
        const int y = (int)((t / g.ni) % g.nj);
        const int z = (int)(t / ((long long)g.ni * g.nj));
        put_img<TF>(f + g.origin, g, x, y, z, (TF)d[t]);
    }
}

template <typename TF, typename TD>
__global__ void k_field_to_dense(const TF* f, TD* d, Geo g) {
    const long long n = (long long)g.ni * g.nj * g.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % g.ni);
        const int y = (int)((t / g.ni) % g.nj);
        const int z = (int)(t / ((long long)g.ni * g.nj));
        d[t] = (TD)f[g.origin + (long long)z * g.plane + (long long)y * g.px + x];
    }
}

cudaError_t launch_dense_to_field(const Geo& g, const void* dense, int dense_prec, void* field, cudaStream_t s) {
    add_launches(1);
    const unsigned gr = grid_for((long long)g.ni * g.nj * g.nk, 256);
    if (g.es == 8) {
        if (dense_prec == 0) k_dense_to_field<double, double><<<gr, 256, 0, s>>>((const double*)dense, (double*)field, g);
        else k_dense_to_field<float, double><<<gr, 256, 0, s>>>((const float*)dense, (double*)field, g);
    } else {
        if (dense_prec == 0) k_dense_to_field<double, float><<<gr, 256, 0, s>>>((const double*)dense, (float*)field, g);
        else k_dense_to_field<float, float><<<gr, 256, 0, s>>>((const float*)dense, (float*)field, g);
    }
    return cudaGetLastError();
}

cudaError_t launch_field_to_dense(const Geo& g, const void* field, void* dense, int dense_prec, cudaStream_t s) {
    add_launches(1);
    const unsigned gr = grid_for((long long)g.ni * g.nj * g.nk, 256);
    if (g.es == 8) {
        if (dense_prec == 0) k_field_to_dense<double, double><<<gr, 256, 0, s>>>((const double*)field, (double*)dense, g);
        else k_field_to_dense<double, float><<<gr, 256, 0, s>>>((const double*)field, (float*)dense, g);
    } else {
        if (dense_prec == 0) k_field_to_dense<float, double><<<gr, 256, 0, s>>>((const float*)field, (double*)dense, g);
        else k_field_to_dense<float, float><<<gr, 256, 0, s>>>((const float*)field, (float*)dense, g);
    }
    return cudaGetLastError();
}

template <typename TD, typename TS>
__global__ void k_convert(TD* dst, Geo gd, const TS* src, Geo gs, const int* item_lo, int item) {
    if (item_lo && item < *item_lo) return;
    const long long n = (long long)gd.ni * gd.nj * gd.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % gd.ni);
        const int y = (int)((t / gd.ni) % gd.nj);
        const int z = (int)(t / ((long long)gd.ni * gd.nj));
        const TS v = src[gs.origin + (long long)z * gs.plane + (long long)y * gs.px + x];
        put_img<TD>(dst + gd.origin, gd, x, y, z, (TD)v);
    }
}

cudaError_t launch_convert(const Geo& gd, void* dst, const Geo& gs, const void* src, cudaStream_t s,
                           const int* item_lo, int item) {
    add_launches(1);
    const unsigned gr = grid_for((long long)gd.ni * gd.nj * gd.nk, 256);
    if (gd.es == 8 && gs.es == 8)
        k_convert<double, double><<<gr, 256, 0, s>>>((double*)dst, gd, (const double*)src, gs, item_lo, item);
    else if (gd.es == 8)
        k_convert<double, float><<<gr, 256, 0, s>>>((double*)dst, gd, (const float*)src, gs, item_lo, item);
    else if (gs.es == 8)
        k_convert<float, double><<<gr, 256, 0, s>>>((float*)dst, gd, (const double*)src, gs, item_lo, item);
    else
        k_convert<float, float><<<gr, 256, 0, s>>>((float*)dst, gd, (const float*)src, gs, item_lo, item);
    return cudaGetLastError();
}

// Parareal correction (UpdateStage, Parareal.h:19-35) fused with the swap of
// the coarse states (Parareal.h:164) and the defect norms.
template <typename TC>
__global__ void k_update(const TC* gnew, const double* f, TC* gold, double* u, double* def, Geo g, Geo gc,
                         const int* item_lo, int item) {
    if (item_lo && item < *item_lo) return;
    const long long n = (long long)g.ni * g.nj * g.nk;
    double s_d = 0., s_q = 0.;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % g.ni);
        const int y = (int)((t / g.ni) % g.nj);
        const int z = (int)(t / ((long long)g.ni * g.nj));
        const long long o = g.origin + (long long)z * g.plane + (long long)y * g.px + x;
        const long long oc = gc.origin + (long long)z * gc.plane + (long long)y * gc.px + x;
        const TC gn = gnew[oc];
        const double q = ((double)gn + f[o]) - (double)gold[oc];
        const double d = q - u[o];
        s_d += d * d;
        s_q += q * q;
        gold[oc] = gn;
        put_img<double>(u + g.origin, g, x, y, z, q);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s_d += __shfl_xor_sync(0xffffffffu, s_d, o);
        s_q += __shfl_xor_sync(0xffffffffu, s_q, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(def, s_d);
        atomicAdd(def + 1, s_q);
    }
}

cudaError_t launch_update(const Geo& g64, const Geo& gc, const void* gnew, const double* f, void* gold,
                          double* u_next, double* def, const int* item_lo, int item, cudaStream_t s) {
    add_launches(1);
    const unsigned gr = grid_for((long long)g64.ni * g64.nj * g64.nk, 256);
    if (gc.es == 8)
        k_update<double><<<gr, 256, 0, s>>>((const double*)gnew, f, (double*)gold, u_next, def, g64, gc, item_lo, item);
    else
        k_update<float><<<gr, 256, 0, s>>>((const float*)gnew, f, (float*)gold, u_next, def, g64, gc, item_lo, item);
    return cudaGetLastError();
}


// Increment form of the correction (linear G): U_{r+1} = F_r + G(delta_r),
// delta_{r+1} = U_{r+1}^new - U_{r+1}^old written, in coarse precision and with
// its periodic images, as the next slice's coarse input; defect sums as k_update.
template <typename TC>
__global__ void k_update_delta(const TC* gd, const double* f, double* u, TC* dnext, double* def, Geo g, Geo gc,
                               const int* item_lo, int item) {
    if (item_lo && item < *item_lo) return;
    const long long n = (long long)g.ni * g.nj * g.nk;
    double s_d = 0., s_q = 0.;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % g.ni);
        const int y = (int)((t / g.ni) % g.nj);
        const int z = (int)(t / ((long long)g.ni * g.nj));
        const long long o = g.origin + (long long)z * g.plane + (long long)y * g.px + x;
        const long long oc = gc.origin + (long long)z * gc.plane + (long long)y * gc.px + x;
        const double q = f[o] + (double)gd[oc];
        const double d = q - u[o];
        s_d += d * d;
        s_q += q * q;
        put_img<double>(u + g.origin, g, x, y, z, q);
        put_img<TC>(dnext + gc.origin, gc, x, y, z, (TC)d);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s_d += __shfl_xor_sync(0xffffffffu, s_d, o);
        s_q += __shfl_xor_sync(0xffffffffu, s_q, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(def, s_d);
        atomicAdd(def + 1, s_q);
    }
}

cudaError_t launch_update_delta(const Geo& g64, const Geo& gc, const void* gd, const double* f, double* u_next,
                                void* d_next, double* def, const int* item_lo, int item, cudaStream_t s) {
    add_launches(1);
    const unsigned gr = grid_for((long long)g64.ni * g64.nj * g64.nk, 256);
    if (gc.es == 8)
        k_update_delta<double><<<gr, 256, 0, s>>>((const double*)gd, f, u_next, (double*)d_next, def, g64, gc,
                                                  item_lo, item);
    else
        k_update_delta<float><<<gr, 256, 0, s>>>((const float*)gd, f, u_next, (float*)d_next, def, g64, gc, item_lo,
                                                 item);
    return cudaGetLastError();
}

// Zeroes field number *item_lo (if in [min_item, nitems)) of an array of fields of `bytes` each.
__global__ void k_zero_item(unsigned char* base, long long bytes, int nitems, const int* item_lo, int min_item) {
    const int it = *item_lo;
    if (it < min_item || it >= nitems) return;
    ulonglong2* p = reinterpret_cast<ulonglong2*>(base + (long long)it * bytes);
    const long long n = bytes / 16;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        p[t] = make_ulonglong2(0ull, 0ull);
}

cudaError_t launch_zero_item(void* base, long long bytes, int nitems, const int* item_lo, cudaStream_t s,
                             int min_item) {
    add_launches(1);
    k_zero_item<<<grid_for(bytes / 16, 256), 256, 0, s>>>(static_cast<unsigned char*>(base), bytes, nitems, item_lo,
                                                         min_item);
    return cudaGetLastError();
}

__device__ __forceinline__ void atomic_max_nonneg(double* p, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

__global__ void k_errors(const double* a, const double* b, double* acc, Geo g) {
    const long long n = (long long)g.ni * g.nj * g.nk;
    double s_d = 0., s_b = 0., m_d = 0., m_a = 0.;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % g.ni);
        const int y = (int)((t / g.ni) % g.nj);
        const int z = (int)(t / ((long long)g.ni * g.nj));
        const long long o = g.origin + (long long)z * g.plane + (long long)y * g.px + x;
        const double va = a[o], vb = b[o], d = va - vb;
        s_d += d * d;
        s_b += vb * vb;
        m_d = fmax(m_d, fabs(d));
        m_a = fmax(m_a, fabs(va));
    }
    for (int o = 16; o > 0; o >>= 1) {
        s_d += __shfl_xor_sync(0xffffffffu, s_d, o);
        s_b += __shfl_xor_sync(0xffffffffu, s_b, o);
        m_d = fmax(m_d, __shfl_xor_sync(0xffffffffu, m_d, o));
        m_a = fmax(m_a, __shfl_xor_sync(0xffffffffu, m_a, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(acc, s_d);
        atomicAdd(acc + 1, s_b);
        atomic_max_nonneg(acc + 2, m_d);
        atomic_max_nonneg(acc + 3, m_a);
    }
}

cudaError_t launch_errors(const Geo& g, const double* a, const double* b, double* acc4, cudaStream_t s) {
    add_launches(1);
    k_errors<<<grid_for((long long)g.ni * g.nj * g.nk, 256), 256, 0, s>>>(a, b, acc4, g);
    return cudaGetLastError();
}

__global__ void k_axpby(double* out, double alpha, const double* x, double beta, const double* y, Geo g) {
    const long long n = (long long)g.ni * g.nj * g.nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.ni);
        const int j = (int)((t / g.ni) % g.nj);
        const int k = (int)(t / ((long long)g.ni * g.nj));
        const long long o = g.origin + (long long)k * g.plane + (long long)j * g.px + i;
        double v = alpha * x[o];
        if (y) v += beta * y[o];
        put_img<double>(out + g.origin, g, i, j, k, v);
    }
}

cudaError_t launch_axpby(const Geo& g, double* out, double alpha, const double* x, double beta, const double* y,
                         cudaStream_t s) {
    add_launches(1);
    k_axpby<<<grid_for((long long)g.ni * g.nj * g.nk, 256), 256, 0, s>>>(out, alpha, x, beta, y, g);
    return cudaGetLastError();
}

__global__ void k_misfit(const double* a, const double* b, double* lam, double* jacc, Geo g) {
    const long long n = (long long)g.ni * g.nj * g.nk;
    double s = 0.;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.ni);
        const int j = (int)((t / g.ni) % g.nj);
        const int k = (int)(t / ((long long)g.ni * g.nj));
        const long long o = g.origin + (long long)k * g.plane + (long long)j * g.px + i;
        const double d = a[o] - b[o];
        s += 0.5 * d * d;
        put_img<double>(lam + g.origin, g, i, j, k, d);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(jacc, s);
}

cudaError_t launch_misfit(const Geo& g, const double* a, const double* b, double* lam, double* jacc, cudaStream_t s) {
    add_launches(1);
    k_misfit<<<grid_for((long long)g.ni * g.nj * g.nk, 256), 256, 0, s>>>(a, b, lam, jacc, g);
    return cudaGetLastError();
}

}  // namespace sp
