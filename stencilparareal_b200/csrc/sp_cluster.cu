// sp_cluster.cu -- many RK4 steps of a small FP64 field in one launch, the
// field held on chip in the distributed shared memory of a thread-block
// cluster.
//
// Small fields (up to ~32^3) are latency-bound on the stage kernels: an RK4
// step of a 32^3 field is four launches of ~3.5 us, most of it pipeline fill
// and drain.  Here one cluster of C = nk / NZ CTAs owns one field: CTA c keeps
// planes [c*NZ, (c+1)*NZ) of the stage input in shared memory, with two halo
// planes below and above that its z-neighbours write into it, and the step
// start q and the accumulator of its cells in registers.  A stage reads the
// 13-point star from shared memory (x and y wrap around inside the plane; z
// from the halo planes), writes the next stage input into the other of two
// shared buffers and stores each value of its two lowest / highest planes, as
// soon as it is computed, into the z-neighbours' halo planes with st.async,
// each store counting its bytes off the transaction count of the receiving
// CTA's mbarrier.  A CTA posts the halo bytes it expects for the next stage,
// and waits (acquire, bounded by %globaltimer) until they have landed: two
// neighbours per stage instead of a barrier over the whole cluster, no fence
// and no separate arrival.  The early stores are safe with two buffers: a
// neighbour's next stage writes into the buffer this stage reads, but only
// after it has received every value of this stage, and every thread sends
// after all its reads (its values depend on them).  Nothing goes to global
// memory between the first load and the last store.
//
// k_rk4_cluster2d splits the field into (y,z) blocks instead of z-slabs: four
// neighbours per CTA and, for the same number of CTAs, fewer halo values per
// stage (half as many at 32^3 on 16 CTAs), which is what bounds the slabs.
// The tuner times both layouts (tune kinds 3 and 5) and keeps the faster.
//
// Every value is computed with the operations, and in the order, of the
// single-stage kernels (rhs_w13 and the 13-access low-storage epilogues of
// sp_kernels.cu), so the result equals theirs bit for bit:
//   S1: y1 = q + dt/2 k1                 S2: y2 = q + dt/2 k2, a = q + (y1-q)/3 + dt/3 k2
//   S3: y3 = q + dt k3                   S4: q' = a + (y3-q)/3 + dt/6 k4
// (src/Convection/Convection.cpp:318-370 in low-storage form).
#include <cuda.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "sp_device.cuh"
#include "sp_internal.h"
#include "sp_stencil.cuh"

namespace sp {

namespace {

using V2 = Vec<double, 2>;
constexpr int kClusterThreads = 512;

struct ClusterArgs {
    const double* in;       // caller layout, items fields back to back
    double* out;
    long long item_stride, origin, px, plane;
    int ni, nj, nk;
    int nsteps;
    const W13<double>* wtab;  // per-step weights (nu(t) varies) or null
    W13<double> w;            // weights of every step when wtab is null
    double dthalf, dt, dt3, dt6;
    const int* item_lo;
    int item_base;
    int* err;
    StoreBounds sb;
    int cy, cz;               // (y,z) blocks: CTAs per field along y and z
};

// Cluster of C = nk / NZ CTAs per field (NZ >= 2, C >= 2); UPT units of two
// x-adjacent cells of one row per thread, every own plane of each unit.
template <int NZ, int UPT>
__global__ void __launch_bounds__(kClusterThreads, 1) k_rk4_cluster(const __grid_constant__ ClusterArgs a) {
    constexpr int NPL = NZ + 4;  // planes per buffer: 2 halo, NZ own, 2 halo
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);  // 2 mbarriers (stage parity)
    double* buf = reinterpret_cast<double*>(smem_raw + 16);
    const int ni = a.ni, nj = a.nj, nk = a.nk;
    const int plane_cells = ni * nj;
    const uint32_t buf_bytes = (uint32_t)NPL * plane_cells * 8u;
    const uint32_t base0 = smem_u32(buf);
    const uint32_t bar0 = smem_u32(bar);

    const uint32_t C = cluster_size();
    const uint32_t rank = cluster_rank();
    const int item = blockIdx.x / (int)C;
    // a converged Parareal slice: the whole cluster leaves before any cluster barrier
    if (a.item_lo && item + a.item_base < *a.item_lo) return;
    const uint32_t lower = (rank + C - 1) % C, upper = (rank + 1) % C;
    const int z0 = (int)rank * NZ;
    const double* fin = a.in + (long long)item * a.item_stride + a.origin;

    const int tid = threadIdx.x;
    if (tid == 0) {
        // per stage: this CTA's own arrival with the halo bytes it expects; the
        // neighbours' stores complete the transaction count
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    const int half = ni / 2;
    const int units = half * nj;
    // own cells: unit u -> cells (2*(u % half), u / half) and (+1, same row)
    int ux[UPT], uy[UPT];
    bool uv[UPT];
#pragma unroll
    for (int j = 0; j < UPT; ++j) {
        const int u = tid + j * kClusterThreads;
        uv[j] = u < units;
        ux[j] = uv[j] ? 2 * (u % half) : 0;
        uy[j] = uv[j] ? u / half : 0;
    }
    const uint32_t plane_bytes = (uint32_t)plane_cells * 8u;
    // byte offsets inside a plane of a unit's cells and of their x- and
    // y-neighbours (periodic): computed once per launch with one unit and up
    // to 3 planes per thread, per stage otherwise (where keeping them would
    // spill registers)
    constexpr bool kKeep = UPT == 1 && NZ < 4;
    // with one unit and two planes per thread, the first own plane's operands
    // are loaded before the wait for the halo planes
    constexpr bool kPreload = UPT == 1 && NZ == 2;
    struct Offs {
        uint32_t c, l, r, ym2, ym1, yp1, yp2;
    };
    auto offsets = [&](int j) {
        const int x = ux[j], y = uy[j];
        Offs o;
        o.c = (uint32_t)((y * ni + x) * 8);
        o.l = (uint32_t)((y * ni + (x + ni - 2) % ni) * 8);
        o.r = (uint32_t)((y * ni + (x + 2) % ni) * 8);
        o.ym2 = (uint32_t)((((y + nj - 2) % nj) * ni + x) * 8);
        o.ym1 = (uint32_t)((((y + nj - 1) % nj) * ni + x) * 8);
        o.yp1 = (uint32_t)((((y + 1) % nj) * ni + x) * 8);
        o.yp2 = (uint32_t)((((y + 2) % nj) * ni + x) * 8);
        return o;
    };
    [[maybe_unused]] Offs off1{};
    if constexpr (kKeep) off1 = offsets(0);
    // load: own planes into registers and buffer 0; the four halo planes of
    // buffer 0 from the field's interior (periodic in z)
    V2 q[UPT][NZ], acc[UPT][NZ];
#pragma unroll
    for (int j = 0; j < UPT; ++j)
#pragma unroll
        for (int p = 0; p < NPL; ++p) {
            if (!uv[j]) continue;
            const int z = (z0 - 2 + p + nk) % nk;
            const V2 v = ld16<double>(fin + (long long)z * a.plane + (long long)uy[j] * a.px + ux[j]);
            sts2(base0 + (uint32_t)((p * plane_cells + uy[j] * ni + ux[j]) * 8), v);
            if (p >= 2 && p < NZ + 2) q[j][p - 2] = v;
        }
#pragma unroll
    for (int j = 0; j < UPT; ++j)
#pragma unroll
        for (int o = 0; o < NZ; ++o) acc[j][o] = V2{};
    __syncthreads();
    cluster_sync_all();  // every CTA runs and its barriers are initialised before any remote access

    bool bad = false;
    const int nstage = 4 * a.nsteps;
    W13<double> w = a.w;
    // halo bytes per stage: two planes from each z-neighbour
    const uint32_t halo_bytes = 4u * (uint32_t)plane_cells * 8u;
    // stage g = 4 * step + ST reads buffer g & 1 and writes buffer (g + 1) & 1
    auto stage = [&](auto stc, int g) {
        constexpr int ST = decltype(stc)::value;
        const uint32_t src = base0 + (uint32_t)(g & 1) * buf_bytes;
        const uint32_t dst = base0 + (uint32_t)((g + 1) & 1) * buf_bytes;
        // NZ = 2, one unit: the first own plane's operands (centre, x- and
        // y-neighbours; written by this CTA before the last barrier) are loaded
        // before the wait for the halo planes (an invalid unit reads cell 0;
        // the second plane's as well would spill registers)
        [[maybe_unused]] V2 pre[1][7];
        if constexpr (kPreload) {
#pragma unroll
            for (int o = 0; o < 1; ++o) {
                const uint32_t row = src + (uint32_t)(o + 2) * plane_bytes;
                pre[o][0] = lds2(row + off1.c);
                pre[o][1] = lds2(row + off1.l);
                pre[o][2] = lds2(row + off1.r);
                pre[o][3] = lds2(row + off1.ym1);
                pre[o][4] = lds2(row + off1.ym2);
                pre[o][5] = lds2(row + off1.yp1);
                pre[o][6] = lds2(row + off1.yp2);
            }
        }
        if (g > 0 && !bad) {
            // halo planes of this stage's input, written by both z-neighbours at the
            // end of stage g-1 (after one wait has given up, none is tried again:
            // the kernel runs to its end, reports the timeout and returns)
            if (!mbar_wait_cluster_bounded(bar0 + 8u * (uint32_t)(g & 1), (uint32_t)(((g - 1) >> 1) & 1))) bad = true;
        }
        const bool exchange = g + 1 < nstage;  // the last stage's output goes to global memory only
        const uint32_t nbar = bar0 + 8u * (uint32_t)((g + 1) & 1);  // completes when stage g+1's halo has landed
        if (exchange && tid == 0) mbar_arrive_expect_tx_u32(nbar, halo_bytes);
#pragma unroll
        for (int j = 0; j < UPT; ++j) {
            if (!uv[j]) continue;
            Offs of;
            if constexpr (kKeep) of = off1;
            else of = offsets(j);
            // the unit's column of stage inputs: planes -2 .. NZ+1 (z-window)
            V2 col[NPL];
#pragma unroll
            for (int p = 0; p < NPL; ++p) {
                if constexpr (kPreload) {
                    if (p == 2) { col[p] = pre[0][0]; continue; }
                }
                col[p] = lds2(src + (uint32_t)p * plane_bytes + of.c);
            }
#pragma unroll
            for (int o = 0; o < NZ; ++o) {
                const int p = o + 2;
                const uint32_t row = src + (uint32_t)p * plane_bytes;
                V2 L, R, Ym1, Ym2, Yp1, Yp2;
                if (kPreload && o == 0) {
                    L = pre[0][1]; R = pre[0][2]; Ym1 = pre[0][3]; Ym2 = pre[0][4]; Yp1 = pre[0][5]; Yp2 = pre[0][6];
                } else {
                    L = lds2(row + of.l);
                    R = lds2(row + of.r);
                    Ym1 = lds2(row + of.ym1);
                    Ym2 = lds2(row + of.ym2);
                    Yp1 = lds2(row + of.yp1);
                    Yp2 = lds2(row + of.yp2);
                }
                const V2& cen = col[p];
                const double rowv[6] = {L.v[0], L.v[1], cen.v[0], cen.v[1], R.v[0], R.v[1]};
                V2 out;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    Nb<double> s;
                    s.c = rowv[2 + e];
                    s.xm1 = rowv[1 + e]; s.xp1 = rowv[3 + e];
                    s.xm2 = rowv[e]; s.xp2 = rowv[4 + e];
                    s.ym1 = Ym1.v[e]; s.yp1 = Yp1.v[e]; s.ym2 = Ym2.v[e]; s.yp2 = Yp2.v[e];
                    s.zm1 = col[p - 1].v[e]; s.zp1 = col[p + 1].v[e];
                    s.zm2 = col[p - 2].v[e]; s.zp2 = col[p + 2].v[e];
                    const double k = rhs_w13(w, s);
                    const double qc = q[j][o].v[e];
                    if constexpr (ST == 0) {
                        out.v[e] = fma(a.dthalf, k, qc);
                    } else if constexpr (ST == 1) {
                        out.v[e] = fma(a.dthalf, k, qc);
                        acc[j][o].v[e] = fma(a.dt3, k, add_third(cen.v[e], qc, qc));
                    } else if constexpr (ST == 2) {
                        out.v[e] = fma(a.dt, k, qc);
                    } else {
                        out.v[e] = fma(a.dt6, k, add_third(cen.v[e], qc, acc[j][o].v[e]));
                    }
                }
                if constexpr (ST == 3) q[j][o] = out;
                sts2(dst + (uint32_t)p * plane_bytes + of.c, out);
                // the plane goes to the z-neighbours at once: the lower neighbour's
                // upper halo planes NZ+2, NZ+3 are our own planes 0, 1; the upper
                // neighbour's lower halo planes 0, 1 our own planes NZ-2, NZ-1.
                // Every thread with a unit sends, each after all its reads of src
                // (its values depend on them), and a neighbour writes into our src
                // halo planes only once its next stage has every byte of ours.
                if (exchange) {
                    if (o < 2)
                        st_async2(map_rank(dst + (uint32_t)(NZ + 2 + o) * plane_bytes + of.c, lower), out,
                                  map_rank(nbar, lower));
                    if (o >= NZ - 2)
                        st_async2(map_rank(dst + (uint32_t)(o - (NZ - 2)) * plane_bytes + of.c, upper), out,
                                  map_rank(nbar, upper));
                }
            }
        }
        // own planes of dst written before the next stage reads them, and every
        // thread of this CTA done reading src before the next stage overwrites it
        __syncthreads();
    };
    for (int i = 0; i < a.nsteps; ++i) {
        if (a.wtab) w = a.wtab[i];
        stage(std::integral_constant<int, 0>{}, 4 * i);
        stage(std::integral_constant<int, 1>{}, 4 * i + 1);
        stage(std::integral_constant<int, 2>{}, 4 * i + 2);
        stage(std::integral_constant<int, 3>{}, 4 * i + 3);
    }
    // result (the last stage's q') to global memory, interior only (the host
    // fills the periodic images)
    double* fout = a.out + (long long)item * a.item_stride + a.origin;
#pragma unroll
    for (int j = 0; j < UPT; ++j)
#pragma unroll
        for (int o = 0; o < NZ; ++o)
            if (uv[j]) gst16<double>(a.sb, fout + (long long)(z0 + o) * a.plane + (long long)uy[j] * a.px + ux[j], q[j][o]);
    if (__syncthreads_or(bad) && tid == 0) atomicExch(a.err, DEV_WAIT_TIMEOUT);
    cluster_sync_all();  // no CTA leaves while a neighbour may still address its shared memory
}

// The same steps on (y,z) blocks: a cluster of C = cy * cz CTAs per field, CTA
// (ry, rz) (cluster rank rz * cy + ry) owning rows [ry*BY, (ry+1)*BY) and
// planes [rz*BZ, (rz+1)*BZ) of every column (BY = nj / cy >= 2, BZ = nk / cz
// >= 2).  A buffer holds the block with two halo rows below and above it
// (over its own planes) and two halo planes below and above it (over its own
// rows): planes of (BY + 4) rows of ni cells, BZ + 4 planes; the corners are
// never operands of the 13-point star.  A stage sends each value of its two
// lowest / highest rows to the y-neighbours and of its two lowest / highest
// planes to the z-neighbours, (4 BY + 4 BZ) ni values per CTA, against
// 4 nj ni for the z-slabs of k_rk4_cluster: at 32^3 on 16 CTAs half as many,
// and the exchange through distributed shared memory is what bounds the slabs
// (32^3 x 1000 steps: 6.6 ms with the slabs' halo, 4.1 ms with half of it sent,
// 3.3 ms with none).  Unit u of a thread: two x-adjacent cells of row
// y = (u / (ni/2)) % BY over ZT consecutive own planes from ZT * (u / (ni/2 * BY)).
// Arithmetic, buffers, barriers and the early sends as in k_rk4_cluster; a
// halo region is read only by threads that send to the neighbour writing it,
// and they send after all their reads, so two buffers suffice here too.
// NT threads per CTA: 256 (up to 255 registers, one unit per thread) where the
// block's units fit, else 512 (128 registers, up to two units per thread); at
// 32^3 and 24^3 the 256-thread form is ~14 % faster, at 40^3 it would spill.
template <int ZT, int UPT, int NT>
__global__ void __launch_bounds__(NT, 1) k_rk4_cluster2d(const __grid_constant__ ClusterArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);  // 2 mbarriers (stage parity)
    double* buf = reinterpret_cast<double*>(smem_raw + 16);
    const int ni = a.ni, nj = a.nj, nk = a.nk;
    const int cy = a.cy, cz = a.cz;
    const int BY = nj / cy, BZ = nk / cz;
    const uint32_t row_bytes = (uint32_t)ni * 8u;
    const uint32_t plane_bytes = (uint32_t)(BY + 4) * row_bytes;
    const uint32_t buf_bytes = (uint32_t)(BZ + 4) * plane_bytes;
    const uint32_t base0 = smem_u32(buf);
    // the accumulator of the own cells (written by stage 2, read by stage 4)
    // lives in shared memory after the two buffers: registers stay for the stars
    const uint32_t accb = base0 + 2u * buf_bytes;
    const uint32_t bar0 = smem_u32(bar);

    const uint32_t C = cluster_size();
    const uint32_t rank = cluster_rank();
    const int item = blockIdx.x / (int)C;
    // a converged Parareal slice: the whole cluster leaves before any cluster barrier
    if (a.item_lo && item + a.item_base < *a.item_lo) return;
    const int ry = (int)rank % cy, rz = (int)rank / cy;
    const int y0 = ry * BY, z0 = rz * BZ;
    const double* fin = a.in + (long long)item * a.item_stride + a.origin;

    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    // neighbours: y-lower, y-upper, z-lower, z-upper; the address of their
    // buffer 0 in the cluster's shared-memory window (a CTA's shared memory is
    // one contiguous range of the window, so its barriers lie 16 bytes below)
    uint32_t rb[4];
    {
        const uint32_t nb[4] = {(uint32_t)(rz * cy + (ry + cy - 1) % cy), (uint32_t)(rz * cy + (ry + 1) % cy),
                                (uint32_t)(((rz + cz - 1) % cz) * cy + ry), (uint32_t)(((rz + 1) % cz) * cy + ry)};
#pragma unroll
        for (int i = 0; i < 4; ++i) rb[i] = map_rank(base0, nb[i]);
    }
    const int half = ni / 2;
    const int units = half * BY * (BZ / ZT);
    int ux[UPT], uy[UPT], uz[UPT];
    bool uv[UPT];
    uint32_t oc[UPT], ol[UPT], orr[UPT];  // byte offsets in a buffer plane: cell, left and right pairs
    bool halo[UPT];                       // the unit's star reaches a halo row or plane
#pragma unroll
    for (int j = 0; j < UPT; ++j) {
        const int u = tid + j * NT;
        uv[j] = u < units;
        const int uu = uv[j] ? u : 0;
        ux[j] = 2 * (uu % half);
        uy[j] = (uu / half) % BY;
        uz[j] = ZT * (uu / (half * BY));
        const uint32_t rowo = (uint32_t)(uy[j] + 2) * row_bytes;
        oc[j] = rowo + (uint32_t)ux[j] * 8u;
        ol[j] = rowo + (uint32_t)((ux[j] + ni - 2) % ni) * 8u;
        orr[j] = rowo + (uint32_t)((ux[j] + 2) % ni) * 8u;
        halo[j] = uy[j] < 2 || uy[j] > BY - 3 || uz[j] < 2 || uz[j] + ZT > BZ - 2;
    }
    // load: the block with its halo rows and planes (corners too: unused) from
    // the field's interior, periodic in y and z; the own cells' step start
    {
        const int rows = BY + 4;
        const int n = (BZ + 4) * rows * half;
        for (int i = tid; i < n; i += NT) {
            const int p = i / (rows * half);
            const int r = i - p * rows * half;
            const int yy = r / half;
            const int x = 2 * (r - yy * half);
            const int gz = (z0 - 2 + p + nk) % nk;
            const int gy = (y0 - 2 + yy + nj) % nj;
            const V2 v = ld16<double>(fin + (long long)gz * a.plane + (long long)gy * a.px + x);
            sts2(base0 + (uint32_t)p * plane_bytes + (uint32_t)yy * row_bytes + (uint32_t)x * 8u, v);
        }
    }
    V2 q[UPT][ZT];
#pragma unroll
    for (int j = 0; j < UPT; ++j)
#pragma unroll
        for (int o = 0; o < ZT; ++o)
            q[j][o] = uv[j] ? ld16<double>(fin + (long long)(z0 + uz[j] + o) * a.plane + (long long)(y0 + uy[j]) * a.px +
                                           ux[j])
                            : V2{};
    __syncthreads();
    cluster_sync_all();  // every CTA runs and its barriers are initialised before any remote access

    bool bad = false;
    const int nstage = 4 * a.nsteps;
    W13<double> w = a.w;
    const uint32_t halo_bytes = (uint32_t)(4 * BY + 4 * BZ) * row_bytes;
    const uint32_t yshift = (uint32_t)BY * row_bytes, zshift = (uint32_t)BZ * plane_bytes;
    auto stage = [&](auto stc, int g) {
        constexpr int ST = decltype(stc)::value;
        const uint32_t dpar = (uint32_t)((g + 1) & 1);
        const uint32_t src = base0 + (uint32_t)(g & 1) * buf_bytes;
        const uint32_t dst = base0 + dpar * buf_bytes;
        // the halo of this stage's input, written by the neighbours in stage g-1:
        // waited for before the first unit whose star reaches it (units inside
        // the block read only cells of this CTA, ordered by the last barrier)
        bool waited = g == 0;
        const bool exchange = g + 1 < nstage;  // the last stage's output goes to global memory only
        if (exchange && tid == 0) mbar_arrive_expect_tx_u32(bar0 + 8u * dpar, halo_bytes);
        const uint32_t rdo = dpar * buf_bytes, rbo = 8u * dpar - (base0 - bar0);
#pragma unroll
        for (int j = 0; j < UPT; ++j) {
            if (!uv[j]) continue;
            if (halo[j] && !waited) {
                // after one wait has given up none is tried again: the kernel
                // runs to its end, reports the timeout and returns
                if (!bad && !mbar_wait_cluster_bounded(bar0 + 8u * (uint32_t)(g & 1), (uint32_t)(((g - 1) >> 1) & 1)))
                    bad = true;
                waited = true;
            }
            // the unit's column of stage inputs: buffer planes uz .. uz+ZT+3
            V2 col[ZT + 4];
#pragma unroll
            for (int p = 0; p < ZT + 4; ++p) col[p] = lds2(src + (uint32_t)(uz[j] + p) * plane_bytes + oc[j]);
#pragma unroll
            for (int o = 0; o < ZT; ++o) {
                const int p = o + 2;
                const uint32_t pl = (uint32_t)(uz[j] + p) * plane_bytes;
                const uint32_t c = src + pl + oc[j];
                const V2 L = lds2(src + pl + ol[j]);
                const V2 R = lds2(src + pl + orr[j]);
                const V2 Ym1 = lds2(c - row_bytes);
                const V2 Ym2 = lds2(c - 2u * row_bytes);
                const V2 Yp1 = lds2(c + row_bytes);
                const V2 Yp2 = lds2(c + 2u * row_bytes);
                const V2& cen = col[p];
                const double rowv[6] = {L.v[0], L.v[1], cen.v[0], cen.v[1], R.v[0], R.v[1]};
                const uint32_t aa = accb + (uint32_t)(((uz[j] + o) * BY + uy[j]) * ni + ux[j]) * 8u;
                V2 out, acc;
                if constexpr (ST == 3) acc = lds2(aa);
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    Nb<double> s;
                    s.c = rowv[2 + e];
                    s.xm1 = rowv[1 + e]; s.xp1 = rowv[3 + e];
                    s.xm2 = rowv[e]; s.xp2 = rowv[4 + e];
                    s.ym1 = Ym1.v[e]; s.yp1 = Yp1.v[e]; s.ym2 = Ym2.v[e]; s.yp2 = Yp2.v[e];
                    s.zm1 = col[p - 1].v[e]; s.zp1 = col[p + 1].v[e];
                    s.zm2 = col[p - 2].v[e]; s.zp2 = col[p + 2].v[e];
                    const double k = rhs_w13(w, s);
                    const double qc = q[j][o].v[e];
                    if constexpr (ST == 0) {
                        out.v[e] = fma(a.dthalf, k, qc);
                    } else if constexpr (ST == 1) {
                        out.v[e] = fma(a.dthalf, k, qc);
                        acc.v[e] = fma(a.dt3, k, add_third(cen.v[e], qc, qc));
                    } else if constexpr (ST == 2) {
                        out.v[e] = fma(a.dt, k, qc);
                    } else {
                        out.v[e] = fma(a.dt6, k, add_third(cen.v[e], qc, acc.v[e]));
                    }
                }
                if constexpr (ST == 1) sts2(aa, acc);
                if constexpr (ST == 3) q[j][o] = out;
                const uint32_t d = pl + oc[j];  // the cell's offset in a buffer
                sts2(dst + d, out);
                // to the neighbours at once: rows y < 2 are the y-lower
                // neighbour's upper halo rows (BY rows further up in its
                // buffer), rows y >= BY-2 the y-upper neighbour's lower halo
                // rows; likewise planes for z
                if (exchange) {
                    const int zo = uz[j] + o;
                    if (uy[j] < 2) st_async2(rb[0] + rdo + d + yshift, out, rb[0] + rbo);
                    if (uy[j] >= BY - 2) st_async2(rb[1] + rdo + d - yshift, out, rb[1] + rbo);
                    if (zo < 2) st_async2(rb[2] + rdo + d + zshift, out, rb[2] + rbo);
                    if (zo >= BZ - 2) st_async2(rb[3] + rdo + d - zshift, out, rb[3] + rbo);
                }
            }
        }
        __syncthreads();
    };
    for (int i = 0; i < a.nsteps; ++i) {
        if (a.wtab) w = a.wtab[i];
        stage(std::integral_constant<int, 0>{}, 4 * i);
        stage(std::integral_constant<int, 1>{}, 4 * i + 1);
        stage(std::integral_constant<int, 2>{}, 4 * i + 2);
        stage(std::integral_constant<int, 3>{}, 4 * i + 3);
    }
    double* fout = a.out + (long long)item * a.item_stride + a.origin;
#pragma unroll
    for (int j = 0; j < UPT; ++j)
#pragma unroll
        for (int o = 0; o < ZT; ++o)
            if (uv[j])
                gst16<double>(a.sb, fout + (long long)(z0 + uz[j] + o) * a.plane + (long long)(y0 + uy[j]) * a.px + ux[j],
                              q[j][o]);
    if (__syncthreads_or(bad) && tid == 0) atomicExch(a.err, DEV_WAIT_TIMEOUT);
    cluster_sync_all();  // no CTA leaves while a neighbour may still address its shared memory
}

template <int NZ, int UPT>
size_t cluster_smem(const Geo& g) {
    return 16 + (size_t)2 * (NZ + 4) * g.ni * g.nj * 8;
}

template <int NZ, int UPT>
cudaError_t set_attr_cluster(const Geo* g) {
    auto k = k_rk4_cluster<NZ, UPT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kClusterSmemMax);
    (void)g;
    return e;
}

// Planes per CTA for a grid and batch: NZ in {2, 3, 4} with a cluster of at
// most 16 CTAs whose buffers fit -- the smallest (the most CTAs per field: a
// single field is bound by the latency of each stage) while the batch's CTAs
// fit on the SMs at once, else the largest (fewer CTAs per field, more fields
// at a time); 0 when the grid is not supported.
int cluster_nz(const Geo& g, int items = 1) {
    if (g.es != 8 || g.ni % 2 != 0 || g.ni < 4 || g.nj < 4 || g.nk < 4) return 0;
    if ((long long)(g.ni / 2) * g.nj > 2LL * kClusterThreads) return 0;
    int first = 0, last = 0;
    for (int nz : {2, 3, 4}) {
        if (g.nk % nz != 0) continue;
        const int c = g.nk / nz;
        if (c < 2 || c > 16) continue;
        if (16 + (size_t)2 * (nz + 4) * g.ni * g.nj * 8 > (size_t)kClusterSmemMax) continue;
        if (!first) first = nz;
        last = nz;
    }
    if (!first) return 0;
    return (long long)items * (g.nk / first) <= 148 ? first : last;
}

template <int NZ, int UPT>
cudaError_t launch_one(const Geo& g, const ClusterArgs& a, int items, cudaStream_t s) {
    const int C = g.nk / NZ;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(C * items));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = cluster_smem<NZ, UPT>(g);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_rk4_cluster<NZ, UPT>, a);
}

// (y,z) blocks for a grid and batch: cy, cz >= 2 with C = cy * cz <= 16, blocks
// of at least 2 rows and 2 planes whose two buffers fit, and a thread form
// (below).  Among those the one with the least estimated time: waves of CTAs
// (one per SM) x (own cells + half the halo cells per CTA; at 32^3 the exchange
// of a halo cell costs about half the stage work of an own cell), x 1.6 for the
// spilling two-unit form; ties go to fewer units per thread.  cy = 0 when the
// grid has no such blocks.
// bytes of shared memory per CTA of k_rk4_cluster2d: barriers, two buffers of
// the block with its halo rows and planes, the accumulator of the own cells
size_t cluster2d_smem(int ni, int by, int bz) {
    return 16 + (size_t)2 * (bz + 4) * (by + 4) * ni * 8 + (size_t)bz * by * ni * 8;
}

struct Blocks2d {
    int cy = 0, cz = 0, zt = 0, upt = 0, nt = 0;
};
Blocks2d blocks_2d(const Geo& g, int items) {
    Blocks2d best;
    if (g.es != 8 || g.ni % 2 != 0 || g.ni < 4 || g.nj < 4 || g.nk < 4 || items < 1) return best;
    double best_cost = 0;
    for (int cy = 2; cy <= 8; ++cy)
        for (int cz = 2; cy * cz <= 16; ++cz) {
            if (g.nj % cy != 0 || g.nk % cz != 0) continue;
            const int by = g.nj / cy, bz = g.nk / cz;
            if (by < 2 || bz < 2) continue;
            if (cluster2d_smem(g.ni, by, bz) > (size_t)kClusterSmemMax) continue;
            // 256 threads with one unit each, of the fewest planes ZT in {1, 2, 4}
            // that fits (the most threads with work), else 512 threads with up
            // to two units of ZT = 2 or 1 planes
            int zt = 0, upt = 0, nt = 0;
            for (int z : {1, 2, 4})
                if (!zt && bz % z == 0 && (long long)(g.ni / 2) * by * (bz / z) <= 256) {
                    zt = z;
                    upt = 1;
                    nt = 256;
                }
            if (!zt) {
                zt = bz % 2 == 0 ? 2 : 1;
                const long long units = (long long)(g.ni / 2) * by * (bz / zt);
                upt = (int)((units + kClusterThreads - 1) / kClusterThreads);
                nt = kClusterThreads;
                if (upt > 2) continue;
            }
            const long long ctas = (long long)items * cy * cz;
            const long long waves = (ctas + 147) / 148;
            // the 512-thread form with two units per thread spills at its
            // 128-register cap: a batch of 16 fields of 32^3 ran its fine sweep
            // at 22.6 GCUPS on (2,4) blocks in one wave of that form, at 40.8 on
            // (4,4) blocks in two waves of the 256-thread form
            const double form = nt == kClusterThreads && upt == 2 ? 1.6 : 1.0;
            const double cost = form * (double)waves * ((double)g.ni * by * bz + 0.5 * (4.0 * by + 4.0 * bz) * g.ni);
            if (!best.cy || cost < best_cost || (cost == best_cost && upt < best.upt)) {
                best = Blocks2d{cy, cz, zt, upt, nt};
                best_cost = cost;
            }
        }
    return best;
}

template <int ZT, int UPT, int NT>
cudaError_t launch_one2d(const Geo& g, const Blocks2d& b, const ClusterArgs& a, int items, cudaStream_t s) {
    auto k = k_rk4_cluster2d<ZT, UPT, NT>;
    const int C = b.cy * b.cz;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(C * items));
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = cluster2d_smem(g.ni, g.nj / b.cy, g.nk / b.cz);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, a);
}

template <int ZT, int UPT, int NT>
cudaError_t set_attr_cluster2d() {
    cudaError_t e = cudaSuccess;
    auto k = k_rk4_cluster2d<ZT, UPT, NT>;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kClusterSmemMax);
    return e;
}

}  // namespace

bool cluster_supported(const Geo& g, int mode) {
    return mode == 2 ? blocks_2d(g, 1).cy != 0 : cluster_nz(g) != 0;
}

cudaError_t prepare_cluster() {
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    chk(set_attr_cluster<2, 1>(nullptr)); chk(set_attr_cluster<2, 2>(nullptr));
    chk(set_attr_cluster<3, 1>(nullptr)); chk(set_attr_cluster<3, 2>(nullptr));
    chk(set_attr_cluster<4, 1>(nullptr)); chk(set_attr_cluster<4, 2>(nullptr));
    chk(set_attr_cluster2d<1, 1, 512>()); chk(set_attr_cluster2d<1, 2, 512>());
    chk(set_attr_cluster2d<2, 1, 512>()); chk(set_attr_cluster2d<2, 2, 512>());
    chk(set_attr_cluster2d<1, 1, 256>()); chk(set_attr_cluster2d<2, 1, 256>());
    chk(set_attr_cluster2d<4, 1, 256>());
    return e;
}

cudaError_t launch_rk4_cluster(const Geo& g, const ClusterLaunch& L, cudaStream_t s, int* err) {
    const int nz = L.mode == 2 ? 0 : cluster_nz(g, L.items);
    const Blocks2d b2 = L.mode == 2 ? blocks_2d(g, L.items) : Blocks2d{};
    if ((L.mode == 2 ? !b2.cy : !nz) || L.nsteps < 1 || L.items < 1) return cudaErrorInvalidValue;
    ClusterArgs a;
    a.in = static_cast<const double*>(L.in);
    a.out = static_cast<double*>(L.out);
    a.item_stride = g.total;
    a.origin = g.origin;
    a.px = g.px;
    a.plane = g.plane;
    a.ni = g.ni; a.nj = g.nj; a.nk = g.nk;
    a.nsteps = L.nsteps;
    a.wtab = static_cast<const W13<double>*>(L.wtab);
    fill_w13(a.w, L.coef, L.nu);
    a.dthalf = L.dt * .5;
    a.dt = L.dt;
    a.dt3 = L.dt / 3.;
    a.dt6 = L.dt / 6.;
    a.item_lo = L.item_lo;
    a.item_base = L.item_base;
    a.err = err;
    a.sb = out_bounds(L.out, g, L.items);
    a.cy = b2.cy;
    a.cz = b2.cz;
    if (L.mode == 2) {
        add_launches(1);
        if (b2.nt == 256) {
            if (b2.zt == 4) return launch_one2d<4, 1, 256>(g, b2, a, L.items, s);
            if (b2.zt == 2) return launch_one2d<2, 1, 256>(g, b2, a, L.items, s);
            return launch_one2d<1, 1, 256>(g, b2, a, L.items, s);
        }
        switch (b2.zt * 2 + b2.upt - 1) {
            case 2: return launch_one2d<1, 1, 512>(g, b2, a, L.items, s);
            case 3: return launch_one2d<1, 2, 512>(g, b2, a, L.items, s);
            case 4: return launch_one2d<2, 1, 512>(g, b2, a, L.items, s);
            default: return launch_one2d<2, 2, 512>(g, b2, a, L.items, s);
        }
    }
    const bool two = (long long)(g.ni / 2) * g.nj > kClusterThreads;
    add_launches(1);
    switch (nz * 2 + (two ? 1 : 0)) {
        case 4: return launch_one<2, 1>(g, a, L.items, s);
        case 5: return launch_one<2, 2>(g, a, L.items, s);
        case 6: return launch_one<3, 1>(g, a, L.items, s);
        case 7: return launch_one<3, 2>(g, a, L.items, s);
        case 8: return launch_one<4, 1>(g, a, L.items, s);
        default: return launch_one<4, 2>(g, a, L.items, s);
    }
}

void fill_cluster_weights(void* w13, const Coef& c, double nu) { fill_w13(*static_cast<W13<double>*>(w13), c, nu); }

size_t cluster_weights_bytes() { return sizeof(W13<double>); }

}  // namespace sp
