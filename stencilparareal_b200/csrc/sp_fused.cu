// sp_fused.cu -- RK4 stages fused in pairs through shared memory.
//
// One low-storage RK4 step (src/Convection/Convection.cpp:286-327) is four
// stencil stages.  Run one by one (sp_kernels.cu) they move 13 field values per
// cell through HBM (104 B in FP64).  Here stages 1+2 and stages 3+4 each run as one kernel:
// the first stage of a pair is evaluated on the CTA tile widened by the
// stencil radius (2 cells in x and y, 2 planes ahead in z) and kept in shared
// memory, where the second stage reads it.  Per step the pairs move 7 values
// per cell (56 B):
//   pair 1+2: reads q;           writes y2 = q + dt/2 R(y1), acc = q + (y1 - q)/3 + dt/3 k2
//   pair 3+4: reads y2, q, acc;  writes q' = acc + (y3 - q)/3 + dt/6 k4
// ((y1 - q)/3 = dt/6 k1 and (y3 - q)/3 = dt/3 k3: the forms the single-stage
// kernels use, where they save the accumulator traffic of stages 1 and 3)
// Every value is computed with the same operations, in the same order, as the
// single-stage kernels, so both paths give bit-identical fields.
//
// The widened first stage reads its input 4 cells beyond the tile, deeper
// than the 2-cell halo of the caller's layout, so the pairs work on internal
// fields with 4-cell periodic images (faces, edges and corners); the step's
// input is widened once per propagation and the last step writes the
// caller's layout directly.
//
// CTA: 32*TY threads; thread (warp w, lane l) owns cells (x0+2l, x0+2l+1) of
// tile row y0+w (tile 64 x TY), and threads below NH also one 2-cell chunk of
// the ring around the tile (two rows above and below over the tile's columns,
// two columns left and right over its rows).  The grid is persistent (one
// wave): groups of up to 4 CTAs take y-adjacent tiles over one range of
// planes, so that they march together and share their halo rows through L2;
// a range is cut into segments at tile boundaries.  In a segment [z0, z1)
// iteration v evaluates the first stage on plane z0-2+v and the second on
// plane z0-4+v.  Shared memory: NSQ slots of the stencil input (TMA boxes of
// (64+8) x (TY+8) cells), 3 slots of the widened first-stage field, NP slots
// of pointwise operands (pair 3+4: q on the widened tile and acc on the tile),
// and the mbarriers of the TMA slots.  z-neighbours of the thread's own cells
// are carried in registers; the ring cells read theirs from the slots.  The
// kernels are launched with programmatic dependent launch and read global
// memory only after griddepcontrol.wait.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <type_traits>
#include <utility>

#include "sp_device.cuh"
#include "sp_internal.h"
#include "sp_stencil.cuh"

namespace sp {

namespace {

using V2 = Vec<double, 2>;

struct PairArgs {
    long long item_stride, origin, px, plane;  // internal geometry (4-cell halo)
    int ni, nj, nk, pz;
    int tiles_x, tiles_y, items;
    int cy;            // CTAs per group: y-adjacent tiles marching the same plane range
    int span;          // planes of the flattened (tile group, z) space per group (total < 2^31)
    const int* item_lo;
    int item_base;
    W13<double> w;
    double c1y;        // first stage:  y = c1y k + base
    double c2y, c2a;   // second stage: y = c2y k + q (pair 1+2), acc / result = c2a k + base
    double* yout;      // pair 1+2: y2 (internal geometry, images 4 deep)
    double* aout;      // pair 1+2: acc (internal geometry, interior only)
    double* qout;      // pair 3+4: step result
    long long o_item_stride, o_origin, o_px, o_plane;
    int o_halo;        // image depth written with qout
    StoreBounds sb_o;  // output allocations (bounds-checked builds): yout or qout,
    StoreBounds sb_a;  // and aout
    int* err;
};

// Stores cells (x, x+1) of a row and their x-images within `hd` cells of the
// x faces; x < ni.
__device__ __forceinline__ void row_pair(const StoreBounds& b, double* row, int ni, int hd, int x, const V2& v) {
    if (x + 2 <= ni) gst16<double>(b, row + x, v);
    else gst1(b, row + x, v.v[0]);
    if (x < hd || x + 2 > ni - hd) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int xe = x + e;
            if (xe >= ni) continue;
            if (xe < hd) gst1(b, row + xe + ni, v.v[e]);
            if (xe >= ni - hd) gst1(b, row + xe - ni, v.v[e]);
        }
    }
}

// Stores cells (x, x+1) of row (y, z) (x < ni) and their periodic images
// within `hd` cells of a face (faces, edges and corners): the path of the
// lanes next to a face; the others store their pair with one 16-byte store.
__device__ __forceinline__ void store_images_pair(const StoreBounds& b, double* base, long long px, long long plane,
                                                  int ni, int nj, int nk, int hd, int x, int y, int z, const V2& v) {
    double* row = base + (long long)z * plane + (long long)y * px;
#pragma unroll
    for (int iz = 0; iz < 3; ++iz) {
        if (iz == 1 && !(z < hd)) continue;
        if (iz == 2 && !(z >= nk - hd)) continue;
        const long long oz = iz == 0 ? 0 : (iz == 1 ? (long long)nk * plane : -(long long)nk * plane);
#pragma unroll
        for (int iy = 0; iy < 3; ++iy) {
            if (iy == 1 && !(y < hd)) continue;
            if (iy == 2 && !(y >= nj - hd)) continue;
            const long long oy = iy == 0 ? 0 : (iy == 1 ? (long long)nj * px : -(long long)nj * px);
            double* r = row + oz + oy;
            row_pair(b, r, ni, hd, x, v);
        }
    }
}

// R4 of cells (at, at+8) of a slot of row width W, `at` a shared-memory byte
// address; the centre values and the z-neighbours are given, the x- and
// y-neighbours are read from the slot.
template <int W>
__device__ __forceinline__ void rhs_s(const W13<double>& wt, uint32_t at, const V2& cen, const V2& zm2,
                                      const V2& zm1, const V2& zp1, const V2& zp2, double k[2]) {
    const V2 r0 = lds2o<-16>(at), r2 = lds2o<16>(at);
    const V2 ym2 = lds2o<-16 * W>(at), ym1 = lds2o<-8 * W>(at);
    const V2 yp1 = lds2o<8 * W>(at), yp2 = lds2o<16 * W>(at);
    const double row[6] = {r0.v[0], r0.v[1], cen.v[0], cen.v[1], r2.v[0], r2.v[1]};
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        Nb<double> s;
        s.c = row[2 + e];
        s.xm1 = row[1 + e]; s.xp1 = row[3 + e];
        s.xm2 = row[e]; s.xp2 = row[4 + e];
        s.ym1 = ym1.v[e]; s.yp1 = yp1.v[e]; s.ym2 = ym2.v[e]; s.yp2 = yp2.v[e];
        s.zm1 = zm1.v[e]; s.zp1 = zp1.v[e]; s.zm2 = zm2.v[e]; s.zp2 = zp2.v[e];
        k[e] = rhs_w13(wt, s);
    }
}

template <int TY, int NSQ, int NP, int PAIR, int TXP = 64>
struct PairShape {
    static constexpr int TX = TXP;                  // tile columns: 64 (one row per warp) or 32 (two)
    static constexpr int NT = TY * TX / 2;          // threads: two cells of one tile row each
    // stencil-input slot (box at x0-4, y0-4).  32-column tiles load a box 4
    // columns wider than they read (44 instead of 40): with rows of 352 instead
    // of 320 bytes, the ring's side columns (2 cells at x0-2 and x0+32, four rows
    // per quarter warp) fall into distinct shared-memory banks; at 256^3 the
    // step runs ~3 % faster per clock
    static constexpr int WB = TX == 32 ? 44 : TX + 8, HB = TY + 8;
    static constexpr int WE = TX + 4, HE = TY + 4;  // widened first-stage slot (origin x0-2, y0-2)
    static constexpr int SB = WB * HB, SE = WE * HE, SA = TX * TY;
    static constexpr int NE = 3;
    static constexpr int NHR = 4 * (TX / 2);        // ring chunks in the two rows above and below (x0 .. x0+63)
    static constexpr int NH = NHR + 2 * TY;         // plus the two columns left and right
    static constexpr int SP = PAIR == 1 ? SE + SA : 0;
    static constexpr size_t smem = 128 + (size_t)(NSQ * SB + NE * SE + NP * SP) * 8 + (NSQ + NP) * 8;
};

template <int PAIR, int TY, int NSQ, int NP, int TXP = 64>
__global__ void __launch_bounds__(TY * TXP / 2, TY * TXP / 2 <= 256 ? 2 : 1)
    k_rk4_pair(const __grid_constant__ CUtensorMap tm_s, const __grid_constant__ CUtensorMap tm_q,
               const __grid_constant__ CUtensorMap tm_a, const PairArgs a) {
    using S = PairShape<TY, NSQ, NP, PAIR, TXP>;
    constexpr int TX = S::TX, WB = S::WB, WE = S::WE, SB = S::SB, SE = S::SE, SP = S::SP;
    constexpr int NE = S::NE, NHR = S::NHR, NH = S::NH;
    constexpr uint32_t SBYTES = SB * 8, PBYTES = SP * 8;
    static_assert(SBYTES % 128 == 0 && (SE * 8) % 128 == 0 && (S::SA * 8) % 128 == 0, "slot alignment");
    static_assert(NH <= S::NT, "ring chunks per CTA");
    static_assert(NSQ >= 6, "five stencil planes in use plus one in flight");

    extern __shared__ unsigned char smem_raw[];
    double* sb = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    double* es = sb + NSQ * SB;
    double* ps = es + NE * SE;
    uint64_t* bar = reinterpret_cast<uint64_t*>(ps + NP * SP);

    // thread -> cells (x0 + 2 px, x0 + 2 px + 1) of tile row `row`
    const int tid = threadIdx.x, px = tid % (TX / 2), row = tid / (TX / 2);
    const bool leader = tid == 0;

    pdl_trigger();  // the next kernel's CTAs may start as this grid's CTAs retire
    if (leader) {
        prefetch_tensormap(&tm_s);
#pragma unroll
        for (int i = 0; i < NSQ + NP; ++i) mbar_init(&bar[i], 1);
        fence_mbar_init();
    }
    __syncthreads();
    pdl_wait();     // fields written by the previous kernel are read from here on

    // own cells and ring chunk
    const bool has_h = tid < NH;
    // the ring: rows y0-2, y0-1, y0+TY, y0+TY+1 over the tile's columns, and
    // columns x0-2..x0-1, x0+64..x0+65 over the tile's rows (the corners are
    // not operands of the second stage)
    int hex = 0, hey = 0;
    if (tid < NHR) {
        const int r = tid / (TX / 2);
        hey = r < 2 ? r : TY + r;
        hex = 2 + 2 * (tid % (TX / 2));
    } else if (has_h) {
        const int d = tid - NHR;
        hey = 2 + (d >> 1);
        hex = (d & 1) ? WE - 2 : 0;
    }
    // byte offsets in the slots
    const uint32_t m_s8 = ((row + 4) * WB + 2 * px + 4) * 8;
    const uint32_t m_e8 = ((row + 2) * WE + 2 * px + 2) * 8;
    [[maybe_unused]] const uint32_t m_a8 = (row * TX + 2 * px) * 8;
    const uint32_t h_s8 = ((hey + 2) * WB + hex + 2) * 8;
    const uint32_t h_e8 = (hey * WE + hex) * 8;
    constexpr uint32_t EBYTES = SE * 8;
    [[maybe_unused]] constexpr uint32_t SEBYTES = SE * 8;
    const uint32_t s_base = smem_u32(sb), e_base = smem_u32(es);
    [[maybe_unused]] const uint32_t p_base = smem_u32(ps);

    // This CTA's planes: [g_lo, g_hi) of all (tile, z) planes, tiles ordered x
    // fastest, then y, then item.  A segment is the part inside one tile; each
    // segment pays 4 extra plane iterations to fill the pipeline.
    // Groups of cy consecutive CTAs take y-adjacent tiles (same x tile, same
    // item) over the same plane range; the grid is one wave, so a group's
    // CTAs march their planes together and the halo rows they share are read
    // from HBM once.
    const int groups_y = (a.tiles_y + a.cy - 1) / a.cy;
    const int groups_xy = a.tiles_x * groups_y;
    const int total = groups_xy * a.items * a.nk;
    const int member = blockIdx.x % a.cy;
    const int g_lo = (blockIdx.x / a.cy) * a.span;
    const int g_hi = min(g_lo + a.span, total);
    unsigned U = 0, VP = 0;  // stencil / pointwise planes this CTA has loaded: ring positions
    for (int g = g_lo; g < g_hi;) {
        const int grp = g / a.nk;
        const int z0 = g - grp * a.nk;
        const int z1 = min(a.nk, z0 + (g_hi - g));
        g += z1 - z0;
        const int b = grp / groups_xy;
        const int gxy = grp - b * groups_xy;
        const int ty = (gxy / a.tiles_x) * a.cy + member;
        if (ty >= a.tiles_y) continue;                             // a partial group's spare CTA
        if (a.item_lo && b + a.item_base < *a.item_lo) continue;  // the same for all threads
        const int x0 = (gxy % a.tiles_x) * TX;
        const int y0 = ty * TY;
        const int nv = z1 - z0 + 4;      // first-stage planes z0-2 .. z1+1
        const int nu = z1 - z0 + 8;      // stencil planes z0-4 .. z1+3
        const int zs = b * a.pz + z0;    // tensor-map plane of stencil plane 0 (interior z0-4)

        // stencil plane u -> ring position U+u; pointwise plane v -> VP+v
        auto issue_s = [&](int u) {
            const int s = (int)((U + u) % NSQ);
            mbar_arrive_expect_tx(&bar[s], SBYTES);
            tma_load_3d(sb + s * SB, &tm_s, x0, y0, zs + u, &bar[s]);  // interior (x0-4, y0-4)
        };
        auto issue_p = [&](int v) {
            const int s = (int)((VP + v) % NP);
            mbar_arrive_expect_tx(&bar[NSQ + s], PBYTES);
            double* d = ps + s * SP;
            tma_load_3d(d, &tm_q, x0 + 2, y0 + 2, zs + 2 + v, &bar[NSQ + s]);       // q, interior (x0-2, y0-2)
            tma_load_3d(d + SE, &tm_a, x0 + 4, y0 + 4, zs + 2 + v, &bar[NSQ + s]);  // acc, interior (x0, y0)
        };
        int s_hi = -1, p_hi = -1;  // highest planes issued (leader)
        if (leader) {
            fence_proxy_async_smem();  // the slots were last read by the previous segment
            for (int u = 0; u < NSQ && u < nu; ++u) { issue_s(u); s_hi = u; }
            if constexpr (PAIR == 1)
                for (int v = 0; v < NP && v < nv; ++v) { issue_p(v); p_hi = v; }
        }
        auto drain = [&](int s_done, int p_done) {
            if (!leader) return;
            for (int u = s_done + 1; u <= s_hi; ++u)
                (void)mbar_wait_bounded(&bar[(U + u) % NSQ], (uint32_t)(((U + u) / NSQ) & 1));
            for (int v = p_done + 1; v <= p_hi; ++v)
                (void)mbar_wait_bounded(&bar[NSQ + (VP + v) % NP], (uint32_t)(((VP + v) / NP) & 1));
        };

        bool bad = false;
        // Register windows of the own cells, indexed by plane mod 5 so that the
        // loop, unrolled by 5, renames registers instead of moving them:
        //   qw[u % 5]: stencil input at stencil plane u (planes v .. v+4 live)
        //   ew[p % 5]: first-stage value at first-stage plane p (p = v-4 .. v)
        //   aw[p % 5]: first-stage accumulator partial (p = v-2 .. v)
        //   sa[u % 5]: shared address of the slot of stencil plane u
        V2 qw[5], ew[5];
        [[maybe_unused]] V2 aw[5];  // pair 3+4 only
        [[maybe_unused]] V2 hw[5];  // pair 1+2: the ring chunk's stencil input, like qw
        uint32_t sa[5];
#pragma unroll
        for (int u = 0; u < 4; ++u) {  // prologue: stencil planes 0..3
            const unsigned gu = U + u;
            if (!mbar_wait_bounded(&bar[gu % NSQ], (gu / NSQ) & 1)) bad = true;
            sa[u] = s_base + (gu % NSQ) * SBYTES;
            qw[u] = lds2(sa[u] + m_s8);
            if constexpr (PAIR == 0) hw[u] = lds2(sa[u] + h_s8);
        }
        sa[4] = 0;
#pragma unroll
        for (int u = 0; u < 5; ++u) ew[u] = aw[u] = V2{};

        const int x = x0 + 2 * px;
        const int y = y0 + row;
        const bool live = x < a.ni && y < a.nj;
        const bool full = x + 2 <= a.ni;
        // whether the cells have periodic images in x or y (image depth hd)
        const int hd = PAIR == 0 ? 4 : a.o_halo;
        // lanes next to an x face add their x-images to the 16-byte store; rows
        // and planes next to a y or z face (and an odd ni's last pair) take the
        // general image path
        const bool x_img = x < hd || x + 2 > a.ni - hd;
        const bool y_img = y < hd || y >= a.nj - hd || !full;
        // the own cells' output columns at plane z0-4 (one plane further per iteration)
        double* ocol;
        [[maybe_unused]] double* acol = nullptr;
        if constexpr (PAIR == 0) {
            const long long ob = (long long)b * a.item_stride + a.origin + (long long)(z0 - 4) * a.plane +
                                 (long long)y * a.px + x;
            ocol = a.yout + ob;
            acol = a.aout + ob;
        } else {
            ocol = a.qout + (long long)b * a.o_item_stride + a.o_origin + (long long)(z0 - 4) * a.o_plane +
                   (long long)y * a.o_px + x;
        }

        int s_4 = (int)((U + 4) % NSQ);             // slot and phase of stencil plane v+4
        uint32_t ph_4 = ((U + 4) / NSQ) & 1;
        uint32_t e_cur = e_base;                    // first-stage slot of plane v (3 slots)
        int sp_v = (int)(VP % NP);                  // pointwise slot and phase of plane v
        uint32_t ph_p = (VP / NP) & 1;

        // One plane iteration; K = v mod 5.  Returns false when the CTA must stop.
        auto iterate = [&](auto kc, int v) -> bool {
            constexpr int K = decltype(kc)::value;
            if (!mbar_wait_bounded(&bar[s_4], ph_4)) bad = true;
            sa[(K + 4) % 5] = s_base + s_4 * SBYTES;
            const uint32_t S0 = sa[K], S1 = sa[(K + 1) % 5], S2 = sa[(K + 2) % 5], S3 = sa[(K + 3) % 5],
                           S4 = sa[(K + 4) % 5];
            qw[(K + 4) % 5] = lds2(S4 + m_s8);
            (void)S0; (void)S1; (void)S3;
            [[maybe_unused]] uint32_t PW = 0;
            if constexpr (PAIR == 1) {
                if (!mbar_wait_bounded(&bar[NSQ + sp_v], ph_p)) bad = true;
                PW = p_base + sp_v * PBYTES;
            }
            const uint32_t E = e_cur;
            const uint32_t E2 = E == e_base + 2 * EBYTES ? e_base : E + EBYTES;  // slot of first-stage plane v-2

            // first stage, own cells (first-stage plane v, stencil centre v+2;
            // the centre value is the window's)
            {
                double k[2];
                rhs_s<WB>(a.w, S2 + m_s8, qw[(K + 2) % 5], qw[K], qw[(K + 1) % 5], qw[(K + 3) % 5], qw[(K + 4) % 5], k);
                V2 en;
                if constexpr (PAIR == 0) {
                    const V2& c = qw[(K + 2) % 5];
#pragma unroll
                    for (int e = 0; e < 2; ++e) en.v[e] = fmaT(a.c1y, k[e], c.v[e]);
                } else {
                    // y3, and acc + (y3 - q)/3 (= acc + dt/3 k3) for the fourth stage
                    const V2 qv = lds2(PW + m_e8);
                    const V2 av = lds2(PW + SEBYTES + m_a8);
                    V2 an;
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        en.v[e] = fmaT(a.c1y, k[e], qv.v[e]);
                        an.v[e] = add_third(en.v[e], qv.v[e], av.v[e]);
                    }
                    aw[K] = an;
                }
                sts2(E + m_e8, en);
                ew[K] = en;
            }
            // first stage, ring chunk
            if (has_h) {
                V2 zm2, zm1, cen, zp1, zp2;
                if constexpr (PAIR == 0) {  // z-window in registers (pair 1+2 has them to spare)
                    hw[(K + 4) % 5] = lds2(S4 + h_s8);
                    zm2 = hw[K]; zm1 = hw[(K + 1) % 5]; cen = hw[(K + 2) % 5];
                    zp1 = hw[(K + 3) % 5]; zp2 = hw[(K + 4) % 5];
                } else {
                    zm2 = lds2(S0 + h_s8); zm1 = lds2(S1 + h_s8);
                    zp1 = lds2(S3 + h_s8); zp2 = lds2(S4 + h_s8);
                    cen = lds2(S2 + h_s8);
                }
                double k[2];
                rhs_s<WB>(a.w, S2 + h_s8, cen, zm2, zm1, zp1, zp2, k);
                V2 base = cen, hv;
                if constexpr (PAIR == 1) base = lds2(PW + h_e8);
#pragma unroll
                for (int e = 0; e < 2; ++e) hv.v[e] = fmaT(a.c1y, k[e], base.v[e]);
                sts2(E + h_e8, hv);
            }
            // second stage on plane z0-4+v (first-stage plane v-2, stencil plane v)
            if (v >= 4) {
                double k[2];
                rhs_s<WE>(a.w, E2 + m_e8, ew[(K + 3) % 5], ew[(K + 1) % 5], ew[(K + 2) % 5], ew[(K + 4) % 5], ew[K], k);
                V2 o;
                [[maybe_unused]] V2 oa;
                if constexpr (PAIR == 0) {
                    // y2, and acc = q + (y1 - q)/3 + dt/3 k2
                    const V2& qc = qw[K];
                    const V2& y1 = ew[(K + 3) % 5];
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        o.v[e] = fmaT(a.c2y, k[e], qc.v[e]);
                        oa.v[e] = fmaT(a.c2a, k[e], add_third(y1.v[e], qc.v[e], qc.v[e]));
                    }
                } else {
                    const V2& ap = aw[(K + 3) % 5];
#pragma unroll
                    for (int e = 0; e < 2; ++e) o.v[e] = fmaT(a.c2a, k[e], ap.v[e]);
                }
                if (live) {
                    const int z = z0 - 4 + v;
                    if (!y_img && z >= hd && z < a.nk - hd) {
                        gst16<double>(a.sb_o, ocol, o);
                        if (x_img) {
#pragma unroll
                            for (int e = 0; e < 2; ++e) {
                                const int xe = x + e;
                                if (xe < hd) gst1(a.sb_o, ocol + e + a.ni, o.v[e]);
                                if (xe >= a.ni - hd) gst1(a.sb_o, ocol + e - a.ni, o.v[e]);
                            }
                        }
                    } else if constexpr (PAIR == 0) {
                        store_images_pair(a.sb_o, a.yout + (long long)b * a.item_stride + a.origin, a.px, a.plane,
                                          a.ni, a.nj, a.nk, 4, x, y, z, o);
                    } else {
                        store_images_pair(a.sb_o, a.qout + (long long)b * a.o_item_stride + a.o_origin, a.o_px,
                                          a.o_plane, a.ni, a.nj, a.nk, a.o_halo, x, y, z, o);
                    }
                    if constexpr (PAIR == 0) {
                        if (full) gst16<double>(a.sb_a, acol, oa);
                        else gst1(a.sb_a, acol, oa.v[0]);
                    }
                }
            }
            ocol += PAIR == 0 ? a.plane : a.o_plane;
            if constexpr (PAIR == 0) acol += a.plane;
            if (__syncthreads_or(bad)) {
                if (leader) atomicExch(a.err, DEV_WAIT_TIMEOUT);
                drain(v + 4, v);
                return false;
            }
            if (leader) {
                fence_proxy_async_smem();
                if (v + NSQ < nu) { issue_s(v + NSQ); s_hi = v + NSQ; }
                if constexpr (PAIR == 1)
                    if (v + NP < nv) { issue_p(v + NP); p_hi = v + NP; }
            }
            if (++s_4 == NSQ) { s_4 = 0; ph_4 ^= 1u; }
            e_cur = E == e_base + 2 * EBYTES ? e_base : E + EBYTES;
            if constexpr (PAIR == 1)
                if (++sp_v == NP) { sp_v = 0; ph_p ^= 1u; }
            return true;
        };

        for (int vb = 0; vb < nv; vb += 5) {  // nv is uniform over the CTA
            if (!iterate(std::integral_constant<int, 0>{}, vb)) return;
            if (vb + 1 < nv && !iterate(std::integral_constant<int, 1>{}, vb + 1)) return;
            if (vb + 2 < nv && !iterate(std::integral_constant<int, 2>{}, vb + 2)) return;
            if (vb + 3 < nv && !iterate(std::integral_constant<int, 3>{}, vb + 3)) return;
            if (vb + 4 < nv && !iterate(std::integral_constant<int, 4>{}, vb + 4)) return;
        }

        U += nu;
        if constexpr (PAIR == 1) VP += nv;
    }
}




// ---------------------------------------------------------------------------
// Widening: interior of a caller-layout field -> internal field with every
// periodic image within 4 cells of a face.
__global__ void k_widen(double* dst, Geo gd, const double* src, Geo gs, int items, const int* item_lo,
                        int item_base, StoreBounds bounds) {
    pdl_trigger();
    pdl_wait();
    const long long n = (long long)gd.ni * gd.nj * gd.nk;
    const int b = blockIdx.y;
    if (item_lo && b + item_base < *item_lo) return;
    const double* sb = src + (long long)b * gs.total + gs.origin;
    double* db = dst + (long long)b * gd.total + gd.origin;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % gd.ni);
        const int y = (int)((t / gd.ni) % gd.nj);
        const int z = (int)(t / ((long long)gd.ni * gd.nj));
        const double v = sb[(long long)z * gs.plane + (long long)y * gs.px + x];
        const int hd = gd.halo;
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
            if (iz == 1 && !(z < hd)) continue;
            if (iz == 2 && !(z >= gd.nk - hd)) continue;
            const int zz = iz == 0 ? z : (iz == 1 ? z + gd.nk : z - gd.nk);
#pragma unroll
            for (int iy = 0; iy < 3; ++iy) {
                if (iy == 1 && !(y < hd)) continue;
                if (iy == 2 && !(y >= gd.nj - hd)) continue;
                const int yy = iy == 0 ? y : (iy == 1 ? y + gd.nj : y - gd.nj);
                double* r = db + (long long)zz * gd.plane + (long long)yy * gd.px;
                gst1(bounds, r + x, v);
                if (x < hd) gst1(bounds, r + x + gd.ni, v);
                if (x >= gd.ni - hd) gst1(bounds, r + x - gd.ni, v);
            }
        }
    }
}

template <int PAIR, int TY, int NSQ, int NP, int TXP>
cudaError_t launch_pair_T(const Geo& g4, const Geo& go, const PairLaunch& L, const Shape& sh, cudaStream_t s,
                          int* err) {
    using S = PairShape<TY, NSQ, NP, PAIR, TXP>;
    CUtensorMap ts{}, tq{}, ta{};
    if (!make_tmap(&ts, g4, PAIR == 0 ? L.q : L.y2, L.items, S::WB, S::HB)) return cudaErrorInvalidValue;
    if (PAIR == 1) {
        if (!make_tmap(&tq, g4, L.q, L.items, S::WE, S::HE)) return cudaErrorInvalidValue;
        if (!make_tmap(&ta, g4, L.acc, L.items, S::TX, TY)) return cudaErrorInvalidValue;
    }
    PairArgs a{};
    a.item_stride = g4.total; a.origin = g4.origin; a.px = g4.px; a.plane = g4.plane;
    a.ni = g4.ni; a.nj = g4.nj; a.nk = g4.nk; a.pz = (int)g4.pz;
    a.tiles_x = (g4.ni + S::TX - 1) / S::TX;
    a.tiles_y = (g4.nj + TY - 1) / TY;
    a.items = L.items;
    a.cy = a.tiles_y % 4 == 0 ? 4 : (a.tiles_y % 2 == 0 ? 2 : 1);
    const long long total = (long long)a.tiles_x * (a.tiles_y / a.cy + (a.tiles_y % a.cy != 0)) * L.items * g4.nk;
    if (total >= 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    if (sh.zchunk > 0) {
        a.span = sh.zchunk;
    } else {  // persistent: one range per resident CTA (resident CTAs per device cached)
        static std::atomic<int> cached[64];  // zero-initialised (static storage)
        int dev = 0;
        cudaGetDevice(&dev);
        int ctas_dev = (dev >= 0 && dev < 64) ? cached[dev].load(std::memory_order_relaxed) : 0;
        if (ctas_dev == 0) {
            int sms = 0, occ = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rk4_pair<PAIR, TY, NSQ, NP, TXP>, S::NT, S::smem);
            ctas_dev = std::max(1, sms) * std::max(1, occ);
            if (dev >= 0 && dev < 64) cached[dev].store(ctas_dev, std::memory_order_relaxed);
        }
        const long long ctas = std::max(1LL, (long long)ctas_dev / a.cy);  // groups
        a.span = (int)std::max(1LL, (total + ctas - 1) / ctas);
    }
    a.item_lo = L.item_lo;
    a.item_base = L.item_base;
    fill_w13<double>(a.w, L.coef, L.nu);
    const double dthalf = L.dt * .5;
    if (PAIR == 0) {  // the coefficients of stages 1 and 2 of the single-stage path
        a.c1y = dthalf; a.c2y = dthalf; a.c2a = L.dt / 3.;
        a.yout = static_cast<double*>(L.y2);
        a.aout = static_cast<double*>(L.acc);
        a.sb_o = out_bounds(a.yout, g4, L.items);
        a.sb_a = out_bounds(a.aout, g4, L.items);
    } else {          // stages 3 and 4
        a.c1y = L.dt; a.c2a = L.dt / 6.;
        a.qout = static_cast<double*>(L.out);
        a.o_item_stride = go.total; a.o_origin = go.origin; a.o_px = go.px; a.o_plane = go.plane;
        a.o_halo = go.halo;
        a.sb_o = out_bounds(a.qout, go, L.items);
    }
    a.err = err;
    const long long nct = (total + a.span - 1) / a.span * a.cy;
    if (nct > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    const dim3 grid((unsigned)nct);
    return launch_pdl(k_rk4_pair<PAIR, TY, NSQ, NP, TXP>, grid, dim3(S::NT), S::smem, s, ts, tq, ta, a);
}

template <int PAIR, int TY, int NSQ, int NP, int TXP = 64>
cudaError_t set_pair_attr() {
    return cudaFuncSetAttribute(k_rk4_pair<PAIR, TY, NSQ, NP, TXP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)PairShape<TY, NSQ, NP, PAIR, TXP>::smem);
}

unsigned grid_cells(long long n) {
    const long long b = (n + 255) / 256;
    return (unsigned)(b < 148 * 16 ? b : 148 * 16);
}

}  // namespace

bool pair_supported(const Geo& g) { return g.es == 8 && g.ni >= 4 && g.nj >= 4 && g.nk >= 4; }

unsigned long long take_store_violations_pairs() {
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_store_violations, sizeof v) != cudaSuccess) return 0;
    const unsigned int zero = 0;
    cudaMemcpyToSymbol(g_store_violations, &zero, sizeof zero);
    return v;
}

cudaError_t prepare_pairs() {
    cudaError_t e = set_pair_attr<0, 8, 7, 2>();
    if (e == cudaSuccess) e = set_pair_attr<1, 8, 7, 2>();
    if (e == cudaSuccess) e = set_pair_attr<0, 16, 7, 2>();
    if (e == cudaSuccess) e = set_pair_attr<1, 16, 7, 2>();
    if (e == cudaSuccess) e = set_pair_attr<0, 16, 7, 2, 32>();
    if (e == cudaSuccess) e = set_pair_attr<1, 16, 7, 2, 32>();
    return e;
}

cudaError_t launch_pair(const Geo& g4, const Geo& go, const PairLaunch& L, const Shape& sh, cudaStream_t s,
                        int* err) {
    add_launches(1);
    if (!pair_supported(g4) || g4.halo != 4 || sh.zchunk < 0) return cudaErrorInvalidValue;
    // tile 64 x 8, 64 x 16 (one row per warp) or 32 x 16 (two rows per warp)
    const bool narrow = sh.tx == 32;
    if (narrow && sh.ty != 16) return cudaErrorInvalidValue;
    if (L.pair == 0) {
        if (narrow) return launch_pair_T<0, 16, 7, 2, 32>(g4, go, L, sh, s, err);
        if (sh.ty == 8) return launch_pair_T<0, 8, 7, 2, 64>(g4, go, L, sh, s, err);
        if (sh.ty == 16) return launch_pair_T<0, 16, 7, 2, 64>(g4, go, L, sh, s, err);
    } else {
        if (narrow) return launch_pair_T<1, 16, 7, 2, 32>(g4, go, L, sh, s, err);
        if (sh.ty == 8) return launch_pair_T<1, 8, 7, 2, 64>(g4, go, L, sh, s, err);
        if (sh.ty == 16) return launch_pair_T<1, 16, 7, 2, 64>(g4, go, L, sh, s, err);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_widen(const Geo& g4, void* dst, const Geo& gs, const void* src, int items, const int* item_lo,
                         int item_base, cudaStream_t s) {
    add_launches(1);
    if (g4.es != 8 || gs.es != 8 || items < 1 || items > 65535) return cudaErrorInvalidValue;
    dim3 grid(grid_cells((long long)g4.ni * g4.nj * g4.nk), items);
    return launch_pdl(k_widen, grid, dim3(256), 0, s, static_cast<double*>(dst), g4,
                      static_cast<const double*>(src), gs, items, item_lo, item_base, out_bounds(dst, g4, items));
}

}  // namespace sp
