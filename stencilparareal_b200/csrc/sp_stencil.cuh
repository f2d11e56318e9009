// sp_stencil.cuh -- the fourth-order right-hand side as 13 per-offset weights,
// shared by the single-stage kernels (sp_kernels.cu) and the fused stage
// pairs (sp_fused.cu), plus the tensor-map helper both use.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdlib>
#include <utility>

#include "sp_device.cuh"
#include "sp_internal.h"

namespace sp {

// R4 as 13 per-offset weights of the reference's coefficients
// (RHS4 of src/Convection/Convection.cpp:40-112):
//   ca_d (8(q[-1]-q[+1]) - (q[-2]-q[+2])) + nl (16 S1 - S2 - 90 q),  nl = nu/(12 dx^2).
template <typename T>
struct W13 {
    T m1[3], p1[3], m2[3], p2[3], c;
};

template <typename T>
inline void fill_w13(W13<T>& w, const Coef& c, double nu) {
    const double nl = nu * c.s4;
    for (int d = 0; d < 3; ++d) {
        w.m1[d] = (T)(8. * c.ca[d] + 16. * nl);
        w.p1[d] = (T)(-8. * c.ca[d] + 16. * nl);
        w.m2[d] = (T)(-c.ca[d] - nl);
        w.p2[d] = (T)(c.ca[d] - nl);
    }
    w.c = (T)(-90. * nl);
}

// The 13 stencil operands of one cell.
template <typename T>
struct Nb {
    T c, xm1, xp1, xm2, xp2, ym1, yp1, ym2, yp2, zm1, zp1, zm2, zp2;
};

// FP64: the 13 products.  FP32 (the coarse propagator): the weights sum to
// zero (the stencils are consistent), so R = sum over the 12 neighbours of
// w_o (q_o - q_c) exactly; the differences of nearby values are exact in FP32
// and small, where the 13 products of O(1) values with weights up to
// 90 nu/(12 dx^2) would cancel to a result ~1e-4 as large as themselves, and
// the FP32-rounded weights would no longer sum to zero (a drift of every
// field, ~7e-7 per 7 coarse steps at 128^3).
template <typename T>
__device__ __forceinline__ T rhs_w13(const W13<T>& w, const Nb<T>& s) {
    if constexpr (sizeof(T) == 4) {
        const T c = s.c;
        const T sx = fmaT(w.m2[0], s.xm2 - c, fmaT(w.m1[0], s.xm1 - c, fmaT(w.p1[0], s.xp1 - c, w.p2[0] * (s.xp2 - c))));
        const T sy = fmaT(w.m2[1], s.ym2 - c, fmaT(w.m1[1], s.ym1 - c, fmaT(w.p1[1], s.yp1 - c, w.p2[1] * (s.yp2 - c))));
        const T sz = fmaT(w.m2[2], s.zm2 - c, fmaT(w.m1[2], s.zm1 - c, fmaT(w.p1[2], s.zp1 - c, w.p2[2] * (s.zp2 - c))));
        return (sx + sy) + sz;
    } else {
        const T sx = fmaT(w.m2[0], s.xm2, fmaT(w.m1[0], s.xm1, fmaT(w.p1[0], s.xp1, w.p2[0] * s.xp2)));
        const T sy = fmaT(w.m2[1], s.ym2, fmaT(w.m1[1], s.ym1, fmaT(w.p1[1], s.yp1, w.p2[1] * s.yp2)));
        const T sz = fmaT(w.m2[2], s.zm2, fmaT(w.m1[2], s.zm1, fmaT(w.p1[2], s.zp1, w.p2[2] * s.zp2)));
        return fmaT(w.c, s.c, (sx + sy) + sz);
    }
}

// The accumulator terms of the low-storage RK4 step recovered from stage
// values: dt/6 k1 = (y1 - q)/3 and dt/3 k3 = (y3 - q)/3, so that no stage
// before the second writes the accumulator and the third neither reads nor
// writes it.  Returns base + (y - q)/3.
template <typename T>
__device__ __forceinline__ T add_third(T y, T q, T base) {
    return fmaT(y - q, T(1.0 / 3.0), base);
}

// Launches a kernel with programmatic stream serialization (kernels launched
// this way call pdl_trigger/pdl_wait), so that in a stream or a captured graph the
// next kernel's CTAs start while this one's last CTAs finish.
template <typename... KP, typename... A>
cudaError_t launch_pdl(void (*k)(KP...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

// Byte range of `items` fields of geometry g from `base`: the allocation a
// launch writes, checked by the bounds-checked build's stores.  In that build
// SP_BOUNDS_SHRINK_PLANES=n (environment) narrows the range by n planes at its
// top, so that a test can see the checker count (and skip) stores that lie
// inside the real allocation.
inline StoreBounds out_bounds(const void* base, const Geo& g, int items) {
    StoreBounds b;
    if (!base) return b;
    b.lo = static_cast<const char*>(base);
    long long bytes = (long long)items * g.total * g.es;
#if SP_BOUNDS_CHECK
    static const long long shrink = [] {
        const char* e = std::getenv("SP_BOUNDS_SHRINK_PLANES");
        return e ? std::atoll(e) : 0LL;
    }();
    bytes -= shrink * g.plane * g.es;
#endif
    b.hi = b.lo + bytes;
    return b;
}

// Tensor map over `items` fields of geometry g starting at `base`: dims
// (px, py, pz*items), box (bw, bh, 1), no swizzle, out-of-range reads as zero.
bool make_tmap(CUtensorMap* tm, const Geo& g, const void* base, int items, int bw, int bh);

}  // namespace sp
