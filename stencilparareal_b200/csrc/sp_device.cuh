// sp_device.cuh -- device-side building blocks: PTX wrappers for mbarriers and
// TMA tensor loads (sm_90+/sm_100a), 16-byte vector access, bounded waits.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace sp {

// A bounded wait gives up after this many nanoseconds of %globaltimer, sets
// the device error word and lets the kernel return (no trap, no endless spin).
constexpr unsigned long long kWaitLimitNs = 2000000000ull;

// Device error word values.
enum : int { DEV_OK = 0, DEV_WAIT_TIMEOUT = 1 };

// Bounds-checked stores (library built with -DSP_BOUNDS_CHECK=1): every global
// store of the stencil-producing kernels is tested against the byte range of
// its output allocation; a store outside it is skipped and counted in this
// module's violation word (read by sp_store_violations).  Without the flag the
// test compiles away.
#ifndef SP_BOUNDS_CHECK
#define SP_BOUNDS_CHECK 0
#endif
struct StoreBounds {
    const char* lo = nullptr;  // first byte of the output allocation
    const char* hi = nullptr;  // one past its last byte
};
static __device__ unsigned int g_store_violations;
__device__ __forceinline__ bool store_ok(const StoreBounds& b, const void* p, int bytes) {
#if SP_BOUNDS_CHECK
    const char* c = static_cast<const char*>(p);
    if (c >= b.lo && c + bytes <= b.hi) return true;
    atomicAdd(&g_store_violations, 1u);
    return false;
#else
    (void)b; (void)p; (void)bytes;
    return true;
#endif
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) accesses to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of the barrier; false after limit_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  unsigned long long limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0 && globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// 3-D tiled TMA load global -> shared, completion signalled on `bar`
// (transaction bytes).  No multicast: the tensor always lies in this GPU's HBM.
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* tm, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Programmatic dependent launch: let the next kernel of the stream start its
// CTAs (they run up to their own pdl_wait), and wait until the previous
// kernel of the stream has completed with its memory visible.  Both are
// no-ops for kernels launched without the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap* tm) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tm)) : "memory");
}

// ---- 16-byte vectors --------------------------------------------------------
template <typename T>
struct V16;
template <>
struct V16<double> {
    static constexpr int N = 2;
};
template <>
struct V16<float> {
    static constexpr int N = 4;
};

template <typename T, int N>
struct Vec {
    T v[N];
};

template <typename T>
__device__ __forceinline__ Vec<T, V16<T>::N> ld16(const T* p) {
    Vec<T, V16<T>::N> r;
    if constexpr (sizeof(T) == 8) {
        const double2 d = *reinterpret_cast<const double2*>(p);
        r.v[0] = d.x;
        r.v[1] = d.y;
    } else {
        const float4 d = *reinterpret_cast<const float4*>(p);
        r.v[0] = d.x;
        r.v[1] = d.y;
        r.v[2] = d.z;
        r.v[3] = d.w;
    }
    return r;
}

template <typename T>
__device__ __forceinline__ void st16(T* p, const Vec<T, V16<T>::N>& r) {
    if constexpr (sizeof(T) == 8) {
        *reinterpret_cast<double2*>(p) = make_double2(r.v[0], r.v[1]);
    } else {
        *reinterpret_cast<float4*>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
    }
}

// Global stores of the stencil-producing kernels, checked against the output
// allocation `b` when the library is built with SP_BOUNDS_CHECK.
template <typename T>
__device__ __forceinline__ void gst1(const StoreBounds& b, T* p, T v) {
    if (store_ok(b, p, (int)sizeof(T))) *p = v;
}
template <typename T>
__device__ __forceinline__ void gst16(const StoreBounds& b, T* p, const Vec<T, V16<T>::N>& r) {
    if (store_ok(b, p, 16)) st16<T>(p, r);
}

// 16-byte shared-memory access by 32-bit shared address (offset OFF bytes).
__device__ __forceinline__ Vec<double, 2> lds2(uint32_t addr) {
    Vec<double, 2> r;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(r.v[0]), "=d"(r.v[1]) : "r"(addr));
    return r;
}
template <int OFF>
__device__ __forceinline__ Vec<double, 2> lds2o(uint32_t addr) {
    Vec<double, 2> r;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2+%3];" : "=d"(r.v[0]), "=d"(r.v[1]) : "r"(addr), "n"(OFF));
    return r;
}
// 16 bytes of T (2 doubles / 4 floats) by 32-bit shared address, plus OFF bytes.
template <typename T, int OFF = 0>
__device__ __forceinline__ Vec<T, V16<T>::N> lds16(uint32_t addr) {
    Vec<T, V16<T>::N> r;
    if constexpr (sizeof(T) == 8) {
        asm volatile("ld.shared.v2.f64 {%0, %1}, [%2+%3];" : "=d"(r.v[0]), "=d"(r.v[1]) : "r"(addr), "n"(OFF));
    } else {
        asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4+%5];"
                     : "=f"(r.v[0]), "=f"(r.v[1]), "=f"(r.v[2]), "=f"(r.v[3])
                     : "r"(addr), "n"(OFF));
    }
    return r;
}
__device__ __forceinline__ void sts2(uint32_t addr, const Vec<double, 2>& v) {
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v.v[0]), "d"(v.v[1]) : "memory");
}

// ---- thread-block clusters ---------------------------------------------------
__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_size() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
// All threads of all CTAs of the cluster (hardware barrier, like __syncthreads).
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Shared-memory address of the same variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t map_rank(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
// 16 bytes into another CTA's shared memory; the store counts its bytes off
// the transaction count of that CTA's mbarrier `rbar` when it lands.
__device__ __forceinline__ void st_async2(uint32_t addr, const Vec<double, 2>& v, uint32_t rbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(addr),
                 "d"(v.v[0]), "d"(v.v[1]), "r"(rbar)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx_u32(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait_cluster(uint32_t addr, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster_bounded(uint32_t addr, uint32_t parity,
                                                          unsigned long long limit_ns = kWaitLimitNs) {
    if (mbar_try_wait_cluster(addr, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait_cluster(addr, parity)) return true;
        if ((it & 63u) == 0 && globaltimer_ns() - t0 > limit_ns) return false;
    }
}
// One arrival (release at cluster scope) on an mbarrier of another CTA of the cluster.
__device__ __forceinline__ void mbar_arrive_remote(uint32_t addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(addr) : "memory");
}


template <typename T>
__device__ __forceinline__ T fmaT(T a, T b, T c) {
    if constexpr (sizeof(T) == 8) return fma(a, b, c);
    else return fmaf(a, b, c);
}

}  // namespace sp
