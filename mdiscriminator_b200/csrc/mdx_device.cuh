// mdx_device.cuh -- device building blocks shared by the partition kernels:
// discriminator functors, bounded waits, mbarrier + bulk-copy (TMA) helpers,
// warp scans.  sm_100a only.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mdx {

constexpr int kMaxClasses = 64;

// Bounded waits: every spin in these kernels gives up after this long, latches
// an error in the workspace and lets the kernel return (no trap, no hang).
constexpr uint64_t kWaitLimitNs = 1000ull * 1000ull * 1000ull;  // 1 s

// Error bits latched in the workspace header.
constexpr uint32_t kErrTimeout = 1u;
constexpr uint32_t kErrSegments = 2u;
constexpr uint32_t kErrCounts = 4u;  // distributed: other ranks' class counts inconsistent

// ----------------------------------------------------------- discriminators --
// The reference's functor concept (HelpersCommon.h:587-596, 840-849,
// 1200-1210) is `static unsigned apply(InType)` with TupleType::cardinal = m.
// Here a discriminator is a small value object so that m can be a run-time
// parameter of a pre-instantiated kernel; the class always comes from the
// element's first 32-bit word (the whole element for u32, the key of an
// 8-byte {key, payload} record -- ModArray<N,2>::apply = x[0] % N,
// MdiscrHost_arrays.cu.h:33-35).

// 16-byte record {u32 key; 12 bytes of payload}: ModArray<N,4> over arrays of
// four unsigned ints (MdiscrHost_arrays.cu.h:26-36, class from x[0]).
struct alignas(16) Rec16 {
    uint32_t w[4];
};

template <class V>
__host__ __device__ __forceinline__ uint32_t key_of(const V& v);
template <>
__host__ __device__ __forceinline__ uint32_t key_of<uint32_t>(const uint32_t& v) { return v; }
template <>
__host__ __device__ __forceinline__ uint32_t key_of<uint64_t>(const uint64_t& v) {
    return static_cast<uint32_t>(v);  // little-endian {u32 key; u32 payload}
}
template <>
__host__ __device__ __forceinline__ uint32_t key_of<Rec16>(const Rec16& v) {
    return v.w[0];
}

// class = key & (m-1): Mod4 / Mod8 (x & 3, x & 7).
struct DiscrMask {
    uint32_t mask;
    template <class V>
    __host__ __device__ __forceinline__ uint32_t operator()(const V& v) const {
        return key_of(v) & mask;
    }
};

// class = key % m: Mod<N> (x % N).  The remainder uses the direct-remainder
// method of Lemire, Kaser and Kurz, "Faster Remainder by Direct Computation"
// (2019): with c = floor((2^64 - 1) / m) + 1, key % m = hi64((c * key mod 2^64) * m),
// exact for every 32-bit key and m >= 1 (c wraps to 0 for m = 1, giving 0).
struct DiscrMod {
    uint64_t c;
    uint32_t m;
    __host__ __device__ static DiscrMod make(uint32_t m_) {
        DiscrMod d;
        d.m = m_;
        d.c = ~0ull / m_ + 1ull;
        return d;
    }
    template <class V>
    __host__ __device__ __forceinline__ uint32_t operator()(const V& v) const {
        const uint64_t low = c * static_cast<uint64_t>(key_of(v));
#ifdef __CUDA_ARCH__
        return static_cast<uint32_t>(__umul64hi(low, static_cast<uint64_t>(m)));
#else
        return static_cast<uint32_t>((static_cast<unsigned __int128>(low) * m) >> 64);
#endif
    }
};

// Adapter for a reference-style functor (static apply, TupleType::cardinal);
// used by the C++ drop-in templates in include/mdx/mdiscr.cuh.  Classes at or
// above the template bound are clamped so a wrong functor cannot write out of
// bounds on the device.
template <class DISCR, int M>
struct DiscrStatic {
    template <class V>
    __host__ __device__ __forceinline__ uint32_t operator()(const V& v) const {
        static_assert(sizeof(typename DISCR::InType) == sizeof(V), "element size");
        const uint32_t c =
            DISCR::apply(*reinterpret_cast<const typename DISCR::InType*>(&v));
        return c < static_cast<uint32_t>(M) ? c : static_cast<uint32_t>(M - 1);
    }
};

// ------------------------------------------------------------------- timing --
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ------------------------------------------------------- mbarrier + bulk copy --
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// Make initialised barriers visible to the async (TMA) proxy.
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar`; false if the wait ran past kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (globaltimer_ns() - t0 > kWaitLimitNs) return false;
    }
    return true;
}

// One bulk (non-tensor) copy global -> this CTA's shared memory, completing
// `bytes` of transaction count on `bar`.  src and dst 16-byte aligned, bytes a
// multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_load_g2s(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// 2-D tiled tensor load (TMA) of the box at coordinates {x, y} of `tmap` into
// this CTA's shared memory, completing on `bar`.  x is always 0 here (boxes
// cover whole 128-byte rows), so the 16-byte rule on the inner coordinate holds.
// No multicast.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int32_t x, int32_t y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// Bulk (non-tensor) store shared -> global, tracked in this thread's bulk
// async-group.  Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_store_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"(smem_addr(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Wait until at most N of this thread's bulk groups still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// Wait until all of this thread's bulk groups have completed.
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
// Order this thread's generic-proxy shared-memory writes before later
// async-proxy (TMA) reads of them.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ------------------------------------------------------------- warp helpers --
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    return x;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t x) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(0xffffffffu, x, d);
    return x;
}

// Acquire / release accesses at GPU scope for cross-CTA publication.
__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

}  // namespace mdx
