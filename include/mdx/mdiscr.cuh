// mdx/mdiscr.cuh -- header-only drop-in for the reference's host templates.
//
// A program written against the reference keeps its functors and calls; it
// swaps the include and compiles with nvcc for sm_100a (-I<repo>/include):
//
//   #include "MdiscrHost_optimized_clean.cu.h"   ->   #include "mdx/mdiscr.cuh"
//   mdiscr<Mod8>(n, 1 << 16, d_in, d_out)          (same call)
//   mdiscrSegm<Mod4>(n, in, segment_sizes, out, new_sizes)   (same call)
//   mdiscr<ModArray<N, LEN>, LEN>(n, hw, d_in, d_out)         (arrays, same call)
//   mdiscr<ModTuple<N>>(n, hw, in1, in2, in3, out1, out2, out3) (tuples, same call)
//
// Signatures (reference):
//   template<class DISCR> typename DISCR::TupleType
//   mdiscr(const unsigned int n, const unsigned int num_hwd_thds,
//          typename DISCR::InType* d_in, typename DISCR::InType* d_out)
//     -- cuda_code/MdiscrHost_optimized_clean.cu.h:9-15
//   template<class DISCR> void
//   mdiscrSegm(unsigned int n, typename DISCR::InType* in, int* segment_sizes,
//              typename DISCR::InType* out, int* new_sizes)
//     -- cuda_code/MdiscrSegmHost.cu.h:36-42
//
// DISCR follows the reference's functor concept (HelpersCommon.h:587-596):
// InType (4 or 8 bytes), TupleType with `cardinal` (m) and operator[], and a
// static `apply(InType) -> unsigned` callable on the device (__host__
// __device__).  Any such functor runs through the same sm_100a kernels as the
// C ABI: m <= 64 for mdiscr, m <= 16 for mdiscrSegm.
//
// Differences from the reference: no per-call cudaMalloc (a workspace per
// device is allocated on first use and grown when a call needs more; it is
// kept until exit); errors print and exit like the reference's gpuErrchk
// (HelpersHost.cu.h:11-19) unless MDX_NO_EXIT is defined, which makes them
// throw std::runtime_error; `num_hwd_thds` is accepted and ignored.  Calls are
// synchronous on the legacy default stream, as the reference's are.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <stdexcept>
#include <type_traits>

#include "../mdx.h"
#include "../../mdiscriminator_b200/csrc/mdx_host.cuh"

namespace mdx {
namespace detail {

inline const char* status_text(mdx_status s) {
    switch (s) {
        case MDX_OK: return "ok";
        case MDX_ERR_INVALID: return "invalid argument";
        case MDX_ERR_WORKSPACE: return "workspace too small or misaligned";
        case MDX_ERR_CUDA: return "CUDA runtime error";
        case MDX_ERR_TIMEOUT: return "device-side bounded wait timed out";
        case MDX_ERR_UNSUPPORTED: return "unsupported request";
        case MDX_ERR_SEGMENTS: return "malformed segment description";
        case MDX_ERR_CANCELLED: return "request cancelled before launch";
    }
    return "unknown status";
}

inline void check(mdx_status s, const char* file, int line) {
    if (s == MDX_OK) return;
#ifdef MDX_NO_EXIT
    (void)file;
    (void)line;
    throw std::runtime_error(status_text(s));
#else
    std::fprintf(stderr, "mdx error (%d): %s (%s, line %d)\n", static_cast<int>(s), status_text(s),
                 file, line);
    std::exit(static_cast<int>(s));
#endif
}

// Host-side fault injection for tests: the nth growth of the workspace from
// now on fails as if cudaMalloc had run out of memory (0: off).
inline std::atomic<int>& workspace_fail_countdown() {
    static std::atomic<int> c{0};
    return c;
}

// One zero-initialised workspace per device, grown on demand.  A failed
// growth leaves none, so the next call tries again.
inline unsigned char* workspace(size_t need) {
    static std::mutex mu;
    static void* ptr[64] = {};
    static size_t bytes[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (bytes[dev] < need) {
        if (ptr[dev] != nullptr) cudaFree(ptr[dev]);  // waits for work still using it
        ptr[dev] = nullptr;
        bytes[dev] = 0;
        const int fc = workspace_fail_countdown().load();
        if (fc > 0 && workspace_fail_countdown().fetch_sub(1) == 1) return nullptr;
        if (cudaMalloc(&ptr[dev], need) != cudaSuccess) return nullptr;
        if (cudaMemset(ptr[dev], 0, need) != cudaSuccess) return nullptr;
        bytes[dev] = need;
    }
    return static_cast<unsigned char*>(ptr[dev]);
}

// Latched device error of a workspace (and clear it), after a synchronise.
inline mdx_status take_error(unsigned char* ws) {
    if (cudaDeviceSynchronize() != cudaSuccess) return MDX_ERR_CUDA;
    uint32_t err = 0;
    if (cudaMemcpy(&err, ws + 4, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return MDX_ERR_CUDA;
    if (err == 0) return MDX_OK;
    cudaMemset(ws + 4, 0, 4);
    return (err & kErrTimeout) ? MDX_ERR_TIMEOUT : MDX_ERR_SEGMENTS;
}

template <unsigned m>
constexpr int class_bound_of() {
    return m <= 2 ? 2 : m <= 4 ? 4 : m <= 8 ? 8 : m <= 16 ? 16 : m <= 32 ? 32 : 64;
}

template <class T>
using elem_of = typename std::conditional<
    sizeof(T) == 4, uint32_t, typename std::conditional<sizeof(T) == 8, uint64_t, Rec16>::type>::type;

template <class T>
constexpr mdx_elem elem_kind() {
    return sizeof(T) == 4 ? MDX_ELEM_U32 : sizeof(T) == 8 ? MDX_ELEM_REC8 : MDX_ELEM_REC16;
}

// Wide rows (arrays of LEN values, or a tuple of three arrays): each row's
// class from the user's functor and its index as one 8-byte record, the stable
// order of those records by class (the 8-byte-record kernels, class < M kept
// by a mask), then every row moved to its place.
constexpr int kRowThreads = 256;
inline uint32_t row_grid(uint64_t work) {
    uint64_t g = (work + kRowThreads - 1) / kRowThreads;
    if (g > 148ull * 16) g = 148ull * 16;
    return static_cast<uint32_t>(g < 1 ? 1 : g);
}

template <class DISCR, unsigned LEN, int M>
__global__ void array_rows(const typename DISCR::InType* in, uint64_t n, uint64_t* rec) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * kRowThreads + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * kRowThreads) {
        uint32_t c = DISCR::apply(const_cast<typename DISCR::InType*>(in + i * LEN));
        c = c < static_cast<uint32_t>(M) ? c : static_cast<uint32_t>(M - 1);
        rec[i] = static_cast<uint64_t>(c) | (i << 32);
    }
}

template <class DISCR, int M>
__global__ void tuple_rows(const typename DISCR::InType1* a, const typename DISCR::InType2* b,
                           const typename DISCR::InType3* c3, uint64_t n, uint64_t* rec) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * kRowThreads + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * kRowThreads) {
        uint32_t c = DISCR::apply(a[i], b[i], c3[i]);
        c = c < static_cast<uint32_t>(M) ? c : static_cast<uint32_t>(M - 1);
        rec[i] = static_cast<uint64_t>(c) | (i << 32);
    }
}

template <class T>
__global__ void gather_rows(const T* in, T* out, const uint64_t* perm, uint64_t n, unsigned len) {
    const uint64_t total = n * len;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * kRowThreads + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * kRowThreads) {
        const uint64_t p = t / len;
        out[t] = in[(perm[p] >> 32) * len + (t - p * len)];
    }
}

template <class T1, class T2, class T3>
__global__ void gather_tuple(const T1* a, const T2* b, const T3* c, T1* oa, T2* ob, T3* oc,
                             const uint64_t* perm, uint64_t n) {
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * kRowThreads + threadIdx.x; p < n;
         p += static_cast<uint64_t>(gridDim.x) * kRowThreads) {
        const uint64_t s = perm[p] >> 32;
        oa[p] = a[s];
        ob[p] = b[s];
        oc[p] = c[s];
    }
}

struct RowsLayout {
    host::PlainLayout L;
    size_t rec_in, rec_out, total;
};
inline RowsLayout rows_layout(uint64_t n, unsigned m) {
    RowsLayout r;
    r.L = host::plain_layout(n, MDX_ELEM_REC8, m);
    r.rec_in = host::align_up(r.L.total, host::kAlign);
    r.rec_out = host::align_up(r.rec_in + 8 * n, host::kAlign);
    r.total = host::align_up(r.rec_out + 8 * n, host::kAlign);
    return r;
}

// Stable order of the {class, row} records in rec_in into rec_out; class sizes.
template <class TupleT, unsigned m>
TupleT order_rows(uint64_t n, unsigned char* ws, const RowsLayout& R) {
    constexpr int M = class_bound_of<m>();
    const uint64_t* rin = reinterpret_cast<const uint64_t*>(ws + R.rec_in);
    uint64_t* rout = reinterpret_cast<uint64_t*>(ws + R.rec_out);
    check(host::run_plain<uint64_t, DiscrMask, M>(rin, rout, n, DiscrMask{M - 1u}, m, nullptr,
                                                  nullptr, ws, R.L, nullptr, nullptr),
          __FILE__, __LINE__);
    check(take_error(ws), __FILE__, __LINE__);
    uint32_t h[64];
    if (cudaMemcpy(h, ws + R.L.class_tot, m * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        check(MDX_ERR_CUDA, __FILE__, __LINE__);
    TupleT result;
    for (unsigned c = 0; c < m; c++) result[c] = h[c];
    return result;
}

}  // namespace detail

// Test hook (no reference counterpart; host side, no GPU fault): the nth
// growth of the per-device workspace from now on fails as if device memory
// were exhausted, so the call reports MDX_ERR_CUDA (exit, or
// std::runtime_error under MDX_NO_EXIT); 0 turns it off.
inline void test_inject_workspace_failure(int nth) { detail::workspace_fail_countdown().store(nth); }

template <class DISCR>
typename DISCR::TupleType mdiscr(const unsigned int num_elems, const unsigned int num_hwd_thds,
                                 typename DISCR::InType* d_in, typename DISCR::InType* d_out) {
    using In = typename DISCR::InType;
    static_assert(sizeof(In) == 4 || sizeof(In) == 8 || sizeof(In) == 16,
                  "4-byte values, 8- or 16-byte records");
    constexpr unsigned m = DISCR::TupleType::cardinal;
    static_assert(m >= 1 && m <= 64, "1 <= m <= 64");
    constexpr int M = detail::class_bound_of<m>();
    using V = detail::elem_of<In>;
    (void)num_hwd_thds;
    typename DISCR::TupleType result;
    for (unsigned c = 0; c < m; c++) result[c] = 0;
    if (num_elems == 0) return result;
    const host::PlainLayout L = host::plain_layout(num_elems, detail::elem_kind<In>(), m);
    unsigned char* ws = detail::workspace(L.total);
    if (ws == nullptr) detail::check(MDX_ERR_CUDA, __FILE__, __LINE__);
    detail::check(host::check_io(d_in, d_out, num_elems, detail::elem_kind<In>()), __FILE__,
                  __LINE__);
    detail::check(host::run_plain<V, DiscrStatic<DISCR, M>, M>(
                      d_in, d_out, num_elems, DiscrStatic<DISCR, M>{}, m, nullptr, nullptr, ws, L,
                      nullptr, nullptr),
                  __FILE__, __LINE__);
    detail::check(detail::take_error(ws), __FILE__, __LINE__);
    uint32_t h[64];
    if (cudaMemcpy(h, ws + L.class_tot, m * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        detail::check(MDX_ERR_CUDA, __FILE__, __LINE__);
    for (unsigned c = 0; c < m; c++) result[c] = h[c];
    return result;
}

// Arrays of LEN values per element, class from the element's values
// (mdiscr<DISCR, LEN>, cuda_code/MdiscrHost_arrays.cu.h:250-430; DISCR::apply
// takes a pointer to the element's first value, as ModArray<N, LEN> does).
template <class DISCR, unsigned int LEN>
typename DISCR::TupleType mdiscr(const unsigned int num_elems, const unsigned int num_hwd_thds,
                                 typename DISCR::InType* d_in, typename DISCR::InType* d_out) {
    using In = typename DISCR::InType;
    constexpr unsigned m = DISCR::TupleType::cardinal;
    static_assert(m >= 1 && m <= 64, "1 <= m <= 64");
    static_assert(LEN >= 1, "LEN >= 1");
    (void)num_hwd_thds;
    typename DISCR::TupleType result;
    for (unsigned c = 0; c < m; c++) result[c] = 0;
    if (num_elems == 0) return result;
    const detail::RowsLayout R = detail::rows_layout(num_elems, m);
    unsigned char* ws = detail::workspace(R.total);
    if (ws == nullptr) detail::check(MDX_ERR_CUDA, __FILE__, __LINE__);
    const char* ib = reinterpret_cast<const char*>(d_in);
    const char* ob = reinterpret_cast<const char*>(d_out);
    const uint64_t bytes = static_cast<uint64_t>(num_elems) * LEN * sizeof(In);
    if (d_in == nullptr || d_out == nullptr || (ib < ob + bytes && ob < ib + bytes))
        detail::check(MDX_ERR_INVALID, __FILE__, __LINE__);
    constexpr int M = detail::class_bound_of<m>();
    uint64_t* rin = reinterpret_cast<uint64_t*>(ws + R.rec_in);
    detail::array_rows<DISCR, LEN, M><<<detail::row_grid(num_elems), detail::kRowThreads>>>(
        d_in, num_elems, rin);
    result = detail::order_rows<typename DISCR::TupleType, m>(num_elems, ws, R);
    detail::gather_rows<In><<<detail::row_grid(static_cast<uint64_t>(num_elems) * LEN),
                              detail::kRowThreads>>>(
        d_in, d_out, reinterpret_cast<const uint64_t*>(ws + R.rec_out), num_elems, LEN);
    detail::check(cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA, __FILE__, __LINE__);
    detail::check(detail::take_error(ws), __FILE__, __LINE__);
    return result;
}

// Three arrays partitioned together by a functor of their values
// (cuda_code/MdiscrHost_tuples.cu.h:262-429: DISCR has InType1..3 and
// apply(x, y, z)).
template <class DISCR>
typename DISCR::TupleType mdiscr(const unsigned int num_elems, const unsigned int num_hwd_thds,
                                 typename DISCR::InType1* d_in1, typename DISCR::InType2* d_in2,
                                 typename DISCR::InType3* d_in3, typename DISCR::InType1* d_out1,
                                 typename DISCR::InType2* d_out2, typename DISCR::InType3* d_out3) {
    constexpr unsigned m = DISCR::TupleType::cardinal;
    static_assert(m >= 1 && m <= 64, "1 <= m <= 64");
    (void)num_hwd_thds;
    typename DISCR::TupleType result;
    for (unsigned c = 0; c < m; c++) result[c] = 0;
    if (num_elems == 0) return result;
    if (!d_in1 || !d_in2 || !d_in3 || !d_out1 || !d_out2 || !d_out3)
        detail::check(MDX_ERR_INVALID, __FILE__, __LINE__);
    const detail::RowsLayout R = detail::rows_layout(num_elems, m);
    unsigned char* ws = detail::workspace(R.total);
    if (ws == nullptr) detail::check(MDX_ERR_CUDA, __FILE__, __LINE__);
    constexpr int M = detail::class_bound_of<m>();
    uint64_t* rin = reinterpret_cast<uint64_t*>(ws + R.rec_in);
    detail::tuple_rows<DISCR, M><<<detail::row_grid(num_elems), detail::kRowThreads>>>(
        d_in1, d_in2, d_in3, num_elems, rin);
    result = detail::order_rows<typename DISCR::TupleType, m>(num_elems, ws, R);
    detail::gather_tuple<<<detail::row_grid(num_elems), detail::kRowThreads>>>(
        d_in1, d_in2, d_in3, d_out1, d_out2, d_out3,
        reinterpret_cast<const uint64_t*>(ws + R.rec_out), num_elems);
    detail::check(cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA, __FILE__, __LINE__);
    detail::check(detail::take_error(ws), __FILE__, __LINE__);
    return result;
}

template <class DISCR>
void mdiscrSegm(const unsigned int num_elems, typename DISCR::InType* in_array, int* segment_sizes,
                typename DISCR::InType* out_array, int* new_sizes) {
    using In = typename DISCR::InType;
    static_assert(sizeof(In) == 4 || sizeof(In) == 8, "4-byte values or 8-byte records");
    constexpr unsigned m = DISCR::TupleType::cardinal;
    static_assert(m >= 1 && m <= 16, "the segmented path takes 1 <= m <= 16");
    constexpr int M = detail::class_bound_of<m>();
    using V = detail::elem_of<In>;
    if (num_elems == 0) return;
    const mdx_elem e = detail::elem_kind<In>();
    detail::check(host::check_io(in_array, out_array, num_elems, e), __FILE__, __LINE__);
    const host::SegLayout L = host::seg_layout(num_elems, num_elems, e, m, true);
    unsigned char* ws = detail::workspace(L.total);
    if (ws == nullptr) detail::check(MDX_ERR_CUDA, __FILE__, __LINE__);
    detail::check(host::launch_flags_to_offsets(segment_sizes, num_elems, ws, L, nullptr), __FILE__,
                  __LINE__);
    const uint64_t* offs = reinterpret_cast<const uint64_t*>(ws + L.offsets);
    detail::check(host::run_segm<V, DiscrStatic<DISCR, M>, M>(
                      in_array, out_array, num_elems, DiscrStatic<DISCR, M>{}, m, offs,
                      kSegsOnDevice, num_elems, segment_sizes, nullptr,
                      reinterpret_cast<uint32_t*>(new_sizes), ws, L, nullptr),
                  __FILE__, __LINE__);
    detail::check(detail::take_error(ws), __FILE__, __LINE__);
}

}  // namespace mdx

#ifndef MDX_NO_GLOBAL_TEMPLATES
// The reference declares these templates at global scope.
using mdx::mdiscr;
using mdx::mdiscrSegm;
#endif
