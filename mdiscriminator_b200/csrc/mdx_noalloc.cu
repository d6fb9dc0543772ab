// mdx_noalloc.cu -- mdx_partition_noalloc: the plain stable partition for
// callers that cannot allocate device memory.
//
// Who needs it: code that has to partition where cudaMalloc is not available
// or not allowed and that cannot keep a workspace of its own -- for example a
// callback running inside a device memory allocator or pool (allocating there
// would re-enter it), a plugin whose host forbids device allocations once it
// has started, or a latency-critical loop that must not pay cudaMalloc's
// implicit device-wide synchronisation.  Such a caller passes only its input,
// output and size arrays; the scratch the kernels need lives in a fixed array
// compiled into this library.
//
// The scratch: g_noalloc_scratch, a file-scope __device__ array of
// kNoAllocScratchBytes = 525,312 bytes.  Every GPU that loads the library
// holds it until the process exits.  It fits the plain partition's chunk
// tables for m <= 16 at any n < 2^32; requests with m > 16 need more and are
// rejected with MDX_ERR_WORKSPACE before anything is launched.
//
// Set-up: in host code the array's name is only a host-side stand-in, not a
// device address, so the first call on each device (with that device
// current) looks the address up with cudaGetSymbolAddress, checks the result
// and caches it; the same first call sets the kernels' shared-memory limit and
// queries their occupancy.  Make that first call on every device before any
// stream capture.
//
// Sharing: every call uses the same array, which keeps whatever the last call
// left in it.  Each call first clears, on its stream, the part that must start
// at zero (the chunk ticket).  Calls whose kernels can overlap on the GPU --
// different streams without ordering between them -- race on the array: issue
// them in one stream or order them.
//
// Errors: a device-side wait that runs out (a tile copy that never lands
// within a second) latches a bit in the array's error word, which no call
// clears; mdx_partition_noalloc_error reads it, clears it and reports it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/mdx.h"
#include "mdx_plain.cuh"

namespace mdx {
namespace noalloc {

constexpr size_t kNoAllocScratchBytes = 525312;  // 2052 * 256
constexpr int kThreadsN = 256;
constexpr int kStagesN = 2;
constexpr uint32_t kMaxChunksN = 4096;
constexpr size_t kHeaderN = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void* g_scratch_dev[kMaxDevices];  // device address of g_noalloc_scratch, per device

// Device address of the scratch on the current device (set up on first use).
cudaError_t scratch_address(void** out) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_scratch_dev[dev] == nullptr) {
        void* p = nullptr;
        err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess) return err;
        g_scratch_dev[dev] = p;
    }
    *out = g_scratch_dev[dev];
    return cudaSuccess;
}

// Resident CTAs per SM and SM count, looked up once per device for each
// kernel instantiation (K tags the instantiation: one pair of statics each).
template <class K>
cudaError_t occupancy_n(const void* fn, size_t smem, int* blocks, int* sms) {
    static int s_blocks[kMaxDevices];
    static int s_sms[kMaxDevices];
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (s_blocks[dev] == 0) {
        if (smem > 48 * 1024) {
            err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
            if (err != cudaSuccess) return err;
        }
        int b = 0, s = 0;
        if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kThreadsN, smem)) !=
            cudaSuccess)
            return err;
        if ((err = cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
            return err;
        s_sms[dev] = s;
        s_blocks[dev] = b < 1 ? 1 : b;
    }
    *blocks = s_blocks[dev];
    *sms = s_sms[dev];
    return cudaSuccess;
}

template <class V, class D, int M>
struct KernelTag {};

typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                             const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                             CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                             CUtensorMapFloatOOBfill);

bool row_map(CUtensorMap* map, const void* base, uint64_t n, size_t elem, uint32_t box_rows) {
    std::memset(map, 0, sizeof(*map));
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                             &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    if (fn == nullptr || reinterpret_cast<uintptr_t>(base) % 16 != 0) return false;
    const uint64_t per_row = 128 / elem, rows = n / per_row;
    if (rows < box_rows) return false;
    const cuuint64_t dims[2] = {per_row, rows};
    const cuuint64_t strides[1] = {128};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(per_row), box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_UINT64, 2,
              const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline uint32_t bound_of(uint32_t m) {
    uint32_t b = 2;
    while (b < m) b <<= 1;
    return b;
}

// Offsets inside the scratch (same roles as the caller workspace of
// mdx_partition): header {ticket, error}, class bases, class totals, [M][G]
// chunk counts and prefixes.
struct Layout {
    size_t class_base, class_tot, chunk_cnt, chunk_pre, total;
};
inline size_t up256(size_t x) { return (x + 255) / 256 * 256; }
inline Layout layout_for(uint32_t M, uint32_t G) {
    Layout L;
    L.class_base = kHeaderN;
    L.class_tot = L.class_base + 64 * 4;
    L.chunk_cnt = up256(L.class_tot + 64 * 4);
    L.chunk_pre = up256(L.chunk_cnt + static_cast<size_t>(M) * G * 4);
    L.total = up256(L.chunk_pre + static_cast<size_t>(M) * G * 4);
    return L;
}

template <class V, class D, int M>
mdx_status run(const void* d_in, void* d_out, uint64_t n, D d, uint32_t m, uint32_t* d_sizes,
               uint32_t* d_headflags, cudaStream_t st) {
    using SL = ScatterTmaSmem<V, kThreadsN, kStagesN, M>;
    constexpr int TILE = SL::kTile;
    auto scatter = plain_scatter_tma_kernel<V, D, M, kThreadsN, kStagesN>;
    auto count = plain_count_kernel<V, D, M, kThreadsN, TILE>;
    void* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) return MDX_ERR_CUDA;
    int blocks = 0, sms = 0;
    if (occupancy_n<KernelTag<V, D, M>>(reinterpret_cast<const void*>(scatter), SL::kBytes,
                                        &blocks, &sms) != cudaSuccess)
        return MDX_ERR_CUDA;
    const uint32_t nt = static_cast<uint32_t>((n + TILE - 1) / TILE);
    uint32_t G = static_cast<uint32_t>(blocks) * static_cast<uint32_t>(sms);
    if (G > nt) G = nt;
    if (G > kMaxChunksN) G = kMaxChunksN;
    const Layout L = layout_for(M, G);
    if (L.total > kNoAllocScratchBytes) return MDX_ERR_WORKSPACE;
    unsigned char* ws = static_cast<unsigned char*>(scratch);
    // the chunk ticket must start at zero (the error word keeps its bits
    // until mdx_partition_noalloc_error reads them)
    if (cudaMemsetAsync(ws, 0, sizeof(uint32_t), st) != cudaSuccess) return MDX_ERR_CUDA;
    if (d_headflags != nullptr &&
        cudaMemsetAsync(d_headflags, 0, n * sizeof(uint32_t), st) != cudaSuccess)
        return MDX_ERR_CUDA;
    PlainArgs a;
    a.in = d_in;
    a.out = d_out;
    a.n = n;
    a.num_tiles = nt;
    a.num_chunks = G;
    a.chunk_cnt = reinterpret_cast<uint32_t*>(ws + L.chunk_cnt);
    a.chunk_pre = reinterpret_cast<uint32_t*>(ws + L.chunk_pre);
    a.class_base = reinterpret_cast<uint32_t*>(ws + L.class_base);
    a.class_tot = reinterpret_cast<uint32_t*>(ws + L.class_tot);
    a.sizes = d_sizes;
    a.headflags = d_headflags;
    a.done = reinterpret_cast<uint32_t*>(ws);
    a.error = reinterpret_cast<uint32_t*>(ws) + 1;
    a.m = m;
    a.skip = nullptr;
    a.chunk_stride = G;
    a.prefix_in_scatter = 0;  // the last counting CTA scans the chunk counts
    CUtensorMap map;
    a.use_tma = row_map(&map, d_in, n, sizeof(V), SL::kRows) ? 1 : 0;
    const OutFlat<V> o{static_cast<V*>(d_out),
                       static_cast<uint32_t>((reinterpret_cast<uintptr_t>(d_out) / sizeof(V)) &
                                             (16u / sizeof(V) - 1u))};
    count<<<G, kThreadsN, 0, st>>>(a, d);
    scatter<<<G, kThreadsN, SL::kBytes, st>>>(a, d, map, o);
    return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
}

template <class V, class D>
mdx_status by_bound(const void* in, void* out, uint64_t n, D d, uint32_t m, uint32_t* sz,
                    uint32_t* hf, cudaStream_t st) {
    switch (bound_of(m)) {
        case 2: return run<V, D, 2>(in, out, n, d, m, sz, hf, st);
        case 4: return run<V, D, 4>(in, out, n, d, m, sz, hf, st);
        case 8: return run<V, D, 8>(in, out, n, d, m, sz, hf, st);
        case 16: return run<V, D, 16>(in, out, n, d, m, sz, hf, st);
        default: return MDX_ERR_WORKSPACE;  // needs more scratch than the built-in array
    }
}

template <class V>
mdx_status by_discr(const void* in, void* out, uint64_t n, mdx_discr dc, uint32_t* sz, uint32_t* hf,
                    cudaStream_t st) {
    const bool pow2 = (dc.m & (dc.m - 1u)) == 0u;
    if (dc.kind == MDX_DISCR_MASK || pow2)
        return by_bound<V>(in, out, n, DiscrMask{dc.m - 1u}, dc.m, sz, hf, st);
    return by_bound<V>(in, out, n, DiscrMod::make(dc.m), dc.m, sz, hf, st);
}

}  // namespace noalloc
}  // namespace mdx

extern "C" mdx_status mdx_partition_noalloc(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                            mdx_discr discr, uint32_t* d_sizes,
                                            uint32_t* d_headflags, mdx_stream_t stream) {
    using namespace mdx::noalloc;
    if (elem == MDX_ELEM_REC16) return MDX_ERR_UNSUPPORTED;  // 4- and 8-byte elements here
    if (elem != MDX_ELEM_U32 && elem != MDX_ELEM_REC8) return MDX_ERR_INVALID;
    if (discr.m < 1 || discr.m > MDX_MAX_CLASSES) return MDX_ERR_INVALID;
    if (discr.kind != MDX_DISCR_MOD && discr.kind != MDX_DISCR_MASK) return MDX_ERR_INVALID;
    if (discr.kind == MDX_DISCR_MASK && (discr.m & (discr.m - 1u)) != 0u) return MDX_ERR_INVALID;
    if (n > MDX_MAX_ELEMS) return MDX_ERR_INVALID;
    if (bound_of(discr.m) > 16) return MDX_ERR_WORKSPACE;  // beyond the built-in scratch
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) {
        if (d_sizes && cudaMemsetAsync(d_sizes, 0, discr.m * sizeof(uint32_t), st) != cudaSuccess)
            return MDX_ERR_CUDA;
        return MDX_OK;
    }
    if (d_in == nullptr || d_out == nullptr) return MDX_ERR_INVALID;
    const size_t w = elem == MDX_ELEM_REC8 ? 8 : 4;
    const char* ib = static_cast<const char*>(d_in);
    const char* ob = static_cast<const char*>(d_out);
    if (ib < ob + n * w && ob < ib + n * w) return MDX_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(d_in) % w || reinterpret_cast<uintptr_t>(d_out) % w)
        return MDX_ERR_INVALID;
    if (elem == MDX_ELEM_U32)
        return by_discr<uint32_t>(d_in, d_out, n, discr, d_sizes, d_headflags, st);
    return by_discr<uint64_t>(d_in, d_out, n, discr, d_sizes, d_headflags, st);
}

extern "C" mdx_status mdx_partition_noalloc_error(mdx_stream_t stream) {
    using namespace mdx::noalloc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    void* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) return MDX_ERR_CUDA;
    uint32_t* word = static_cast<uint32_t*>(scratch) + 1;
    uint32_t bits = 0;  // pageable: the copy completes before cudaMemcpyAsync returns
    if (cudaMemcpyAsync(&bits, word, sizeof(bits), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemsetAsync(word, 0, sizeof(uint32_t), st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return MDX_ERR_CUDA;
    if (bits & mdx::kErrTimeout) return MDX_ERR_TIMEOUT;
    return bits ? MDX_ERR_INVALID : MDX_OK;
}
