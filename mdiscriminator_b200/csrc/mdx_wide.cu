// mdx_wide.cu -- stable partition of wide elements: arrays of records of any
// width (the reference's _arrays variant, ModArray<N,LEN> over LEN u32 words,
// cuda_code/MdiscrHost_arrays.cu.h:26-36,250-430) and several columns that
// are permuted together (the _tuples variant's u32 / u8 / bool arrays,
// cuda_code/MdiscrHost_tuples.cu.h:13-48,262-429).
//
// Both go through the 8-byte record path:
//   1. build:     rec[i] = {key_i, i}        (key: the record's first u32 word,
//                                            or column 0)
//   2. partition: the REC8 kernels with the caller's discriminator on the key
//                 give the stable order of (key, row) and the class sizes;
//   3. gather:    output row p = input row (rec_out[p] >> 32), for the whole
//                 record or for every column; the key comes from rec_out[p].
// Traffic per row: 4 + 8 (build) + 24 (partition) + 8 + 2R (gather) bytes for
// R bytes of row data, against 2R for a kernel specialised to the width; 4-,
// 8- and (16-byte aligned) 16-byte records take the direct record kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "mdx_host.cuh"

namespace mdx {
namespace wide {

constexpr int kThreads = 256;
constexpr int kMaxCols = 8;

struct Cols {
    const void* in[kMaxCols];
    void* out[kMaxCols];
    uint32_t bytes[kMaxCols];
    uint32_t num;
};

// rec[i] = key_i | (i << 32), key_i = the u32 at byte offset stride * i of keys
__global__ void __launch_bounds__(kThreads) build_key_index(const unsigned char* keys, uint64_t stride,
                                                            uint64_t n, uint64_t* rec) {
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * kThreads) {
        const uint32_t k = *reinterpret_cast<const uint32_t*>(keys + stride * i);
        rec[i] = static_cast<uint64_t>(k) | (i << 32);
    }
}

// Records of `words` u32 words: out row p = in row (perm[p] >> 32).  One
// thread per (row, word) pair, so a warp reads and writes consecutive words.
__global__ void __launch_bounds__(kThreads) gather_records(const uint32_t* in, uint32_t* out,
                                                           const uint64_t* perm, uint64_t n,
                                                           uint32_t words) {
    const uint64_t total = n * words;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x; t < total;
         t += static_cast<uint64_t>(gridDim.x) * kThreads) {
        const uint64_t p = t / words;
        const uint32_t w = static_cast<uint32_t>(t - p * words);
        const uint64_t src = perm[p] >> 32;
        out[t] = in[src * words + w];
    }
}

template <class T>
__device__ __forceinline__ void move_one(const void* in, void* out, uint64_t src, uint64_t p) {
    static_cast<T*>(out)[p] = static_cast<const T*>(in)[src];
}

// Columns: out_c[p] = in_c[perm[p] >> 32]; column 0 (the u32 key) from perm[p].
__global__ void __launch_bounds__(kThreads) gather_columns(Cols cols, const uint64_t* perm, uint64_t n) {
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x; p < n;
         p += static_cast<uint64_t>(gridDim.x) * kThreads) {
        const uint64_t r = perm[p];
        const uint64_t src = r >> 32;
        static_cast<uint32_t*>(cols.out[0])[p] = static_cast<uint32_t>(r);
        for (uint32_t c = 1; c < cols.num; c++) {
            switch (cols.bytes[c]) {
                case 1: move_one<uint8_t>(cols.in[c], cols.out[c], src, p); break;
                case 2: move_one<uint16_t>(cols.in[c], cols.out[c], src, p); break;
                case 4: move_one<uint32_t>(cols.in[c], cols.out[c], src, p); break;
                default: move_one<uint64_t>(cols.in[c], cols.out[c], src, p); break;
            }
        }
    }
}

struct Layout {
    size_t rec_in, rec_out, plain, total;
    host::PlainLayout L;
};

// The REC8 partition's own workspace comes first, so its header (and the
// error word mdx_workspace_error reads) is the caller's; the two record
// arrays follow.
inline Layout layout(uint64_t n, uint32_t m) {
    Layout w;
    w.L = host::plain_layout(n, MDX_ELEM_REC8, m);
    w.plain = 0;
    w.rec_in = host::align_up(w.L.total, host::kAlign);
    w.rec_out = host::align_up(w.rec_in + 8 * n, host::kAlign);
    w.total = host::align_up(w.rec_out + 8 * n, host::kAlign);
    return w;
}

inline uint32_t grid_for(uint64_t work) {
    uint64_t g = (work + kThreads - 1) / kThreads;
    if (g > 148ull * 16) g = 148ull * 16;
    return static_cast<uint32_t>(g < 1 ? 1 : g);
}

// Steps 1-2: the stable order of (key, row) into rec_out, sizes and head flags.
inline mdx_status key_order(const unsigned char* keys, uint64_t stride, uint64_t n, mdx_discr discr,
                            uint32_t* d_sizes, uint32_t* d_headflags, unsigned char* ws,
                            const Layout& w, cudaStream_t st) {
    uint64_t* rec_in = reinterpret_cast<uint64_t*>(ws + w.rec_in);
    uint64_t* rec_out = reinterpret_cast<uint64_t*>(ws + w.rec_out);
    build_key_index<<<grid_for(n), kThreads, 0, st>>>(keys, stride, n, rec_in);
    if (cudaGetLastError() != cudaSuccess) return MDX_ERR_CUDA;
    return mdx_partition(rec_in, rec_out, n, MDX_ELEM_REC8, discr, d_sizes, d_headflags,
                         ws + w.plain, w.L.total, reinterpret_cast<mdx_stream_t>(st));
}

}  // namespace wide
}  // namespace mdx

using namespace mdx;

extern "C" {

size_t mdx_records_workspace_size(uint64_t n, uint32_t record_bytes, uint32_t m) {
    if (record_bytes < 4 || record_bytes % 4 != 0 || m < 1 || m > MDX_MAX_CLASSES) return 0;
    if (record_bytes == 4) return mdx_workspace_size(n, MDX_ELEM_U32, m);
    if (record_bytes == 8) return mdx_workspace_size(n, MDX_ELEM_REC8, m);
    const size_t gathered = wide::layout(n, m).total;  // unaligned 16-byte records use it too
    if (record_bytes == 16) return std::max(gathered, mdx_workspace_size(n, MDX_ELEM_REC16, m));
    return gathered;
}

mdx_status mdx_partition_records(const void* d_in, void* d_out, uint64_t n, uint32_t record_bytes,
                                 mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                                 void* d_ws, size_t ws_bytes, mdx_stream_t stream) {
    if (record_bytes < 4 || record_bytes % 4 != 0) return MDX_ERR_INVALID;
    if (record_bytes == 4)
        return mdx_partition(d_in, d_out, n, MDX_ELEM_U32, discr, d_sizes, d_headflags, d_ws,
                             ws_bytes, stream);
    if (record_bytes == 8)
        return mdx_partition(d_in, d_out, n, MDX_ELEM_REC8, discr, d_sizes, d_headflags, d_ws,
                             ws_bytes, stream);
    if (record_bytes == 16 && reinterpret_cast<uintptr_t>(d_in) % 16 == 0 &&
        reinterpret_cast<uintptr_t>(d_out) % 16 == 0)  // the 16-byte record kernels
        return mdx_partition(d_in, d_out, n, MDX_ELEM_REC16, discr, d_sizes, d_headflags, d_ws,
                             ws_bytes, stream);
    mdx_status s = host::check_discr(discr);
    if (s != MDX_OK) return s;
    if (n > MDX_MAX_ELEMS) return MDX_ERR_INVALID;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) {
        if (d_sizes && cudaMemsetAsync(d_sizes, 0, discr.m * sizeof(uint32_t), st) != cudaSuccess)
            return MDX_ERR_CUDA;
        return MDX_OK;
    }
    if (d_in == nullptr || d_out == nullptr) return MDX_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(d_in) % 4 || reinterpret_cast<uintptr_t>(d_out) % 4)
        return MDX_ERR_INVALID;
    const char* ib = static_cast<const char*>(d_in);
    const char* ob = static_cast<const char*>(d_out);
    if (ib < ob + n * record_bytes && ob < ib + n * record_bytes) return MDX_ERR_INVALID;
    const wide::Layout w = wide::layout(n, discr.m);
    if (d_ws == nullptr || ws_bytes < w.total || reinterpret_cast<uintptr_t>(d_ws) % host::kAlign)
        return MDX_ERR_WORKSPACE;
    unsigned char* ws = static_cast<unsigned char*>(d_ws);
    s = wide::key_order(static_cast<const unsigned char*>(d_in), record_bytes, n, discr, d_sizes,
                        d_headflags, ws, w, st);
    if (s != MDX_OK) return s;
    const uint32_t words = record_bytes / 4;
    wide::gather_records<<<wide::grid_for(n * words), wide::kThreads, 0, st>>>(
        static_cast<const uint32_t*>(d_in), static_cast<uint32_t*>(d_out),
        reinterpret_cast<const uint64_t*>(ws + w.rec_out), n, words);
    return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
}

size_t mdx_columns_workspace_size(uint64_t n, uint32_t m) {
    if (m < 1 || m > MDX_MAX_CLASSES) return 0;
    return wide::layout(n, m).total;
}

mdx_status mdx_partition_columns(const mdx_column* cols, uint32_t num_cols, uint64_t n,
                                 mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                                 void* d_ws, size_t ws_bytes, mdx_stream_t stream) {
    if (cols == nullptr || num_cols < 1 || num_cols > static_cast<uint32_t>(wide::kMaxCols))
        return MDX_ERR_INVALID;
    mdx_status s = host::check_discr(discr);
    if (s != MDX_OK) return s;
    if (n > MDX_MAX_ELEMS || cols[0].elem_bytes != 4) return MDX_ERR_INVALID;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) {
        if (d_sizes && cudaMemsetAsync(d_sizes, 0, discr.m * sizeof(uint32_t), st) != cudaSuccess)
            return MDX_ERR_CUDA;
        return MDX_OK;
    }
    wide::Cols c{};
    c.num = num_cols;
    for (uint32_t i = 0; i < num_cols; i++) {
        const uint32_t b = cols[i].elem_bytes;
        if ((b != 1 && b != 2 && b != 4 && b != 8) || cols[i].in == nullptr || cols[i].out == nullptr ||
            reinterpret_cast<uintptr_t>(cols[i].in) % b || reinterpret_cast<uintptr_t>(cols[i].out) % b)
            return MDX_ERR_INVALID;
        for (uint32_t j = 0; j < num_cols; j++) {  // no output may overlap any input or output
            const char* o = static_cast<const char*>(cols[i].out);
            const char* x = static_cast<const char*>(cols[j].in);
            if (o < x + n * cols[j].elem_bytes && x < o + n * b) return MDX_ERR_INVALID;
            if (j != i) {
                const char* y = static_cast<const char*>(cols[j].out);
                if (o < y + n * cols[j].elem_bytes && y < o + n * b) return MDX_ERR_INVALID;
            }
        }
        c.in[i] = cols[i].in;
        c.out[i] = cols[i].out;
        c.bytes[i] = b;
    }
    const wide::Layout w = wide::layout(n, discr.m);
    if (d_ws == nullptr || ws_bytes < w.total || reinterpret_cast<uintptr_t>(d_ws) % host::kAlign)
        return MDX_ERR_WORKSPACE;
    unsigned char* ws = static_cast<unsigned char*>(d_ws);
    s = wide::key_order(static_cast<const unsigned char*>(cols[0].in), 4, n, discr, d_sizes,
                        d_headflags, ws, w, st);
    if (s != MDX_OK) return s;
    wide::gather_columns<<<wide::grid_for(n), wide::kThreads, 0, st>>>(
        c, reinterpret_cast<const uint64_t*>(ws + w.rec_out), n);
    return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
}

}  // extern "C"
