// mdx_capi.cu -- the C ABI (include/mdx.h) over pre-instantiated kernels.
//
// Instantiated families: element U32 / REC8 / REC16 (plain only) x discriminator MOD / MASK x class
// bound M in {2, 4, 8, 16, 32, 64} (the smallest bound >= m is used; m itself
// is a run-time parameter of the functor).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "mdx_host.cuh"


using namespace mdx;
using namespace mdx::host;

extern "C" {

size_t mdx_workspace_size(uint64_t n, mdx_elem elem, uint32_t m) {
    if (check_elem(elem) != MDX_OK || m < 1 || m > MDX_MAX_CLASSES) return 0;
    return plain_layout(n, elem, m).total;
}

mdx_status mdx_workspace_init(void* d_ws, size_t ws_bytes, mdx_stream_t stream) {
    if (d_ws == nullptr || ws_bytes < kHeaderBytes) return MDX_ERR_WORKSPACE;
    if (reinterpret_cast<uintptr_t>(d_ws) % kAlign) return MDX_ERR_WORKSPACE;
    return cudaMemsetAsync(d_ws, 0, ws_bytes, reinterpret_cast<cudaStream_t>(stream)) == cudaSuccess
               ? MDX_OK
               : MDX_ERR_CUDA;
}

mdx_status mdx_workspace_error(void* d_ws, mdx_stream_t stream) {
    if (d_ws == nullptr) return MDX_ERR_WORKSPACE;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (cudaStreamSynchronize(st) != cudaSuccess) return MDX_ERR_CUDA;
    uint32_t err = 0;
    uint32_t* d_err = &reinterpret_cast<WsHeader*>(d_ws)->error;
    if (cudaMemcpy(&err, d_err, sizeof(err), cudaMemcpyDeviceToHost) != cudaSuccess)
        return MDX_ERR_CUDA;
    if (err != 0 && cudaMemset(d_err, 0, sizeof(err)) != cudaSuccess) return MDX_ERR_CUDA;
    if (err & kErrTimeout) return MDX_ERR_TIMEOUT;
    if (err & kErrSegments) return MDX_ERR_SEGMENTS;
    if (err & kErrCounts) return MDX_ERR_INVALID;
    return MDX_OK;
}

static mdx_status partition_impl(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                 mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                                 void* d_ws, size_t ws_bytes, mdx_stream_t stream,
                                 void* ev_count_done, bool allow_fused) {
    cudaEvent_t ev = reinterpret_cast<cudaEvent_t>(ev_count_done);
    mdx_status s = check_elem(elem);
    if (s != MDX_OK) return s;
    if ((s = check_discr(discr)) != MDX_OK) return s;
    if (n > MDX_MAX_ELEMS) return MDX_ERR_INVALID;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) {
        if (d_sizes && cudaMemsetAsync(d_sizes, 0, discr.m * sizeof(uint32_t), st) != cudaSuccess)
            return MDX_ERR_CUDA;
        return MDX_OK;
    }
    if (d_in == nullptr || d_out == nullptr) return MDX_ERR_INVALID;
    const size_t w = elem_bytes(elem);
    const char* ib = static_cast<const char*>(d_in);
    const char* ob = static_cast<const char*>(d_out);
    if (ib < ob + n * w && ob < ib + n * w) return MDX_ERR_INVALID;  // overlapping in/out
    if (reinterpret_cast<uintptr_t>(d_in) % w || reinterpret_cast<uintptr_t>(d_out) % w)
        return MDX_ERR_INVALID;  // elements must be naturally aligned
    const PlainLayout L = plain_layout(n, elem, discr.m);
    if (d_ws == nullptr || ws_bytes < L.total) return MDX_ERR_WORKSPACE;
    if (reinterpret_cast<uintptr_t>(d_ws) % kAlign) return MDX_ERR_WORKSPACE;
    unsigned char* ws = static_cast<unsigned char*>(d_ws);
    if (elem == MDX_ELEM_U32)
        return dispatch_plain<uint32_t>(d_in, d_out, n, discr, d_sizes, d_headflags, ws, L, st, ev,
                                        PlainStep::kBoth, nullptr, allow_fused);
    if (elem == MDX_ELEM_REC16)
        return dispatch_plain<Rec16>(d_in, d_out, n, discr, d_sizes, d_headflags, ws, L, st, ev,
                                     PlainStep::kBoth, nullptr, allow_fused);
    return dispatch_plain<uint64_t>(d_in, d_out, n, discr, d_sizes, d_headflags, ws, L, st, ev,
                                    PlainStep::kBoth, nullptr, allow_fused);
}

mdx_status mdx_partition_timed(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                               mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                               void* d_ws, size_t ws_bytes, mdx_stream_t stream,
                               void* ev_count_done) {
    return partition_impl(d_in, d_out, n, elem, discr, d_sizes, d_headflags, d_ws, ws_bytes, stream,
                          ev_count_done, true);
}


mdx_status mdx_partition(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                         mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags, void* d_ws,
                         size_t ws_bytes, mdx_stream_t stream) {
    return mdx_partition_timed(d_in, d_out, n, elem, discr, d_sizes, d_headflags, d_ws, ws_bytes,
                               stream, nullptr);
}

mdx_status mdx_dist_count(const void* d_in, uint64_t n_local, mdx_elem elem, mdx_discr discr,
                          uint32_t* d_counts, void* d_ws, size_t ws_bytes, mdx_stream_t stream) {
    mdx_status s = check_elem(elem);
    if (s != MDX_OK) return s;
    if (elem == MDX_ELEM_REC16) return MDX_ERR_UNSUPPORTED;
    if ((s = check_discr(discr)) != MDX_OK) return s;
    if (n_local > MDX_MAX_ELEMS || d_counts == nullptr) return MDX_ERR_INVALID;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (n_local == 0)
        return cudaMemsetAsync(d_counts, 0, discr.m * sizeof(uint32_t), st) == cudaSuccess
                   ? MDX_OK
                   : MDX_ERR_CUDA;
    if (d_in == nullptr || reinterpret_cast<uintptr_t>(d_in) % elem_bytes(elem)) return MDX_ERR_INVALID;
    const PlainLayout L = plain_layout(n_local, elem, discr.m);
    if (d_ws == nullptr || ws_bytes < L.total) return MDX_ERR_WORKSPACE;
    if (reinterpret_cast<uintptr_t>(d_ws) % kAlign) return MDX_ERR_WORKSPACE;
    unsigned char* ws = static_cast<unsigned char*>(d_ws);
    if (elem == MDX_ELEM_U32)
        return dispatch_plain<uint32_t>(d_in, nullptr, n_local, discr, d_counts, nullptr, ws, L, st,
                                        nullptr, PlainStep::kCount);
    return dispatch_plain<uint64_t>(d_in, nullptr, n_local, discr, d_counts, nullptr, ws, L, st,
                                    nullptr, PlainStep::kCount);
}

mdx_status mdx_dist_scatter(const void* d_in, uint64_t n_local, mdx_elem elem, mdx_discr discr,
                            const uint32_t* d_all_counts, uint32_t num_ranks, uint32_t rank,
                            void* const* out_chunks, uint64_t out_chunk, uint64_t n_total,
                            uint32_t* d_sizes, void* d_ws, size_t ws_bytes, mdx_stream_t stream) {
    mdx_status s = check_elem(elem);
    if (s != MDX_OK) return s;
    if (elem == MDX_ELEM_REC16) return MDX_ERR_UNSUPPORTED;
    if ((s = check_discr(discr)) != MDX_OK) return s;
    if (num_ranks == 0 || num_ranks > static_cast<uint32_t>(kMaxRanks) || rank >= num_ranks ||
        d_all_counts == nullptr || out_chunks == nullptr)
        return MDX_ERR_INVALID;
    const uint64_t w = elem_bytes(elem);
    if (n_total > MDX_MAX_ELEMS || n_local > n_total || out_chunk == 0 ||
        out_chunk % (16 / w) != 0 || out_chunk > MDX_MAX_ELEMS)
        return MDX_ERR_INVALID;
    // chunk q: [q * out_chunk, (q + 1) * out_chunk) within [0, n_total); the
    // last chunk: everything from (R - 1) * out_chunk on
    auto chunk_len = [&](uint32_t q) -> uint64_t {
        const uint64_t a = static_cast<uint64_t>(q) * out_chunk;
        if (a >= n_total) return 0;
        return q + 1 < num_ranks ? std::min<uint64_t>(out_chunk, n_total - a) : n_total - a;
    };
    DistOut dist;
    dist.all_counts = d_all_counts;
    dist.R = num_ranks;
    dist.rank = rank;
    dist.n_total = n_total;
    dist.chunk = out_chunk;
    for (uint32_t q = 0; q < num_ranks; q++) {
        if (chunk_len(q) > 0 &&
            (out_chunks[q] == nullptr || reinterpret_cast<uintptr_t>(out_chunks[q]) % 16))
            return MDX_ERR_INVALID;
        dist.chunks[q] = out_chunks[q];
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (d_ws == nullptr || reinterpret_cast<uintptr_t>(d_ws) % kAlign) return MDX_ERR_WORKSPACE;
    unsigned char* ws = static_cast<unsigned char*>(d_ws);
    if (n_local == 0) {  // nothing to send; still check the counts and give the sizes
        if (ws_bytes < kHeaderBytes) return MDX_ERR_WORKSPACE;
        uint32_t* skip = reinterpret_cast<uint32_t*>(ws + kDistSkipOffset);
        uint32_t* err = &reinterpret_cast<WsHeader*>(ws)->error;
        switch (class_bound(discr.m)) {
            case 2: plain_dist_bases_kernel<2><<<1, 64, 0, st>>>(d_all_counts, num_ranks, rank, discr.m, n_total, nullptr, nullptr, d_sizes, skip, err); break;
            case 4: plain_dist_bases_kernel<4><<<1, 64, 0, st>>>(d_all_counts, num_ranks, rank, discr.m, n_total, nullptr, nullptr, d_sizes, skip, err); break;
            case 8: plain_dist_bases_kernel<8><<<1, 64, 0, st>>>(d_all_counts, num_ranks, rank, discr.m, n_total, nullptr, nullptr, d_sizes, skip, err); break;
            case 16: plain_dist_bases_kernel<16><<<1, 64, 0, st>>>(d_all_counts, num_ranks, rank, discr.m, n_total, nullptr, nullptr, d_sizes, skip, err); break;
            case 32: plain_dist_bases_kernel<32><<<1, 64, 0, st>>>(d_all_counts, num_ranks, rank, discr.m, n_total, nullptr, nullptr, d_sizes, skip, err); break;
            default: plain_dist_bases_kernel<64><<<1, 64, 0, st>>>(d_all_counts, num_ranks, rank, discr.m, n_total, nullptr, nullptr, d_sizes, skip, err); break;
        }
        return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
    }
    if (d_in == nullptr || reinterpret_cast<uintptr_t>(d_in) % w) return MDX_ERR_INVALID;
    {  // the input must not overlap this rank's own output chunk
        const uint64_t own = chunk_len(rank);
        const char* ib = static_cast<const char*>(d_in);
        const char* ob = static_cast<const char*>(out_chunks[rank]);
        if (own > 0 && ib < ob + own * w && ob < ib + n_local * w) return MDX_ERR_INVALID;
    }
    const PlainLayout L = plain_layout(n_local, elem, discr.m);
    if (ws_bytes < L.total) return MDX_ERR_WORKSPACE;
    if (elem == MDX_ELEM_U32)
        return dispatch_plain<uint32_t>(d_in, nullptr, n_local, discr, d_sizes, nullptr, ws, L, st,
                                        nullptr, PlainStep::kScatter, &dist);
    return dispatch_plain<uint64_t>(d_in, nullptr, n_local, discr, d_sizes, nullptr, ws, L, st,
                                    nullptr, PlainStep::kScatter, &dist);
}

mdx_status mdx_ipc_get_handle(const void* d_ptr, void* handle, uint64_t* offset) {
    if (d_ptr == nullptr || handle == nullptr || offset == nullptr) return MDX_ERR_INVALID;
    using RangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
    static RangeFn range = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &p, 12000, cudaEnableDefault,
                                             &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            range = reinterpret_cast<RangeFn>(p);
    });
    if (range == nullptr) return MDX_ERR_UNSUPPORTED;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (range(&base, &size, reinterpret_cast<CUdeviceptr>(d_ptr)) != CUDA_SUCCESS)
        return MDX_ERR_INVALID;
    cudaIpcMemHandle_t h;
    if (cudaIpcGetMemHandle(&h, reinterpret_cast<void*>(base)) != cudaSuccess) return MDX_ERR_CUDA;
    std::memcpy(handle, &h, sizeof(h));
    *offset = reinterpret_cast<CUdeviceptr>(d_ptr) - base;
    return MDX_OK;
}

mdx_status mdx_ipc_open(const void* handle, uint64_t offset, void** d_ptr) {
    if (handle == nullptr || d_ptr == nullptr) return MDX_ERR_INVALID;
    cudaIpcMemHandle_t h;
    std::memcpy(&h, handle, sizeof(h));
    void* p = nullptr;
    if (cudaIpcOpenMemHandle(&p, h, cudaIpcMemLazyEnablePeerAccess) != cudaSuccess)
        return MDX_ERR_CUDA;
    *d_ptr = static_cast<unsigned char*>(p) + offset;
    return MDX_OK;
}

mdx_status mdx_ipc_close(void* d_ptr, uint64_t offset) {
    if (d_ptr == nullptr) return MDX_ERR_INVALID;
    return cudaIpcCloseMemHandle(static_cast<unsigned char*>(d_ptr) - offset) == cudaSuccess
               ? MDX_OK
               : MDX_ERR_CUDA;
}

mdx_status mdx_mdiscr(uint32_t n, uint32_t num_hwd_thds, const void* d_in, void* d_out,
                      mdx_elem elem, mdx_discr discr, uint32_t* h_sizes, void* d_ws,
                      size_t ws_bytes, mdx_stream_t stream) {
    (void)num_hwd_thds;
    if (h_sizes == nullptr) return MDX_ERR_INVALID;
    mdx_status s = check_discr(discr);
    if (s != MDX_OK) return s;
    const PlainLayout L = plain_layout(n, elem, discr.m);
    if (d_ws == nullptr || ws_bytes < L.total) return MDX_ERR_WORKSPACE;
    // The class totals land in the workspace (class_tot); copy them back.
    s = mdx_partition(d_in, d_out, n, elem, discr, nullptr, nullptr, d_ws, ws_bytes, stream);
    if (s != MDX_OK) return s;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) {
        memset(h_sizes, 0, discr.m * sizeof(uint32_t));
        return MDX_OK;
    }
    const uint32_t* tot = reinterpret_cast<const uint32_t*>(static_cast<unsigned char*>(d_ws) +
                                                            L.class_tot);
    if (cudaMemcpyAsync(h_sizes, tot, discr.m * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
        return MDX_ERR_CUDA;
    return mdx_workspace_error(d_ws, stream);
}

size_t mdx_segmented_workspace_size(uint64_t n, uint64_t num_segments, mdx_elem elem,
                                    uint32_t m) {
    if (check_elem(elem) != MDX_OK || elem == MDX_ELEM_REC16 || m < 1 || m > MDX_MAX_CLASSES)
        return 0;
    return seg_layout(n, num_segments, elem, m, false).total;
}

size_t mdx_mdiscr_segm_workspace_size(uint64_t n, mdx_elem elem, uint32_t m) {
    if (check_elem(elem) != MDX_OK || elem == MDX_ELEM_REC16 || m < 1 || m > MDX_MAX_CLASSES)
        return 0;
    return seg_layout(n, n, elem, m, true).total;
}

mdx_status mdx_partition_segmented(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                   mdx_discr discr, const uint64_t* d_offsets,
                                   uint64_t num_segments, uint32_t* d_seg_sizes,
                                   uint32_t* d_headflags, void* d_ws, size_t ws_bytes,
                                   mdx_stream_t stream) {
    mdx_status s = check_elem(elem);
    if (s != MDX_OK) return s;
    if (elem == MDX_ELEM_REC16) return MDX_ERR_UNSUPPORTED;  // plain path only
    if ((s = check_discr(discr)) != MDX_OK) return s;
    if (n > MDX_MAX_ELEMS || num_segments > MDX_MAX_ELEMS) return MDX_ERR_INVALID;
    if ((s = check_io(d_in, d_out, n, elem)) != MDX_OK) return s;
    if (num_segments == 0) return n == 0 ? MDX_OK : MDX_ERR_SEGMENTS;
    if (d_offsets == nullptr) return MDX_ERR_INVALID;
    if (class_bound(discr.m) > 16) return MDX_ERR_UNSUPPORTED;
    const SegLayout L = seg_layout(n, num_segments, elem, discr.m, false);
    if (d_ws == nullptr || ws_bytes < L.total) return MDX_ERR_WORKSPACE;
    if (reinterpret_cast<uintptr_t>(d_ws) % kAlign) return MDX_ERR_WORKSPACE;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* ws = static_cast<unsigned char*>(d_ws);
    if (elem == MDX_ELEM_U32)
        return dispatch_segm<uint32_t>(d_in, d_out, n, discr, d_offsets, num_segments, num_segments,
                                       nullptr, d_seg_sizes, d_headflags, ws, L, st);
    return dispatch_segm<uint64_t>(d_in, d_out, n, discr, d_offsets, num_segments, num_segments,
                                   nullptr, d_seg_sizes, d_headflags, ws, L, st);
}

mdx_status mdx_partition_segmented_multi(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                         const uint32_t* d_seg_m, uint32_t m_max,
                                         const uint64_t* d_offsets, uint64_t num_segments,
                                         uint32_t* d_seg_sizes, uint32_t* d_headflags,
                                         void* d_ws, size_t ws_bytes, mdx_stream_t stream) {
    mdx_status s = check_elem(elem);
    if (s != MDX_OK) return s;
    if (elem == MDX_ELEM_REC16) return MDX_ERR_UNSUPPORTED;  // plain path only
    if (m_max < 1 || m_max > 16) return m_max > 16 ? MDX_ERR_UNSUPPORTED : MDX_ERR_INVALID;
    if (n > MDX_MAX_ELEMS || num_segments > MDX_MAX_ELEMS) return MDX_ERR_INVALID;
    if ((s = check_io(d_in, d_out, n, elem)) != MDX_OK) return s;
    if (num_segments == 0) return n == 0 ? MDX_OK : MDX_ERR_SEGMENTS;
    if (d_offsets == nullptr || d_seg_m == nullptr) return MDX_ERR_INVALID;
    const SegLayout L = seg_layout(n, num_segments, elem, m_max, false);
    if (d_ws == nullptr || ws_bytes < L.total) return MDX_ERR_WORKSPACE;
    if (reinterpret_cast<uintptr_t>(d_ws) % kAlign) return MDX_ERR_WORKSPACE;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* ws = static_cast<unsigned char*>(d_ws);
    const DiscrMod d = DiscrMod::make(m_max);  // replaced per segment by key % m_s
    auto go = [&](auto tag) -> mdx_status {
        using V = decltype(tag);
        switch (class_bound(m_max)) {
            case 2: return run_segm<V, DiscrMod, 2>(d_in, d_out, n, d, m_max, d_offsets, num_segments, num_segments, nullptr, d_seg_sizes, d_headflags, ws, L, st, d_seg_m);
            case 4: return run_segm<V, DiscrMod, 4>(d_in, d_out, n, d, m_max, d_offsets, num_segments, num_segments, nullptr, d_seg_sizes, d_headflags, ws, L, st, d_seg_m);
            case 8: return run_segm<V, DiscrMod, 8>(d_in, d_out, n, d, m_max, d_offsets, num_segments, num_segments, nullptr, d_seg_sizes, d_headflags, ws, L, st, d_seg_m);
            default: return run_segm<V, DiscrMod, 16>(d_in, d_out, n, d, m_max, d_offsets, num_segments, num_segments, nullptr, d_seg_sizes, d_headflags, ws, L, st, d_seg_m);
        }
    };
    return elem == MDX_ELEM_U32 ? go(uint32_t{}) : go(uint64_t{});
}

mdx_status mdx_mdiscr_segm(uint32_t n, const void* d_in, const int32_t* d_segment_sizes,
                           void* d_out, int32_t* d_new_sizes, mdx_elem elem, mdx_discr discr,
                           void* d_ws, size_t ws_bytes, mdx_stream_t stream) {
    mdx_status s = check_elem(elem);
    if (s != MDX_OK) return s;
    if (elem == MDX_ELEM_REC16) return MDX_ERR_UNSUPPORTED;  // plain path only
    if ((s = check_discr(discr)) != MDX_OK) return s;
    if ((s = check_io(d_in, d_out, n, elem)) != MDX_OK) return s;
    if (n == 0) return MDX_OK;
    if (d_segment_sizes == nullptr) return MDX_ERR_INVALID;
    if (class_bound(discr.m) > 16) return MDX_ERR_UNSUPPORTED;
    const SegLayout L = seg_layout(n, n, elem, discr.m, true);
    if (d_ws == nullptr || ws_bytes < L.total) return MDX_ERR_WORKSPACE;
    if (reinterpret_cast<uintptr_t>(d_ws) % kAlign) return MDX_ERR_WORKSPACE;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    unsigned char* ws = static_cast<unsigned char*>(d_ws);
    uint64_t* offs = reinterpret_cast<uint64_t*>(ws + L.offsets);
    if ((s = launch_flags_to_offsets(d_segment_sizes, n, ws, L, st)) != MDX_OK) return s;
    uint32_t* hf = reinterpret_cast<uint32_t*>(d_new_sizes);
    if (elem == MDX_ELEM_U32)
        return dispatch_segm<uint32_t>(d_in, d_out, n, discr, offs, kSegsOnDevice, n,
                                       d_segment_sizes, nullptr, hf, ws, L, st);
    return dispatch_segm<uint64_t>(d_in, d_out, n, discr, offs, kSegsOnDevice, n, d_segment_sizes,
                                   nullptr, hf, ws, L, st);
}

}  // extern "C"

namespace mdx {
// The plain partition without the one-kernel cooperative path, for callers
// whose calls run side by side with other kernels (the serving loop's
// in-place lanes): a cooperative grid needs the whole GPU at once, so it would
// wait for every concurrent kernel to drain instead of interleaving with them.
mdx_status partition_two_kernel(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                                void* d_ws, size_t ws_bytes, mdx_stream_t stream) {
    return partition_impl(d_in, d_out, n, elem, discr, d_sizes, d_headflags, d_ws, ws_bytes, stream,
                          nullptr, false);
}
}  // namespace mdx


struct mdx_graph_st {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

namespace {
// Capture what `issue` launches on a private stream into a graph.  Relaxed
// mode: a kernel family's first call may set attributes and query occupancy
// while capturing.
template <class F>
mdx_status capture_graph(mdx_graph* out, F&& issue) {
    if (out == nullptr) return MDX_ERR_INVALID;
    *out = nullptr;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return MDX_ERR_CUDA;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaStreamDestroy(s);
        return MDX_ERR_CUDA;
    }
    const mdx_status st = issue(s);
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(s, &g);
    cudaStreamDestroy(s);
    if (st != MDX_OK || end != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return st != MDX_OK ? st : MDX_ERR_CUDA;
    }
    cudaGraphExec_t exec = nullptr;
    if (cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return MDX_ERR_CUDA;
    }
    *out = new mdx_graph_st{g, exec};
    return MDX_OK;
}
}  // namespace

extern "C" {

mdx_status mdx_graph_partition(mdx_graph* graph, const void* d_in, void* d_out, uint64_t n,
                               mdx_elem elem, mdx_discr discr, uint32_t* d_sizes,
                               uint32_t* d_headflags, void* d_ws, size_t ws_bytes) {
    return capture_graph(graph, [&](cudaStream_t s) {
        return mdx_partition(d_in, d_out, n, elem, discr, d_sizes, d_headflags, d_ws, ws_bytes,
                             reinterpret_cast<mdx_stream_t>(s));
    });
}

mdx_status mdx_graph_partition_segmented(mdx_graph* graph, const void* d_in, void* d_out,
                                         uint64_t n, mdx_elem elem, mdx_discr discr,
                                         const uint64_t* d_offsets, uint64_t num_segments,
                                         uint32_t* d_seg_sizes, uint32_t* d_headflags,
                                         void* d_ws, size_t ws_bytes) {
    return capture_graph(graph, [&](cudaStream_t s) {
        return mdx_partition_segmented(d_in, d_out, n, elem, discr, d_offsets, num_segments,
                                       d_seg_sizes, d_headflags, d_ws, ws_bytes,
                                       reinterpret_cast<mdx_stream_t>(s));
    });
}

mdx_status mdx_graph_launch(mdx_graph graph, mdx_stream_t stream) {
    if (graph == nullptr) return MDX_ERR_INVALID;
    return cudaGraphLaunch(graph->exec, reinterpret_cast<cudaStream_t>(stream)) == cudaSuccess
               ? MDX_OK
               : MDX_ERR_CUDA;
}

mdx_status mdx_graph_destroy(mdx_graph graph) {
    if (graph == nullptr) return MDX_OK;
    const bool ok = cudaGraphExecDestroy(graph->exec) == cudaSuccess &&
                    cudaGraphDestroy(graph->graph) == cudaSuccess;
    delete graph;
    return ok ? MDX_OK : MDX_ERR_CUDA;
}

mdx_status mdx_set_tuning(mdx_elem elem, uint32_t m, uint32_t log2_n_lo, uint32_t log2_n_hi,
                          const mdx_tuning* t) {
    if (check_elem(elem) != MDX_OK || t == nullptr || m < 1 || m > MDX_MAX_CLASSES ||
        log2_n_lo > log2_n_hi || log2_n_hi > 33)
        return MDX_ERR_INVALID;
    if (t->run_tiles > 64 || t->group_batch > 1024 || t->plain_two_kernel > 1 || t->pool_pct > 100 ||
        t->mid_tiles > static_cast<uint32_t>(kMidTiles) ||
        (t->tile_bytes != 0 && t->tile_bytes != 32 && t->tile_bytes != 64) ||
        (t->tile_threads != 0 && t->tile_threads != 256 && t->tile_threads != 512))
        return MDX_ERR_INVALID;
    TuningTable& tt = tuning_table();
    std::lock_guard<std::mutex> lk(tt.mu);
    for (uint32_t b = log2_n_lo; b <= log2_n_hi; b++) {
        Tuning& x = tt.t[elem == MDX_ELEM_REC8 ? 1 : 0][bound_index(class_bound(m))][b];
        x.plain_ctas_per_sm = t->plain_ctas_per_sm;
        x.run_tiles = t->run_tiles ? t->run_tiles : kRunTiles;
        x.group_batch = t->group_batch ? t->group_batch : kGroupBatch;
        x.plain_two_kernel = t->plain_two_kernel;
        x.pool_pct = t->pool_pct;
        x.mid_tiles = t->mid_tiles;
        x.tile_bytes = t->tile_bytes;
        x.tile_threads = t->tile_threads;
    }
    return MDX_OK;
}

mdx_status mdx_get_tuning(mdx_elem elem, uint32_t m, uint64_t n, mdx_tuning* t) {
    if (check_elem(elem) != MDX_OK || t == nullptr || m < 1 || m > MDX_MAX_CLASSES)
        return MDX_ERR_INVALID;
    const Tuning x = tuning_for(elem, class_bound(m), n);
    t->plain_ctas_per_sm = x.plain_ctas_per_sm;
    t->run_tiles = x.run_tiles;
    t->group_batch = x.group_batch;
    t->plain_two_kernel = x.plain_two_kernel;
    t->pool_pct = x.pool_pct ? x.pool_pct : kFusedPoolPct;
    t->mid_tiles = x.mid_tiles >= 2 ? x.mid_tiles : 1u;
    t->tile_bytes = x.tile_bytes == 32 ? 32u : 64u;
    t->tile_threads = x.tile_threads == 512 ? 512u : 256u;
    return MDX_OK;
}

void mdx_test_set_barrier_shortfall(uint32_t extra_arrivals, uint64_t wait_limit_ns) {
    g_test_bar_extra.store(extra_arrivals);
    g_test_wait_ns.store(wait_limit_ns);
}

const char* mdx_strerror(mdx_status s) {
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

const char* mdx_version(void) { return "mdx 0.1.0 sm_100a"; }

}  // extern "C"
