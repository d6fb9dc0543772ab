// mdx_host.cuh -- host-side launch code shared by the C ABI (mdx_capi.cu)
// and the header-only C++ templates (include/mdx/mdiscr.cuh): workspace
// layouts, occupancy cache, tensor-map encoding, per-family kernel dispatch.
#pragma once

#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched from the runtime)
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/mdx.h"
#include "mdx_fused.cuh"
#include "mdx_plain.cuh"
#include "mdx_segm.cuh"
#include "mdx_tile.cuh"

namespace mdx {
namespace host {

constexpr int kThreads = 256;
constexpr uint32_t kMaxChunks = 4096;
constexpr int kStages = 2;
constexpr size_t kHeaderBytes = 256;  // done, error, ... (see WsHeader)
constexpr size_t kAlign = 256;

struct WsHeader {  // first bytes of every workspace (the segmented header extends it)
    uint32_t seg_ticket;  // segmented kernel's ticket (SegHeader::ticket)
    uint32_t error;       // latched error bits, shared by every entry point
};
// The plain path's chunk ticket has a slot of its own, outside the 64-byte
// segmented header: one workspace may serve plain and segmented calls in turn,
// and each path leaves its own counters as the next call of that path expects.
constexpr size_t kPlainDoneOffset = 192;
static_assert(sizeof(SegHeader) <= kPlainDoneOffset, "plain ticket outside the segmented header");

template <class V>
struct ElemCfg;
template <>
struct ElemCfg<uint32_t> {
    static constexpr int kItems = 16;  // 4096-element tiles, 16 KB
};
template <>
struct ElemCfg<uint64_t> {
    static constexpr int kItems = 8;  // 2048-record tiles, 16 KB
};
template <>
struct ElemCfg<Rec16> {
    static constexpr int kItems = 4;  // 1024-record tiles, 16 KB
};

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

inline uint32_t class_bound(uint32_t m) {
    uint32_t b = 2;
    while (b < m) b <<= 1;
    return b;
}

inline size_t elem_bytes(mdx_elem e) { return e == MDX_ELEM_REC16 ? 16 : e == MDX_ELEM_REC8 ? 8 : 4; }
inline uint32_t tile_elems(mdx_elem e) {  // 64 bytes per thread
    return static_cast<uint32_t>(kThreads * 64 / elem_bytes(e));
}

inline uint32_t num_tiles_of(uint64_t n, mdx_elem e) {
    const uint64_t t = tile_elems(e);
    return static_cast<uint32_t>((n + t - 1) / t);
}

inline uint32_t max_chunks_of(uint64_t n, mdx_elem e) {
    const uint32_t nt = num_tiles_of(n, e);
    return nt < kMaxChunks ? (nt == 0 ? 1u : nt) : kMaxChunks;
}

struct PlainLayout {
    size_t class_base, class_tot, chunk_cnt, chunk_pre;
    size_t ready, tile_cnt, tile_pre;  // the one-kernel path's ready words and [tile][class] tables
    size_t total;
};

inline PlainLayout plain_layout(uint64_t n, mdx_elem e, uint32_t m) {
    const uint32_t M = class_bound(m);
    // rows of the [class][chunk] tables padded to 4 chunks (16-byte loads)
    const size_t G = (max_chunks_of(n, e) + 3u) & ~size_t{3};
    PlainLayout L;
    L.class_base = kHeaderBytes;
    L.class_tot = L.class_base + kMaxClasses * 4;
    L.chunk_cnt = align_up(L.class_tot + kMaxClasses * 4, kAlign);
    // [class][chunk] counts, then the chunks' ready words right after them
    // (one memset clears both), then the [class][chunk] prefixes
    L.ready = L.chunk_cnt + M * G * 4;
    L.chunk_pre = align_up(L.ready + 4 * G, kAlign);
    const size_t T = num_tiles_of(n, e);
    L.tile_cnt = align_up(L.chunk_pre + M * G * 4, kAlign);
    L.tile_pre = align_up(L.tile_cnt + M * T * 4, kAlign);
    L.total = align_up(L.tile_pre + M * T * 4, kAlign);
    return L;
}

inline bool is_pow2(uint32_t x) { return x && !(x & (x - 1)); }

inline mdx_status check_discr(mdx_discr d) {
    if (d.m < 1 || d.m > MDX_MAX_CLASSES) return MDX_ERR_INVALID;
    if (d.kind != MDX_DISCR_MOD && d.kind != MDX_DISCR_MASK) return MDX_ERR_INVALID;
    if (d.kind == MDX_DISCR_MASK && !is_pow2(d.m)) return MDX_ERR_INVALID;
    return MDX_OK;
}

inline mdx_status check_elem(mdx_elem e) {
    return (e == MDX_ELEM_U32 || e == MDX_ELEM_REC8 || e == MDX_ELEM_REC16) ? MDX_OK
                                                                               : MDX_ERR_INVALID;
}

// Resident CTAs per SM of a kernel, cached per (device, kernel).
struct OccEntry {
    int device;
    const void* fn;
    int blocks;
    int sms;
};
struct OccCache {
    std::mutex mu;
    OccEntry e[256];
    int n = 0;
};
inline OccCache& occ_cache() {
    static OccCache c;
    return c;
}

inline cudaError_t occupancy(const void* fn, size_t dyn_smem, int* blocks, int* sms,
                             int threads = kThreads) {
    OccCache& C = occ_cache();
    std::mutex& g_occ_mu = C.mu;
    OccEntry* g_occ = C.e;
    int& g_occ_n = C.n;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        for (int i = 0; i < g_occ_n; i++)
            if (g_occ[i].device == dev && g_occ[i].fn == fn) {
                *blocks = g_occ[i].blocks;
                *sms = g_occ[i].sms;
                return cudaSuccess;
            }
    }
    if (dyn_smem > 48 * 1024) {
        err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(dyn_smem));
        if (err != cudaSuccess) return err;
    }
    int b = 0, s = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, threads, dyn_smem);
    if (err != cudaSuccess) return err;
    err = cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
    if (err != cudaSuccess) return err;
    if (b < 1) b = 1;
    std::lock_guard<std::mutex> lk(g_occ_mu);
    if (g_occ_n < 256) g_occ[g_occ_n++] = OccEntry{dev, fn, b, s};
    *blocks = b;
    *sms = s;
    return cudaSuccess;
}

// cuTensorMapEncodeTiled, fetched through the runtime so the library needs no
// direct libcuda link.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn tensor_map_encoder() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                             &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// The n elements viewed as rows of 128 bytes (n * sizeof(V) / 128 whole rows),
// boxes of `box_rows` rows, 128-byte swizzle (thread-contiguous tile steps
// read 16-byte chunks of every row) or none (the warp-rank step of more than
// 16 classes reads the tile striped, one word per lane).  False if TMA
// cannot be used (unaligned base, fewer rows than one box, encoder
// unavailable).
inline bool make_row_map(CUtensorMap* map, const void* base, uint64_t n, size_t elem, uint32_t box_rows,
                         bool swizzle = true) {
    std::memset(map, 0, sizeof(*map));
    if (reinterpret_cast<uintptr_t>(base) % 16 != 0) return false;
    const uint64_t rows = n * elem / 128;  // whole 128-byte rows
    if (rows < box_rows) return false;
    EncodeTiledFn enc = tensor_map_encoder();
    if (enc == nullptr) return false;
    // the rows as 32 u32 words each, whatever the element width
    const cuuint64_t dims[2] = {32, rows};
    const cuuint64_t strides[1] = {128};
    const cuuint32_t box[2] = {32, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_UINT32;
    return enc(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE,
               swizzle ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ------------------------------------------------------------------ tuning --
// Run-time knobs per (element width, class bound, log2 n), installed by
// mdx_set_tuning (the package loads the autotuner's table at import).
struct Tuning {
    uint32_t plain_ctas_per_sm = 0;  // 0: as many as fit
    uint32_t run_tiles = kRunTiles;
    uint32_t group_batch = kGroupBatch;
    uint32_t plain_two_kernel = 0;  // 1: count and scatter as two kernels
    uint32_t pool_pct = 0;          // one-kernel path: % of every chunk drained by ticket (0: default)
    uint32_t mid_tiles = 0;         // segmented: medium segments up to this many tiles (0, 1: none)
    uint32_t tile_bytes = 0;        // plain path: tile bytes per thread (0, 64: 64; 32: 32)
    uint32_t tile_threads = 0;      // plain path: threads of a scatter CTA (0, 256: 256; 512)
};
struct TuningTable {
    std::mutex mu;
    Tuning t[2][7][34];  // [elem][log2 class bound - 1][ceil log2 n]
};
inline TuningTable& tuning_table() {
    static TuningTable tt;
    return tt;
}
inline uint32_t log2_ceil(uint64_t x) {
    uint32_t b = 0;
    while ((1ull << b) < x && b < 33) b++;
    return b;
}
inline int bound_index(uint32_t M) {
    int i = 0;
    while ((2u << i) < M && i < 6) i++;
    return i;
}
inline Tuning tuning_for(mdx_elem e, uint32_t M, uint64_t n) {
    TuningTable& tt = tuning_table();
    std::lock_guard<std::mutex> lk(tt.mu);
    return tt.t[e == MDX_ELEM_REC8 ? 1 : 0][bound_index(M)][log2_ceil(n)];
}

// Steps of a plain call: both kernels, or (distributed partition) the count
// alone and later the scatter alone into a sharded output.
enum class PlainStep { kBoth, kCount, kScatter };

// Sharded output of a distributed partition (kScatter).
struct DistOut {
    const uint32_t* all_counts;  // [R][m] class counts of every rank (device)
    uint32_t R, rank;
    uint64_t n_total;            // elements over all ranks
    void* chunks[kMaxRanks];     // output chunk of each rank (device pointers, peers' included)
    uint64_t chunk;              // elements per chunk (the last chunk: the rest)
};
// Set by plain_dist_bases_kernel when the counts are inconsistent.
constexpr size_t kDistSkipOffset = 196;
static_assert(kDistSkipOffset >= kPlainDoneOffset + 4 && kDistSkipOffset + 4 <= kHeaderBytes,
              "skip word inside the header, clear of the plain ticket");
// Test setting of the one-kernel plain path (mdx_test_set_barrier_shortfall):
// arrivals its grid barrier expects beyond the grid, and the wait's limit.
inline std::atomic<uint32_t> g_test_bar_extra{0};
inline std::atomic<uint64_t> g_test_wait_ns{0};
// Grid barrier and chunk tickets of the one-kernel plain path: arrival
// counter, generation, count-phase and scatter-phase tickets.
constexpr size_t kFusedBarOffset = 200;
constexpr uint32_t kFusedPoolPct = 10;  // share of every chunk drained by ticket (default)
static_assert(kFusedBarOffset >= kDistSkipOffset + 4 && kFusedBarOffset + 16 <= kHeaderBytes,
              "barrier words inside the header");

// BPT: bytes of a tile per thread (64: the tiles of every path; 32: tiles
// half as long); TS: threads of a scatter CTA (256, or 512 for tiles twice
// as long).  Geometries other than 64 bytes x 256 threads run the two-kernel
// path only, for the sizes where the tuning table picks them.
template <class V, class D, int M, int BPT, int TS>
mdx_status run_plain_g(const void* d_in, void* d_out, uint64_t n, D d, uint32_t m,
                       uint32_t* d_sizes, uint32_t* d_headflags, unsigned char* ws,
                       const PlainLayout& L, cudaStream_t stream, cudaEvent_t ev_mid,
                       PlainStep step, const DistOut* dist, bool allow_fused) {
    constexpr int ITEMS = BPT / static_cast<int>(sizeof(V));
    constexpr int TILE = TS * ITEMS;
    constexpr bool kBase = BPT == 64 && TS == kThreads;  // the geometry of every path
    static_assert(BPT != 64 || ITEMS == ElemCfg<V>::kItems, "64-byte tiles");
    auto count = plain_count_kernel<V, D, M, kThreads, TILE>;
    const void* scatter_fn;
    size_t smem;
    {
        using SL = ScatterTmaSmem<V, TS, kStages, M, BPT>;
        static_assert(SL::kTile == TILE, "both kernels use the same tiles");
        scatter_fn = reinterpret_cast<const void*>(
            plain_scatter_tma_kernel<V, D, M, TS, kStages, OutFlat<V>, BPT>);
        smem = SL::kBytes;
    }
    int blocks = 0, sms = 0;
    if (occupancy(scatter_fn, smem, &blocks, &sms, TS) != cudaSuccess) return MDX_ERR_CUDA;
    const uint32_t nt = static_cast<uint32_t>((n + TILE - 1) / TILE);
    const Tuning tun = tuning_for(sizeof(V) == 8 ? MDX_ELEM_REC8 : MDX_ELEM_U32, M, n);
    if (tun.plain_ctas_per_sm > 0 && static_cast<int>(tun.plain_ctas_per_sm) < blocks)
        blocks = static_cast<int>(tun.plain_ctas_per_sm);
    uint32_t G = static_cast<uint32_t>(blocks) * static_cast<uint32_t>(sms);
    if (G > nt) G = nt;
    if (G > kMaxChunks) G = kMaxChunks;

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
    a.done = reinterpret_cast<uint32_t*>(ws + kPlainDoneOffset);
    a.error = &reinterpret_cast<WsHeader*>(ws)->error;
    a.m = m;
    a.use_tma = 0;
    a.skip = nullptr;
    a.chunk_stride = (G + 3u) & ~3u;
    // a whole call: every scatter CTA forms its own prefixes (no serial scan);
    // the distributed steps keep the scan in the count kernel, whose class
    // totals go to the other ranks before the scatter
    a.prefix_in_scatter = step == PlainStep::kBoth ? 1 : 0;
    if (m == 1 && step == PlainStep::kBoth) {  // one class: the partition is a copy
        if ((d_headflags != nullptr &&
             cudaMemsetAsync(d_headflags, 0, n * sizeof(uint32_t), stream) != cudaSuccess) ||
            cudaMemcpyAsync(d_out, d_in, n * sizeof(V), cudaMemcpyDeviceToDevice, stream) !=
                cudaSuccess)
            return MDX_ERR_CUDA;
        plain_single_class_kernel<<<1, 32, 0, stream>>>(n, a.class_base, a.class_tot, d_sizes,
                                                         d_headflags);
        if (ev_mid != nullptr && cudaEventRecord(ev_mid, stream) != cudaSuccess) return MDX_ERR_CUDA;
        return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
    }
    if constexpr (kBase) {  // the one-kernel path has the base geometry only
        if (step == PlainStep::kBoth && dist == nullptr && ev_mid == nullptr && allow_fused &&
            tun.plain_two_kernel == 0) {
            // one cooperative kernel: count, grid barrier, scatter (mdx_fused.cuh)
            using SL = ScatterTmaSmem<V, kThreads, kStages, M>;
            CUtensorMap map;
            if (make_row_map(&map, d_in, n, sizeof(V), SL::kRows, M <= 16)) {
                auto fused = plain_fused_kernel<V, D, M, kThreads, kStages>;
                int fb = 0, fs = 0;
                if (occupancy(reinterpret_cast<const void*>(fused), smem, &fb, &fs) != cudaSuccess)
                    return MDX_ERR_CUDA;
                if (tun.plain_ctas_per_sm > 0 && static_cast<int>(tun.plain_ctas_per_sm) < fb)
                    fb = static_cast<int>(tun.plain_ctas_per_sm);
                uint32_t FG = static_cast<uint32_t>(fb) * static_cast<uint32_t>(fs);
                if (FG > nt) FG = nt;
                if (FG > kMaxChunks) FG = kMaxChunks;
                if (d_headflags != nullptr &&
                    cudaMemsetAsync(d_headflags, 0, n * sizeof(uint32_t), stream) != cudaSuccess)
                    return MDX_ERR_CUDA;
                FusedArgs fa;
                fa.p = a;
                fa.p.num_chunks = FG;
                fa.p.use_tma = 1;
                fa.chunk_stride = (FG + 3u) & ~3u;
                // pool: this share of every chunk's tiles is drained by ticket
                const uint32_t min_len = nt / FG;
                const uint32_t pct = tun.pool_pct ? tun.pool_pct : kFusedPoolPct;
                fa.pool = pct >= 100u ? 0u : min_len * pct / 100u;
                if (fa.pool >= min_len) fa.pool = min_len > 0 ? min_len - 1u : 0u;
                fa.tile_cnt = reinterpret_cast<uint32_t*>(ws + L.tile_cnt);
                fa.tile_pre = reinterpret_cast<uint32_t*>(ws + L.tile_pre);
                fa.ready = reinterpret_cast<uint32_t*>(ws + L.ready);
                fa.bar_count = reinterpret_cast<uint32_t*>(ws + kFusedBarOffset);
                fa.bar_gen = reinterpret_cast<uint32_t*>(ws + kFusedBarOffset + 4);
                fa.cnt_ticket = reinterpret_cast<uint32_t*>(ws + kFusedBarOffset + 8);
                fa.sct_ticket = reinterpret_cast<uint32_t*>(ws + kFusedBarOffset + 12);
                fa.bar_extra = g_test_bar_extra.load();
                const uint64_t lim = g_test_wait_ns.load();
                fa.wait_ns = lim != 0 ? lim : kWaitLimitNs;
                // chunk sums are added up by atomics; ready words start unset
                if (cudaMemsetAsync(ws + L.chunk_cnt, 0, L.ready + 4 * FG - L.chunk_cnt, stream) !=
                    cudaSuccess)
                    return MDX_ERR_CUDA;
                const OutFlat<V> o{static_cast<V*>(d_out),
                                   static_cast<uint32_t>((reinterpret_cast<uintptr_t>(d_out) / sizeof(V)) &
                                                         (16u / sizeof(V) - 1u))};
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3(FG);
                cfg.blockDim = dim3(kThreads);
                cfg.dynamicSmemBytes = smem;
                cfg.stream = stream;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeCooperative;
                attr[0].val.cooperative = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                if (cudaLaunchKernelEx(&cfg, fused, fa, d, map, o) != cudaSuccess) return MDX_ERR_CUDA;
                return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
            }
        }
    }
    if (step != PlainStep::kScatter) {
        // head flags: all zero but for count_c at offset_c, which the last
        // counting CTA writes
        if (d_headflags != nullptr &&
            cudaMemsetAsync(d_headflags, 0, n * sizeof(uint32_t), stream) != cudaSuccess)
            return MDX_ERR_CUDA;
        count<<<G, kThreads, 0, stream>>>(a, d);
        if (ev_mid != nullptr && cudaEventRecord(ev_mid, stream) != cudaSuccess) return MDX_ERR_CUDA;
    }
    if (step == PlainStep::kCount) return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
    {
        using SL = ScatterTmaSmem<V, TS, kStages, M, BPT>;
        CUtensorMap map;
        a.use_tma = make_row_map(&map, d_in, n, sizeof(V), SL::kRows, M <= 16) ? 1 : 0;
        if (dist == nullptr) {
            const OutFlat<V> o{static_cast<V*>(d_out),
                               static_cast<uint32_t>((reinterpret_cast<uintptr_t>(d_out) / sizeof(V)) &
                                                     (16u / sizeof(V) - 1u))};
            auto scatter = plain_scatter_tma_kernel<V, D, M, TS, kStages, OutFlat<V>, BPT>;
            if (step == PlainStep::kBoth && ev_mid == nullptr) {
                // programmatic dependent launch: scheduled while the count grid
                // drains, it starts its first tile copies before waiting for it
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3(G);
                cfg.blockDim = dim3(TS);
                cfg.dynamicSmemBytes = smem;
                cfg.stream = stream;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                attr[0].val.programmaticStreamSerializationAllowed = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                if (cudaLaunchKernelEx(&cfg, scatter, a, d, map, o) != cudaSuccess) return MDX_ERR_CUDA;
            } else {
                scatter<<<G, TS, smem, stream>>>(a, d, map, o);
            }
        } else if constexpr (sizeof(V) == 16 || !kBase) {
            return MDX_ERR_UNSUPPORTED;  // no sharded 16-byte record kernels; sharded: base tiles
        } else {
            // the sharded instantiation is a kernel of its own: give it the
            // shared-memory attribute too (the grid stays the count's G, the
            // chunks of both steps must match)
            int b2 = 0, s2 = 0;
            if (occupancy(reinterpret_cast<const void*>(
                              plain_scatter_tma_kernel<V, D, M, kThreads, kStages, OutSharded<V>>),
                          smem, &b2, &s2) != cudaSuccess)
                return MDX_ERR_CUDA;
            uint32_t* skip = reinterpret_cast<uint32_t*>(ws + kDistSkipOffset);
            plain_dist_bases_kernel<M><<<1, 64, 0, stream>>>(
                dist->all_counts, dist->R, dist->rank, m, dist->n_total, a.class_base, a.class_tot,
                d_sizes, skip, a.error);
            a.skip = skip;
            OutSharded<V> o;
            for (uint32_t q = 0; q < dist->R; q++) o.chunks[q] = static_cast<V*>(dist->chunks[q]);
            for (uint32_t q = dist->R; q < static_cast<uint32_t>(kMaxRanks); q++) o.chunks[q] = nullptr;
            o.chunk = static_cast<uint32_t>(dist->chunk);
            o.R = dist->R;
            plain_scatter_tma_kernel<V, D, M, kThreads, kStages, OutSharded<V>>
                <<<G, kThreads, smem, stream>>>(a, d, map, o);
        }
    }
    return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
}

template <class V, class D, int M>
mdx_status run_plain(const void* d_in, void* d_out, uint64_t n, D d, uint32_t m, uint32_t* d_sizes,
                     uint32_t* d_headflags, unsigned char* ws, const PlainLayout& L,
                     cudaStream_t stream, cudaEvent_t ev_mid, PlainStep step = PlainStep::kBoth,
                     const DistOut* dist = nullptr, bool allow_fused = true) {
    if constexpr (sizeof(V) <= 8) {
        const Tuning tun = tuning_for(sizeof(V) == 8 ? MDX_ELEM_REC8 : MDX_ELEM_U32, M, n);
        if (dist == nullptr && step == PlainStep::kBoth) {
            if constexpr (M <= 16) {  // the warp-rank step spills at 512 threads
                if (tun.tile_threads == 512)
                    return run_plain_g<V, D, M, 64, 512>(d_in, d_out, n, d, m, d_sizes, d_headflags,
                                                         ws, L, stream, ev_mid, step, dist,
                                                         allow_fused);
            }
            if (tun.tile_bytes == 32)
                return run_plain_g<V, D, M, 32, kThreads>(d_in, d_out, n, d, m, d_sizes,
                                                          d_headflags, ws, L, stream, ev_mid, step,
                                                          dist, allow_fused);
        }
    }
    return run_plain_g<V, D, M, 64, kThreads>(d_in, d_out, n, d, m, d_sizes, d_headflags, ws, L,
                                              stream, ev_mid, step, dist, allow_fused);
}

template <class V, class D>
mdx_status dispatch_plain_m(const void* in, void* out, uint64_t n, D d, uint32_t m, uint32_t* sz,
                            uint32_t* hf, unsigned char* ws, const PlainLayout& L,
                            cudaStream_t st, cudaEvent_t ev, PlainStep step, const DistOut* dist,
                            bool fu) {
    switch (class_bound(m)) {
        case 2: return run_plain<V, D, 2>(in, out, n, d, m, sz, hf, ws, L, st, ev, step, dist, fu);
        case 4: return run_plain<V, D, 4>(in, out, n, d, m, sz, hf, ws, L, st, ev, step, dist, fu);
        case 8: return run_plain<V, D, 8>(in, out, n, d, m, sz, hf, ws, L, st, ev, step, dist, fu);
        case 16: return run_plain<V, D, 16>(in, out, n, d, m, sz, hf, ws, L, st, ev, step, dist, fu);
        case 32: return run_plain<V, D, 32>(in, out, n, d, m, sz, hf, ws, L, st, ev, step, dist, fu);
        case 64: return run_plain<V, D, 64>(in, out, n, d, m, sz, hf, ws, L, st, ev, step, dist, fu);
        default: return MDX_ERR_INVALID;
    }
}

// key % m == key & (m - 1) for unsigned keys when m is a power of two (Mod<4>
// and Mod4 agree), so such MOD requests take the mask functor.
inline bool use_mask(mdx_discr dc) { return dc.kind == MDX_DISCR_MASK || is_pow2(dc.m); }

template <class V>
mdx_status dispatch_plain(const void* in, void* out, uint64_t n, mdx_discr dc, uint32_t* sz,
                          uint32_t* hf, unsigned char* ws, const PlainLayout& L, cudaStream_t st,
                          cudaEvent_t ev, PlainStep step = PlainStep::kBoth,
                          const DistOut* dist = nullptr, bool allow_fused = true) {
    if (use_mask(dc))
        return dispatch_plain_m<V>(in, out, n, DiscrMask{dc.m - 1u}, dc.m, sz, hf, ws, L, st, ev,
                                   step, dist, allow_fused);
    return dispatch_plain_m<V>(in, out, n, DiscrMod::make(dc.m), dc.m, sz, hf, ws, L, st, ev, step,
                               dist, allow_fused);
}

// ------------------------------------------------------------- segmented --
constexpr int kPlanThreads = 256;
constexpr uint32_t kMaxPlanBlocks = 1024;
constexpr int kFlagsTile = 4096;
constexpr uint32_t kMaxFlagChunks = 4096;

inline uint32_t window_elems(mdx_elem e) { return tile_elems(e); }

struct SegLayout {
    size_t run_loc, grp_loc, blk_runs, blk_grps, runs, groups, groups_end, run_cnt, run_base,
        mid_loc, blk_mids, mids, offsets, flag_stage, flag_cnt, flag_pre, total;
    uint64_t max_runs, max_groups, max_mids;
};

// flags_form: room for n+1 offsets and the converter's tile status words.
inline SegLayout seg_layout(uint64_t n, uint64_t S, mdx_elem e, uint32_t m, bool flags_form) {
    const uint32_t M = class_bound(m);
    const uint64_t P = window_elems(e);
    const uint64_t NW = (n + P - 1) / P;
    SegLayout L;
    L.max_runs = 2 * NW + 2;    // runs of segments that tile [0, n): far fewer
    // a group starts at a new window of P elements or after kGroupSegs segments
    const uint64_t GW = P;  // group_window<P>()
    L.max_groups = (n + GW - 1) / GW + S / kGroupSegs + 2;
    L.run_loc = kHeaderBytes;
    L.grp_loc = align_up(L.run_loc + 4 * (S + 1), kAlign);
    L.blk_runs = align_up(L.grp_loc + 4 * (S + 1), kAlign);
    L.blk_grps = align_up(L.blk_runs + 4 * kMaxPlanBlocks, kAlign);
    L.runs = align_up(L.blk_grps + 4 * kMaxPlanBlocks, kAlign);
    L.groups = align_up(L.runs + sizeof(RunEntry) * L.max_runs, kAlign);
    L.groups_end = align_up(L.groups + 4 * L.max_groups, kAlign);
    L.run_cnt = align_up(L.groups_end + 4 * L.max_groups, kAlign);
    L.run_base = align_up(L.run_cnt + 4ull * M * L.max_runs, kAlign);
    L.max_mids = n / (P + 1) + 2;  // a medium segment holds more than P elements
    L.mid_loc = align_up(L.run_base + 4ull * M * L.max_runs, kAlign);
    L.blk_mids = align_up(L.mid_loc + 4 * (S + 1), kAlign);
    L.mids = align_up(L.blk_mids + 4 * kMaxPlanBlocks, kAlign);
    L.offsets = align_up(L.mids + 4 * L.max_mids, kAlign);
    L.flag_stage = L.flag_cnt = L.flag_pre = L.offsets;
    L.total = L.offsets;
    if (flags_form) {  // offsets, staged start positions, per-chunk counts and prefixes
        L.flag_stage = align_up(L.offsets + 8 * (n + 1), kAlign);
        L.flag_cnt = align_up(L.flag_stage + 4 * n, kAlign);
        L.flag_pre = align_up(L.flag_cnt + 4 * kMaxFlagChunks, kAlign);
        L.total = align_up(L.flag_pre + 4 * kMaxFlagChunks, kAlign);
    }
    return L;
}

inline uint32_t plan_blocks_for(uint64_t S_bound) {
    uint64_t g = (S_bound + 511) / 512;
    if (g < 1) g = 1;
    if (g > kMaxPlanBlocks) g = kMaxPlanBlocks;
    return static_cast<uint32_t>(g);
}

template <class V, class D, int M>
mdx_status run_segm(const void* d_in, void* d_out, uint64_t n, D d, uint32_t m,
                    const uint64_t* d_offsets, uint64_t S, uint64_t S_bound, const int32_t* in_flags,
                    uint32_t* d_seg_sizes, uint32_t* d_headflags, unsigned char* ws,
                    const SegLayout& L, cudaStream_t st, const uint32_t* d_seg_m = nullptr) {
    using SL = SegSmem<V, M, kThreads, kStages>;
    constexpr int P = SL::kTile;
    using ML = MidSmem<V, M, kThreads, kMidTiles>;
    auto main_fn = seg_main<V, D, M, kThreads, kStages>;
    auto scatter_fn = seg_run_scatter<V, D, M, kThreads, kStages>;
    auto mid_fn = seg_mid<V, D, M, kThreads, kMidTiles>;
    int blocks = 0, sms = 0, sblocks = 0, mblocks = 0;
    if (occupancy(reinterpret_cast<const void*>(main_fn), SL::kBytes, &blocks, &sms) != cudaSuccess ||
        occupancy(reinterpret_cast<const void*>(scatter_fn), SL::kRunBytes, &sblocks, &sms) !=
            cudaSuccess ||
        occupancy(reinterpret_cast<const void*>(mid_fn), ML::kBytes, &mblocks, &sms) != cudaSuccess)
        return MDX_ERR_CUDA;
    SegArgs a;
    a.in = d_in;
    a.out = d_out;
    a.n = n;
    a.offsets = d_offsets;
    a.num_segs = S;
    a.seg_sizes = d_seg_sizes;
    a.headflags = d_headflags;
    a.in_flags = in_flags;
    a.m = m;
    a.hdr = reinterpret_cast<SegHeader*>(ws);
    a.run_loc = reinterpret_cast<uint32_t*>(ws + L.run_loc);
    a.grp_loc = reinterpret_cast<uint32_t*>(ws + L.grp_loc);
    a.blk_runs = reinterpret_cast<uint32_t*>(ws + L.blk_runs);
    a.blk_grps = reinterpret_cast<uint32_t*>(ws + L.blk_grps);
    a.runs = reinterpret_cast<RunEntry*>(ws + L.runs);
    a.groups = reinterpret_cast<uint32_t*>(ws + L.groups);
    a.groups_end = reinterpret_cast<uint32_t*>(ws + L.groups_end);
    a.run_cnt = reinterpret_cast<uint32_t*>(ws + L.run_cnt);
    a.run_base = reinterpret_cast<uint32_t*>(ws + L.run_base);
    a.mid_loc = reinterpret_cast<uint32_t*>(ws + L.mid_loc);
    a.blk_mids = reinterpret_cast<uint32_t*>(ws + L.blk_mids);
    a.mids = reinterpret_cast<uint32_t*>(ws + L.mids);
    a.max_mids = static_cast<uint32_t>(L.max_mids);
    a.plan_blocks = plan_blocks_for(S_bound);
    a.max_runs = static_cast<uint32_t>(L.max_runs);
    a.max_groups = static_cast<uint32_t>(L.max_groups);
    a.seg_m = d_seg_m;
    a.m_bound = m;
    {
        const Tuning tun = tuning_for(sizeof(V) == 8 ? MDX_ELEM_REC8 : MDX_ELEM_U32, M, n);
        a.run_tiles = tun.run_tiles >= 1 ? tun.run_tiles : kRunTiles;
        a.group_batch = tun.group_batch >= 1 ? tun.group_batch : kGroupBatch;
        if (a.group_batch > static_cast<uint32_t>(kMaxGroupBatch)) a.group_batch = kMaxGroupBatch;
        // 0 (default) and 1: no medium segments
        a.mid_tiles = tun.mid_tiles >= 2 ? tun.mid_tiles : 0u;
        if (a.mid_tiles > static_cast<uint32_t>(kMidTiles)) a.mid_tiles = kMidTiles;
    }
    CUtensorMap map;
    a.use_tma = make_row_map(&map, d_in, n, sizeof(V), SL::G::kRows) ? 1 : 0;
    if (d_headflags != nullptr &&
        cudaMemsetAsync(d_headflags, 0, n * sizeof(uint32_t), st) != cudaSuccess)
        return MDX_ERR_CUDA;
    if (cudaMemsetAsync(a.groups_end, 0xff, L.max_groups * sizeof(uint32_t), st) != cudaSuccess)
        return MDX_ERR_CUDA;
    seg_plan_spans<P, kPlanThreads><<<a.plan_blocks, kPlanThreads, 0, st>>>(a);
    seg_plan_emit<P, kPlanThreads><<<a.plan_blocks, kPlanThreads, 0, st>>>(a);
    main_fn<<<static_cast<uint32_t>(blocks) * sms, kThreads, SL::kBytes, st>>>(a, d);
    if (a.mid_tiles > 0)
        mid_fn<<<static_cast<uint32_t>(mblocks) * sms, kThreads, ML::kBytes, st>>>(a, d, map);
    {
        auto count_fn = seg_run_count<V, D, M, kThreads>;
        int cblocks = 0;
        if (occupancy(reinterpret_cast<const void*>(count_fn), 0, &cblocks, &sms) != cudaSuccess)
            return MDX_ERR_CUDA;
        count_fn<<<static_cast<uint32_t>(cblocks) * sms, kThreads, 0, st>>>(a, d);
    }
    // a warp per 32 runs (the run count is on the device: enough for the capacity)
    const uint64_t scan_blocks = std::min<uint64_t>((L.max_runs + 255) / 256, 4096);
    seg_run_scan<M><<<static_cast<uint32_t>(scan_blocks), 256, 0, st>>>(a);
    scatter_fn<<<static_cast<uint32_t>(sblocks) * sms, kThreads, SL::kRunBytes, st>>>(a, d, map);
    return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
}

template <class V, class D>
mdx_status dispatch_segm_m(const void* in, void* out, uint64_t n, D d, uint32_t m,
                           const uint64_t* offs, uint64_t S, uint64_t Sb, const int32_t* fl,
                           uint32_t* sz, uint32_t* hf, unsigned char* ws, const SegLayout& L,
                           cudaStream_t st) {
    switch (class_bound(m)) {
        case 2: return run_segm<V, D, 2>(in, out, n, d, m, offs, S, Sb, fl, sz, hf, ws, L, st);
        case 4: return run_segm<V, D, 4>(in, out, n, d, m, offs, S, Sb, fl, sz, hf, ws, L, st);
        case 8: return run_segm<V, D, 8>(in, out, n, d, m, offs, S, Sb, fl, sz, hf, ws, L, st);
        case 16: return run_segm<V, D, 16>(in, out, n, d, m, offs, S, Sb, fl, sz, hf, ws, L, st);
        default: return MDX_ERR_UNSUPPORTED;
    }
}

template <class V>
mdx_status dispatch_segm(const void* in, void* out, uint64_t n, mdx_discr dc, const uint64_t* offs,
                         uint64_t S, uint64_t Sb, const int32_t* fl, uint32_t* sz, uint32_t* hf,
                         unsigned char* ws, const SegLayout& L, cudaStream_t st) {
    if (use_mask(dc))
        return dispatch_segm_m<V>(in, out, n, DiscrMask{dc.m - 1u}, dc.m, offs, S, Sb, fl, sz, hf,
                                  ws, L, st);
    return dispatch_segm_m<V>(in, out, n, DiscrMod::make(dc.m), dc.m, offs, S, Sb, fl, sz, hf, ws,
                              L, st);
}

// Head-flag segment sizes -> offsets (written into the workspace's offsets
// area) and S into the header, ahead of run_segm with kSegsOnDevice.
inline mdx_status launch_flags_to_offsets(const int32_t* d_flags, uint64_t n, unsigned char* ws,
                                          const SegLayout& L, cudaStream_t st) {
    auto stage_fn = seg_flags_stage<kThreads, kFlagsTile>;
    int blocks = 0, sms = 0;
    if (occupancy(reinterpret_cast<const void*>(stage_fn), 0, &blocks, &sms) != cudaSuccess)
        return MDX_ERR_CUDA;
    const uint64_t tiles = (n + kFlagsTile - 1) / kFlagsTile;
    uint64_t G = static_cast<uint64_t>(blocks) * sms;
    if (G > tiles) G = tiles;
    if (G > kMaxFlagChunks) G = kMaxFlagChunks;
    if (G < 1) G = 1;
    FlagsArgs fa;
    fa.flags = d_flags;
    fa.n = n;
    fa.chunk = ((n + G - 1) / G + 3u) & ~uint64_t{3};
    fa.stage = reinterpret_cast<uint32_t*>(ws + L.flag_stage);
    fa.cnt = reinterpret_cast<uint32_t*>(ws + L.flag_cnt);
    fa.pre = reinterpret_cast<uint32_t*>(ws + L.flag_pre);
    fa.offsets = reinterpret_cast<uint64_t*>(ws + L.offsets);
    fa.hdr = reinterpret_cast<SegHeader*>(ws);
    stage_fn<<<static_cast<uint32_t>(G), kThreads, 0, st>>>(fa);
    seg_flags_compact<kThreads><<<static_cast<uint32_t>(G), kThreads, 0, st>>>(fa);
    return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
}

inline mdx_status check_io(const void* d_in, void* d_out, uint64_t n, mdx_elem elem) {
    if (n == 0) return MDX_OK;
    if (d_in == nullptr || d_out == nullptr) return MDX_ERR_INVALID;
    const size_t w = elem_bytes(elem);
    const char* ib = static_cast<const char*>(d_in);
    const char* ob = static_cast<const char*>(d_out);
    if (ib < ob + n * w && ob < ib + n * w) return MDX_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(d_in) % w || reinterpret_cast<uintptr_t>(d_out) % w)
        return MDX_ERR_INVALID;
    return MDX_OK;
}

}  // namespace host
}  // namespace mdx
