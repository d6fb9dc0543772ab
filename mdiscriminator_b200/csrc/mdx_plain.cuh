// mdx_plain.cuh -- plain (unsegmented) stable m-way partition for sm_100a.
//
// Replaces the reference's four-phase pipeline of mdiscr<DISCR>
// (cuda_code/MdiscrHost_optimized_clean.cu.h:9-150: transposePad ->
// mapVctKernel -> recursive scanInc with a mid-pipeline D2H copy ->
// writeMultiKernel, ~32 B of HBM traffic per int32 element, four host syncs and
// per-call cudaMalloc) by two kernels and no host round trip:
//
//   plain_count_kernel   reads each element once (4 B/elem for int32) and
//                        counts classes per chunk; the last CTA to finish
//                        (ticket on a workspace counter, no waiting) scans the
//                        per-chunk counts into per-chunk class prefixes, the
//                        class bases (exclusive scan of the totals, the
//                        `offsets` of SeqMdiscr.h:34-38) and the class sizes.
//   plain_scatter_tma_kernel (m <= 16) / plain_scatter_kernel (m <= 64)
//                        re-read each element (4 B) and write it once (4 B):
//                        per tile, element ranks (thread-local byte counters
//                        and a block scan; or warp ranks from __match_any_sync
//                        + __popc for more classes),
//                        a block scan of the per-warp class counts, a
//                        shared-memory staged scatter so every class run leaves
//                        the SM as coalesced stores.  Tiles are staged into
//                        shared memory by TMA bulk copies (cp.async.bulk, no
//                        multicast) through an mbarrier ring.  Each CTA walks
//                        its chunk from the end backwards, so the tiles the
//                        count kernel read last are still in L2.
//
// Why two passes: the output position of a class-c element is
// base_c + prefix_c(tile) + rank, and base_c = sum of the totals of classes
// below c depends on every element of the input, the last one included.  With
// on-chip storage (~33 MB shared memory + 126 MB L2) far below the 1 GiB input
// of N = 2^28 int32, no element of class >= 1 can be stored before the whole
// input has been read, so the minimum traffic is read + re-read + write
// (12 B/elem), minus whatever the re-read finds in L2.
#pragma once

#include <cuda.h>  // CUtensorMap (type only; maps are encoded by the host)

#include "mdx_device.cuh"

namespace mdx {

struct PlainArgs {
    const void* in;
    void* out;
    uint64_t n;
    uint32_t num_tiles;   // ceil(n / TILE)
    uint32_t num_chunks;  // G: one chunk of consecutive tiles per CTA
    uint32_t* chunk_cnt;  // [M][G] class counts per chunk
    uint32_t* chunk_pre;  // [M][G] exclusive prefix of chunk_cnt over chunks
    uint32_t* class_base; // [M]    exclusive scan of the class totals
    uint32_t* class_tot;  // [M]    class totals
    uint32_t* sizes;      // [m]    user output (tuple form) or null
    uint32_t* headflags;  // [n]    user output (head-flag form) or null
    uint32_t* done;       // chunk ticket counter (0 on entry, reset to 0 by the last CTA)
    uint32_t* error;      // latched error bits
    uint32_t m;
    int use_tma;          // the tensor map passed to the scatter kernel is valid
};

// Chunk k covers tiles [k*T/G, (k+1)*T/G).
__device__ __forceinline__ void chunk_tiles(uint32_t k, uint32_t T, uint32_t G, uint32_t& t0,
                                            uint32_t& t1) {
    t0 = static_cast<uint32_t>(static_cast<uint64_t>(k) * T / G);
    t1 = static_cast<uint32_t>(static_cast<uint64_t>(k + 1) * T / G);
}

template <class V>
__device__ __forceinline__ void unpack16(const uint4& r, V (&e)[16 / sizeof(V)]);
template <>
__device__ __forceinline__ void unpack16<uint32_t>(const uint4& r, uint32_t (&e)[4]) {
    e[0] = r.x; e[1] = r.y; e[2] = r.z; e[3] = r.w;
}
template <>
__device__ __forceinline__ void unpack16<uint64_t>(const uint4& r, uint64_t (&e)[2]) {
    e[0] = static_cast<uint64_t>(r.x) | (static_cast<uint64_t>(r.y) << 32);
    e[1] = static_cast<uint64_t>(r.z) | (static_cast<uint64_t>(r.w) << 32);
}

// Per-thread class counters for M <= 16: 8-bit lanes packed in u64 words,
// flushed into u32 accumulators before any lane can reach 256.
template <int M>
struct PackedCounts {
    static_assert(M <= 16, "packed counters cover at most 16 classes");
    static constexpr int NW = (M + 7) / 8;
    uint64_t pk[NW];
    uint32_t acc[M];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int w = 0; w < NW; w++) pk[w] = 0;
#pragma unroll
        for (int c = 0; c < M; c++) acc[c] = 0;
    }
    __device__ __forceinline__ void add(uint32_t c) {
        if constexpr (NW == 1) {
            pk[0] += 1ull << (c << 3);
        } else {
            const uint64_t inc = 1ull << ((c & 7u) << 3);
            pk[0] += (c < 8u) ? inc : 0ull;
            pk[1] += (c < 8u) ? 0ull : inc;
        }
    }
    __device__ __forceinline__ void flush() {
#pragma unroll
        for (int c = 0; c < M; c++)
            acc[c] += static_cast<uint32_t>(pk[c >> 3] >> ((c & 7) * 8)) & 0xffu;
#pragma unroll
        for (int w = 0; w < NW; w++) pk[w] = 0;
    }
};

// After every CTA has published its chunk counts, the last CTA turns them into
// per-chunk exclusive prefixes, class totals, class bases and the user's sizes,
// then resets the ticket counter for the next call.
template <int M, int THREADS>
__device__ void plain_finish_scan(const PlainArgs& a, uint32_t* tot_sh) {
    constexpr int W = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t G = a.num_chunks;
    for (int c = warp; c < M; c += W) {
        uint32_t run = 0;
        for (uint32_t k0 = 0; k0 < G; k0 += 32) {
            const uint32_t kk = k0 + lane;
            const uint32_t x = kk < G ? __ldcg(&a.chunk_cnt[c * G + kk]) : 0u;
            const uint32_t incl = warp_incl_scan(x);
            if (kk < G) a.chunk_pre[c * G + kk] = run + incl - x;
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) tot_sh[c] = run;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int c = 0; c < M; c++) {
            a.class_base[c] = acc;
            a.class_tot[c] = tot_sh[c];
            if (a.sizes != nullptr && static_cast<uint32_t>(c) < a.m) a.sizes[c] = tot_sh[c];
            // head-flag form (SeqMdiscr.h:47-49): count_c at offset_c; the
            // rest of the array was zeroed before this kernel
            if (a.headflags != nullptr && tot_sh[c] > 0) a.headflags[acc] = tot_sh[c];
            acc += tot_sh[c];
        }
        *a.done = 0u;
    }
}

template <class V, class D, int M, int THREADS, int TILE>
__global__ void __launch_bounds__(THREADS) plain_count_kernel(PlainArgs a, D d) {
    constexpr int W = THREADS / 32;
    constexpr int VEC = 16 / static_cast<int>(sizeof(V));
    constexpr int UNROLL = 4;
    __shared__ uint32_t red[W][M];
    __shared__ uint32_t tot_sh[M];
    __shared__ int am_last;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t G = a.num_chunks, k = blockIdx.x;
    uint32_t t0, t1;
    chunk_tiles(k, a.num_tiles, G, t0, t1);
    const uint64_t e0 = static_cast<uint64_t>(t0) * TILE;
    const uint64_t e1 = min(static_cast<uint64_t>(t1) * TILE, a.n);
    const V* in = static_cast<const V*>(a.in);
    const bool vec_ok = (reinterpret_cast<uintptr_t>(in) & 15u) == 0;

    if constexpr (M <= 16) {
        PackedCounts<M> pc;
        pc.init();
        if (vec_ok) {
            const uint4* vp = reinterpret_cast<const uint4*>(in + e0);
            const uint64_t nv = (e1 - e0) / VEC;
            int since_flush = 0;
            for (uint64_t i = tid; i < nv; i += static_cast<uint64_t>(THREADS) * UNROLL) {
                uint4 r[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; u++) {
                    const uint64_t j = i + static_cast<uint64_t>(u) * THREADS;
                    if (j < nv) r[u] = __ldg(vp + j);
                }
#pragma unroll
                for (int u = 0; u < UNROLL; u++) {
                    const uint64_t j = i + static_cast<uint64_t>(u) * THREADS;
                    if (j < nv) {
                        V e[VEC];
                        unpack16<V>(r[u], e);
#pragma unroll
                        for (int q = 0; q < VEC; q++) pc.add(d(e[q]));
                    }
                }
                if (++since_flush == 15) {  // <= 15 * 16 = 240 increments per lane
                    pc.flush();
                    since_flush = 0;
                }
            }
            for (uint64_t e = e0 + nv * VEC + tid; e < e1; e += THREADS) pc.add(d(in[e]));
        } else {
            int since_flush = 0;
            for (uint64_t e = e0 + tid; e < e1; e += THREADS) {
                pc.add(d(in[e]));
                if (++since_flush == 255) {
                    pc.flush();
                    since_flush = 0;
                }
            }
        }
        pc.flush();
#pragma unroll
        for (int c = 0; c < M; c++) {
            const uint32_t s = warp_sum(pc.acc[c]);
            if (lane == 0) red[warp][c] = s;
        }
    } else {
        for (int c = lane; c < M; c += 32) red[warp][c] = 0;
        __syncwarp();
        if (vec_ok) {
            const uint4* vp = reinterpret_cast<const uint4*>(in + e0);
            const uint64_t nv = (e1 - e0) / VEC;
            for (uint64_t i = tid; i < nv; i += static_cast<uint64_t>(THREADS) * UNROLL) {
                uint4 r[UNROLL];
#pragma unroll
                for (int u = 0; u < UNROLL; u++) {
                    const uint64_t j = i + static_cast<uint64_t>(u) * THREADS;
                    if (j < nv) r[u] = __ldg(vp + j);
                }
#pragma unroll
                for (int u = 0; u < UNROLL; u++) {
                    const uint64_t j = i + static_cast<uint64_t>(u) * THREADS;
                    if (j < nv) {
                        V e[VEC];
                        unpack16<V>(r[u], e);
#pragma unroll
                        for (int q = 0; q < VEC; q++) atomicAdd(&red[warp][d(e[q])], 1u);
                    }
                }
            }
            for (uint64_t e = e0 + nv * VEC + tid; e < e1; e += THREADS)
                atomicAdd(&red[warp][d(in[e])], 1u);
        } else {
            for (uint64_t e = e0 + tid; e < e1; e += THREADS) atomicAdd(&red[warp][d(in[e])], 1u);
        }
    }
    __syncthreads();
    if (tid < M) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < W; w++) s += red[w][tid];
        a.chunk_cnt[tid * G + k] = s;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) am_last = (atomicAdd(a.done, 1u) == G - 1u);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    plain_finish_scan<M, THREADS>(a, tot_sh);
}

// Shared-memory bytes of plain_scatter_kernel's dynamic part.
template <class V, int TILE, int STAGES>
constexpr size_t plain_scatter_smem() {
    return static_cast<size_t>(STAGES + 1) * TILE * sizeof(V) + TILE;  // ring + stage + class bytes
}

template <class V, class D, int M, int THREADS, int ITEMS, int STAGES>
__global__ void __launch_bounds__(THREADS) plain_scatter_kernel(PlainArgs a, D d) {
    constexpr int TILE = THREADS * ITEMS;
    constexpr int W = THREADS / 32;
    constexpr int WSPAN = 32 * ITEMS;  // elements per warp per tile
    static_assert(WSPAN <= 65536, "warp-local ranks are packed in 16 bits");
    static_assert(M <= 64 && M >= 2, "class bound");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    V* ring = reinterpret_cast<V*>(smem_raw);       // STAGES tiles, filled by TMA
    V* stage = ring + STAGES * TILE;                // one tile, class-sorted
    uint8_t* stage_cls = reinterpret_cast<uint8_t*>(stage + TILE);

    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ uint32_t whist[W][M];  // per-warp running class counts
    __shared__ uint32_t wbase[W][M];  // tile-local start of warp w's class-c run
    __shared__ uint32_t cursor[M];    // global end cursor of this chunk's class-c run
    __shared__ uint32_t delta[M];     // dst = slot + delta[c] (mod 2^32)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t G = a.num_chunks, k = blockIdx.x;
    uint32_t t0, t1;
    chunk_tiles(k, a.num_tiles, G, t0, t1);
    const uint32_t cnt = t1 - t0;
    if (cnt == 0) return;
    const V* in = static_cast<const V*>(a.in);
    V* out = static_cast<V*>(a.out);
    const bool tma_ok = (reinterpret_cast<uintptr_t>(in) & 15u) == 0;

    if (tid < M) cursor[tid] = a.class_base[tid] + a.chunk_pre[tid * G + k] + a.chunk_cnt[tid * G + k];
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();

    // Issue the load of the i-th tile in processing order (tile t1-1-i) into
    // ring slot i % STAGES.  Full tiles go by TMA; the partial last tile of
    // the array (or any tile when `in` is not 16-byte aligned) is read by the
    // threads straight from global memory, and the barrier is only arrived on
    // so that its phase still advances once per use.
    auto issue = [&](uint32_t i) {
        const uint32_t tile = t1 - 1u - i;
        const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
        uint64_t* bar = &bars[i % STAGES];
        if (tma_ok && ts + TILE <= a.n) {
            mbar_arrive_expect_tx(bar, TILE * sizeof(V));
            bulk_load_g2s(ring + (i % STAGES) * TILE, in + ts, TILE * sizeof(V), bar);
        } else {
            mbar_arrive(bar);
        }
    };
    if (tid == 0)
        for (uint32_t i = 0; i < STAGES && i < cnt; i++) issue(i);

    for (uint32_t i = 0; i < cnt; i++) {
        const uint32_t tile = t1 - 1u - i;
        const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
        const uint32_t valid = static_cast<uint32_t>(min(static_cast<uint64_t>(TILE), a.n - ts));
        const bool from_ring = tma_ok && valid == TILE;
        const V* src = ring + (i % STAGES) * TILE;
        const bool ok = mbar_wait_bounded(&bars[i % STAGES], (i / STAGES) & 1u);

        // ---- warp ranks: element (warp, j, lane) is tile slot warp*WSPAN + j*32 + lane
        for (int c = lane; c < M; c += 32) whist[warp][c] = 0;
        __syncwarp();
        V vals[ITEMS];
        uint32_t info[ITEMS];  // class << 16 | warp-local rank
        const uint32_t lt = lanemask_lt();
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const uint32_t idx = warp * WSPAN + j * 32 + lane;
            const bool live = idx < valid;
            V v = V();
            if (live) v = from_ring ? src[idx] : in[ts + idx];
            const uint32_t c = live ? d(v) : static_cast<uint32_t>(M);
            const uint32_t peers = __match_any_sync(0xffffffffu, c);
            const uint32_t before = live ? whist[warp][c] : 0u;
            const uint32_t rank = before + __popc(peers & lt);
            __syncwarp();
            if (live && (peers >> lane) == 1u) whist[warp][c] = rank + 1u;  // last lane of its class
            __syncwarp();
            vals[j] = v;
            info[j] = (c << 16) | rank;
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(a.error, kErrTimeout);
            // drain: wait (bounded) for the copies this CTA still has in flight
            for (uint32_t q = i + 1; q < cnt && q < i + STAGES; q++)
                if (tid == 0) (void)mbar_wait_bounded(&bars[q % STAGES], (q / STAGES) & 1u);
            return;
        }

        // ---- block scan: per class, over warps (wprefix) and over classes (tile start)
        if (warp == 0) {
            uint32_t carry = 0;
#pragma unroll
            for (int c0 = 0; c0 < M; c0 += 32) {
                const int c = c0 + lane;
                uint32_t tcnt = 0;
                if (c < M) {
#pragma unroll
                    for (int w = 0; w < W; w++) {
                        const uint32_t x = whist[w][c];
                        wbase[w][c] = tcnt;
                        tcnt += x;
                    }
                }
                const uint32_t incl = warp_incl_scan(tcnt);
                const uint32_t tstart = carry + incl - tcnt;
                carry += __shfl_sync(0xffffffffu, incl, 31);
                if (c < M) {
                    const uint32_t cur = cursor[c] - tcnt;
                    cursor[c] = cur;
                    delta[c] = cur - tstart;
#pragma unroll
                    for (int w = 0; w < W; w++) wbase[w][c] += tstart;
                }
            }
        }
        __syncthreads();

        // ---- scatter into the class-sorted stage
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const uint32_t c = info[j] >> 16;
            if (c < static_cast<uint32_t>(M)) {
                const uint32_t slot = wbase[warp][c] + (info[j] & 0xffffu);
                stage[slot] = vals[j];
                stage_cls[slot] = static_cast<uint8_t>(c);
            }
        }
        __syncthreads();
        if (tid == 0 && i + STAGES < cnt) issue(i + STAGES);

        // ---- coalesced write-out of the class runs
        for (uint32_t slot = tid; slot < valid; slot += THREADS) {
            const uint32_t c = stage_cls[slot];
            const uint32_t dst = slot + delta[c];
            out[dst] = stage[slot];
        }
    }
}

// Per-thread class counters in 4-bit lanes: one u32 holds 8 classes, two
// hold 16.  A lane never reaches 16: with 16 elements per thread only the
// first 15 are counted in the lanes and the 16th is added when the counts are
// published.
template <int M>
struct NibbleCounts {
    static_assert(M <= 16, "nibble counters cover at most 16 classes");
    static constexpr int NW = (M + 7) / 8;
    uint32_t w[NW];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int q = 0; q < NW; q++) w[q] = 0;
    }
    __device__ __forceinline__ uint32_t get(uint32_t c) const {
        if constexpr (NW == 1) {
            return (w[0] >> (c << 2)) & 15u;
        } else {
            return (((c < 8u) ? w[0] : w[1]) >> ((c & 7u) << 2)) & 15u;
        }
    }
    __device__ __forceinline__ void inc(uint32_t c) {
        if constexpr (NW == 1) {
            w[0] += 1u << (c << 2);
        } else {
            const uint32_t one = 1u << ((c & 7u) << 2);
            if (c < 8u) w[0] += one; else w[1] += one;
        }
    }
};

template <class V>
__device__ __forceinline__ void unpack16_to(const uint4& r, V* e);
template <>
__device__ __forceinline__ void unpack16_to<uint32_t>(const uint4& r, uint32_t* e) {
    e[0] = r.x; e[1] = r.y; e[2] = r.z; e[3] = r.w;
}
template <>
__device__ __forceinline__ void unpack16_to<uint64_t>(const uint4& r, uint64_t* e) {
    e[0] = static_cast<uint64_t>(r.x) | (static_cast<uint64_t>(r.y) << 32);
    e[1] = static_cast<uint64_t>(r.z) | (static_cast<uint64_t>(r.w) << 32);
}

template <class V, int THREADS, int STAGES, int M>
struct ScatterTmaSmem {
    static constexpr int kItems = 64 / static_cast<int>(sizeof(V));  // 64 bytes per thread
    static constexpr int kTile = THREADS * kItems;
    static constexpr int kRows = kTile * static_cast<int>(sizeof(V)) / 128;  // 128-byte rows
    static constexpr uint32_t kAU = 16 / sizeof(V);                 // elements per 16 bytes
    // every class run gets kAU slots of slack for its 16-byte phase
    static constexpr int kStageElems = kTile + static_cast<int>(kAU) * M;
    static constexpr size_t kRingBytes = static_cast<size_t>(STAGES) * kTile * sizeof(V);
    static constexpr size_t kStageBytes = static_cast<size_t>(kStageElems) * sizeof(V);
    static constexpr size_t kCntBytes = static_cast<size_t>(M) * THREADS * 2;  // u16 counts
    // +1024: the ring is re-aligned to 1024 bytes (128-byte swizzle atoms)
    static constexpr size_t kBytes = 1024 + kRingBytes + kStageBytes + kCntBytes;
};

// Scatter kernel for m <= 16.  Same contract as plain_scatter_kernel; faster
// per element:
//  * tiles arrive by tensor TMA (one 2-D box of 128-byte rows per tile) with
//    the 128-byte swizzle, so the four 16-byte shared loads with which a thread
//    takes its 64 contiguous bytes are free of bank conflicts;
//  * a thread ranks its own consecutive elements with 4-bit counters in a
//    register (local rank = count of its earlier same-class elements); a block
//    scan over the [class][thread] count matrix in shared memory then gives
//    every thread its exclusive class prefix (stable: thread order = input
//    order), with the tile's class-run start folded in;
//  * every class run is placed in the stage at the same 16-byte phase as its
//    destination, so its aligned interior leaves by one bulk store
//    (cp.async.bulk shared->global) and only the < 16-byte head and tail of a
//    run are written by threads.  The stage is rewritten only after the bulk
//    stores of the previous tile have read it (they have the whole next pass 1
//    and row scan to do so).
template <class V, class D, int M, int THREADS, int STAGES>
__global__ void __launch_bounds__(THREADS, 4)  // 4 CTAs (32 warps) per SM: <= 64 registers
    plain_scatter_tma_kernel(PlainArgs a, D d, const __grid_constant__ CUtensorMap tmap) {
    using L = ScatterTmaSmem<V, THREADS, STAGES, M>;
    constexpr int ITEMS = L::kItems;
    constexpr int TILE = L::kTile;
    constexpr int ROWS = L::kRows;
    constexpr uint32_t AU = L::kAU;
    constexpr int W = THREADS / 32;
    constexpr int PER = THREADS / 32;  // count-matrix entries per lane in a row scan
    constexpr int LR = (ITEMS + 7) / 8;
    static_assert(M <= 16 && M >= 2, "class bound");
    static_assert(M <= W * 2, "each warp scans at most two rows");
    static_assert(ITEMS == 16 || ITEMS == 8, "64 bytes of 4- or 8-byte elements");
    static_assert(PER == 8, "row scan loads 8 entries per lane");
    static_assert(ROWS <= 256, "TMA box height");
    static_assert(L::kStageElems < 65536, "stage slots are kept in 16 bits");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    V* ring = reinterpret_cast<V*>(base);
    V* stage = reinterpret_cast<V*>(base + L::kRingBytes);
    uint16_t* cnt_sm = reinterpret_cast<uint16_t*>(base + L::kRingBytes + L::kStageBytes);

    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ uint32_t cursor[2][M];  // ping-pong by tile parity
    __shared__ uint32_t run_start[M], run_cnt[M], run_dst[M], rowtot[M];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t G = a.num_chunks, k = blockIdx.x;
    uint32_t t0, t1;
    chunk_tiles(k, a.num_tiles, G, t0, t1);
    const uint32_t cnt = t1 - t0;
    if (cnt == 0) return;
    const V* in = static_cast<const V*>(a.in);
    V* out = static_cast<V*>(a.out);
    const uint32_t out_phase =
        static_cast<uint32_t>(reinterpret_cast<uintptr_t>(out) / sizeof(V)) & (AU - 1u);
    const bool tma_ok = a.use_tma != 0;

    if (tid < M)
        cursor[0][tid] = a.class_base[tid] + a.chunk_pre[tid * G + k] + a.chunk_cnt[tid * G + k];
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();

    // i-th tile in processing order is tile t1-1-i (the chunk is walked backwards).
    auto issue = [&](uint32_t i) {
        const uint32_t tile = t1 - 1u - i;
        uint64_t* bar = &bars[i % STAGES];
        if (tma_ok && static_cast<uint64_t>(tile + 1) * TILE <= a.n) {
            mbar_arrive_expect_tx(bar, TILE * sizeof(V));
            tma_load_2d(ring + (i % STAGES) * TILE, &tmap, 0, static_cast<int32_t>(tile * ROWS), bar);
        } else {
            mbar_arrive(bar);
        }
    };
    if (tid == 0)
        for (uint32_t i = 0; i < STAGES && i < cnt; i++) issue(i);

    const uint32_t e0 = tid * ITEMS;  // this thread's first tile-local element
    uint16_t* my_cnt = cnt_sm + tid;  // column of this thread: my_cnt[c * THREADS]
    for (uint32_t i = 0; i < cnt; i++) {
        const uint32_t tile = t1 - 1u - i;
        const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
        const uint32_t valid = static_cast<uint32_t>(min(static_cast<uint64_t>(TILE), a.n - ts));
        const bool full = valid == TILE;
        const bool ok = mbar_wait_bounded(&bars[i % STAGES], (i / STAGES) & 1u);

        // ---- pass 1: take 64 contiguous bytes, classify, local ranks
        V v[ITEMS];
        if (tma_ok && full) {
            const unsigned char* tb =
                reinterpret_cast<const unsigned char*>(ring + (i % STAGES) * TILE);
            const uint32_t row = static_cast<uint32_t>(tid) >> 1;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t chunk = ((static_cast<uint32_t>(tid) & 1u) * 4u + q) ^ (row & 7u);
                const uint4 r = *reinterpret_cast<const uint4*>(tb + row * 128u + chunk * 16u);
                unpack16_to<V>(r, &v[q * AU]);
            }
        } else if (full) {
#pragma unroll
            for (int j = 0; j < ITEMS; j++) v[j] = in[ts + e0 + j];
        } else {
#pragma unroll
            for (int j = 0; j < ITEMS; j++) v[j] = (e0 + j < valid) ? in[ts + e0 + j] : V();
        }
        NibbleCounts<M> nc;
        nc.init();
        uint32_t lr[LR];
#pragma unroll
        for (int q = 0; q < LR; q++) lr[q] = 0;
        uint32_t last_c = M;  // class of element 15 (not in the nibbles)
        if (full) {
#pragma unroll
            for (int j = 0; j < ITEMS; j++) {
                const uint32_t c = d(v[j]);
                lr[j >> 3] += nc.get(c) << (4 * (j & 7));
                if (j < 15) nc.inc(c); else last_c = c;
            }
        } else {
#pragma unroll
            for (int j = 0; j < ITEMS; j++) {
                if (e0 + j < valid) {
                    const uint32_t c = d(v[j]);
                    lr[j >> 3] += nc.get(c) << (4 * (j & 7));
                    if (j < 15) nc.inc(c); else last_c = c;
                }
            }
        }
#pragma unroll
        for (int c = 0; c < M; c++) my_cnt[c * THREADS] = static_cast<uint16_t>(nc.get(c));
        if (last_c < static_cast<uint32_t>(M)) my_cnt[last_c * THREADS] += 1;
        if (__syncthreads_or(!ok)) {  // (A)
            if (tid == 0) {
                atomicOr(a.error, kErrTimeout);
                for (uint32_t q = i; q < cnt && q < i + STAGES; q++)
                    (void)mbar_wait_bounded(&bars[q % STAGES], (q / STAGES) & 1u);
            }
            if (tid < M) bulk_wait_all();
            return;
        }
        // The ring slot is consumed (values are in registers): refill it now.
        if (tid == 0 && i + STAGES < cnt) issue(i + STAGES);

        // ---- row scans of the [class][thread] count matrix: warp w owns
        // rows w and w + W; the prefixes stay in registers until the class
        // runs are known
        uint32_t pre[2][PER];
        uint32_t rtot[2] = {0u, 0u};
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int c = warp + h * W;
            if (c < M) {
                const uint4 xw = *reinterpret_cast<const uint4*>(cnt_sm + c * THREADS + lane * PER);
                const uint32_t x[8] = {xw.x & 0xffffu, xw.x >> 16, xw.y & 0xffffu, xw.y >> 16,
                                       xw.z & 0xffffu, xw.z >> 16, xw.w & 0xffffu, xw.w >> 16};
                uint32_t tot = 0;
#pragma unroll
                for (int q = 0; q < 8; q++) tot += x[q];
                const uint32_t incl = warp_incl_scan(tot);
                uint32_t run = incl - tot;
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    pre[h][q] = run;
                    run += x[q];
                }
                rtot[h] = __shfl_sync(0xffffffffu, incl, 31);
                if (lane == 31) rowtot[c] = incl;
            }
        }
        __syncthreads();  // (B)

        // ---- class runs (every warp, lanes = classes): destination of run c
        // (chunk walked backwards) and its stage slot, at the destination's
        // 16-byte phase within kAU slots of slack per run
        {
            const uint32_t par = i & 1u;
            const uint32_t c = static_cast<uint32_t>(lane);
            const uint32_t cc = c < static_cast<uint32_t>(M) ? rowtot[c] : 0u;
            const uint32_t dst = c < static_cast<uint32_t>(M) ? cursor[par][c] - cc : 0u;
            const uint32_t room = cc + (c < static_cast<uint32_t>(M) ? AU : 0u);
            const uint32_t q0 = warp_incl_scan(room) - room;
            const uint32_t st = q0 + (((out_phase + dst) - q0) & (AU - 1u));
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int row = warp + h * W;
                if (row < M) {
                    // slots < kStageElems < 2^16: pairs of u16 prefixes per word
                    const uint32_t add = __shfl_sync(0xffffffffu, st, row);
                    const uint32_t add2 = add | (add << 16);
                    *reinterpret_cast<uint4*>(cnt_sm + row * THREADS + lane * PER) =
                        make_uint4((pre[h][0] | (pre[h][1] << 16)) + add2,
                                   (pre[h][2] | (pre[h][3] << 16)) + add2,
                                   (pre[h][4] | (pre[h][5] << 16)) + add2,
                                   (pre[h][6] | (pre[h][7] << 16)) + add2);
                }
            }
            if (warp == 0 && c < static_cast<uint32_t>(M)) {
                cursor[par ^ 1u][c] = dst;
                run_start[c] = st;
                run_cnt[c] = cc;
                run_dst[c] = dst;
            }
            (void)rtot;
        }
        // the stage is about to be rewritten: the bulk stores of the previous
        // tile must have finished reading it
        if (tid < M) bulk_wait_read<0>();
        __syncthreads();  // (C)

        // ---- pass 2: scatter into the class-sorted stage
        V* stg = stage;
        if (full) {
#pragma unroll
            for (int j = 0; j < ITEMS; j++) {
                const uint32_t c = d(v[j]);
                const uint32_t slot = my_cnt[c * THREADS] + ((lr[j >> 3] >> (4 * (j & 7))) & 15u);
                stg[slot] = v[j];
            }
        } else {
#pragma unroll
            for (int j = 0; j < ITEMS; j++) {
                if (e0 + j < valid) {
                    const uint32_t c = d(v[j]);
                    const uint32_t slot =
                        my_cnt[c * THREADS] + ((lr[j >> 3] >> (4 * (j & 7))) & 15u);
                    stg[slot] = v[j];
                }
            }
        }
        fence_proxy_async_smem();
        __syncthreads();  // (D)

        // ---- write-out: bulk store of each run's aligned interior, threads
        // store the unaligned head and tail elements
        if (tid < M) {
            const uint32_t s = run_start[tid], cc = run_cnt[tid];
            uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
            if (head > cc) head = cc;
            const uint32_t body = ((cc - head) / AU) * AU;
            if (body > 0)
                bulk_store_s2g(out + run_dst[tid] + head, stg + s + head, body * sizeof(V));
            bulk_commit();
        } else if (tid >= 32 && tid < 32 + M * 2 * static_cast<int>(AU)) {
            const uint32_t c = (tid - 32) / (2 * AU), q = (tid - 32) % (2 * AU);
            const uint32_t s = run_start[c], cc = run_cnt[c];
            uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
            if (head > cc) head = cc;
            const uint32_t body = ((cc - head) / AU) * AU;
            uint32_t off = 0xffffffffu;
            if (q < AU) {
                if (q < head) off = q;
            } else if (head + body + (q - AU) < cc) {
                off = head + body + (q - AU);
            }
            if (off != 0xffffffffu) out[run_dst[c] + off] = stg[s + off];
        }
    }
    if (tid < M) bulk_wait_all();
}

}  // namespace mdx
