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
//   plain_scatter_tma_kernel
//                        re-reads each element (4 B) and writes it once (4 B):
//                        per tile, element ranks (m <= 16: thread-local
//                        nibble counters and a block scan, mdx_tile.cuh
//                        tile_scatter; more classes: warp ranks from ballots
//                        of the class bits + __popc, tile_scatter_wide), a
//                        shared-memory staged scatter so every class run
//                        leaves the SM as bulk stores.  Tiles are staged into
//                        shared memory by TMA (cp.async.bulk.tensor, no
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

#include <type_traits>

#include "mdx_device.cuh"
#include "mdx_tile.cuh"

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
    const uint32_t* skip; // scatter: return at once if *skip != 0 (null: never)
    uint32_t chunk_stride;   // row stride of chunk_cnt / chunk_pre (>= num_chunks; a multiple
                             // of 4 when prefix_in_scatter)
    int prefix_in_scatter;   // 1: the count kernel only counts; every scatter CTA forms its
                             // own chunk prefix and the class bases (CTA 0 writes sizes and
                             // head flags).  0: the last counting CTA scans them for all.
};

// Programmatic dependent launch: the count kernel lets the scatter grid be
// scheduled at once; the scatter waits for the count grid's results (its
// memory operations complete and visible) only where it needs them.  Both are
// no-ops in a launch without the programmatic attribute.
__device__ __forceinline__ void pdl_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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
template <>
__device__ __forceinline__ void unpack16<Rec16>(const uint4& r, Rec16 (&e)[1]) {
    unpack16_to<Rec16>(r, e);
}

// 1 << s with the shift clamped as PTX defines it (s >= 32 gives 0), so one
// increment is added to the right 32-bit word without a select.
__device__ __forceinline__ uint32_t shl1_clamped(uint32_t s) {
    uint32_t r;
    asm("shl.b32 %0, 1, %1;" : "=r"(r) : "r"(s));
    return r;
}

// Per-thread class counters for M <= 16: 4-bit lanes in one or two u32 words
// (an increment is one shift and one add per word), folded into 8-bit lanes
// (even / odd classes of each nibble word) at least every 8 increments and
// into u32 totals at least every 31 folds, before any lane can overflow.
template <int M>
struct PackedCounts {
    static_assert(M <= 16, "packed counters cover at most 16 classes");
    static constexpr int NW = (M + 7) / 8;
    uint32_t nib[NW];
    uint32_t byt[2 * NW];
    uint32_t acc[M];
    uint32_t folds;
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int w = 0; w < NW; w++) nib[w] = 0;
#pragma unroll
        for (int w = 0; w < 2 * NW; w++) byt[w] = 0;
#pragma unroll
        for (int c = 0; c < M; c++) acc[c] = 0;
        folds = 0;
    }
    // At most 8 calls between fold() calls.
    __device__ __forceinline__ void add(uint32_t c) {
        if constexpr (NW == 1) {
            nib[0] += 1u << (c << 2);
        } else {
            const uint32_t s = c << 2;
            nib[0] += shl1_clamped(s);
            nib[1] += shl1_clamped(s - 32u);
        }
    }
    __device__ __forceinline__ void flush() {  // bytes -> u32 totals
#pragma unroll
        for (int w = 0; w < NW; w++) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (8 * w + 2 * j < M) acc[8 * w + 2 * j] += (byt[2 * w] >> (8 * j)) & 0xffu;
                if (8 * w + 2 * j + 1 < M) acc[8 * w + 2 * j + 1] += (byt[2 * w + 1] >> (8 * j)) & 0xffu;
            }
            byt[2 * w] = 0;
            byt[2 * w + 1] = 0;
        }
        folds = 0;
    }
    __device__ __forceinline__ void fold() {  // nibbles -> bytes
#pragma unroll
        for (int w = 0; w < NW; w++) {
            byt[2 * w] += nib[w] & 0x0f0f0f0fu;
            byt[2 * w + 1] += (nib[w] >> 4) & 0x0f0f0f0fu;
            nib[w] = 0;
        }
        if (++folds == 31u) flush();
    }
    __device__ __forceinline__ void finish() {
        fold();
        flush();
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
    // a warp per class; each lane takes PER consecutive chunk counts with all
    // its loads in flight at once (this runs while the rest of the GPU waits)
    constexpr uint32_t PER = 8;
    for (int c = warp; c < M; c += W) {
        uint32_t run = 0;
        for (uint32_t k0 = 0; k0 < G; k0 += 32 * PER) {
            const uint32_t kb = k0 + lane * PER;
            uint32_t x[PER];
#pragma unroll
            for (uint32_t q = 0; q < PER; q++)
                x[q] = kb + q < G ? __ldcg(&a.chunk_cnt[c * a.chunk_stride + kb + q]) : 0u;
            uint32_t s = 0;
#pragma unroll
            for (uint32_t q = 0; q < PER; q++) s += x[q];
            const uint32_t incl = warp_incl_scan(s);
            uint32_t pre = run + incl - s;
#pragma unroll
            for (uint32_t q = 0; q < PER; q++) {
                if (kb + q < G) a.chunk_pre[c * a.chunk_stride + kb + q] = pre;
                pre += x[q];
            }
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
__global__ void __launch_bounds__(THREADS, 4) plain_count_kernel(PlainArgs a, D d) {
    constexpr int W = THREADS / 32;
    constexpr int VEC = 16 / static_cast<int>(sizeof(V));
    constexpr int UNROLL = M <= 8 ? 8 : 4;  // 16-byte loads in flight per thread (registers allowing)
    __shared__ uint32_t red[W][M];
    __shared__ uint32_t tot_sh[M];
    __shared__ int am_last;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t G = a.num_chunks, k = blockIdx.x;
    pdl_launch_dependents();  // the scatter grid may be scheduled as CTAs here finish
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
                    if (VEC == 4 ? (u & 1) : ((u & 3) == 3)) pc.fold();  // <= 8 increments
                }
            }
            uint32_t k = 0;
            for (uint64_t e = e0 + nv * VEC + tid; e < e1; e += THREADS) {
                pc.add(d(in[e]));
                if (++k == 8u) {
                    pc.fold();
                    k = 0;
                }
            }
        } else {
            uint32_t k = 0;
            for (uint64_t e = e0 + tid; e < e1; e += THREADS) {
                pc.add(d(in[e]));
                if (++k == 8u) {
                    pc.fold();
                    k = 0;
                }
            }
        }
        pc.finish();
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
        a.chunk_cnt[tid * a.chunk_stride + k] = s;
    }
    if (a.prefix_in_scatter) return;  // the scatter CTAs form the prefixes
    __threadfence();
    __syncthreads();
    if (tid == 0) am_last = (atomicAdd(a.done, 1u) == G - 1u);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    plain_finish_scan<M, THREADS>(a, tot_sh);
}

template <class V, int THREADS, int STAGES, int M, int BPT = 64>
struct ScatterTmaSmem {
    using G = TileGeom<V, THREADS, M, BPT>;
    static constexpr int kItems = G::kItems;
    static constexpr int kTile = G::kTile;
    static constexpr int kRows = G::kRows;
    static constexpr size_t kRingBytes = static_cast<size_t>(STAGES) * kTile * sizeof(V);
    // +1024: the ring is re-aligned to 1024 bytes (128-byte swizzle atoms)
    static constexpr size_t kBytes = 1024 + kRingBytes + G::kStageBytes + G::kCntBytes;
};

// Scatter kernel: CTA k re-reads chunk k (tiles in reverse order) and writes
// every element at class_base[c] + chunk_pre[c][k] + its rank in the chunk.
// Tiles arrive by tensor TMA (one 2-D box of 128-byte rows per tile, 128-byte
// swizzle for m <= 16 and none above, STAGES-deep mbarrier ring) and go
// through tile_filter (m = 2), tile_scatter (m <= 16:
// thread-local nibble ranks, a block scan over the [class][thread] count
// matrix) or tile_scatter_wide (17..64 classes: warp ranks from ballots),
// then a shared-memory stage at the destination's 16-byte phase and bulk
// stores of every class run (mdx_tile.cuh).  OUT: one output array, or the
// output chunks of several ranks (distributed partition).  BPT: bytes of a
// tile per thread (64, or 32 for tiles half as long).
template <class V, class D, int M, int THREADS, int STAGES, class OUT = OutFlat<V>, int BPT = 64>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)  // 32 warps per SM: <= 64 registers
    plain_scatter_tma_kernel(PlainArgs a, D d, const __grid_constant__ CUtensorMap tmap,
                             const __grid_constant__ OUT out) {
    using L = ScatterTmaSmem<V, THREADS, STAGES, M, BPT>;
    constexpr int ITEMS = L::kItems;
    constexpr int TILE = L::kTile;
    constexpr int ROWS = L::kRows;
    static_assert(ROWS <= 256, "TMA box height");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    V* ring = reinterpret_cast<V*>(base);
    V* stage = reinterpret_cast<V*>(base + L::kRingBytes);
    uint16_t* cnt_sm = reinterpret_cast<uint16_t*>(base + L::kRingBytes + L::G::kStageBytes);

    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ TileShared<M> sh;
    __shared__ uint32_t tot_sh[M], pre_sh[M];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t G = a.num_chunks, k = blockIdx.x;
    uint32_t t0, t1;
    chunk_tiles(k, a.num_tiles, G, t0, t1);
    const uint32_t cnt = t1 - t0;
    if (cnt == 0) return;
    const V* in = static_cast<const V*>(a.in);
    const bool tma_ok = a.use_tma != 0;
    // sharded output: the class bases came from other ranks' counts; a
    // mismatch found by plain_dist_bases_kernel leaves everything unwritten
    if (a.skip != nullptr && *a.skip != 0u) return;

    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    if (tid < M) {
        tot_sh[tid] = 0u;
        pre_sh[tid] = 0u;
    }
    __syncthreads();

    // i-th tile in processing order is tile t1-1-i (the chunk is walked
    // backwards, so the tiles the counting kernel read last are still in L2).
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
    // the first tiles only read the input: their copies start before the
    // count grid's results are needed
    if (tid == 0)
        for (uint32_t i = 0; i < STAGES && i < cnt; i++) issue(i);
    pdl_wait();
    const uint32_t stride = a.chunk_stride;
    if (a.prefix_in_scatter) {
        // this chunk's exclusive class prefix and the class totals from the
        // [class][chunk] counts (TPC threads per class, 16-byte loads)
        constexpr int TPC = THREADS / M;
        constexpr int RW = TPC < 32 ? TPC : 32;
        const uint32_t c = static_cast<uint32_t>(tid / TPC), l = static_cast<uint32_t>(tid % TPC);
        const uint4* row = reinterpret_cast<const uint4*>(a.chunk_cnt + static_cast<uint64_t>(c) * stride);
        uint32_t tot = 0, pre = 0;
        for (uint32_t q4 = l; q4 < stride / 4u; q4 += TPC) {
            const uint4 x = __ldcg(row + q4);
            const uint32_t j = 4u * q4;
            const uint32_t xv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (uint32_t u = 0; u < 4; u++) {
                const uint32_t v = (j + u < G) ? xv[u] : 0u;
                tot += v;
                pre += (j + u < k) ? v : 0u;
            }
        }
#pragma unroll
        for (int off = RW / 2; off > 0; off >>= 1) {
            tot += __shfl_xor_sync(0xffffffffu, tot, off);
            pre += __shfl_xor_sync(0xffffffffu, pre, off);
        }
        if ((lane % RW) == 0) {
            atomicAdd(&tot_sh[c], tot);
            atomicAdd(&pre_sh[c], pre);
        }
        __syncthreads();
        if (warp == 0) {  // class bases: exclusive scan of the totals
            uint32_t carry = 0;
#pragma unroll
            for (int h = 0; h < (M + 31) / 32; h++) {
                const uint32_t cc = static_cast<uint32_t>(lane + 32 * h);
                const uint32_t x = cc < static_cast<uint32_t>(M) ? tot_sh[cc] : 0u;
                const uint32_t incl = warp_incl_scan(x);
                const uint32_t bc = carry + incl - x;
                if (cc < static_cast<uint32_t>(M)) {
                    sh.cursor[0][cc] = bc + pre_sh[cc] + __ldcg(a.chunk_cnt + static_cast<uint64_t>(cc) * stride + k);
                    if (k == 0) {
                        a.class_base[cc] = bc;
                        a.class_tot[cc] = x;
                        if (a.sizes != nullptr && cc < a.m) a.sizes[cc] = x;
                        // head-flag form (SeqMdiscr.h:47-49); zeroed before the count kernel
                        if (a.headflags != nullptr && x > 0) a.headflags[bc] = x;
                    }
                }
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
    } else if (tid < M) {
        const uint64_t o = static_cast<uint64_t>(tid) * stride + k;
        sh.cursor[0][tid] = a.class_base[tid] + a.chunk_pre[o] + a.chunk_cnt[o];
    }
    __syncthreads();

    const uint32_t e0 = tid * ITEMS;
    for (uint32_t i = 0; i < cnt; i++) {
        const uint32_t tile = t1 - 1u - i;
        const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
        const uint32_t valid = static_cast<uint32_t>(min(static_cast<uint64_t>(TILE), a.n - ts));
        const bool full = valid == TILE;
        const bool ok = mbar_wait_bounded(&bars[i % STAGES], (i / STAGES) & 1u);
        V v[ITEMS];
        // the ring slot is consumed (values are in registers): refill it
        auto refill = [&] {
            if (tid == 0 && i + STAGES < cnt) issue(i + STAGES);
        };
        bool done;
        if constexpr (M <= 16) {  // thread-contiguous elements
            if (tma_ok && full) {
                take_swizzled<V, ITEMS>(ring + (i % STAGES) * TILE, v);
            } else if (full) {
#pragma unroll
                for (int j = 0; j < ITEMS; j++) v[j] = in[ts + e0 + j];
            } else {
#pragma unroll
                for (int j = 0; j < ITEMS; j++) v[j] = (e0 + j < valid) ? in[ts + e0 + j] : V();
            }
            if constexpr (M == 2)
                done = tile_filter<V, D, THREADS, false>(d, v, 0u, valid, full, stage,
                                                         reinterpret_cast<uint32_t*>(cnt_sm), sh,
                                                         i & 1u, out, ok, refill);
            else
                done = tile_scatter<V, D, M, THREADS, false>(d, v, 0u, valid, full, stage, cnt_sm,
                                                             sh, i & 1u, out, ok, refill);
        } else {  // striped elements (warp ranks)
            const uint32_t w0 = static_cast<uint32_t>(tid >> 5) * 32u * ITEMS + (tid & 31);
            if (tma_ok && full) {
                take_striped<V, ITEMS>(ring + (i % STAGES) * TILE, v);
            } else {
#pragma unroll
                for (int j = 0; j < ITEMS; j++)
                    v[j] = (w0 + j * 32u < valid) ? in[ts + w0 + j * 32u] : V();
            }
            done = tile_scatter_wide<V, D, M, THREADS, false>(
                d, v, 0u, valid, full, stage, reinterpret_cast<uint32_t*>(cnt_sm), sh, i & 1u, out,
                ok, refill);
        }
        if (!done) {
            if (tid == 0) {
                atomicOr(a.error, kErrTimeout);
                for (uint32_t q = i; q < cnt && q < i + STAGES; q++)
                    (void)mbar_wait_bounded(&bars[q % STAGES], (q / STAGES) & 1u);
            }
            break;
        }
    }
    if (tid < M) bulk_wait_all();
    if constexpr (!std::is_same<OUT, OutFlat<V>>::value) {
        // writes into other GPUs' memory: make them visible system-wide
        // before the kernel ends
        __threadfence_system();
    }
}

// m = 1: every element is in class 0, the partition is a copy (made by the
// host with cudaMemcpyAsync); this kernel fills in the class total and base,
// the sizes and the head flag (count_0 at offset 0; the array was zeroed).
static __global__ void plain_single_class_kernel(uint64_t n, uint32_t* class_base, uint32_t* class_tot,
                                          uint32_t* sizes, uint32_t* headflags) {
    if (threadIdx.x == 0) {
        class_base[0] = 0u;
        class_tot[0] = static_cast<uint32_t>(n);
        if (sizes != nullptr) sizes[0] = static_cast<uint32_t>(n);
        if (headflags != nullptr) headflags[0] = static_cast<uint32_t>(n);
    }
}

// Sharded output (distributed partition): this rank's class bases in the
// whole output from the class counts of all ranks, all_counts[r * m + c]:
// base_c = (elements of classes < c on every rank) + (elements of class c on
// ranks < rank).  The counts of this rank must equal its own count (class_tot,
// from plain_count_kernel; null: a rank without elements, all zero) and all
// counts must add up to n_total; otherwise *skip = 1, the error is latched and
// the scatter writes nothing.  class_base may be null (no elements to place).
template <int M>
__global__ void plain_dist_bases_kernel(const uint32_t* all_counts, uint32_t R, uint32_t rank,
                                        uint32_t m, uint64_t n_total, uint32_t* class_base,
                                        const uint32_t* class_tot, uint32_t* sizes, uint32_t* skip,
                                        uint32_t* error) {
    __shared__ uint64_t tot[M];
    __shared__ uint32_t bad;
    const uint32_t c = threadIdx.x;
    if (c == 0) bad = 0u;
    __syncthreads();
    uint64_t below = 0;
    if (c < static_cast<uint32_t>(M)) {
        uint64_t t = 0;
        for (uint32_t r = 0; r < R; r++) {
            const uint32_t x = c < m ? all_counts[static_cast<uint64_t>(r) * m + c] : 0u;
            t += x;
            if (r < rank) below += x;
            const uint32_t own = (c < m && class_tot != nullptr) ? class_tot[c] : 0u;
            if (r == rank && x != own) atomicOr(&bad, 1u);
        }
        tot[c] = t;
    }
    __syncthreads();
    if (c == 0) {
        uint64_t sum = 0;
        for (int q = 0; q < M; q++) sum += tot[q];
        if (sum != n_total) bad = 1u;
    }
    __syncthreads();
    if (c < static_cast<uint32_t>(M)) {
        uint64_t base = below;
        for (uint32_t q = 0; q < c; q++) base += tot[q];
        if (class_base != nullptr) class_base[c] = static_cast<uint32_t>(base);
        if (sizes != nullptr && c < m) sizes[c] = static_cast<uint32_t>(tot[c]);
    }
    if (c == 0) {
        *skip = bad;
        if (bad) atomicOr(error, kErrCounts);
    }
}

}  // namespace mdx
