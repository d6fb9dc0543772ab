// mdx_fused.cuh -- the plain stable partition as ONE cooperative kernel.
//
// CTA k owns chunk k of the tiles (chunk_tiles) and streams it in both phases,
// so each CTA reads and writes its own regions of the arrays -- the access
// pattern that keeps the scatter at its copy-bandwidth rate.  Per-SM HBM
// bandwidth is uneven, though: with fixed chunks alone the CTAs finished the
// count phase over a ~35 us spread and the scatter over ~70 us.  So the first
// q tiles of every chunk form a shared pool that the CTAs drain by ticket
// after their own part, at the end of each phase:
//
//   count phase   own part [t0 + q, t1) through the CTA's TMA ring
//                 (cp.async.bulk.tensor, 128-byte swizzle -- none for more
//                 than 16 classes -- no multicast),
//                 counted from shared memory with 4-bit packed counters; then
//                 pool tiles by ticket (tile idx of chunk j for ticket
//                 idx * G + j, so concurrent tiles lie far apart), each reduced
//                 with redux.sync into the [tile][class] count table; chunk
//                 sums are added into [class][chunk] (zeroed by the host);
//   grid barrier  one arrival counter and a generation word (bounded spin,
//                 kErrTimeout latched when it runs out); a CTA whose copies
//                 failed arrives with a failure mark and the release then says
//                 "abort", so nobody scatters from incomplete counts;
//   prefixes      every CTA reads the chunk sums (16-byte loads from L2): its
//                 chunk's exclusive prefix, the class bases (CTA 0 writes the
//                 sizes and head flags), the prefixes of its pool tiles inside
//                 the chunk; it publishes them with its chunk's ready word
//                 (the barrier's generation);
//   scatter phase own part from its last tile down (running cursors, the tile
//                 step of plain_scatter_tma_kernel), then pool tiles by ticket,
//                 each with cursors chunk base + tile prefix + tile count read
//                 once its chunk is ready.
//
// The grid must be co-resident (every CTA waits for every other at the
// barrier): the host launches it cooperatively with at most the occupancy
// bound of CTAs.  After a timeout the barrier words are left behind:
// re-initialise the workspace.  Outputs are those of the two-kernel path
// (SeqMdiscr.h:10-57): stable order, class sizes, head flags.
#pragma once

#include <cuda.h>

#include "mdx_device.cuh"
#include "mdx_plain.cuh"
#include "mdx_tile.cuh"

namespace mdx {

struct FusedArgs {
    PlainArgs p;            // num_chunks = chunks = the grid
    uint32_t chunk_stride;  // row stride of chunk_cnt / chunk_pre (a multiple of 4 >= chunks)
    uint32_t pool;          // q: pool tiles at the start of every chunk
    uint32_t* tile_cnt;     // [tiles][M] class counts of every pool tile
    uint32_t* tile_pre;     // [tiles][M] class prefix of every pool tile inside its chunk
    uint32_t* ready;        // [chunks] generation at which the chunk's prefixes were published
                            // (zeroed by the host with chunk_cnt)
    uint32_t* bar_count;    // grid barrier: arrivals (low 16 bits) and failures (high 16 bits)
    uint32_t* bar_gen;      // grid barrier: generation (+2 per call), bit 0 = the call aborted
    uint32_t* cnt_ticket;   // count-phase pool tickets (reset by the last arrival)
    uint32_t* sct_ticket;   // scatter-phase pool tickets (reset by the last arrival)
    uint32_t bar_extra;     // arrivals expected beyond the grid (0; tests set 1 to make the wait run out)
    uint64_t wait_ns;       // limit of a wait
};

constexpr uint32_t kSlotEnd = 0xffffffffu;
constexpr uint32_t kSlotPool = 0x80000000u;  // meta flag: a pool tile

// Bounded spin until *p == want; false when the wait ran out.
__device__ __forceinline__ bool wait_word(const uint32_t* p, uint32_t want, uint64_t limit_ns) {
    if (ld_acquire_u32(p) == want) return true;
    const uint64_t t0 = globaltimer_ns();
    while (ld_acquire_u32(p) != want)
        if (globaltimer_ns() - t0 > limit_ns) return false;
    return true;
}

// The chunk holding `tile` (chunks of chunk_tiles over T tiles, G chunks).
__device__ __forceinline__ uint32_t chunk_of(uint32_t tile, uint32_t T, uint32_t G) {
    uint32_t j = static_cast<uint32_t>((static_cast<uint64_t>(tile) * G + G - 1u) / T);
    if (j >= G) j = G - 1u;
    uint32_t c0, c1;
    chunk_tiles(j, T, G, c0, c1);
    while (tile < c0 && j > 0) chunk_tiles(--j, T, G, c0, c1);
    while (tile >= c1 && j + 1 < G) chunk_tiles(++j, T, G, c0, c1);
    return j;
}

template <class V, class D, int M, int THREADS, int STAGES>
__global__ void __launch_bounds__(THREADS, 4)  // 4 CTAs (32 warps) per SM: <= 64 registers
    plain_fused_kernel(FusedArgs fa, D d, const __grid_constant__ CUtensorMap tmap,
                       const __grid_constant__ OutFlat<V> out) {
    using L = ScatterTmaSmem<V, THREADS, STAGES, M>;
    constexpr int ITEMS = L::kItems;
    constexpr int TILE = L::kTile;
    constexpr int ROWS = L::kRows;
    constexpr int W = THREADS / 32;
    constexpr int HW = (M + 1) / 2;  // 16-bit class-count pairs per pool tile (M <= 16)
    static_assert(ROWS <= 256, "TMA box height");
    static_assert(THREADS % M == 0, "threads per class");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    V* ring = reinterpret_cast<V*>(base);
    V* stage = reinterpret_cast<V*>(base + L::kRingBytes);
    uint16_t* cnt_sm = reinterpret_cast<uint16_t*>(base + L::kRingBytes + L::G::kStageBytes);
    // count-phase tables in the (still unused) stage: chunk reduction [W][M];
    // pool-tile counts by tile parity, M <= 16: [2][W][HW] pairs, else [2][W][M]
    uint32_t* red = reinterpret_cast<uint32_t*>(stage);
    constexpr int PRED = M <= 16 ? W * HW : W * M;
    uint32_t* pred = red + W * M;

    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ uint32_t meta[STAGES];  // tile (| kSlotPool) in the slot, or kSlotEnd
    __shared__ TileShared<M> sh;
    __shared__ uint32_t tot_sh[M], pre_sh[M];
    __shared__ uint32_t gen_sh;
    __shared__ int go_sh;

    const PlainArgs& a = fa.p;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t G = a.num_chunks, T = a.num_tiles, k = blockIdx.x, q = fa.pool;
    const uint32_t stride = fa.chunk_stride;
    uint32_t t0, t1;
    chunk_tiles(k, T, G, t0, t1);
    const uint32_t own_lo = t0 + q;  // own part [own_lo, t1) (q < chunk length)
    const V* in = static_cast<const V*>(a.in);

    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    if (tid < M) {
        tot_sh[tid] = 0u;
        pre_sh[tid] = 0u;
    }
    if constexpr (M > 16) {
        for (int i = tid; i < W * M + 2 * PRED; i += THREADS) red[i] = 0u;
    }
    __syncthreads();

    auto in_map = [&](uint32_t tile) {
        return a.use_tma != 0 && static_cast<uint64_t>(tile + 1) * TILE <= a.n;
    };
    // pool ticket t: tile t / G of chunk t % G's pool part (scatter: from the top)
    auto pool_tile = [&](uint32_t t, bool top_down) {
        const uint32_t j = t % G, idx = t / G;
        uint32_t c0, c1;
        chunk_tiles(j, T, G, c0, c1);
        return top_down ? c0 + q - 1u - idx : c0 + idx;
    };
    // producer (thread 0): own tiles, then pool tickets
    uint32_t p_own = 0;  // own tiles issued
    bool p_done = false;
    // the next pool ticket is taken one tile ahead, so the atomic's round trip
    // overlaps a tile instead of delaying the copy it names
    uint32_t p_ticket = 0;
    bool p_have = false;
    auto produce = [&](uint32_t slot, bool scatter) {
        uint32_t m = kSlotEnd;
        const uint32_t own_n = t1 - own_lo;
        uint32_t* tk = scatter ? fa.sct_ticket : fa.cnt_ticket;
        if (p_own < own_n) {
            m = scatter ? t1 - 1u - p_own : own_lo + p_own;
            p_own++;
            if (p_own == own_n && q > 0) {
                p_ticket = atomicAdd(tk, 1u);
                p_have = true;
            }
        } else if (!p_done) {
            const uint32_t t = p_have ? p_ticket : atomicAdd(tk, 1u);
            if (t < G * q) {
                m = pool_tile(t, scatter) | kSlotPool;
                p_ticket = atomicAdd(tk, 1u);
                p_have = true;
            } else {
                p_done = true;
            }
        }
        meta[slot] = m;
        const uint32_t tile = m & ~kSlotPool;
        if (m != kSlotEnd && in_map(tile)) {
            mbar_arrive_expect_tx(&bars[slot], TILE * sizeof(V));
            tma_load_2d(ring + slot * TILE, &tmap, 0, static_cast<int32_t>(tile * ROWS), &bars[slot]);
        } else {
            mbar_arrive(&bars[slot]);  // end marker, or a tile read from global memory
        }
    };
    uint32_t par = 0;  // bit q: parity of the next wait on ring slot q (uniform over the CTA)
    uint32_t seq = 0;  // ring uses so far: slot = seq % STAGES
    uint32_t par_before = 0;
    auto drain = [&]() {  // thread 0, after a wait that did not complete: the copies in flight
        for (uint32_t u = seq; u < seq + STAGES; u++) {
            const uint32_t su = u % STAGES;
            if (u == seq && ((par >> su) & 1u) != ((par_before >> su) & 1u)) continue;
            if (mbar_wait_bounded(&bars[su], (par >> su) & 1u)) par ^= 1u << su;
        }
    };
    auto take_ends = [&]() {  // all threads: the uses after an end marker are end markers too
        for (uint32_t u = seq + 1; u < seq + STAGES; u++) {
            const uint32_t su = u % STAGES;
            if (mbar_wait_bounded(&bars[su], (par >> su) & 1u)) par ^= 1u << su;
        }
        seq += STAGES;
    };
    const uint32_t e0 = tid * ITEMS;

    // ---------------------------------------------------------- count phase
    if (tid == 0)
        for (uint32_t s = 0; s < STAGES; s++) produce(s, false);
    bool failed = false;
    bool own_open = true;  // the own part's counts are not reduced yet
    PackedCounts<M <= 16 ? M : 16> pc;  // own part, M <= 16
    pc.init();
    for (uint32_t i = 0;; i++, seq++) {
        const uint32_t slot = seq % STAGES;
        par_before = par;
        const bool ok = mbar_wait_bounded(&bars[slot], (par >> slot) & 1u);
        if (ok) par ^= 1u << slot;
        const uint32_t m = meta[slot];  // written before the slot's copy was issued
        const bool pool_t = m != kSlotEnd && (m & kSlotPool) != 0u;
        if (own_open && (m == kSlotEnd || pool_t)) {
            // the own part is counted: its class sums go to the chunk
            if constexpr (M <= 16) {
                pc.finish();
#pragma unroll
                for (int c = 0; c < M; c++) {
                    const uint32_t s = warp_sum(pc.acc[c]);
                    if (lane == 0) red[warp * M + c] = s;
                }
            }
            __syncthreads();
            if (tid < M) {
                uint32_t s = 0;
#pragma unroll
                for (int w = 0; w < W; w++) s += red[w * M + tid];
                atomicAdd(a.chunk_cnt + static_cast<uint64_t>(tid) * stride + k, s);
            }
            own_open = false;
        }
        const uint32_t tp = i & 1u;
        if (m != kSlotEnd) {
            const uint32_t tile = m & ~kSlotPool;
            const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
            const bool tma_tile = in_map(tile);
            const uint32_t valid = static_cast<uint32_t>(min(static_cast<uint64_t>(TILE), a.n - ts));
            V v[ITEMS];
            if (tma_tile) {
                // counts do not depend on the order within a tile: for more
                // than 16 classes the tile is unswizzled and read striped
                if constexpr (M <= 16) take_swizzled<V, ITEMS>(ring + slot * TILE, v);
                else take_striped<V, ITEMS>(ring + slot * TILE, v);
            } else {
#pragma unroll
                for (int j = 0; j < ITEMS; j++) v[j] = (e0 + j < valid) ? in[ts + e0 + j] : V();
            }
            if (!pool_t) {  // own tile: into the running counters
#pragma unroll
                for (int j = 0; j < ITEMS; j++) {
                    if constexpr (M <= 16) {
                        if (tma_tile || e0 + j < valid) pc.add(d(v[j]));
                        if ((j & 7) == 7) pc.fold();
                    } else {
                        if (tma_tile || e0 + j < valid) atomicAdd(&red[warp * M + d(v[j])], 1u);
                    }
                }
                if constexpr (M <= 16 && ITEMS % 8 != 0) pc.fold();
            } else if constexpr (M <= 16) {  // pool tile: its own counts, reduced per warp
                NibbleCounts<M> nc;
                nc.init();
                uint32_t last_c = M;
#pragma unroll
                for (int j = 0; j < ITEMS; j++) {
                    if (tma_tile || e0 + j < valid) {
                        const uint32_t c = d(v[j]);
                        if (j < 15) nc.inc(c); else last_c = c;
                    }
                }
                uint32_t* rw = pred + tp * PRED + warp * HW;
#pragma unroll
                for (int h = 0; h < HW; h++) {
                    uint32_t x = nc.get(2 * h);
                    if (2 * h + 1 < M) x |= nc.get(2 * h + 1) << 16;
                    if (last_c == static_cast<uint32_t>(2 * h)) x += 1u;
                    if (last_c == static_cast<uint32_t>(2 * h + 1)) x += 1u << 16;
                    const uint32_t sum = __reduce_add_sync(0xffffffffu, x);  // <= 4096 per half
                    if (lane == 0) rw[h] = sum;
                }
            } else {
                uint32_t* rw = pred + tp * PRED + warp * M;
#pragma unroll
                for (int j = 0; j < ITEMS; j++)
                    if (tma_tile || e0 + j < valid) atomicAdd(&rw[d(v[j])], 1u);
            }
        }
        // every thread has read the slot; a copy that did not land stops the CTA
        if (__syncthreads_or(!ok)) {
            failed = true;
            if (tid == 0) drain();
            break;
        }
        if (m == kSlotEnd) {
            take_ends();
            break;
        }
        if (tid == 0) produce(slot, false);
        if (pool_t) {  // the pool tile's counts (tables of parity tp are complete)
            const uint32_t tile = m & ~kSlotPool;
            const uint32_t jj = chunk_of(tile, T, G);
            uint32_t* dst = fa.tile_cnt + static_cast<uint64_t>(tile) * M;
            if constexpr (M <= 16) {
                if (tid < HW) {
                    uint32_t s = 0;
#pragma unroll
                    for (int w = 0; w < W; w++) s += pred[tp * PRED + w * HW + tid];
                    dst[2 * tid] = s & 0xffffu;
                    atomicAdd(a.chunk_cnt + static_cast<uint64_t>(2 * tid) * stride + jj, s & 0xffffu);
                    if (2 * tid + 1 < M) {
                        dst[2 * tid + 1] = s >> 16;
                        atomicAdd(a.chunk_cnt + static_cast<uint64_t>(2 * tid + 1) * stride + jj, s >> 16);
                    }
                }
            } else {
                if (tid < M) {
                    uint32_t s = 0;
#pragma unroll
                    for (int w = 0; w < W; w++) {
                        s += pred[tp * PRED + w * M + tid];
                        pred[tp * PRED + w * M + tid] = 0u;  // reused two tiles on
                    }
                    dst[tid] = s;
                    atomicAdd(a.chunk_cnt + static_cast<uint64_t>(tid) * stride + jj, s);
                }
            }
        }
    }

    // ---------------------------------------------------------- grid barrier
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        const uint32_t g = ld_acquire_u32(fa.bar_gen);  // moves on only after every arrival
        __threadfence();
        const uint32_t old = atomicAdd(fa.bar_count, failed ? 0x10001u : 1u);
        bool go;
        uint32_t w;
        if ((old & 0xffffu) == G - 1u + fa.bar_extra) {
            go = !failed && (old >> 16) == 0u;
            *fa.cnt_ticket = 0u;
            *fa.sct_ticket = 0u;
            atomicExch(fa.bar_count, 0u);
            w = ((g + 2u) & ~1u) | (go ? 0u : 1u);
            __threadfence();
            st_release_u32(fa.bar_gen, w);
        } else {
            w = ld_acquire_u32(fa.bar_gen);
            go = true;
            if ((w & ~1u) == (g & ~1u)) {
                const uint64_t tw = globaltimer_ns();
                for (;;) {
                    w = ld_acquire_u32(fa.bar_gen);
                    if ((w & ~1u) != (g & ~1u)) break;
                    if (globaltimer_ns() - tw > fa.wait_ns) {
                        atomicOr(a.error, kErrTimeout);
                        go = false;
                        break;
                    }
                }
            }
            go = go && (w & 1u) == 0u;
        }
        go_sh = go ? 1 : 0;
        gen_sh = w & ~1u;  // this call's ready word: >= 2 after a release (the host zeroes them)
    }
    __syncthreads();
    if (!go_sh) return;  // every copy this CTA issued has landed or was waited for
    const uint32_t gen = gen_sh;

    // ---------------------------------------------- prefixes and class bases
    {
        constexpr int TPC = THREADS / M;          // threads per class
        constexpr int RW = TPC < 32 ? TPC : 32;   // lanes of one class in a warp
        const uint32_t c = static_cast<uint32_t>(tid / TPC), l = static_cast<uint32_t>(tid % TPC);
        const uint32_t G4 = stride / 4u;
        const uint4* row = reinterpret_cast<const uint4*>(a.chunk_cnt + static_cast<uint64_t>(c) * stride);
        uint32_t tot = 0, pre = 0;
        for (uint32_t q4 = l; q4 < G4; q4 += TPC) {
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
    }
    __syncthreads();
    if (warp == 0) {
        // class bases: exclusive scan of the totals (lanes = classes, two
        // passes for 64 classes)
        uint32_t carry = 0;
#pragma unroll
        for (int h = 0; h < (M + 31) / 32; h++) {
            const uint32_t c = static_cast<uint32_t>(lane + 32 * h);
            const uint32_t x = c < static_cast<uint32_t>(M) ? tot_sh[c] : 0u;
            const uint32_t incl = warp_incl_scan(x);
            const uint32_t bc = carry + incl - x;
            if (c < static_cast<uint32_t>(M)) {
                const uint64_t o = static_cast<uint64_t>(c) * stride + k;
                // end of this chunk's class-c run: the own part walks back from it
                sh.cursor[0][c] = bc + pre_sh[c] + __ldcg(a.chunk_cnt + o);
                a.chunk_pre[o] = bc + pre_sh[c];  // this chunk's base, for its pool tiles
                if (k == 0) {
                    a.class_base[c] = bc;
                    a.class_tot[c] = x;
                    if (a.sizes != nullptr && c < a.m) a.sizes[c] = x;
                    // head-flag form (SeqMdiscr.h:47-49); zeroed before the kernel
                    if (a.headflags != nullptr && x > 0) a.headflags[bc] = x;
                }
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    // the class prefixes of this chunk's pool tiles inside the chunk: TPC
    // threads per class, each a run of the q tiles
    if (q > 0) {
        constexpr int TPC = THREADS / M < 32 ? THREADS / M : 32;
        const uint32_t c = static_cast<uint32_t>(tid / TPC), l = static_cast<uint32_t>(tid % TPC);
        const bool scan_thread = tid < M * TPC;
        const uint32_t per = (q + TPC - 1) / TPC;
        const uint32_t r0 = min(t0 + l * per, own_lo), r1 = min(r0 + per, own_lo);
        constexpr int KEEP = 8;
        uint32_t keep[KEEP];
        uint32_t part = 0;
        if (scan_thread) {
#pragma unroll
            for (int u = 0; u < KEEP; u++) {
                keep[u] = r0 + u < r1 ? __ldcg(fa.tile_cnt + static_cast<uint64_t>(r0 + u) * M + c) : 0u;
                part += keep[u];
            }
            for (uint32_t t = r0 + KEEP; t < r1; t++) part += __ldcg(fa.tile_cnt + static_cast<uint64_t>(t) * M + c);
        }
        uint32_t incl = part;
#pragma unroll
        for (int off = 1; off < TPC; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, off, TPC);
            if (static_cast<int>(l) >= off) incl += y;
        }
        if (scan_thread) {
            uint32_t run = incl - part;
#pragma unroll
            for (int u = 0; u < KEEP; u++) {
                if (r0 + u < r1) {
                    fa.tile_pre[static_cast<uint64_t>(r0 + u) * M + c] = run;
                    run += keep[u];
                }
            }
            for (uint32_t t = r0 + KEEP; t < r1; t++) {
                const uint64_t o = static_cast<uint64_t>(t) * M + c;
                fa.tile_pre[o] = run;
                run += __ldcg(fa.tile_cnt + o);
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) st_release_u32(fa.ready + k, gen);  // this chunk's prefixes are out

    // --------------------------------------------------------- scatter phase
    p_own = 0;
    p_done = false;
    p_have = false;
    if (tid == 0)
        for (uint32_t s = 0; s < STAGES; s++) produce((seq + s) % STAGES, true);
    // a pool tile's cursors (thread c < M): its chunk's base + its prefix in
    // the chunk + its count -- the end of its class runs, the tile step walks
    // back; false in `rdy` if the chunk's prefixes never appeared
    auto pool_cursor = [&](uint32_t tile, uint32_t c, bool& rdy) {
        const uint32_t j = chunk_of(tile, T, G);
        rdy = wait_word(fa.ready + j, gen, fa.wait_ns);
        const uint64_t o = static_cast<uint64_t>(tile) * M + c;
        return __ldcg(a.chunk_pre + static_cast<uint64_t>(c) * stride + j) + __ldcg(fa.tile_pre + o) +
               __ldcg(fa.tile_cnt + o);
    };
    uint32_t next_cur = 0;  // thread c < M: cursor of the next pool tile, loaded one tile ahead
    bool have_next = false, next_rdy = true;
    for (uint32_t i = 0;; i++, seq++) {
        const uint32_t slot = seq % STAGES;
        par_before = par;
        const bool ok0 = mbar_wait_bounded(&bars[slot], (par >> slot) & 1u);
        if (ok0) par ^= 1u << slot;
        const uint32_t m = meta[slot];
        if (m == kSlotEnd) {
            take_ends();
            break;
        }
        const uint32_t tile = m & ~kSlotPool;
        const uint32_t tp = i & 1u;  // parity of the tile step's cursor ping-pong
        bool rdy = true;
        if (tid < M) {
            if ((m & kSlotPool) != 0u) {
                if (have_next) {
                    sh.cursor[tp][tid] = next_cur;
                    rdy = next_rdy;
                } else {
                    sh.cursor[tp][tid] = pool_cursor(tile, tid, rdy);
                }
            }
            // a pool tile next in the ring: its cursors while this tile is placed
            const uint32_t nm = meta[(seq + 1) % STAGES];
            have_next = nm != kSlotEnd && (nm & kSlotPool) != 0u;
            if (have_next) next_cur = pool_cursor(nm & ~kSlotPool, tid, next_rdy);
        }
        const bool ok = ok0 && rdy;
        const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
        const uint32_t valid = static_cast<uint32_t>(min(static_cast<uint64_t>(TILE), a.n - ts));
        const bool full = valid == static_cast<uint32_t>(TILE);
        V v[ITEMS];
        auto refill = [&] {
            if (tid == 0) produce(slot, true);
        };
        const bool tma_tile = in_map(tile);
        bool done;
        if constexpr (M <= 16) {
            if (tma_tile) {
                take_swizzled<V, ITEMS>(ring + slot * TILE, v);
            } else {
#pragma unroll
                for (int j = 0; j < ITEMS; j++) v[j] = (e0 + j < valid) ? in[ts + e0 + j] : V();
            }
            // m = 2 keeps the nibble step here: tile_filter measured 1 % slower
            // in this kernel (N = 2^28 u32: 0.544 against 0.538 ms per call)
            done = tile_scatter<V, D, M, THREADS, false>(d, v, 0u, valid, full, stage, cnt_sm, sh, tp,
                                                         out, ok, refill);
        } else {
            const uint32_t w0 = static_cast<uint32_t>(tid >> 5) * 32u * ITEMS + (tid & 31);
            if (tma_tile) {
                take_striped<V, ITEMS>(ring + slot * TILE, v);
            } else {
#pragma unroll
                for (int j = 0; j < ITEMS; j++)
                    v[j] = (w0 + j * 32u < valid) ? in[ts + w0 + j * 32u] : V();
            }
            done = tile_scatter_wide<V, D, M, THREADS, false>(
                d, v, 0u, valid, full, stage, reinterpret_cast<uint32_t*>(cnt_sm), sh, tp, out, ok,
                refill);
        }
        if (!done) {  // a copy did not land or a chunk never got ready: nothing of this tile written
            if (tid == 0) {
                atomicOr(a.error, kErrTimeout);
                drain();
            }
            break;
        }
    }
    if (tid < M) bulk_wait_all();
}

}  // namespace mdx
