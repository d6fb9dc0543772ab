// mdx_fused.cuh -- the plain stable partition as ONE cooperative kernel.
//
// The two-kernel path (mdx_plain.cuh) pays, per call, a kernel boundary, a
// serial scan of the chunk counts by the last counting CTA, and a re-read of
// every tile.  Here each CTA owns one chunk of consecutive tiles and runs
//
//   count phase   its chunk's tiles arrive through the CTA's TMA ring
//                 (cp.async.bulk.tensor, 128-byte swizzle, no multicast) and
//                 are counted from shared memory with 4-bit packed counters;
//                 the ring is refilled except for its last STAGES tiles,
//                 which stay resident for the scatter phase;
//   grid barrier  the chunk counts go to the workspace; one arrival counter
//                 and a generation word (bounded spin, error latched on
//                 timeout); a CTA whose copies failed arrives with a failure
//                 mark and the last arrival publishes "abort" with the new
//                 generation, so no CTA scatters from incomplete counts;
//   prefixes      every CTA reads the [class][chunk] count table (16-byte
//                 loads from L2) and forms its own exclusive chunk prefix and
//                 the class bases in parallel -- no serial scan, no launch;
//   scatter phase the chunk walked backwards (the resident tiles first, then
//                 the tiles the count phase read last, still in L2) through
//                 the same ring and tile step as plain_scatter_tma_kernel.
//
// The grid must be co-resident (every CTA waits for every other at the
// barrier): the host launches it cooperatively with at most the occupancy
// bound of CTAs.  A barrier wait that runs out latches kErrTimeout and leaves
// the arrival counter behind: re-initialise the workspace after a timeout.  Semantics and outputs are those of the two-kernel path
// (SeqMdiscr.h:10-57): stable order, class sizes, head flags.
#pragma once

#include <cuda.h>

#include "mdx_device.cuh"
#include "mdx_plain.cuh"
#include "mdx_tile.cuh"

namespace mdx {

struct FusedArgs {
    PlainArgs p;            // in, out, n, tiles, chunks, class_base/tot, sizes, headflags, error, m
    uint32_t chunk_stride;  // row stride of chunk_cnt (a multiple of 4 >= num_chunks)
    uint32_t* bar_count;    // grid barrier: arrivals (low 16 bits) and failures (high 16 bits)
    uint32_t* bar_gen;      // grid barrier: generation (+2 per call), bit 0 = the call aborted
    uint32_t bar_extra;     // arrivals expected beyond the grid (0; tests set 1 to make the wait run out)
    uint64_t wait_ns;       // limit of the barrier wait
};

// Bounded grid barrier (thread 0 of each CTA).  Returns true when the call
// may go on; false when a CTA failed before arriving or the wait ran out.
__device__ __forceinline__ bool fused_grid_barrier(const FusedArgs& a, bool failed) {
    const uint32_t G = a.p.num_chunks;
    const uint32_t g = ld_acquire_u32(a.bar_gen);  // read before arriving: the last
                                                   // arrival moves it on only after this
    __threadfence();                               // this CTA's chunk counts, then the arrival
    const uint32_t old = atomicAdd(a.bar_count, failed ? 0x10001u : 1u);
    if ((old & 0xffffu) == G - 1u + a.bar_extra) {
        const bool any_fail = failed || (old >> 16) != 0u;
        atomicExch(a.bar_count, 0u);
        __threadfence();
        st_release_u32(a.bar_gen, ((g + 2u) & ~1u) | (any_fail ? 1u : 0u));
        return !any_fail;
    }
    uint32_t w = ld_acquire_u32(a.bar_gen);
    if ((w & ~1u) == (g & ~1u)) {
        const uint64_t t0 = globaltimer_ns();
        for (;;) {
            w = ld_acquire_u32(a.bar_gen);
            if ((w & ~1u) != (g & ~1u)) break;
            if (globaltimer_ns() - t0 > a.wait_ns) {
                atomicOr(a.p.error, kErrTimeout);
                return false;
            }
        }
    }
    return (w & 1u) == 0u;
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
    static_assert(ROWS <= 256, "TMA box height");
    static_assert(THREADS % M == 0, "threads per class");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    V* ring = reinterpret_cast<V*>(base);
    V* stage = reinterpret_cast<V*>(base + L::kRingBytes);
    uint16_t* cnt_sm = reinterpret_cast<uint16_t*>(base + L::kRingBytes + L::G::kStageBytes);
    // count-phase reduction table [W][M] in the (still unused) stage
    uint32_t* red = reinterpret_cast<uint32_t*>(stage);

    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ TileShared<M> sh;
    __shared__ uint32_t own_sh[M], tot_sh[M], pre_sh[M];
    __shared__ int go_sh;

    const PlainArgs& a = fa.p;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t G = a.num_chunks, k = blockIdx.x;
    uint32_t t0, t1;
    chunk_tiles(k, a.num_tiles, G, t0, t1);
    const uint32_t cnt = t1 - t0;  // >= 1: G <= number of tiles
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
    __syncthreads();

    uint32_t par = 0;  // bit q: parity of the next wait on ring slot q (uniform over the CTA)
    auto in_map = [&](uint32_t tile) {
        return a.use_tma != 0 && static_cast<uint64_t>(tile + 1) * TILE <= a.n;
    };
    auto issue_tile = [&](uint32_t tile, uint32_t slot) {  // thread 0
        if (in_map(tile)) {
            mbar_arrive_expect_tx(&bars[slot], TILE * sizeof(V));
            tma_load_2d(ring + slot * TILE, &tmap, 0, static_cast<int32_t>(tile * ROWS), &bars[slot]);
        } else {
            mbar_arrive(&bars[slot]);  // read from global memory by the consumer
        }
    };

    // ---------------------------------------------------------- count phase
    // count index i = tile t0 + i, ring slot i % STAGES
    if (tid == 0)
        for (uint32_t i = 0; i < STAGES && i < cnt; i++) issue_tile(t0 + i, i % STAGES);
    bool failed = false;
    uint32_t fail_at = 0;
    const uint32_t e0 = tid * ITEMS;
    if constexpr (M <= 16) {
        PackedCounts<M> pc;
        pc.init();
        for (uint32_t i = 0; i < cnt; i++) {
            const uint32_t tile = t0 + i, slot = i % STAGES;
            const bool ok = mbar_wait_bounded(&bars[slot], (par >> slot) & 1u);
            if (ok) par ^= 1u << slot;
            if (__syncthreads_or(!ok)) {
                failed = true;
                fail_at = i;
                break;
            }
            const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
            if (in_map(tile)) {
                V v[ITEMS];
                take_swizzled<V, ITEMS>(ring + slot * TILE, v);
#pragma unroll
                for (int j = 0; j < ITEMS; j++) {
                    pc.add(d(v[j]));
                    if ((j & 7) == 7) pc.fold();
                }
            } else {
                const uint32_t valid = static_cast<uint32_t>(min(static_cast<uint64_t>(TILE), a.n - ts));
#pragma unroll
                for (int j = 0; j < ITEMS; j++) {
                    if (e0 + j < valid) pc.add(d(in[ts + e0 + j]));
                    if ((j & 7) == 7) pc.fold();
                }
            }
            if constexpr (ITEMS % 8 != 0) pc.fold();
            __syncthreads();  // every thread has read the slot
            if (tid == 0 && i + STAGES < cnt) issue_tile(t0 + i + STAGES, slot);
        }
        pc.finish();
#pragma unroll
        for (int c = 0; c < M; c++) {
            const uint32_t s = warp_sum(pc.acc[c]);
            if (lane == 0) red[warp * M + c] = s;
        }
    } else {
        for (int c = lane; c < M; c += 32) red[warp * M + c] = 0u;
        __syncwarp();
        for (uint32_t i = 0; i < cnt; i++) {
            const uint32_t tile = t0 + i, slot = i % STAGES;
            const bool ok = mbar_wait_bounded(&bars[slot], (par >> slot) & 1u);
            if (ok) par ^= 1u << slot;
            if (__syncthreads_or(!ok)) {
                failed = true;
                fail_at = i;
                break;
            }
            const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
            if (in_map(tile)) {
                V v[ITEMS];
                take_swizzled<V, ITEMS>(ring + slot * TILE, v);
#pragma unroll
                for (int j = 0; j < ITEMS; j++) atomicAdd(&red[warp * M + d(v[j])], 1u);
            } else {
                const uint32_t valid = static_cast<uint32_t>(min(static_cast<uint64_t>(TILE), a.n - ts));
#pragma unroll
                for (int j = 0; j < ITEMS; j++)
                    if (e0 + j < valid) atomicAdd(&red[warp * M + d(in[ts + e0 + j])], 1u);
            }
            __syncthreads();
            if (tid == 0 && i + STAGES < cnt) issue_tile(t0 + i + STAGES, slot);
        }
    }
    if (failed && tid == 0) {
        atomicOr(a.error, kErrTimeout);
        // the copies issued for count indices fail_at .. fail_at + STAGES - 1
        // that have not landed (distinct slots, parity bits still pending):
        // wait for them (bounded) so none outlives the kernel
        for (uint32_t q = fail_at; q < cnt && q < fail_at + STAGES; q++) {
            const uint32_t sq = q % STAGES;
            if (mbar_wait_bounded(&bars[sq], (par >> sq) & 1u)) par ^= 1u << sq;
        }
    }
    __syncthreads();
    if (tid < M) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < W; w++) s += red[w * M + tid];
        own_sh[tid] = s;
        a.chunk_cnt[static_cast<uint64_t>(tid) * fa.chunk_stride + k] = s;
        __threadfence();
    }
    __syncthreads();

    // ---------------------------------------------------------- grid barrier
    if (tid == 0) go_sh = fused_grid_barrier(fa, failed) ? 1 : 0;
    __syncthreads();
    if (!go_sh) return;  // every copy this CTA issued has landed or was waited for above

    // ---------------------------------------------- prefixes and class bases
    {
        constexpr int TPC = THREADS / M;          // threads per class
        constexpr int RW = TPC < 32 ? TPC : 32;   // lanes of one class in a warp
        const uint32_t c = static_cast<uint32_t>(tid / TPC), l = static_cast<uint32_t>(tid % TPC);
        const uint32_t G4 = fa.chunk_stride / 4u;
        const uint4* row = reinterpret_cast<const uint4*>(a.chunk_cnt + static_cast<uint64_t>(c) * fa.chunk_stride);
        uint32_t tot = 0, pre = 0;
        for (uint32_t q = l; q < G4; q += TPC) {
            const uint4 x = __ldcg(row + q);
            const uint32_t j = 4u * q;
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
                sh.cursor[0][c] = bc + pre_sh[c] + own_sh[c];  // end of this chunk's class-c run
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
    __syncthreads();

    // --------------------------------------------------------- scatter phase
    // scatter index s = tile t1 - 1 - s = count index cnt - 1 - s, in ring
    // slot (cnt - 1 - s) % STAGES; the first min(STAGES, cnt) are resident
    auto slot_of = [&](uint32_t s) { return (cnt - 1u - s) % STAGES; };
    const uint32_t resident = cnt < static_cast<uint32_t>(STAGES) ? cnt : static_cast<uint32_t>(STAGES);
    for (uint32_t s = 0; s < cnt; s++) {
        const uint32_t tile = t1 - 1u - s, slot = slot_of(s);
        const uint64_t ts = static_cast<uint64_t>(tile) * TILE;
        const uint32_t valid = static_cast<uint32_t>(min(static_cast<uint64_t>(TILE), a.n - ts));
        const bool full = valid == static_cast<uint32_t>(TILE);
        const uint32_t par_before = par;
        bool ok = true;
        if (s >= resident) {
            ok = mbar_wait_bounded(&bars[slot], (par >> slot) & 1u);
            if (ok) par ^= 1u << slot;
        }
        V v[ITEMS];
        auto refill = [&] {
            if (tid == 0 && s + STAGES < cnt) issue_tile(t1 - 1u - (s + STAGES), slot);
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
            done = tile_scatter<V, D, M, THREADS, false>(d, v, 0u, valid, full, stage, cnt_sm, sh,
                                                         s & 1u, out, ok, refill);
        } else {
            const uint32_t w0 = static_cast<uint32_t>(tid >> 5) * 32u * ITEMS + (tid & 31);
            if (tma_tile) {
                take_striped_swizzled<V, ITEMS>(ring + slot * TILE, v);
            } else {
#pragma unroll
                for (int j = 0; j < ITEMS; j++)
                    v[j] = (w0 + j * 32u < valid) ? in[ts + w0 + j * 32u] : V();
            }
            done = tile_scatter_wide<V, D, M, THREADS, false>(
                d, v, 0u, valid, full, stage, reinterpret_cast<uint32_t*>(cnt_sm), sh, s & 1u, out,
                ok, refill);
        }
        if (!done) {
            if (tid == 0) {
                atomicOr(a.error, kErrTimeout);
                // copies that may still be in flight: scatter indices s .. s +
                // STAGES - 1 past the resident ones (distinct slots); s itself
                // only if this thread's wait on it did not complete
                for (uint32_t q = s; q < cnt && q < s + STAGES; q++) {
                    if (q < resident) continue;
                    const uint32_t sq = slot_of(q);
                    if (q == s && ((par >> sq) & 1u) != ((par_before >> sq) & 1u)) continue;
                    if (mbar_wait_bounded(&bars[sq], (par >> sq) & 1u)) par ^= 1u << sq;
                }
            }
            break;
        }
    }
    if (tid < M) bulk_wait_all();
}

}  // namespace mdx
