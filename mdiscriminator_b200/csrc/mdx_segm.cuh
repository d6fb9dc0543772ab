// mdx_segm.cuh -- segmented (batched) stable m-way partition for sm_100a.
//
// Replaces mdiscrSegm<DISCR> (cuda_code/MdiscrSegmHost.cu.h:36-230: a chain
// of ~12 kernels -- segmented scans of head flags and of N one-hot m-tuples,
// per-element reductions, class offsets, indices, permute, sizes -- with nine
// N-sized temporaries, four of them N*m tuples) by three launches:
//
//   seg_plan_spans  per segment: its length.  Segments longer than one tile
//                   (P elements) are "large" and are cut into runs of up to
//                   RUN_TILES tiles; the other ("small") segments are grouped
//                   by the tile their first element falls in (a group spans
//                   at most 2P elements).  Block-local scans of the run and
//                   group counts; the last CTA scans the block totals and
//                   records the counts, the largest number of runs of one
//                   segment (the lag below) and a new look-back epoch, and
//                   resets the persistent kernel's ticket.
//   seg_plan_emit   writes the run entries {segment, [p0, p1), last run of
//                   the segment} and the group heads, in element order.
//   seg_main        one persistent launch.  CTAs take tickets in order, a
//                   ticket only when the CTA is ready to work on it:
//                     * batches of small-segment groups: each group's range is
//                       read into shared memory by one bulk copy (the next
//                       group's copy overlaps the current group's work), warps
//                       partition one segment each (lanes own odd-stride
//                       contiguous sub-ranges: per-lane 16-bit class counters,
//                       a warp scan, a second pass places the elements) into a
//                       shared output image, and the CTA writes the range back
//                       with 16-byte stores -- one HBM read and one write per
//                       element;
//                     * then, per run j of a large segment, a count item C(j)
//                       (class counts of the run with 16-byte loads, published
//                       to epoch-tagged per-class status words; decoupled
//                       look-back over the segment's earlier runs gives the
//                       run's exclusive prefix, the last run gives the
//                       segment's class totals) and a scatter item S(j) (the
//                       run's tiles through a TMA ring and tile_scatter).
//                       S(j) is issued D tickets after C(j), D = the most runs
//                       of one segment, so it waits only on earlier tickets (no
//                       deadlock) and re-reads its run from L2.
//
// Every wait is bounded (kWaitLimitNs); a wait that runs out latches
// kErrTimeout and publishes what it has so no other CTA waits forever.
//
// Output per segment equals seqMdiscr (SeqMdiscr.h:10-57) applied to the
// segment, which is exactly what MdiscrSegmTest.cu:8-41 validates; sizes are
// emitted as an S x m tuple table and/or per-segment head flags
// (MdiscrSegmKernels.cu.h:89-114 writes the latter into new_sizes).
#pragma once

#include <cuda.h>  // CUtensorMap

#include <type_traits>

#include "mdx_device.cuh"
#include "mdx_plain.cuh"  // PackedCounts
#include "mdx_tile.cuh"

namespace mdx {

// Defaults of the run-time knobs (the autotuner may choose others):
constexpr int kRunTiles = 8;     // tiles per run of a large segment
constexpr int kGroupBatch = 8;   // small-segment groups per work item (pipelined)
constexpr int kLagSlackPct = 50; // extra lag of scatter items, in % of the grid

// status word: [63:34] epoch (30 bits), [33:32] state, [31:0] count
constexpr uint64_t kStAgg = 1ull;
constexpr uint64_t kStInc = 2ull;

__device__ __forceinline__ uint64_t st_pack(uint32_t epoch, uint64_t state, uint32_t v) {
    return (static_cast<uint64_t>(epoch & 0x3fffffffu) << 34) | (state << 32) | v;
}
__device__ __forceinline__ uint32_t st_epoch(uint64_t w) { return static_cast<uint32_t>(w >> 34); }
__device__ __forceinline__ uint64_t st_state(uint64_t w) { return (w >> 32) & 3ull; }

struct SegHeader {      // lives at the start of the segmented workspace
    uint32_t ticket;    // persistent-kernel ticket counter (reset by the planner)
    uint32_t error;     // latched error bits
    uint32_t epoch;     // look-back epoch of the current call (1 .. 2^30-1)
    uint32_t num_runs;  // large-segment runs this call
    uint32_t lag;       // most runs of one segment (max over the planner's blocks)
    uint32_t plan_done; // planner CTA ticket
    uint64_t num_segs;  // S (written by the flags converter for the head-flag form)
    uint32_t lag_cur;   // lag of the current call (snapshot taken by the planner)
    uint32_t flags_ticket;  // tile ticket of the flags converter
    uint32_t flags_done;    // finished tiles of the flags converter
    uint32_t flags_epoch;   // look-back epoch of the flags converter
    uint32_t num_groups;    // small-segment groups this call
    uint32_t pad[3];
};

struct RunEntry {       // a run of up to run_tiles tiles of one large segment
    uint32_t seg;       // segment index
    uint32_t p0, p1;    // element range of the run
    uint32_t jlast;     // entry index of the segment's last run
};

struct SegArgs {
    const void* in;
    void* out;
    uint64_t n;
    const uint64_t* offsets;   // S+1
    uint64_t num_segs;         // S, or kSegsOnDevice: read hdr->num_segs
    uint32_t* seg_sizes;       // S*m or null
    uint32_t* headflags;       // n or null (zeroed before the main kernel)
    const int32_t* in_flags;   // head-flag input (validated by the planner) or null
    uint32_t m;
    SegHeader* hdr;
    uint32_t* run_loc;         // [S] block-local exclusive run offsets
    uint32_t* grp_loc;         // [S] block-local exclusive group-head offsets
    uint32_t* blk_runs;        // [plan blocks] run totals, then offsets
    uint32_t* blk_grps;        // [plan blocks] group totals, then offsets
    RunEntry* runs;            // [max_runs]
    uint32_t* groups;          // [max_groups] first segment of each group
    uint32_t* groups_end;      // [max_groups] one past its last segment (0xffffffff: none
                               // marked, the group runs to S; reset every call)
    uint64_t* status;          // [max_runs][M]
    uint32_t* excl;            // [max_runs][M] exclusive prefix of each run
    uint32_t plan_blocks;
    uint32_t max_runs;         // capacity (enough for segments that tile [0, n))
    uint32_t max_groups;
    int use_tma;               // the tensor map passed to seg_main is valid
    const uint32_t* seg_m;     // per-segment class counts (remainder discriminator), or null:
                               // every segment uses the launch's discriminator
    uint32_t m_bound;          // classes of any segment are < m_bound (per-segment m clamped)
    uint32_t run_tiles;        // tiles per run of a large segment
    uint32_t group_batch;      // small-segment groups per work item
    uint32_t lag_slack_pct;    // extra lag of scatter items, in % of the grid
};

// The discriminator of segment s: the launch's, or -- when the call carries
// per-segment class counts -- key % m_s (m_s clamped to [1, m_bound]).
template <class D>
__device__ __forceinline__ D seg_discr(const SegArgs& a, const D& d, uint64_t s) {
    if constexpr (std::is_same<D, DiscrMod>::value) {
        if (a.seg_m != nullptr) {
            const uint32_t m = min(max(a.seg_m[s], 1u), a.m_bound);
            return DiscrMod::make(m);
        }
    }
    return d;
}

constexpr uint64_t kSegsOnDevice = ~0ull;

__device__ __forceinline__ uint64_t seg_count(const SegArgs& a) {
    return a.num_segs == kSegsOnDevice ? a.hdr->num_segs : a.num_segs;
}

// --------------------------------------------------------------- planning --
// Block b of the planner owns segments [b*R, min((b+1)*R, S)), R = ceil(S/G).
template <int P, int THREADS>
__global__ void __launch_bounds__(THREADS) seg_plan_spans(SegArgs a) {
    constexpr int W = THREADS / 32;
    __shared__ uint32_t warp_runs[W], warp_grps[W];
    __shared__ int am_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t S = seg_count(a);
    const uint64_t G = gridDim.x;
    const uint64_t R = (S + G - 1) / G;
    const uint64_t s0 = blockIdx.x * R, s1 = min(s0 + R, S);
    uint32_t carry_r = 0, carry_g = 0, maxruns = 0;
    for (uint64_t base = s0; base < s1; base += THREADS) {
        const uint64_t s = base + tid;
        uint32_t runs = 0, head = 0;
        if (s < s1) {
            const uint64_t a0 = a.offsets[s], a1 = a.offsets[s + 1];
            if (a1 < a0 || a1 > a.n || (s == 0 && a0 != 0) || (s + 1 == S && a1 != a.n)) {
                atomicOr(&a.hdr->error, kErrSegments);
            } else if (a1 - a0 > static_cast<uint64_t>(P)) {
                const uint32_t span = static_cast<uint32_t>((a1 - 1) / P - a0 / P + 1);
                runs = (span + a.run_tiles - 1) / a.run_tiles;
            } else {
                head = (s == 0 || a.offsets[s - 1] / (P / 2) != a0 / (P / 2)) ? 1u : 0u;
            }
            if (a.in_flags != nullptr && a1 > a0 && a1 <= a.n &&
                static_cast<uint64_t>(a.in_flags[a0]) != a1 - a0)
                atomicOr(&a.hdr->error, kErrSegments);
            if (a.seg_m != nullptr && (a.seg_m[s] < 1u || a.seg_m[s] > a.m_bound))
                atomicOr(&a.hdr->error, kErrSegments);
        }
        maxruns = max(maxruns, runs);
        const uint32_t ir = warp_incl_scan(runs);
        const uint32_t ig = warp_incl_scan(head);
        if (lane == 31) {
            warp_runs[warp] = ir;
            warp_grps[warp] = ig;
        }
        __syncthreads();
        uint32_t pr = 0, pg = 0, tr = 0, tg = 0;
        for (int w = 0; w < W; w++) {
            const uint32_t xr = warp_runs[w], xg = warp_grps[w];
            pr += (w < warp) ? xr : 0u;
            pg += (w < warp) ? xg : 0u;
            tr += xr;
            tg += xg;
        }
        if (s < s1) {
            a.run_loc[s] = carry_r + pr + ir - runs;
            a.grp_loc[s] = carry_g + pg + ig - head;
        }
        carry_r += tr;
        carry_g += tg;
        __syncthreads();
    }
    for (int d = 16; d > 0; d >>= 1) maxruns = max(maxruns, __shfl_xor_sync(0xffffffffu, maxruns, d));
    if (lane == 0 && maxruns > 0) atomicMax(&a.hdr->lag, maxruns);
    if (tid == 0) {
        a.blk_runs[blockIdx.x] = carry_r;
        a.blk_grps[blockIdx.x] = carry_g;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) am_last = (atomicAdd(&a.hdr->plan_done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    // last CTA: exclusive scans of the block totals (in place)
    if (warp < 2) {
        uint32_t* arr = warp == 0 ? a.blk_runs : a.blk_grps;
        uint32_t run = 0;
        for (uint32_t b0 = 0; b0 < gridDim.x; b0 += 32) {
            const uint32_t b = b0 + lane;
            const uint32_t x = b < gridDim.x ? __ldcg(&arr[b]) : 0u;
            const uint32_t incl = warp_incl_scan(x);
            if (b < gridDim.x) arr[b] = run + incl - x;
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) {
            if (warp == 0) {
                a.hdr->num_runs = run <= a.max_runs ? run : 0u;  // over capacity: malformed
                a.hdr->lag_cur = a.hdr->lag;  // every block's atomicMax preceded its ticket
                a.hdr->lag = 0u;
            } else {
                a.hdr->num_groups = run <= a.max_groups ? run : 0u;
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t e = a.hdr->epoch + 1u;
        if (e >= (1u << 30) || e == 0u) e = 1u;
        a.hdr->epoch = e;
        a.hdr->ticket = 0u;
        a.hdr->plan_done = 0u;
        // head-flag converter state for its next call
        a.hdr->flags_ticket = 0u;
        a.hdr->flags_done = 0u;
        uint32_t fe = a.hdr->flags_epoch + 1u;
        if (fe >= (1u << 30)) fe = 1u;
        a.hdr->flags_epoch = fe;
    }
}

template <int P, int THREADS>
__global__ void __launch_bounds__(THREADS) seg_plan_emit(SegArgs a) {
    __shared__ uint32_t list_seg[THREADS], list_pos[THREADS], list_runs[THREADS];
    __shared__ uint32_t list_n;
    const int tid = threadIdx.x;
    const uint64_t S = seg_count(a);
    const uint64_t G = gridDim.x;
    const uint64_t R = (S + G - 1) / G;
    const uint64_t s0 = blockIdx.x * R, s1 = min(s0 + R, S);
    const uint32_t roff = a.blk_runs[blockIdx.x], goff = a.blk_grps[blockIdx.x];
    const uint32_t num_runs = a.hdr->num_runs, num_groups = a.hdr->num_groups;
    for (uint64_t base = s0; base < s1; base += THREADS) {
        if (tid == 0) list_n = 0;
        __syncthreads();
        const uint64_t s = base + tid;
        if (s < s1) {
            const uint64_t a0 = a.offsets[s], a1 = a.offsets[s + 1];
            if (a1 >= a0 && a1 <= a.n) {
                if (a1 - a0 > static_cast<uint64_t>(P)) {
                    const uint32_t span = static_cast<uint32_t>((a1 - 1) / P - a0 / P + 1);
                    const uint32_t nr = (span + a.run_tiles - 1) / a.run_tiles;
                    const uint32_t pos = roff + a.run_loc[s];
                    if (nr <= 16) {  // this thread emits the runs itself
                        if (static_cast<uint64_t>(pos) + nr <= num_runs) {
                            const uint64_t w0 = a0 / P;
                            for (uint32_t r = 0; r < nr; r++) {
                                const uint64_t wa = w0 + static_cast<uint64_t>(r) * a.run_tiles;
                                RunEntry e;
                                e.seg = static_cast<uint32_t>(s);
                                e.p0 = static_cast<uint32_t>(max(a0, wa * P));
                                e.p1 = static_cast<uint32_t>(min(a1, (wa + a.run_tiles) * P));
                                e.jlast = pos + nr - 1u;
                                a.runs[pos + r] = e;
                            }
                        }
                    } else {  // long segments: the whole block emits them below
                        const uint32_t q = atomicAdd(&list_n, 1u);
                        list_seg[q] = static_cast<uint32_t>(s);
                        list_pos[q] = pos;
                        list_runs[q] = nr;
                    }
                } else if (s == 0 || a.offsets[s - 1] / (P / 2) != a0 / (P / 2)) {
                    const uint32_t g = goff + a.grp_loc[s];
                    if (g < num_groups) a.groups[g] = static_cast<uint32_t>(s);
                }
            }
            // the group before segment s ends at s at the latest when s starts
            // a group, is large or is malformed
            const bool small_ok = (a1 >= a0 && a1 <= a.n && a1 - a0 <= static_cast<uint64_t>(P));
            const bool is_head = small_ok && (s == 0 || a.offsets[s - 1] / (P / 2) != a0 / (P / 2));
            const uint32_t before = goff + a.grp_loc[s];  // groups starting before s
            if ((is_head || !small_ok) && before >= 1u && before - 1u < num_groups)
                atomicMin(&a.groups_end[before - 1u], static_cast<uint32_t>(s));
        }
        __syncthreads();
        const uint32_t cnt = list_n;
        for (uint32_t q = 0; q < cnt; q++) {  // the block emits each large segment's runs
            const uint32_t seg = list_seg[q], pos = list_pos[q], nr = list_runs[q];
            if (static_cast<uint64_t>(pos) + nr > num_runs) continue;  // malformed offsets
            const uint64_t a0 = a.offsets[seg], a1 = a.offsets[seg + 1];
            const uint64_t w0 = a0 / P;
            for (uint32_t r = tid; r < nr; r += THREADS) {
                const uint64_t wa = w0 + static_cast<uint64_t>(r) * a.run_tiles;
                RunEntry e;
                e.seg = seg;
                e.p0 = static_cast<uint32_t>(max(a0, wa * P));
                e.p1 = static_cast<uint32_t>(min(a1, (wa + a.run_tiles) * P));
                e.jlast = pos + nr - 1u;
                a.runs[pos + r] = e;
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------- main kernel --
template <class V, int M, int THREADS, int STAGES>
struct SegSmem {
    using G = TileGeom<V, THREADS, M>;
    static constexpr int kTile = G::kTile;  // == P
    static constexpr uint32_t kAU = G::kAU;
    // small groups (segments starting in one half-tile window, each <= P):
    // two input buffers (one being filled by TMA) and an output image, each
    // for a range of <= P/2 + P elements plus 16-byte alignment slack
    static constexpr int kGroupElems = kTile / 2 + kTile + 2 * static_cast<int>(kAU);
    static constexpr size_t kGroupBytes = 3ull * kGroupElems * sizeof(V);
    // runs: TMA ring + tile stage + count matrix
    static constexpr size_t kRingBytes = static_cast<size_t>(STAGES) * kTile * sizeof(V);
    static constexpr size_t kRunBytes = kRingBytes + G::kStageBytes + G::kCntBytes;
    static constexpr size_t kBytes = 1024 + (kGroupBytes > kRunBytes ? kGroupBytes : kRunBytes);
};

// Bounded spin on a status word until it carries this epoch with state >=
// `want`.  Returns false on timeout.
__device__ __forceinline__ bool wait_status(const uint64_t* p, uint32_t epoch, uint64_t want,
                                            uint64_t& w) {
    w = ld_acquire_u64(p);
    if (st_epoch(w) == epoch && st_state(w) >= want) return true;
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        w = ld_acquire_u64(p);
        if (st_epoch(w) == epoch && st_state(w) >= want) return true;
        if (globaltimer_ns() - t0 > kWaitLimitNs) return false;
    }
}

// Per-lane class counters in 16-bit fields (M <= 16: (M+1)/2 words), wide
// enough for a whole segment's totals after a warp scan (<= 2P < 2^16).
template <int M>
struct HalfCounts {
    static constexpr int NW = (M + 1) / 2;
    uint32_t w[NW];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int q = 0; q < NW; q++) w[q] = 0;
    }
    __device__ __forceinline__ uint32_t get(uint32_t c) const {
        uint32_t x = w[0];
#pragma unroll
        for (int q = 1; q < NW; q++) x = (c >> 1) == static_cast<uint32_t>(q) ? w[q] : x;
        return (x >> ((c & 1u) << 4)) & 0xffffu;
    }
    __device__ __forceinline__ void inc(uint32_t c) {
        const uint32_t one = 1u << ((c & 1u) << 4);
#pragma unroll
        for (int q = 0; q < NW; q++) w[q] += (c >> 1) == static_cast<uint32_t>(q) ? one : 0u;
    }
};

// One warp partitions one segment held in shared memory (element e at
// src[e], 0 <= e < L <= 2P) into the shared output image dst[0 .. L) and
// writes the segment's sizes.  Lane l owns the contiguous elements
// [l*k, (l+1)*k) with k odd (so the 32 lanes read 32 different banks):
// pass 1 counts them, a warp scan of the counters gives every lane its
// per-class prefix (stable: lane order = input order) and the segment's
// class offsets, pass 2 places them.
template <class V, class D, int M>
__device__ void seg_small_warp(const SegArgs& a, const D& d, uint64_t s, uint64_t a0, uint32_t L,
                               const V* src, V* dst) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t k = (L + 31u) >> 5;
    k |= 1u;  // odd stride
    const uint32_t b = min(lane * k, L), e1 = min(b + k, L);
    HalfCounts<M> cnt;
    cnt.zero();
    for (uint32_t e = b; e < e1; e++) cnt.inc(d(src[e]));
    // warp inclusive scan of the packed counters
    HalfCounts<M> incl = cnt;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
#pragma unroll
        for (int q = 0; q < HalfCounts<M>::NW; q++) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl.w[q], dd);
            if (lane >= static_cast<uint32_t>(dd)) incl.w[q] += y;
        }
    }
    // segment totals (lane 31's inclusive) -> class offsets
    HalfCounts<M> tot;
#pragma unroll
    for (int q = 0; q < HalfCounts<M>::NW; q++) tot.w[q] = __shfl_sync(0xffffffffu, incl.w[q], 31);
    HalfCounts<M> base;  // class offset + this lane's exclusive prefix, per class
    base.zero();
    uint32_t off = 0;
#pragma unroll
    for (int c = 0; c < M; c++) {
        const uint32_t t = tot.get(c);
        const uint32_t mine = incl.get(c) - cnt.get(c) + off;
        base.w[c >> 1] |= mine << ((c & 1) << 4);
        if (static_cast<uint32_t>(c) == lane) {
            if (a.seg_sizes != nullptr && static_cast<uint32_t>(c) < a.m) a.seg_sizes[s * a.m + c] = t;
            if (a.headflags != nullptr && t > 0) a.headflags[a0 + off] = t;
        }
        off += t;
    }
    for (uint32_t e = b; e < e1; e++) {
        const V v = src[e];
        const uint32_t c = d(v);
        dst[base.get(c)] = v;
        base.inc(c);
    }
}

template <class V, class D, int M, int THREADS, int STAGES>
__global__ void __launch_bounds__(THREADS, 3)
    seg_main(SegArgs a, D d, const __grid_constant__ CUtensorMap tmap) {
    using L = SegSmem<V, M, THREADS, STAGES>;
    using TG = typename L::G;
    constexpr int ITEMS = TG::kItems;
    constexpr int P = L::kTile;
    constexpr int ROWS = TG::kRows;
    constexpr uint32_t AU = L::kAU;
    constexpr int W = THREADS / 32;
    static_assert(M <= 16 && M >= 2, "class bound");
    static_assert(ROWS <= 256, "TMA box height");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    // small groups
    V* g_in0 = reinterpret_cast<V*>(base);
    V* g_out = g_in0 + 2 * L::kGroupElems;
    // runs (aliases the group buffers)
    V* ring = reinterpret_cast<V*>(base);
    V* stage = reinterpret_cast<V*>(base + L::kRingBytes);
    uint16_t* cnt_sm = reinterpret_cast<uint16_t*>(base + L::kRingBytes + TG::kStageBytes);

    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ __align__(8) uint64_t gbars[2];
    __shared__ TileShared<M> sh;
    __shared__ uint32_t ticket_sh[2];
    __shared__ uint32_t gi_h[2], gi_he[2], gi_next[2];  // group pipeline slots
    __shared__ uint64_t gi_r0[2], gi_r1[2], gi_as[2], gi_tail[2];
    __shared__ uint32_t red[W][M];
    __shared__ int fail_sh;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const V* in = static_cast<const V*>(a.in);
    V* out = static_cast<V*>(a.out);
    const uint32_t out_phase =
        static_cast<uint32_t>(reinterpret_cast<uintptr_t>(out) / sizeof(V)) & (AU - 1u);
    const bool in_vec = (reinterpret_cast<uintptr_t>(in) & 15u) == 0;
    const bool out_vec = (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
    const bool tma_ok = a.use_tma != 0;
    const uint64_t S = seg_count(a);
    const uint32_t epoch = a.hdr->epoch;
    const uint32_t num_runs = a.hdr->num_runs;
    const uint32_t num_groups = a.hdr->num_groups;
    // S(j) trails C(j) by the most runs of one segment (so it only waits on
    // earlier tickets) plus half a grid of slack (so those are mostly done)
    const uint32_t lag =
        min(max(a.hdr->lag_cur, 1u) + gridDim.x * a.lag_slack_pct / 100u, max(num_runs, 1u));
    const uint32_t num_batches = (num_groups + a.group_batch - 1) / a.group_batch;
    const uint32_t total = num_batches + 2u * num_runs;
    uint32_t ring_uses = 0;   // mbarrier phase bookkeeping across items
    uint32_t group_uses = 0;

    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; s++) mbar_init(&bars[s], 1);
        mbar_init(&gbars[0], 1);
        mbar_init(&gbars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();

    // A ticket is taken only when the CTA is ready to work on it: a ticket held
    // while its CTA waits on another item would delay every item that waits on
    // it in turn.
    for (uint32_t it = 0;; it++) {
        if (tid == 0) ticket_sh[it & 1u] = atomicAdd(&a.hdr->ticket, 1u);
        __syncthreads();
        const uint32_t t = ticket_sh[it & 1u];
        if (t >= total) break;

        if (t < num_batches) {
            // ---------------- a batch of small-segment groups ----------------
            // group i of the batch: segments [h, he), elements [r0, r1); its
            // range is fetched by one bulk copy while the previous group is
            // partitioned
            const uint32_t g0 = t * a.group_batch;
            const uint32_t gcnt = min(a.group_batch, num_groups - g0);
            auto issue_group = [&](uint32_t i) {  // thread 0 only
                const uint32_t slot = (group_uses + i) & 1u;
                const uint32_t h = a.groups[g0 + i];
                const uint32_t he = static_cast<uint32_t>(min(static_cast<uint64_t>(a.groups_end[g0 + i]), S));
                const uint64_t r0 = a.offsets[h], r1 = a.offsets[he];
                const uint64_t as = r0 & ~static_cast<uint64_t>(AU - 1u);
                uint64_t ve = min((r1 + AU - 1u) & ~static_cast<uint64_t>(AU - 1u),
                                  a.n & ~static_cast<uint64_t>(AU - 1u));
                if (!in_vec || ve < as) ve = as;
                gi_h[slot] = h;
                gi_he[slot] = he;
                gi_next[slot] = h;
                gi_r0[slot] = r0;
                gi_r1[slot] = r1;
                gi_as[slot] = as;
                gi_tail[slot] = max(ve, r0);
                V* dst = g_in0 + slot * L::kGroupElems;
                const uint32_t bytes = static_cast<uint32_t>((ve - as) * sizeof(V));
                if (bytes > 0) {
                    mbar_arrive_expect_tx(&gbars[slot], bytes);
                    bulk_load_g2s(dst, in + as, bytes, &gbars[slot]);
                } else {
                    mbar_arrive(&gbars[slot]);
                }
            };
            if (tid == 0) issue_group(0);
            bool failed = false;
            for (uint32_t i = 0; i < gcnt; i++) {
                const uint32_t use = group_uses + i;
                const uint32_t slot = use & 1u;
                const bool ok = mbar_wait_bounded(&gbars[slot], (use >> 1) & 1u);
                __syncthreads();  // slot info visible
                V* gin = g_in0 + slot * L::kGroupElems;
                const uint64_t as = gi_as[slot], r0 = gi_r0[slot], r1 = gi_r1[slot];
                for (uint64_t e = gi_tail[slot] + tid; e < r1; e += THREADS) gin[e - as] = in[e];
                if (__syncthreads_or(!ok)) {
                    failed = true;
                    if (tid == 0) {  // only this group's copy can be in flight
                        atomicOr(&a.hdr->error, kErrTimeout);
                        (void)mbar_wait_bounded(&gbars[slot], (use >> 1) & 1u);
                    }
                    break;
                }
                if (tid == 0 && i + 1 < gcnt) issue_group(i + 1);  // the other buffer is free
                const uint32_t he = gi_he[slot];
                for (;;) {
                    uint32_t s = 0;
                    if (lane == 0) s = atomicAdd(&gi_next[slot], 1u);
                    s = __shfl_sync(0xffffffffu, s, 0);
                    if (s >= he) break;
                    const uint64_t a0 = a.offsets[s], a1 = a.offsets[s + 1];
                    seg_small_warp<V, D, M>(a, seg_discr(a, d, s), s, a0, static_cast<uint32_t>(a1 - a0),
                                            gin + (a0 - as), g_out + (a0 - as));
                }
                __syncthreads();
                // write the range back from the output image
                if (out_vec && out_phase == 0u) {
                    const uint64_t vs = (r0 + AU - 1u) & ~static_cast<uint64_t>(AU - 1u);
                    const uint64_t ve = r1 & ~static_cast<uint64_t>(AU - 1u);
                    if (vs < ve) {
                        const uint4* srcv = reinterpret_cast<const uint4*>(g_out + (vs - as));
                        uint4* dstv = reinterpret_cast<uint4*>(out + vs);
                        const uint32_t nv = static_cast<uint32_t>((ve - vs) / AU);
                        for (uint32_t q = tid; q < nv; q += THREADS) dstv[q] = srcv[q];
                        for (uint64_t e = r0 + tid; e < vs; e += THREADS) out[e] = g_out[e - as];
                        for (uint64_t e = ve + tid; e < r1; e += THREADS) out[e] = g_out[e - as];
                    } else {
                        for (uint64_t e = r0 + tid; e < r1; e += THREADS) out[e] = g_out[e - as];
                    }
                } else {
                    for (uint64_t e = r0 + tid; e < r1; e += THREADS) out[e] = g_out[e - as];
                }
                // generic-proxy accesses of these buffers precede the next TMA writes
                fence_proxy_async_smem();
            }
            group_uses += gcnt;
            __syncthreads();
            if (failed) break;
            continue;
        }

        // ---------------- runs of large segments ----------------
        const uint32_t u = t - num_batches;
        uint32_t j;
        bool is_count;
        if (u < lag) {
            j = u;
            is_count = true;
        } else {
            const uint32_t v = u - lag;
            const uint32_t pairs = num_runs - lag;
            if (v < 2u * pairs) {
                is_count = (v & 1u) != 0u;
                j = is_count ? lag + (v >> 1) : (v >> 1);
            } else {
                is_count = false;
                j = pairs + (v - 2u * pairs);
                if (lag >= num_runs) j = num_runs - 1u - j;  // all counts first: walk back (L2)
            }
        }
        const RunEntry ent = a.runs[j];
        const uint64_t seg_start = a.offsets[ent.seg];
        const D dj = seg_discr(a, d, ent.seg);
        const bool first_run = (ent.p0 == static_cast<uint32_t>(seg_start));
        const bool last_run = (j == ent.jlast);

        if (is_count) {
            // ---------------- C(j): class counts of the run + look-back ----
            PackedCounts<M> pc;
            pc.init();
            const uint64_t p0 = ent.p0, p1 = ent.p1;
            const uint64_t vs = in_vec ? ((p0 + AU - 1u) & ~static_cast<uint64_t>(AU - 1u)) : p1;
            const uint64_t ve = in_vec ? max(vs, p1 & ~static_cast<uint64_t>(AU - 1u)) : p1;
            {
                uint32_t k = 0;
                for (uint64_t e = p0 + tid; e < min(vs, p1); e += THREADS) {
                    pc.add(dj(in[e]));
                    if (++k == 8u) {
                        pc.fold();
                        k = 0;
                    }
                }
                for (uint64_t e = ve + tid; e < p1 && vs < p1; e += THREADS) {
                    pc.add(dj(in[e]));
                    if (++k == 8u) {
                        pc.fold();
                        k = 0;
                    }
                }
                pc.fold();
            }
            {
                const uint4* vp = reinterpret_cast<const uint4*>(in + vs);
                const uint32_t nv = static_cast<uint32_t>((ve - vs) / AU);
                constexpr int UNROLL = 4;
                for (uint32_t q = tid; q < nv; q += THREADS * UNROLL) {
                    uint4 r[UNROLL];
#pragma unroll
                    for (int uu = 0; uu < UNROLL; uu++)
                        if (q + uu * THREADS < nv) r[uu] = __ldg(vp + q + uu * THREADS);
#pragma unroll
                    for (int uu = 0; uu < UNROLL; uu++) {
                        if (q + uu * THREADS < nv) {
                            V e[AU];
                            unpack16_to<V>(r[uu], e);
#pragma unroll
                            for (uint32_t z = 0; z < AU; z++) pc.add(dj(e[z]));
                        }
                        if (uu & 1) pc.fold();  // every two vectors: <= 8 increments
                    }
                }
            }
            pc.finish();
#pragma unroll
            for (int c = 0; c < M; c++) {
                const uint32_t x = warp_sum(pc.acc[c]);
                if (lane == 0) red[warp][c] = x;
            }
            __syncthreads();
            if (warp == 0) {
                const uint32_t c = lane;
                const bool cls = c < static_cast<uint32_t>(M);
                uint32_t agg = 0;
                if (cls)
                    for (int w = 0; w < W; w++) agg += red[w][c];
                uint64_t* st = a.status + static_cast<uint64_t>(j) * M;
                uint32_t prefix = 0;
                bool ok = true;
                if (cls) {
                    if (first_run) {
                        a.excl[static_cast<uint64_t>(j) * M + c] = 0u;
                        __threadfence();
                        st_release_u64(st + c, st_pack(epoch, kStInc, agg));
                    } else {
                        st_release_u64(st + c, st_pack(epoch, kStAgg, agg));
                        // decoupled look-back over this segment's earlier runs
                        for (uint32_t jj = j - 1u;; jj--) {
                            uint64_t w;
                            if (!wait_status(a.status + static_cast<uint64_t>(jj) * M + c, epoch,
                                             kStAgg, w)) {
                                ok = false;
                                break;
                            }
                            prefix += static_cast<uint32_t>(w);
                            if (st_state(w) == kStInc) break;
                        }
                        a.excl[static_cast<uint64_t>(j) * M + c] = prefix;
                        __threadfence();
                        st_release_u64(st + c, st_pack(epoch, kStInc, prefix + agg));
                    }
                }
                if (__any_sync(0xffffffffu, !ok) && lane == 0) atomicOr(&a.hdr->error, kErrTimeout);
                if (last_run) {
                    // segment totals -> sizes (tuple and head-flag forms)
                    const uint32_t tot = cls ? prefix + agg : 0u;
                    const uint32_t incl = warp_incl_scan(tot);
                    if (cls) {
                        if (a.seg_sizes != nullptr && c < a.m)
                            a.seg_sizes[static_cast<uint64_t>(ent.seg) * a.m + c] = tot;
                        if (a.headflags != nullptr && tot > 0)
                            a.headflags[seg_start + incl - tot] = tot;
                    }
                }
            }
            __syncthreads();
            continue;
        }

        // ---------------- S(j): scatter the run ----------------
        if (warp == 0) {
            const uint32_t c = lane;
            bool ok = true;
            uint32_t tot = 0, pre = 0;
            if (c < static_cast<uint32_t>(M)) {
                uint64_t w;
                ok = wait_status(a.status + static_cast<uint64_t>(ent.jlast) * M + c, epoch, kStInc, w);
                tot = static_cast<uint32_t>(w);
                uint64_t w2;
                ok = wait_status(a.status + static_cast<uint64_t>(j) * M + c, epoch, kStInc, w2) && ok;
                pre = __ldcg(a.excl + static_cast<uint64_t>(j) * M + c);
            }
            const uint32_t incl = warp_incl_scan(tot);
            if (c < static_cast<uint32_t>(M))
                sh.cursor[0][c] = static_cast<uint32_t>(seg_start) + (incl - tot) + pre;
            const bool bad = __any_sync(0xffffffffu, !ok);
            if (lane == 0) {
                fail_sh = bad ? 1 : 0;
                if (bad) atomicOr(&a.hdr->error, kErrTimeout);
            }
        }
        __syncthreads();
        if (fail_sh) continue;  // uniform: nothing was issued
        const uint32_t wf = ent.p0 / P, wl = (ent.p1 - 1u) / P;
        const uint32_t ntiles = wl - wf + 1u;
        auto issue = [&](uint32_t i) {  // tile wf+i into ring slot (ring_uses+i) % STAGES
            const uint32_t w = wf + i;
            const uint32_t slot = (ring_uses + i) % STAGES;
            const bool whole = static_cast<uint64_t>(w) * P >= ent.p0 &&
                               static_cast<uint64_t>(w + 1) * P <= ent.p1;
            if (tma_ok && whole) {
                mbar_arrive_expect_tx(&bars[slot], P * sizeof(V));
                tma_load_2d(ring + slot * P, &tmap, 0, static_cast<int32_t>(w * ROWS), &bars[slot]);
            } else {
                mbar_arrive(&bars[slot]);
            }
        };
        if (tid == 0)
            for (uint32_t i = 0; i < STAGES && i < ntiles; i++) issue(i);
        const uint32_t e0 = tid * ITEMS;
        bool failed = false;
        for (uint32_t i = 0; i < ntiles; i++) {
            const uint32_t w = wf + i;
            const uint64_t ts = static_cast<uint64_t>(w) * P;
            const uint32_t lo = static_cast<uint32_t>(max(static_cast<uint64_t>(ent.p0), ts) - ts);
            const uint32_t hi = static_cast<uint32_t>(min(static_cast<uint64_t>(ent.p1), ts + P) - ts);
            const bool full = lo == 0u && hi == static_cast<uint32_t>(P);
            const uint32_t use = ring_uses + i;
            const bool ok = mbar_wait_bounded(&bars[use % STAGES], (use / STAGES) & 1u);
            V v[ITEMS];
            if (tma_ok && full) {
                take_swizzled<V, ITEMS>(ring + (use % STAGES) * P, v);
            } else {
#pragma unroll
                for (int q = 0; q < ITEMS; q++)
                    v[q] = (e0 + q >= lo && e0 + q < hi) ? in[ts + e0 + q] : V();
            }
            const bool done = tile_scatter<V, D, M, THREADS, true>(
                dj, v, lo, hi, full, stage, cnt_sm, sh, i & 1u, OutFlat<V>{out, out_phase}, ok, [&] {
                    if (tid == 0 && i + STAGES < ntiles) issue(i + STAGES);
                });
            if (!done) {
                failed = true;
                if (tid == 0) {
                    atomicOr(&a.hdr->error, kErrTimeout);
                    for (uint32_t q = i; q < ntiles && q < i + STAGES; q++)
                        (void)mbar_wait_bounded(&bars[(ring_uses + q) % STAGES],
                                                ((ring_uses + q) / STAGES) & 1u);
                }
                break;
            }
        }
        ring_uses += ntiles;
        // the ring and the stage alias the group buffers: the bulk stores must
        // have read the stage before a group item may overwrite it
        if (tid < M) bulk_wait_read<0>();
        __syncthreads();
        if (failed) break;
    }
    if (tid < M) bulk_wait_all();
}

// ------------------------------------------------ head flags -> offsets --
// The reference's segment descriptor (MdiscrSegmHost.cu.h:36-42,
// populateSizesArray HelpersCommon.h:105-151) is an n-entry array holding each
// segment's length at its first element and 0 elsewhere.  One pass of a
// decoupled look-back compaction writes the start positions (offsets[0..S-1]),
// offsets[S] = n, and S into the header; the planner then checks that every
// flag equals the distance to the next start.  Tiles of FT flags, dynamic tile
// tickets, per-tile status words tagged with the converter's epoch.
template <int THREADS, int FT>
__global__ void __launch_bounds__(THREADS) seg_flags_to_offsets(const int32_t* flags, uint64_t n,
                                                                uint64_t* offsets, SegHeader* hdr,
                                                                uint64_t* tile_status) {
    constexpr int ITEMS = FT / THREADS;
    constexpr int W = THREADS / 32;
    static_assert(ITEMS * THREADS == FT, "tile");
    __shared__ uint32_t tile_sh, base_sh, warp_tot[W];
    __shared__ int last_sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t num_tiles = static_cast<uint32_t>((n + FT - 1) / FT);
    const uint32_t epoch = hdr->flags_epoch;
    for (;;) {
        if (tid == 0) tile_sh = atomicAdd(&hdr->flags_ticket, 1u);
        __syncthreads();
        const uint32_t t = tile_sh;
        if (t >= num_tiles) break;
        const uint64_t ts = static_cast<uint64_t>(t) * FT;
        // blocked: thread holds flags ts + tid*ITEMS .. +ITEMS-1
        uint32_t nz = 0;
        int32_t f[ITEMS];
#pragma unroll
        for (int q = 0; q < ITEMS; q++) {
            const uint64_t i = ts + static_cast<uint64_t>(tid) * ITEMS + q;
            f[q] = i < n ? flags[i] : 0;
            nz += f[q] != 0 ? 1u : 0u;
        }
        const uint32_t incl = warp_incl_scan(nz);
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        uint32_t wpre = 0, agg = 0;
        for (int w = 0; w < W; w++) {
            wpre += w < warp ? warp_tot[w] : 0u;
            agg += warp_tot[w];
        }
        if (warp == 0) {
            uint32_t prefix = 0;
            bool ok = true;
            if (lane == 0) {
                uint64_t* st = tile_status + t;
                if (t == 0) {
                    st_release_u64(st, st_pack(epoch, kStInc, agg));
                } else {
                    st_release_u64(st, st_pack(epoch, kStAgg, agg));
                    for (uint32_t tt = t - 1u;; tt--) {
                        uint64_t w;
                        if (!wait_status(tile_status + tt, epoch, kStAgg, w)) {
                            ok = false;
                            break;
                        }
                        prefix += static_cast<uint32_t>(w);
                        if (st_state(w) == kStInc) break;
                    }
                    st_release_u64(st, st_pack(epoch, kStInc, prefix + agg));
                }
                if (!ok) atomicOr(&hdr->error, kErrTimeout);
                base_sh = prefix;
            }
        }
        __syncthreads();
        uint32_t pos = base_sh + wpre + incl - nz;
#pragma unroll
        for (int q = 0; q < ITEMS; q++) {
            if (f[q] != 0) {
                if (f[q] < 0) atomicOr(&hdr->error, kErrSegments);
                offsets[pos++] = ts + static_cast<uint64_t>(tid) * ITEMS + q;
            }
        }
        // the tile that finishes last writes S and offsets[S]
        if (tid == 0) {
            __threadfence();
            last_sh = (atomicAdd(&hdr->flags_done, 1u) == num_tiles - 1u);
        }
        __syncthreads();
        if (last_sh && tid == 0) {
            const uint64_t w = ld_acquire_u64(tile_status + (num_tiles - 1u));
            const uint64_t S = static_cast<uint32_t>(w);
            hdr->num_segs = S;
            offsets[S] = n;
            if (n > 0 && flags[0] == 0) atomicOr(&hdr->error, kErrSegments);
            // the ticket, done counter and epoch are reset by the planner,
            // which runs after every CTA of this kernel has left its loop
        }
        __syncthreads();
    }
}

}  // namespace mdx
