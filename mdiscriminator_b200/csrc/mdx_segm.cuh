// mdx_segm.cuh -- segmented (batched) stable m-way partition for sm_100a.
//
// Replaces mdiscrSegm<DISCR> (cuda_code/MdiscrSegmHost.cu.h:36-230: a chain
// of ~12 kernels -- segmented scans of head flags and of N one-hot m-tuples,
// per-element reductions, class offsets, indices, permute, sizes -- with nine
// N-sized temporaries, four of them N*m tuples) by six launches:
//
//   seg_plan_spans  per segment: its length.  Segments longer than one tile
//                   (P elements) are "large" and are cut into runs of up to
//                   RUN_TILES tiles; the other ("small") segments are grouped
//                   (consecutive small segments starting in one window of
//                   P elements, at most kGroupSegs of them).  Block-local
//                   scans of the run and group counts; the last CTA scans the
//                   block totals, records the counts and resets the tickets.
//   seg_plan_emit   writes the run entries {segment, [p0, p1), last run of
//                   the segment} and the group heads, in element order.
//   seg_main        persistent; CTAs take tickets for batches of groups.
//                   Each group's range is read into shared memory by one bulk
//                   copy and partitioned by the whole CTA (seg_group_cta:
//                   every thread owns ~L/256 consecutive elements whatever the
//                   segment lengths; a segmented scan of per-thread class
//                   counts, the segments' class bases in shared memory) into
//                   a shared output image written back with 16-byte stores --
//                   one HBM read and one write per element;
//   seg_run_count   the class counts of every run of the large segments,
//                   one CTA per run (16-byte loads, warp reductions).
//   seg_run_scan    per large segment (a lane, or a warp for many runs):
//                   the runs' exclusive class prefixes, the segment's sizes
//                   and head flags, and every run's output position per class.
//   seg_run_scatter persistent; the runs in reverse order through a TMA ring
//                   and tile_scatter (as the plain scatter), from those
//                   positions.
//
// The partition kernels and the head-flag converter wait on no other CTA, only
// on their own bulk copies.
// Every wait is bounded by kWaitLimitNs; one that runs out latches
// kErrTimeout and publishes what it has, so no other CTA waits forever.
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
constexpr int kMidTiles = 2;     // most tiles a medium segment may span (seg_mid's slab)
constexpr int kGroupBatch = 8;   // small-segment groups per ticket of seg_main
constexpr int kMaxGroupBatch = 32;

struct SegHeader {      // lives at the start of the segmented workspace
    uint32_t ticket;    // seg_main's group-batch tickets (reset by the planner)
    uint32_t error;     // latched error bits
    uint32_t num_mids;  // medium segments this call
    uint32_t num_runs;  // large-segment runs this call
    uint32_t ticket4;   // seg_mid's segment tickets (reset by the planner)
    uint32_t plan_done; // planner CTA ticket
    uint64_t num_segs;  // S (written by the flags converter for the head-flag form)
    uint32_t reserved2;
    uint32_t reserved3;
    uint32_t flags_done;    // finished chunks of the flags converter (reset by its last CTA)
    uint32_t reserved4;
    uint32_t num_groups;    // small-segment groups this call
    uint32_t ticket2;       // run-scatter ticket counter (reset by the planner)
    uint32_t ticket3;       // run-count ticket counter (reset by the planner)
    uint32_t pad[1];
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
    uint32_t* run_cnt;         // [max_runs][M] class counts of each run
    uint32_t* run_base;        // [max_runs][M] output position of each run's first element per class
    uint32_t plan_blocks;
    uint32_t max_runs;         // capacity (enough for segments that tile [0, n))
    uint32_t max_groups;
    int use_tma;               // the tensor map passed to seg_run_scatter is valid
    const uint32_t* seg_m;     // per-segment class counts (remainder discriminator), or null:
                               // every segment uses the launch's discriminator
    uint32_t m_bound;          // classes of any segment are < m_bound (per-segment m clamped)
    uint32_t run_tiles;        // tiles per run of a large segment
    uint32_t group_batch;      // small-segment groups per work item
    uint32_t mid_tiles;        // a segment of more than one tile that spans at most this
                               // many row-aligned tiles is medium (0: none are)
    uint32_t* mid_loc;         // [S] block-local exclusive medium-segment offsets
    uint32_t* blk_mids;        // [plan blocks] medium-segment totals, then offsets
    uint32_t* mids;            // [max_mids] the medium segments, in order
    uint32_t max_mids;
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

// Small segments are grouped: a group is a run of consecutive small segments
// whose first elements lie in one window of P elements, cut after at most
// kGroupSegs segments, so a group spans < 2P elements.
constexpr uint32_t kGroupSegs = 128;
template <int P>
__host__ __device__ constexpr uint64_t group_window() {
    return static_cast<uint64_t>(P);
}
template <int P>
__device__ __forceinline__ bool group_head(const SegArgs& a, uint64_t s, uint64_t a0) {
    constexpr uint64_t GW = group_window<P>();
    return s == 0 || a.offsets[s - 1] / GW != a0 / GW || (s % kGroupSegs) == 0;
}

// A segment's tiles start at the 128-byte row holding its first element (a
// tile is P * sizeof(V) = 16 KB, so a row is P / 128 elements): the TMA box
// needs a row start, and tiles counted from there leave only the last one
// short.
template <int P>
__device__ __forceinline__ uint64_t seg_row_start(uint64_t a0) {
    return a0 & ~(static_cast<uint64_t>(P) / 128u - 1u);
}
template <int P>
__device__ __forceinline__ uint32_t seg_tiles(uint64_t a0, uint64_t a1) {
    return static_cast<uint32_t>((a1 - seg_row_start<P>(a0) + P - 1u) / P);
}

// A segment [a0, a1) longer than one tile is medium when its tiles number at
// most mid_tiles: seg_mid then reads it once.  The longer ones are cut into
// runs of run_tiles of those tiles (every run but the last is whole tiles).
template <int P>
__device__ __forceinline__ bool is_mid(const SegArgs& a, uint64_t a0, uint64_t a1) {
    return a.mid_tiles > 0u && seg_tiles<P>(a0, a1) <= a.mid_tiles;
}

__device__ __forceinline__ uint64_t seg_count(const SegArgs& a) {
    return a.num_segs == kSegsOnDevice ? a.hdr->num_segs : a.num_segs;
}

// --------------------------------------------------------------- planning --
// Block b of the planner owns segments [b*R, min((b+1)*R, S)), R = ceil(S/G).
template <int P, int THREADS>
__global__ void __launch_bounds__(THREADS) seg_plan_spans(SegArgs a) {
    constexpr int W = THREADS / 32;
    __shared__ uint32_t warp_runs[W], warp_grps[W], warp_mids[W];
    __shared__ int am_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t S = seg_count(a);
    const uint64_t G = gridDim.x;
    const uint64_t R = (S + G - 1) / G;
    const uint64_t s0 = blockIdx.x * R, s1 = min(s0 + R, S);
    uint32_t carry_r = 0, carry_g = 0, carry_m = 0;
    for (uint64_t base = s0; base < s1; base += THREADS) {
        const uint64_t s = base + tid;
        uint32_t runs = 0, head = 0, mid = 0;
        if (s < s1) {
            const uint64_t a0 = a.offsets[s], a1 = a.offsets[s + 1];
            if (a1 < a0 || a1 > a.n || (s == 0 && a0 != 0) || (s + 1 == S && a1 != a.n)) {
                atomicOr(&a.hdr->error, kErrSegments);
            } else if (a1 - a0 > static_cast<uint64_t>(P)) {
                if (is_mid<P>(a, a0, a1)) {
                    mid = 1;
                } else {
                    runs = (seg_tiles<P>(a0, a1) + a.run_tiles - 1) / a.run_tiles;
                }
            } else {
                head = group_head<P>(a, s, a0) ? 1u : 0u;
            }
            if (a.in_flags != nullptr && a1 > a0 && a1 <= a.n &&
                static_cast<uint64_t>(a.in_flags[a0]) != a1 - a0)
                atomicOr(&a.hdr->error, kErrSegments);
            if (a.seg_m != nullptr && (a.seg_m[s] < 1u || a.seg_m[s] > a.m_bound))
                atomicOr(&a.hdr->error, kErrSegments);
        }
        const uint32_t ir = warp_incl_scan(runs);
        const uint32_t ig = warp_incl_scan(head);
        const uint32_t im = warp_incl_scan(mid);
        if (lane == 31) {
            warp_runs[warp] = ir;
            warp_grps[warp] = ig;
            warp_mids[warp] = im;
        }
        __syncthreads();
        uint32_t pr = 0, pg = 0, pm = 0, tr = 0, tg = 0, tm = 0;
        for (int w = 0; w < W; w++) {
            const uint32_t xr = warp_runs[w], xg = warp_grps[w], xm = warp_mids[w];
            pr += (w < warp) ? xr : 0u;
            pg += (w < warp) ? xg : 0u;
            pm += (w < warp) ? xm : 0u;
            tr += xr;
            tg += xg;
            tm += xm;
        }
        if (s < s1) {
            a.run_loc[s] = carry_r + pr + ir - runs;
            a.grp_loc[s] = carry_g + pg + ig - head;
            a.mid_loc[s] = carry_m + pm + im - mid;
        }
        carry_r += tr;
        carry_g += tg;
        carry_m += tm;
        __syncthreads();
    }
    if (tid == 0) {
        a.blk_runs[blockIdx.x] = carry_r;
        a.blk_grps[blockIdx.x] = carry_g;
        a.blk_mids[blockIdx.x] = carry_m;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) am_last = (atomicAdd(&a.hdr->plan_done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    // last CTA: exclusive scans of the block totals (in place)
    if (warp < 3) {
        uint32_t* arr = warp == 0 ? a.blk_runs : warp == 1 ? a.blk_grps : a.blk_mids;
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
            } else if (warp == 1) {
                a.hdr->num_groups = run <= a.max_groups ? run : 0u;
            } else {
                a.hdr->num_mids = run <= a.max_mids ? run : 0u;
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        a.hdr->ticket = 0u;
        a.hdr->ticket2 = 0u;
        a.hdr->ticket3 = 0u;
        a.hdr->ticket4 = 0u;
        a.hdr->plan_done = 0u;
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
    const uint32_t moff = a.blk_mids[blockIdx.x];
    const uint32_t num_runs = a.hdr->num_runs, num_groups = a.hdr->num_groups;
    const uint32_t num_mids = a.hdr->num_mids;
    for (uint64_t base = s0; base < s1; base += THREADS) {
        if (tid == 0) list_n = 0;
        __syncthreads();
        const uint64_t s = base + tid;
        if (s < s1) {
            const uint64_t a0 = a.offsets[s], a1 = a.offsets[s + 1];
            if (a1 >= a0 && a1 <= a.n) {
                if (a1 - a0 > static_cast<uint64_t>(P) && is_mid<P>(a, a0, a1)) {
                    const uint32_t pos = moff + a.mid_loc[s];
                    if (pos < num_mids) a.mids[pos] = static_cast<uint32_t>(s);
                } else if (a1 - a0 > static_cast<uint64_t>(P)) {
                    const uint32_t nr = (seg_tiles<P>(a0, a1) + a.run_tiles - 1) / a.run_tiles;
                    const uint32_t pos = roff + a.run_loc[s];
                    if (nr <= 16) {  // this thread emits the runs itself
                        if (static_cast<uint64_t>(pos) + nr <= num_runs) {
                            const uint64_t rb = seg_row_start<P>(a0);
                            const uint64_t len = static_cast<uint64_t>(a.run_tiles) * P;
                            for (uint32_t r = 0; r < nr; r++) {
                                RunEntry e;
                                e.seg = static_cast<uint32_t>(s);
                                e.p0 = static_cast<uint32_t>(max(a0, rb + r * len));
                                e.p1 = static_cast<uint32_t>(min(a1, rb + (r + 1) * len));
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
                } else if (group_head<P>(a, s, a0)) {
                    const uint32_t g = goff + a.grp_loc[s];
                    if (g < num_groups) a.groups[g] = static_cast<uint32_t>(s);
                }
            }
            // the group before segment s ends at s at the latest when s starts
            // a group, is large or is malformed
            const bool small_ok = (a1 >= a0 && a1 <= a.n && a1 - a0 <= static_cast<uint64_t>(P));
            const bool is_head = small_ok && group_head<P>(a, s, a0);
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
            const uint64_t rb = seg_row_start<P>(a0);
            const uint64_t len = static_cast<uint64_t>(a.run_tiles) * P;
            for (uint32_t r = tid; r < nr; r += THREADS) {
                RunEntry e;
                e.seg = seg;
                e.p0 = static_cast<uint32_t>(max(a0, rb + r * len));
                e.p1 = static_cast<uint32_t>(min(a1, rb + (r + 1) * len));
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
    // small groups (segments starting in one window of P, each <= P): an
    // input buffer and an output image, each for a range of < 2P elements plus
    // 16-byte alignment slack (the next group's copy overlaps the current
    // group's write-out; the other resident CTAs cover the rest of its latency)
    static constexpr int kGroupElems =
        static_cast<int>(group_window<kTile>()) + kTile + 2 * static_cast<int>(kAU);
    static constexpr size_t kGroupBytes = 2ull * kGroupElems * sizeof(V);
    static constexpr size_t kBytes = 128 + kGroupBytes;  // seg_main
    // seg_run_scatter: TMA ring + tile stage + count matrix
    static constexpr size_t kRingBytes = static_cast<size_t>(STAGES) * kTile * sizeof(V);
    static constexpr size_t kRunBytes = 1024 + kRingBytes + G::kStageBytes + G::kCntBytes;
};

// Per-thread class counters in 16-bit fields (M <= 16: (M+1)/2 words), wide
// enough for any count within one group (< 2P < 2^16 elements).
template <int M>
struct HalfCounts {
    static constexpr int NW = (M + 1) / 2;
    uint32_t w[NW];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int q = 0; q < NW; q++) w[q] = 0;
    }
    __device__ __forceinline__ uint32_t get(uint32_t c) const {
        if constexpr (NW == 2) {  // four fields: one 64-bit shift
            const uint64_t x = (static_cast<uint64_t>(w[1]) << 32) | w[0];
            return static_cast<uint32_t>(x >> (c << 4)) & 0xffffu;
        } else if constexpr (NW == 4) {  // eight fields: two 64-bit halves
            const uint64_t lo = (static_cast<uint64_t>(w[1]) << 32) | w[0];
            const uint64_t hi = (static_cast<uint64_t>(w[3]) << 32) | w[2];
            return static_cast<uint32_t>(((c & 4u) ? hi : lo) >> ((c & 3u) << 4)) & 0xffffu;
        } else if constexpr (NW == 8) {  // sixteen fields: four 64-bit quarters
            uint64_t x = (static_cast<uint64_t>(w[1]) << 32) | w[0];
#pragma unroll
            for (int q = 1; q < 4; q++)
                x = (c >> 2) == static_cast<uint32_t>(q)
                        ? (static_cast<uint64_t>(w[2 * q + 1]) << 32) | w[2 * q]
                        : x;
            return static_cast<uint32_t>(x >> ((c & 3u) << 4)) & 0xffffu;
        } else {
            uint32_t x = w[0];
#pragma unroll
            for (int q = 1; q < NW; q++) x = (c >> 1) == static_cast<uint32_t>(q) ? w[q] : x;
            return (x >> ((c & 1u) << 4)) & 0xffffu;
        }
    }
    __device__ __forceinline__ void inc(uint32_t c) {
        if constexpr (NW == 2) {
            uint64_t x = (static_cast<uint64_t>(w[1]) << 32) | w[0];
            x += 1ull << (c << 4);
            w[0] = static_cast<uint32_t>(x);
            w[1] = static_cast<uint32_t>(x >> 32);
        } else if constexpr (NW == 4) {
            uint64_t lo = (static_cast<uint64_t>(w[1]) << 32) | w[0];
            uint64_t hi = (static_cast<uint64_t>(w[3]) << 32) | w[2];
            const uint64_t one = 1ull << ((c & 3u) << 4);
            if (c & 4u) hi += one; else lo += one;
            w[0] = static_cast<uint32_t>(lo);
            w[1] = static_cast<uint32_t>(lo >> 32);
            w[2] = static_cast<uint32_t>(hi);
            w[3] = static_cast<uint32_t>(hi >> 32);
        } else if constexpr (NW == 8) {
            const uint64_t one = 1ull << ((c & 3u) << 4);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint64_t x = (static_cast<uint64_t>(w[2 * q + 1]) << 32) | w[2 * q];
                if ((c >> 2) == static_cast<uint32_t>(q)) x += one;
                w[2 * q] = static_cast<uint32_t>(x);
                w[2 * q + 1] = static_cast<uint32_t>(x >> 32);
            }
        } else {
            const uint32_t one = 1u << ((c & 1u) << 4);
#pragma unroll
            for (int q = 0; q < NW; q++) w[q] += (c >> 1) == static_cast<uint32_t>(q) ? one : 0u;
        }
    }
};

// Shared state of one group partition (at most kGroupSegs non-empty
// segments).
template <int M, int THREADS>
struct GroupScratch {
    static constexpr int NW = HalfCounts<M>::NW;
    uint32_t base[kGroupSegs][NW];  // class bases of each non-empty segment (u16 pairs)
    uint32_t wagg[THREADS / 32][NW + 1];
    uint16_t hpos[kGroupSegs + 1];  // head of each non-empty segment in the group; [nseg] = L
    uint16_t sidx[kGroupSegs];      // its index - h
    uint8_t msz[kGroupSegs];        // its class count (per-segment m)
};

// Offsets (and class count) of segment h + threadIdx.x of the next group,
// loaded by each thread while the current group is partitioned.
struct GroupPrefetch {
    uint64_t o0, o1;
    uint32_t m;
    bool valid;
};

// The discriminator of a group's segment with class count m: per-segment
// remainders use the precomputed constants cmod[m] (DiscrMod::make).
template <class D>
__device__ __forceinline__ D group_discr(const SegArgs& a, const D& d, const uint64_t* cmod,
                                         uint32_t m) {
    if constexpr (std::is_same<D, DiscrMod>::value) {
        if (a.seg_m != nullptr) {
            DiscrMod x;
            x.m = min(m, 16u);
            x.c = cmod[x.m];
            return x;
        }
    }
    return d;
}

// One CTA partitions one group of small segments held in shared memory
// (element x of the group at src[x], 0 <= x < L) into the output image
// dst[0 .. L) and writes the segments' sizes.  Every thread owns k = ~L/256
// consecutive elements whatever the segment lengths (k odd: the threads'
// strided shared-memory reads fall in different banks):
//   P0  one thread per segment: ordinals of the non-empty segments and their
//       heads; each thread finds the segment holding its first element by a
//       binary search over the heads;
//   P1  the class counts of the fragment after the thread's last segment
//       head; a segment that begins and ends inside the thread's range is
//       closed here (its class bases to shared memory, its sizes and head
//       flags to global memory);
//   P2  a segmented exclusive scan of those counts over the threads gives the
//       counts of the thread's first segment before its first element;
//   P3  the thread's first segment, if it ends in the thread's range, is
//       closed with the scanned counts plus its part in the range;
//   P4  every element goes to head + base[class] + its rank in the segment.
template <class V, class D, int M, int THREADS>
__device__ void seg_group_cta(const SegArgs& a, const D& d, const uint64_t* cmod, uint32_t h,
                              uint32_t he, uint64_t r0, uint32_t L, const V* src, V* dst,
                              GroupScratch<M, THREADS>& gs, GroupPrefetch& pf,
                              const uint32_t* next_h, const uint32_t* next_he) {
    using HC = HalfCounts<M>;
    constexpr int NW = HC::NW;
    constexpr int W = THREADS / 32;
    static_assert(static_cast<int>(kGroupSegs) <= THREADS, "one thread per segment");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t k = ((L + THREADS - 1) / THREADS) | 1u;
    const uint32_t lo = min(tid * k, L), hi = min(lo + k, L);

    // ---- P0
    const uint64_t sg = static_cast<uint64_t>(h) + tid;
    uint32_t ne = 0, x0 = 0, x1 = 0, ms = a.m;
    if (sg < he && tid < static_cast<int>(kGroupSegs)) {
        uint64_t o0, o1;
        if (pf.valid) {
            o0 = pf.o0;
            o1 = pf.o1;
            ms = pf.m;
        } else {
            o0 = a.offsets[sg];
            o1 = a.offsets[sg + 1];
            if (a.seg_m != nullptr) ms = min(max(a.seg_m[sg], 1u), a.m_bound);
        }
        x0 = static_cast<uint32_t>(o0 - r0);
        x1 = static_cast<uint32_t>(o1 - r0);
        ne = (o1 > o0 && o0 >= r0 && x1 <= L) ? 1u : 0u;
        if (o1 == o0 && a.seg_sizes != nullptr)
            for (uint32_t c = 0; c < a.m; c++) a.seg_sizes[sg * a.m + c] = 0u;
    }
    const uint32_t incl = warp_incl_scan(ne);
    if (lane == 31) gs.wagg[warp][0] = incl;
    __syncthreads();
    // the next group's head and end are visible now: start its loads
    pf.valid = next_h != nullptr;
    if (pf.valid) {
        const uint64_t ns = static_cast<uint64_t>(*next_h) + tid;
        pf.m = a.m;
        if (ns < *next_he && tid < static_cast<int>(kGroupSegs)) {
            pf.o0 = a.offsets[ns];
            pf.o1 = a.offsets[ns + 1];
            if (a.seg_m != nullptr) pf.m = min(max(a.seg_m[ns], 1u), a.m_bound);
        }
    }
    uint32_t before = 0, nseg = 0;
#pragma unroll
    for (int w = 0; w < W; w++) {
        const uint32_t x = gs.wagg[w][0];
        before += w < warp ? x : 0u;
        nseg += x;
    }
    if (ne) {
        const uint32_t q = before + incl - 1u;
        gs.hpos[q] = static_cast<uint16_t>(x0);
        gs.sidx[q] = static_cast<uint16_t>(tid);
        gs.msz[q] = static_cast<uint8_t>(ms);
    }
    if (tid == 0) gs.hpos[nseg] = static_cast<uint16_t>(L);
    __syncthreads();

    // ---- P1
    const bool active = lo < hi && nseg > 0;
    uint32_t q0 = 0;  // the last non-empty segment with head <= lo (hpos[nseg] = L > lo)
    if (active) {
        uint32_t qb = nseg;
        while (qb - q0 > 1u) {
            const uint32_t mid = (q0 + qb) >> 1;
            if (gs.hpos[mid] <= lo) q0 = mid; else qb = mid;
        }
    }
    const bool head_at_lo = active && gs.hpos[q0] == lo;
    const D d0 = active ? group_discr(a, d, cmod, gs.msz[q0]) : d;
    // segment qq ends here with class totals `tot`: its class bases (shared),
    // sizes and head flags (global)
    auto close = [&](uint32_t qq, const HC& tot) {
        const uint64_t s = static_cast<uint64_t>(h) + gs.sidx[qq];
        const uint64_t xh = r0 + gs.hpos[qq];
        uint32_t off = 0;
        uint32_t bw[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) bw[w] = 0;
#pragma unroll
        for (int c = 0; c < M; c++) {
            const uint32_t t = tot.get(c);
            bw[c >> 1] |= off << (16 * (c & 1));
            if (a.seg_sizes != nullptr && static_cast<uint32_t>(c) < a.m) a.seg_sizes[s * a.m + c] = t;
            if (a.headflags != nullptr && t > 0) a.headflags[xh + off] = t;
            off += t;
        }
#pragma unroll
        for (int w = 0; w < NW; w++) gs.base[qq][w] = bw[w];
    };
    // the counts of the fragment after the last head in (lo, hi) (all of the
    // range without one); segments that begin and end inside the range are
    // closed on the way, the first segment's part is kept for after the scan
    HC tail, pre;
    tail.zero();
    pre.zero();
    bool inner = false;  // a segment head in (lo, hi)
    if (active) {
        uint32_t q = q0, nxt = gs.hpos[q0 + 1];
        D dc = d0;
        for (uint32_t x = lo; x < hi; x++) {
            if (x == nxt) {
                if (inner) close(q, tail);
                else pre = tail;
                inner = true;
                tail.zero();
                q++;
                nxt = gs.hpos[q + 1];
                dc = group_discr(a, d, cmod, gs.msz[q]);
            }
            tail.inc(dc(src[x]));
        }
        if (inner && hi == nxt) close(q, tail);
        if (!inner) pre = tail;
    }

    // ---- P2: segmented exclusive scan of (reset, counts) over the threads
    uint32_t f = (head_at_lo || inner) ? 1u : 0u;
    HC v = tail;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        const uint32_t fu = __shfl_up_sync(0xffffffffu, f, dd);
        HC vu;
#pragma unroll
        for (int w = 0; w < NW; w++) vu.w[w] = __shfl_up_sync(0xffffffffu, v.w[w], dd);
        if (lane >= dd) {
            if (!f) {
#pragma unroll
                for (int w = 0; w < NW; w++) v.w[w] += vu.w[w];
            }
            f |= fu;
        }
    }
    if (lane == 31) {
        gs.wagg[warp][0] = f;
#pragma unroll
        for (int w = 0; w < NW; w++) gs.wagg[warp][1 + w] = v.w[w];
    }
    const uint32_t fe = __shfl_up_sync(0xffffffffu, f, 1);
    HC ve;
#pragma unroll
    for (int w = 0; w < NW; w++) ve.w[w] = __shfl_up_sync(0xffffffffu, v.w[w], 1);
    __syncthreads();
    HC carry;
    carry.zero();
    for (int w = 0; w < warp; w++) {
        const bool fw = gs.wagg[w][0] != 0u;
#pragma unroll
        for (int q = 0; q < NW; q++) carry.w[q] = (fw ? 0u : carry.w[q]) + gs.wagg[w][1 + q];
    }
    if (lane > 0) {
#pragma unroll
        for (int q = 0; q < NW; q++) carry.w[q] = (fe ? 0u : carry.w[q]) + ve.w[q];
    }
    if (head_at_lo) carry.zero();

    // ---- P3: the first segment ends at the first head inside, or exactly at hi
    if (active) {
        const bool ends = inner || hi == gs.hpos[q0 + 1];
        if (ends) {
            HC t;
#pragma unroll
            for (int w = 0; w < NW; w++) t.w[w] = carry.w[w] + pre.w[w];
            close(q0, t);
        }
    }
    __syncthreads();

    // ---- P4: positions = head + class base + rank in the segment (packed per class)
    if (active) {
        uint32_t q = q0, nxt = gs.hpos[q0 + 1], xh = gs.hpos[q0];
        HC cur;
#pragma unroll
        for (int w = 0; w < NW; w++) cur.w[w] = gs.base[q0][w] + carry.w[w];
        D dc = d0;
        for (uint32_t x = lo; x < hi; x++) {
            if (x == nxt) {
                q++;
                xh = x;
                nxt = gs.hpos[q + 1];
#pragma unroll
                for (int w = 0; w < NW; w++) cur.w[w] = gs.base[q][w];
                dc = group_discr(a, d, cmod, gs.msz[q]);
            }
            const V v = src[x];
            const uint32_t c = dc(v);
            const uint32_t pos = xh + cur.get(c);
            cur.inc(c);
            if (pos < L) dst[pos] = v;
        }
    }
}

template <class V, class D, int M, int THREADS, int STAGES>
__global__ void __launch_bounds__(THREADS, 3)
    seg_main(SegArgs a, D d) {
    using L = SegSmem<V, M, THREADS, STAGES>;
    constexpr uint32_t AU = L::kAU;
    static_assert(M <= 16 && M >= 2, "class bound");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* base = smem_raw + (((raw + 127u) & ~127u) - raw);
    V* g_in0 = reinterpret_cast<V*>(base);
    V* g_out = g_in0 + L::kGroupElems;

    __shared__ __align__(8) uint64_t gbars[2];
    __shared__ uint32_t ticket_sh[2];
    __shared__ uint32_t gi_h[2], gi_he[2];  // group pipeline slots
    __shared__ uint64_t gi_r0[2], gi_r1[2], gi_as[2], gi_tail[2];
    __shared__ GroupScratch<M, THREADS> gs;
    __shared__ uint32_t gb_h[kMaxGroupBatch], gb_he[kMaxGroupBatch];  // the batch's groups
    __shared__ uint64_t gb_r0[kMaxGroupBatch], gb_r1[kMaxGroupBatch];
    __shared__ uint64_t cmod[17];  // DiscrMod constants for m = 1 .. 16

    const int tid = threadIdx.x;
    const V* in = static_cast<const V*>(a.in);
    V* out = static_cast<V*>(a.out);
    const uint32_t out_phase =
        static_cast<uint32_t>(reinterpret_cast<uintptr_t>(out) / sizeof(V)) & (AU - 1u);
    const bool in_vec = (reinterpret_cast<uintptr_t>(in) & 15u) == 0;
    const bool out_vec = (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
    const uint64_t S = seg_count(a);
    const uint32_t num_groups = a.hdr->num_groups;
    // groups per ticket: the tuned batch, but no more than spreads the groups
    // over every CTA (a few groups must not queue up on one CTA)
    const uint32_t batch =
        max(1u, min(a.group_batch, (num_groups + gridDim.x - 1) / gridDim.x));
    const uint32_t num_batches = (num_groups + batch - 1) / batch;
    const uint32_t total = num_batches;
    uint32_t group_uses = 0;

    if (tid == 0) {
        mbar_init(&gbars[0], 1);
        mbar_init(&gbars[1], 1);
        mbar_fence_init();
    }
    if (tid >= 1 && tid <= 16) cmod[tid] = DiscrMod::make(static_cast<uint32_t>(tid)).c;
    if (tid == 0) cmod[0] = 0;
    __syncthreads();

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
            const uint32_t g0 = t * batch;
            const uint32_t gcnt = min(batch, num_groups - g0);
            // the batch's group heads, ends and element ranges, loaded once
            if (tid < static_cast<int>(gcnt)) {
                const uint32_t h = a.groups[g0 + tid];
                const uint32_t he =
                    static_cast<uint32_t>(min(static_cast<uint64_t>(a.groups_end[g0 + tid]), S));
                gb_h[tid] = h;
                gb_he[tid] = he;
                gb_r0[tid] = a.offsets[h];
                gb_r1[tid] = a.offsets[he];
            }
            __syncthreads();
            auto issue_group = [&](uint32_t i) {  // thread 0 only
                const uint32_t slot = (group_uses + i) & 1u;
                const uint32_t h = gb_h[i], he = gb_he[i];
                const uint64_t r0 = gb_r0[i], r1 = gb_r1[i];
                const uint64_t as = r0 & ~static_cast<uint64_t>(AU - 1u);
                uint64_t ve = min((r1 + AU - 1u) & ~static_cast<uint64_t>(AU - 1u),
                                  a.n & ~static_cast<uint64_t>(AU - 1u));
                if (!in_vec || ve < as) ve = as;
                gi_h[slot] = h;
                gi_he[slot] = he;
                gi_r0[slot] = r0;
                gi_r1[slot] = r1;
                gi_as[slot] = as;
                gi_tail[slot] = max(ve, r0);
                V* dst = g_in0;
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
            GroupPrefetch pf;
            pf.valid = false;
            for (uint32_t i = 0; i < gcnt; i++) {
                const uint32_t use = group_uses + i;
                const uint32_t slot = use & 1u;
                const bool ok = mbar_wait_bounded(&gbars[slot], (use >> 1) & 1u);
                __syncthreads();  // slot info visible
                V* gin = g_in0;
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
                const bool more = i + 1 < gcnt;
                seg_group_cta<V, D, M, THREADS>(
                    a, d, cmod, gi_h[slot], gi_he[slot], r0, static_cast<uint32_t>(r1 - r0),
                    gin + (r0 - as), g_out + (r0 - as), gs, pf, more ? &gb_h[i + 1] : nullptr,
                    more ? &gb_he[i + 1] : nullptr);
                // every read of the input buffer precedes the next group's copy
                fence_proxy_async_smem();
                __syncthreads();
                if (tid == 0 && more) issue_group(i + 1);
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
    }
}

// Class counts of every run of the large segments: one CTA per run (run
// tickets), 16-byte loads four deep per thread, per-thread packed counters,
// warp reductions and one barrier per run.  A few hundred bytes of shared
// memory, so more CTAs per SM than the group kernel keep loads in flight.
template <class V, class D, int M, int THREADS>
__global__ void __launch_bounds__(THREADS, 4) seg_run_count(SegArgs a, D d) {
    constexpr uint32_t AU = 16 / sizeof(V);
    constexpr int W = THREADS / 32;
    __shared__ uint32_t red[W][M];
    __shared__ uint32_t ticket_sh[2];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const V* in = static_cast<const V*>(a.in);
    const bool in_vec = (reinterpret_cast<uintptr_t>(in) & 15u) == 0;
    const uint32_t num_runs = a.hdr->num_runs;
    for (uint32_t it = 0;; it++) {
        if (tid == 0) ticket_sh[it & 1u] = atomicAdd(&a.hdr->ticket3, 1u);
        __syncthreads();
        const uint32_t j = ticket_sh[it & 1u];
        if (j >= num_runs) break;
        const RunEntry ent = a.runs[j];
        const D dj = seg_discr(a, d, ent.seg);
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
        if (tid < static_cast<uint32_t>(M)) {
            uint32_t agg = 0;
#pragma unroll
            for (int w = 0; w < W; w++) agg += red[w][tid];
            a.run_cnt[static_cast<uint64_t>(j) * M + tid] = agg;
        }
    }
}

// One large segment's runs [j, jl]: lane l takes a contiguous share of the
// runs, class counts in registers; warp scans per class give each run's
// output position per class, the segment's sizes and head flags.
template <int M>
__device__ __forceinline__ void scan_segment_runs(const SegArgs& a, uint32_t j, uint32_t jl,
                                                  uint32_t seg, uint32_t seg_start) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t R = jl - j + 1u;
    const uint32_t per = (R + 31u) >> 5;
    const uint32_t rb = j + min(lane * per, R), re = j + min(lane * per + per, R);
    uint32_t acc[M];
#pragma unroll
    for (int c = 0; c < M; c++) acc[c] = 0;
    for (uint32_t r = rb; r < re; r++) {
        const uint32_t* row = a.run_cnt + static_cast<uint64_t>(r) * M;
#pragma unroll
        for (int c = 0; c < M; c++) acc[c] += __ldcg(row + c);
    }
    uint32_t cur[M];
    uint32_t off = seg_start;
#pragma unroll
    for (int c = 0; c < M; c++) {
        const uint32_t incl = warp_incl_scan(acc[c]);
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        cur[c] = off + incl - acc[c];
        if (lane == static_cast<uint32_t>(c)) {
            if (a.seg_sizes != nullptr && static_cast<uint32_t>(c) < a.m)
                a.seg_sizes[static_cast<uint64_t>(seg) * a.m + c] = tot;
            if (a.headflags != nullptr && tot > 0) a.headflags[off] = tot;
        }
        off += tot;
    }
    for (uint32_t r = rb; r < re; r++) {
        const uint32_t* row = a.run_cnt + static_cast<uint64_t>(r) * M;
        uint32_t* dst = a.run_base + static_cast<uint64_t>(r) * M;
#pragma unroll
        for (int c = 0; c < M; c++) {
            const uint32_t x = __ldcg(row + c);
            dst[c] = cur[c];
            cur[c] += x;
        }
    }
}

// One large segment with few runs [j, jl], by one lane alone.
template <int M>
__device__ __forceinline__ void scan_segment_runs_lane(const SegArgs& a, uint32_t j, uint32_t jl,
                                                       uint32_t seg, uint32_t seg_start) {
    uint32_t tot[M];
#pragma unroll
    for (int c = 0; c < M; c++) tot[c] = 0;
    for (uint32_t r = j; r <= jl; r++) {
        const uint32_t* row = a.run_cnt + static_cast<uint64_t>(r) * M;
#pragma unroll
        for (int c = 0; c < M; c++) tot[c] += __ldcg(row + c);
    }
    uint32_t cur[M];
    uint32_t off = seg_start;
#pragma unroll
    for (int c = 0; c < M; c++) {
        cur[c] = off;
        if (a.seg_sizes != nullptr && static_cast<uint32_t>(c) < a.m)
            a.seg_sizes[static_cast<uint64_t>(seg) * a.m + c] = tot[c];
        if (a.headflags != nullptr && tot[c] > 0) a.headflags[off] = tot[c];
        off += tot[c];
    }
    for (uint32_t r = j; r <= jl; r++) {
        const uint32_t* row = a.run_cnt + static_cast<uint64_t>(r) * M;
        uint32_t* dst = a.run_base + static_cast<uint64_t>(r) * M;
#pragma unroll
        for (int c = 0; c < M; c++) {
            const uint32_t x = __ldcg(row + c);
            dst[c] = cur[c];
            cur[c] += x;
        }
    }
}

// Every warp looks at 32 consecutive runs at a time: the lane holding a
// segment's first run scans a segment of at most 4 runs by itself, the whole
// warp takes the longer ones in turn.
template <int M>
__global__ void __launch_bounds__(256) seg_run_scan(SegArgs a) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t num_runs = a.hdr->num_runs;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t j0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32u; j0 < num_runs;
         j0 += warps * 32u) {
        const uint32_t j = j0 + lane;
        RunEntry e{};
        bool first = false;
        if (j < num_runs) {
            e = a.runs[j];
            first = e.p0 == static_cast<uint32_t>(a.offsets[e.seg]);
        }
        const uint32_t jl = min(e.jlast, num_runs - 1u);
        const bool shortseg = first && jl >= j && jl - j < 4u;
        if (shortseg) scan_segment_runs_lane<M>(a, j, jl, e.seg, e.p0);
        uint32_t longs = __ballot_sync(0xffffffffu, first && !shortseg);
        while (longs != 0u) {
            const int l = __ffs(longs) - 1;
            longs &= longs - 1u;
            const uint32_t jll = __shfl_sync(0xffffffffu, jl, l);
            const uint32_t seg = __shfl_sync(0xffffffffu, e.seg, l);
            const uint32_t p0 = __shfl_sync(0xffffffffu, e.p0, l);
            if (jll >= j0 + l) scan_segment_runs<M>(a, j0 + l, jll, seg, p0);
        }
    }
}

// Every run of a large segment through the TMA ring and tile_scatter, from
// the run_base positions.  Runs are taken in reverse order of the counts, so
// the first re-reads find the runs counted last still in L2.
template <class V, class D, int M, int THREADS, int STAGES>
__global__ void __launch_bounds__(THREADS, 4)  // 4 CTAs (32 warps) per SM: <= 64 registers
    seg_run_scatter(SegArgs a, D d, const __grid_constant__ CUtensorMap tmap) {
    using L = SegSmem<V, M, THREADS, STAGES>;
    using TG = typename L::G;
    constexpr int ITEMS = TG::kItems;
    constexpr int P = L::kTile;
    constexpr int ROWS = TG::kRows;
    constexpr uint32_t AU = L::kAU;
    static_assert(M <= 16 && M >= 2, "class bound");
    static_assert(ROWS <= 256, "TMA box height");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    V* ring = reinterpret_cast<V*>(base);
    V* stage = reinterpret_cast<V*>(base + L::kRingBytes);
    uint16_t* cnt_sm = reinterpret_cast<uint16_t*>(base + L::kRingBytes + TG::kStageBytes);

    __shared__ __align__(8) uint64_t bars[STAGES];
    __shared__ TileShared<M> sh;
    __shared__ uint32_t ticket_sh[2];

    const int tid = threadIdx.x;
    const V* in = static_cast<const V*>(a.in);
    V* out = static_cast<V*>(a.out);
    const uint32_t out_phase =
        static_cast<uint32_t>(reinterpret_cast<uintptr_t>(out) / sizeof(V)) & (AU - 1u);
    const bool tma_ok = a.use_tma != 0;
    constexpr uint32_t kPerRow = 128u / sizeof(V);  // elements per 128-byte row
    const uint64_t map_elems = (a.n * sizeof(V) / 128u) * kPerRow;
    const uint32_t num_runs = a.hdr->num_runs;
    uint32_t ring_uses = 0;  // mbarrier phase bookkeeping across runs

    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; s++) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    __syncthreads();

    for (uint32_t it = 0;; it++) {
        if (tid == 0) ticket_sh[it & 1u] = atomicAdd(&a.hdr->ticket2, 1u);
        __syncthreads();
        const uint32_t t = ticket_sh[it & 1u];
        if (t >= num_runs) break;
        const uint32_t j = num_runs - 1u - t;
        const RunEntry ent = a.runs[j];
        const D dj = seg_discr(a, d, ent.seg);
        if (tid < M) sh.cursor[0][tid] = __ldcg(a.run_base + static_cast<uint64_t>(j) * M + tid);
        __syncthreads();
        // the run's tiles start at the 128-byte row holding its first element
        // (not at multiples of P), so only its last tile is short
        const uint64_t rb = ent.p0 & ~static_cast<uint64_t>(kPerRow - 1u);
        const uint32_t ntiles = static_cast<uint32_t>((ent.p1 - rb + P - 1u) / P);
        // a tile comes by TMA when the run's part of it lies inside the tensor
        // map (the input's whole 128-byte rows; rows past the map read as zeros
        // and lie outside the run)
        auto via_tma = [&](uint32_t i) {
            return tma_ok && min(static_cast<uint64_t>(ent.p1), rb + static_cast<uint64_t>(i + 1) * P) <= map_elems;
        };
        auto issue = [&](uint32_t i) {  // tile i of the run into ring slot (ring_uses+i) % STAGES
            const uint32_t slot = (ring_uses + i) % STAGES;
            if (via_tma(i)) {
                mbar_arrive_expect_tx(&bars[slot], P * sizeof(V));
                tma_load_2d(ring + slot * P, &tmap, 0,
                            static_cast<int32_t>(rb / kPerRow + static_cast<uint64_t>(i) * ROWS), &bars[slot]);
            } else {
                mbar_arrive(&bars[slot]);
            }
        };
        if (tid == 0)
            for (uint32_t i = 0; i < STAGES && i < ntiles; i++) issue(i);
        const uint32_t e0 = tid * ITEMS;
        bool failed = false;
        for (uint32_t i = 0; i < ntiles; i++) {
            const uint64_t ts = rb + static_cast<uint64_t>(i) * P;
            const uint32_t lo = static_cast<uint32_t>(max(static_cast<uint64_t>(ent.p0), ts) - ts);
            const uint32_t hi = static_cast<uint32_t>(min(static_cast<uint64_t>(ent.p1), ts + P) - ts);
            const bool full = lo == 0u && hi == static_cast<uint32_t>(P);
            const uint32_t use = ring_uses + i;
            const bool ok = mbar_wait_bounded(&bars[use % STAGES], (use / STAGES) & 1u);
            V v[ITEMS];
            if (via_tma(i)) {
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
        if (failed) break;
    }
    if (tid < M) bulk_wait_all();
}

// ------------------------------------------------------- medium segments --
// A medium segment (more than one tile, at most mid_tiles <= KMAX row-aligned
// tiles) is read from HBM once: all its tiles come by TMA into a shared slab;
// a count pass over the slab gives the segment's class totals (its sizes, head
// flags and the class cursors at its start); tile_scatter then places the
// tiles from the slab in order with forward cursors, as the plain scatter
// does.  The run path reads the same elements twice (count, then scatter).
//
// CTA b takes the medium segments b, b + G, b + 2G, ... (G CTAs), so it knows
// its next segment in advance: the next segment's offsets are loaded during
// the current count pass, and its tiles are requested while the current
// segment is scattered -- a tile slot as soon as the current segment's tile
// in it has been taken into registers, the slots the current segment does not
// use at once.  The loads of one segment thus overlap the scatter of the one
// before.  A slab of two tiles keeps the kernel at four CTAs per SM (a slab of
// four at two CTAs per SM was slower: the tile step needs the occupancy).
//
// Measured (100,000 LogNormal(ln 1024, 1.5) segments, u32, m = 4): the
// segments of two tiles take 165 us here against 152 us less in the run
// kernels, so the single read does not pay for itself there -- the tile step,
// not the re-read, bounds those segments (a segment of ~1.5 tiles costs two
// tile steps either way).  It stays a tuned option (mid_tiles) and is off by
// default.
template <class V, int M, int THREADS, int KMAX>
struct MidSmem {
    using G = TileGeom<V, THREADS, M>;
    static constexpr size_t kSlabBytes = static_cast<size_t>(KMAX) * G::kTile * sizeof(V);
    static constexpr size_t kBytes = 1024 + kSlabBytes + G::kStageBytes + G::kCntBytes;
};

template <class V, class D, int M, int THREADS, int KMAX>
__global__ void __launch_bounds__(THREADS, 4)
    seg_mid(SegArgs a, D d, const __grid_constant__ CUtensorMap tmap) {
    using L = MidSmem<V, M, THREADS, KMAX>;
    using TG = typename L::G;
    constexpr int ITEMS = TG::kItems;
    constexpr int P = TG::kTile;
    constexpr int ROWS = TG::kRows;
    constexpr uint32_t AU = TG::kAU;
    constexpr int W = THREADS / 32;
    constexpr uint32_t kPerRow = 128u / sizeof(V);
    static_assert(M <= 16 && M >= 2, "class bound");
    static_assert(KMAX >= 2 && KMAX <= 32, "one phase bit per slab tile");
    static_assert(ROWS <= 256, "TMA box height");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    unsigned char* base = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    V* slab = reinterpret_cast<V*>(base);
    V* stage = reinterpret_cast<V*>(base + L::kSlabBytes);
    uint16_t* cnt_sm = reinterpret_cast<uint16_t*>(base + L::kSlabBytes + TG::kStageBytes);

    __shared__ __align__(8) uint64_t bars[KMAX];
    __shared__ TileShared<M> sh;
    __shared__ uint32_t red[W][M];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const V* in = static_cast<const V*>(a.in);
    V* out = static_cast<V*>(a.out);
    const uint32_t out_phase =
        static_cast<uint32_t>(reinterpret_cast<uintptr_t>(out) / sizeof(V)) & (AU - 1u);
    const bool tma_ok = a.use_tma != 0;
    const uint64_t map_elems = (a.n * sizeof(V) / 128u) * kPerRow;
    const uint32_t num_mids = a.hdr->num_mids;
    const uint32_t G = gridDim.x;
    const uint32_t e0 = tid * ITEMS;
    uint32_t parity = 0;  // bit i: the phase of bars[i] that completes next

    // A segment's element range and its tiles from the 128-byte row of a0 (at
    // most mid_tiles <= KMAX by the planner's classification).
    struct Seg {
        uint64_t a0, a1, rb;
        uint32_t s, ntiles;
    };
    auto make_seg = [&](uint32_t s, uint64_t a0, uint64_t a1) {
        Seg g;
        g.s = s;
        g.a0 = a0;
        g.a1 = a1;
        g.rb = a0 & ~static_cast<uint64_t>(kPerRow - 1u);
        g.ntiles = static_cast<uint32_t>(
            min((a1 - g.rb + P - 1u) / P, static_cast<uint64_t>(KMAX)));
        return g;
    };
    // a tile comes by TMA when the segment's part of it lies inside the
    // tensor map (the input's whole 128-byte rows; rows past the map read as
    // zeros and lie outside the segment)
    auto via_tma = [&](const Seg& g, uint32_t i) {
        return tma_ok && min(g.a1, g.rb + static_cast<uint64_t>(i + 1) * P) <= map_elems;
    };
    auto issue = [&](const Seg& g, uint32_t i) {  // tile i of g into slab slot i
        if (via_tma(g, i)) {
            mbar_arrive_expect_tx(&bars[i], P * sizeof(V));
            tma_load_2d(slab + static_cast<size_t>(i) * P, &tmap, 0,
                        static_cast<int32_t>(g.rb / kPerRow + static_cast<uint64_t>(i) * ROWS),
                        &bars[i]);
        } else {
            mbar_arrive(&bars[i]);
        }
    };
    auto range = [&](const Seg& g, uint32_t i, uint32_t& lo, uint32_t& hi) {
        const uint64_t ts = g.rb + static_cast<uint64_t>(i) * P;
        lo = static_cast<uint32_t>(max(g.a0, ts) - ts);
        hi = static_cast<uint32_t>(min(g.a1, ts + P) - ts);
    };
    auto take = [&](const Seg& g, uint32_t i, uint32_t lo, uint32_t hi, V (&v)[ITEMS]) {
        if (via_tma(g, i)) {
            take_swizzled<V, ITEMS>(slab + static_cast<size_t>(i) * P, v);
        } else {
            const uint64_t ts = g.rb + static_cast<uint64_t>(i) * P;
#pragma unroll
            for (int q = 0; q < ITEMS; q++)
                v[q] = (e0 + q >= lo && e0 + q < hi) ? in[ts + e0 + q] : V();
        }
    };

    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < KMAX; q++) mbar_init(&bars[q], 1);
        mbar_fence_init();
    }
    __syncthreads();

    uint32_t t = blockIdx.x;
    if (t >= num_mids) return;
    Seg cur;
    {
        const uint32_t s = a.mids[t];
        cur = make_seg(s, a.offsets[s], a.offsets[s + 1]);
    }
    if (tid == 0)
        for (uint32_t i = 0; i < cur.ntiles; i++) issue(cur, i);
    // the segment after the next one: its index is loaded one iteration early
    uint32_t s_next = t + G < num_mids ? a.mids[t + G] : 0u;

    for (; t < num_mids; t += G) {
        const bool has_next = t + G < num_mids;
        uint64_t n0 = 0, n1 = 0;
        if (has_next) {  // used after the count pass
            n0 = a.offsets[s_next];
            n1 = a.offsets[s_next + 1];
        }
        const uint32_t s_after = t + 2u * G < num_mids ? a.mids[t + 2u * G] : 0u;
        const D dj = seg_discr(a, d, cur.s);

        // ---- count pass: lane c of every warp keeps the warp's count of class c
        uint32_t wt = 0;
        bool ok = true;
        for (uint32_t i = 0; i < cur.ntiles; i++) {
            ok = mbar_wait_bounded(&bars[i], (parity >> i) & 1u) && ok;
            uint32_t lo, hi;
            range(cur, i, lo, hi);
            const bool full = lo == 0u && hi == static_cast<uint32_t>(P);
            V v[ITEMS];
            take(cur, i, lo, hi, v);
            NibbleCounts<M> nc;
            nc.init();
            uint32_t last_c = M;  // element 15 stays out of the nibbles (a nibble holds 15)
#pragma unroll
            for (int j = 0; j < ITEMS; j++) {
                if (full || (e0 + j >= lo && e0 + j < hi)) {
                    const uint32_t c = dj(v[j]);
                    if (j < 15) nc.inc(c); else last_c = c;
                }
            }
#pragma unroll
            for (int c = 0; c < M; c++) {
                const uint32_t x = __reduce_add_sync(
                    0xffffffffu, nc.get(c) + (last_c == static_cast<uint32_t>(c) ? 1u : 0u));
                if (lane == c) wt += x;
            }
        }
        if (lane < M) red[warp][lane] = wt;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(&a.hdr->error, kErrTimeout);
                for (uint32_t i = 0; i < cur.ntiles; i++)  // copies still in flight
                    (void)mbar_wait_bounded(&bars[i], (parity >> i) & 1u);
            }
            break;
        }
        parity ^= cur.ntiles >= 32u ? 0xffffffffu : ((1u << cur.ntiles) - 1u);
        Seg nxt{};
        if (has_next) nxt = make_seg(s_next, n0, n1);

        // ---- the segment's class totals: sizes, head flags, cursors
        if (warp == 0) {
            uint32_t tot = 0;
            if (lane < M) {
#pragma unroll
                for (int w = 0; w < W; w++) tot += red[w][lane];
            }
            const uint32_t excl = warp_incl_scan(tot) - tot;
            if (lane < M) {
                sh.cursor[0][lane] = static_cast<uint32_t>(cur.a0) + excl;
                if (a.seg_sizes != nullptr && static_cast<uint32_t>(lane) < a.m)
                    a.seg_sizes[static_cast<uint64_t>(cur.s) * a.m + lane] = tot;
                if (a.headflags != nullptr && tot > 0) a.headflags[cur.a0 + excl] = tot;
            }
            // the next segment's tiles in the slots this one leaves unused
            if (lane == 0 && has_next)
                for (uint32_t i = cur.ntiles; i < nxt.ntiles; i++) issue(nxt, i);
        }
        __syncthreads();

        // ---- scatter pass from the slab; slot i takes the next segment's tile
        // i once this segment's tile i is in registers
        for (uint32_t i = 0; i < cur.ntiles; i++) {
            uint32_t lo, hi;
            range(cur, i, lo, hi);
            const bool full = lo == 0u && hi == static_cast<uint32_t>(P);
            V v[ITEMS];
            take(cur, i, lo, hi, v);
            (void)tile_scatter<V, D, M, THREADS, true>(
                dj, v, lo, hi, full, stage, cnt_sm, sh, i & 1u, OutFlat<V>{out, out_phase}, true,
                [&] {
                    if (tid == 0 && has_next && i < nxt.ntiles) issue(nxt, i);
                });
        }
        cur = nxt;
        s_next = s_after;
    }
    if (tid < M) bulk_wait_all();
}

// ------------------------------------------------ head flags -> offsets --
// The reference's segment descriptor (MdiscrSegmHost.cu.h:36-42,
// populateSizesArray HelpersCommon.h:105-151) is an n-entry array holding each
// segment's length at its first element and 0 elsewhere.  Two launches turn it
// into offsets[0..S] and S (in the header); the planner then checks that every
// flag equals the distance to the next start.
//
//   seg_flags_stage    CTA k reads chunk k of the flags once (tiles of FT
//                      flags, 16 per thread), writes the positions of its
//                      non-zero flags in order into its own part of a staging
//                      array (stage[chunk start + j]) and its count; the last
//                      CTA to finish (ticket, no waiting) scans the chunk
//                      counts into chunk prefixes, S and offsets[S] = n.
//   seg_flags_compact  CTA k moves its staged positions to offsets[prefix + j].
//
// No CTA waits on another: the single pass with a decoupled look-back that
// this replaces spent most of its time walking predecessors, because ~10^3
// tiles of a few microseconds each were in flight at once.
struct FlagsArgs {
    const int32_t* flags;
    uint64_t n;
    uint64_t chunk;      // flags per chunk (a multiple of 4)
    uint32_t* stage;     // [n] staged start positions, chunk k's from k * chunk
    uint32_t* cnt;       // [G] start positions per chunk
    uint32_t* pre;       // [G] exclusive prefix of cnt
    uint64_t* offsets;   // [S + 1]
    SegHeader* hdr;
};

template <int THREADS, int FT>
__global__ void __launch_bounds__(THREADS) seg_flags_stage(FlagsArgs fa) {
    constexpr int ITEMS = FT / THREADS;
    constexpr int W = THREADS / 32;
    static_assert(ITEMS * THREADS == FT && ITEMS % 4 == 0, "tile");
    __shared__ uint32_t warp_tot[W];
    __shared__ int last_sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t c0 = min(static_cast<uint64_t>(blockIdx.x) * fa.chunk, fa.n);
    const uint64_t c1 = min(c0 + fa.chunk, fa.n);
    const bool vec = (reinterpret_cast<uintptr_t>(fa.flags) & 15u) == 0;
    uint32_t running = 0;  // start positions of this chunk so far
    bool bad = false;
    for (uint64_t ts = c0; ts < c1; ts += FT) {
        const uint64_t e0 = ts + static_cast<uint64_t>(tid) * ITEMS;
        int32_t f[ITEMS];
        if (vec && e0 + ITEMS <= c1) {
#pragma unroll
            for (int q = 0; q < ITEMS / 4; q++) {
                const int4 r = __ldg(reinterpret_cast<const int4*>(fa.flags + e0) + q);
                f[4 * q] = r.x; f[4 * q + 1] = r.y; f[4 * q + 2] = r.z; f[4 * q + 3] = r.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < ITEMS; q++) f[q] = e0 + q < c1 ? __ldg(fa.flags + e0 + q) : 0;
        }
        uint32_t nz = 0;
#pragma unroll
        for (int q = 0; q < ITEMS; q++) {
            nz += f[q] != 0 ? 1u : 0u;
            bad |= f[q] < 0;
        }
        const uint32_t incl = warp_incl_scan(nz);
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        uint32_t wpre = 0, agg = 0;
#pragma unroll
        for (int w = 0; w < W; w++) {
            const uint32_t x = warp_tot[w];
            wpre += w < warp ? x : 0u;
            agg += x;
        }
        uint32_t pos = running + wpre + incl - nz;
#pragma unroll
        for (int q = 0; q < ITEMS; q++)
            if (f[q] != 0) fa.stage[c0 + pos++] = static_cast<uint32_t>(e0 + q);
        running += agg;
        __syncthreads();  // warp_tot is rewritten by the next tile
    }
    if (bad) atomicOr(&fa.hdr->error, kErrSegments);
    if (tid == 0) {
        fa.cnt[blockIdx.x] = running;
        __threadfence();
        last_sh = (atomicAdd(&fa.hdr->flags_done, 1u) == gridDim.x - 1u);
    }
    __syncthreads();
    if (!last_sh) return;
    __threadfence();
    // last CTA: exclusive scan of the chunk counts (one warp), S, offsets[S]
    if (warp == 0) {
        uint64_t run = 0;
        for (uint32_t b0 = 0; b0 < gridDim.x; b0 += 32) {
            const uint32_t b = b0 + lane;
            const uint32_t x = b < gridDim.x ? __ldcg(&fa.cnt[b]) : 0u;
            const uint32_t inc = warp_incl_scan(x);
            if (b < gridDim.x) fa.pre[b] = static_cast<uint32_t>(run) + inc - x;
            run += __shfl_sync(0xffffffffu, inc, 31);
        }
        if (lane == 0) {
            fa.hdr->num_segs = run;
            fa.offsets[run] = fa.n;
            if (fa.n > 0 && __ldg(fa.flags) == 0) atomicOr(&fa.hdr->error, kErrSegments);
            fa.hdr->flags_done = 0u;  // for the next call
        }
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) seg_flags_compact(FlagsArgs fa) {
    const uint64_t c0 = min(static_cast<uint64_t>(blockIdx.x) * fa.chunk, fa.n);
    const uint32_t k = fa.cnt[blockIdx.x], p = fa.pre[blockIdx.x];
    for (uint32_t j = threadIdx.x; j < k; j += THREADS) fa.offsets[p + j] = fa.stage[c0 + j];
}

}  // namespace mdx
