// mdx_segm.cuh -- segmented (batched) stable m-way partition for sm_100a.
//
// Replaces mdiscrSegm<DISCR> (cuda_code/MdiscrSegmHost.cu.h:36-230: a chain
// of ~12 kernels -- segmented scans of head flags and of N one-hot m-tuples,
// per-element reductions, class offsets, indices, permute, sizes -- with nine
// N-sized temporaries, four of them N*m tuples) by three launches:
//
//   seg_plan_spans  per segment: its length; segments longer than one window
//                   (P elements) are "large" and get one work entry per
//                   window they touch.  Block-local scan of the entry counts;
//                   the last CTA scans the block totals and records the
//                   number of entries, the largest span (the lag below), a new
//                   epoch for the look-back words, and resets the ticket.
//   seg_plan_emit   writes the work entries {segment, piece [p0, p1), last
//                   entry of the segment} in element order.
//   seg_main        one persistent launch.  CTAs take tickets in order:
//                     * small-segment groups first: each segment of length
//                       <= P is partitioned on its own by one warp (count
//                       pass, then rank pass with __match_any_sync + __popc
//                       ranks and running class counts), single HBM read;
//                     * then, for every large-segment window entry j, a
//                       count item C(j) (class counts of the piece, published
//                       to epoch-tagged per-class status words; decoupled
//                       look-back over the segment's earlier entries gives the
//                       piece's exclusive prefix, the segment's last entry
//                       gives its class totals) and a scatter item S(j)
//                       (re-reads the piece, ranks it CTA-wide, writes it
//                       through a shared-memory stage).  S(j) is issued D
//                       tickets after C(j), D = the longest span, so S(j)
//                       only waits on earlier tickets (no deadlock) and finds
//                       its piece still in L2 (D * P elements of lag).
//
// Every wait is bounded (kWaitLimitNs); a wait that runs out latches
// kErrTimeout and publishes what it has so that no other CTA waits forever.
//
// Output per segment equals seqMdiscr (SeqMdiscr.h:10-57) applied to the
// segment, which is exactly what MdiscrSegmTest.cu:8-41 validates; sizes are
// emitted as an S x m tuple table and/or per-segment head flags
// (MdiscrSegmKernels.cu.h:89-114 writes the latter into new_sizes).
#pragma once

#include "mdx_device.cuh"
#include "mdx_plain.cuh"  // NibbleCounts, unpack16_to

namespace mdx {

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
    uint32_t num_lw;    // large-window entries this call
    uint32_t lag;       // longest span of a large segment, in windows
    uint32_t plan_done; // planner CTA ticket
    uint64_t num_segs;  // S (written by the flags converter for the head-flag form)
    uint32_t lag_cur;   // lag of the current call (snapshot taken by the planner)
    uint32_t flags_ticket;  // tile ticket of the flags converter
    uint32_t flags_done;    // finished tiles of the flags converter
    uint32_t flags_epoch;   // look-back epoch of the flags converter
    uint32_t pad[4];
};

struct LwEntry {        // one window piece of a large segment
    uint32_t seg;       // segment index
    uint32_t p0, p1;    // element range of the piece
    uint32_t jlast;     // entry index of the segment's last piece
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
    uint32_t* span_loc;        // [S] block-local exclusive entry offsets
    uint32_t* blk_tot;         // [plan blocks] entry totals, then offsets
    LwEntry* lw;               // [max entries]
    uint64_t* status;          // [max entries][M]
    uint32_t* excl;            // [max entries][M] exclusive prefix of each piece
    uint32_t plan_blocks;
    uint32_t max_entries;      // capacity of lw / status / excl (2 per window: enough
                               // for segments that tile [0, n); malformed ones are cut)
};

constexpr uint64_t kSegsOnDevice = ~0ull;

__device__ __forceinline__ uint64_t seg_count(const SegArgs& a) {
    return a.num_segs == kSegsOnDevice ? a.hdr->num_segs : a.num_segs;
}

// --------------------------------------------------------------- planning --
// Block b of the planner owns segments [b*R, min((b+1)*R, S)), R = ceil(S/G).
template <int P, int THREADS>
__global__ void __launch_bounds__(THREADS) seg_plan_spans(SegArgs a) {
    __shared__ uint32_t warp_tot[THREADS / 32];
    __shared__ uint32_t carry_sh;
    __shared__ int am_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t S = seg_count(a);
    const uint64_t G = gridDim.x;
    const uint64_t R = (S + G - 1) / G;
    const uint64_t s0 = blockIdx.x * R, s1 = min(s0 + R, S);
    uint32_t carry = 0, maxspan = 0;
    for (uint64_t base = s0; base < s1; base += THREADS) {
        const uint64_t s = base + tid;
        uint32_t span = 0;
        if (s < s1) {
            const uint64_t a0 = a.offsets[s], a1 = a.offsets[s + 1];
            if (a1 < a0 || a1 > a.n || (s == 0 && a0 != 0) || (s + 1 == S && a1 != a.n)) {
                atomicOr(&a.hdr->error, kErrSegments);
            } else if (a1 - a0 > static_cast<uint64_t>(P)) {
                span = static_cast<uint32_t>((a1 - 1) / P - a0 / P + 1);
            }
            if (a.in_flags != nullptr && a1 > a0 &&
                static_cast<uint64_t>(a.in_flags[a0]) != a1 - a0)
                atomicOr(&a.hdr->error, kErrSegments);
        }
        maxspan = max(maxspan, span);
        const uint32_t incl = warp_incl_scan(span);
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        uint32_t wpre = 0, btot = 0;
        for (int w = 0; w < THREADS / 32; w++) {
            const uint32_t x = warp_tot[w];
            wpre += (w < warp) ? x : 0u;
            btot += x;
        }
        if (s < s1) a.span_loc[s] = carry + wpre + incl - span;
        carry += btot;
        __syncthreads();
    }
    for (int d = 16; d > 0; d >>= 1) maxspan = max(maxspan, __shfl_xor_sync(0xffffffffu, maxspan, d));
    if (lane == 0 && maxspan > 0) atomicMax(&a.hdr->lag, maxspan);
    if (tid == 0) a.blk_tot[blockIdx.x] = carry;
    __threadfence();
    __syncthreads();
    if (tid == 0) am_last = (atomicAdd(&a.hdr->plan_done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    // last CTA: exclusive scan of the block totals (in place)
    if (warp == 0) {
        uint32_t run = 0;
        for (uint32_t b0 = 0; b0 < gridDim.x; b0 += 32) {
            const uint32_t b = b0 + lane;
            const uint32_t x = b < gridDim.x ? __ldcg(&a.blk_tot[b]) : 0u;
            const uint32_t incl = warp_incl_scan(x);
            if (b < gridDim.x) a.blk_tot[b] = run + incl - x;
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) {
            carry_sh = run;
            a.hdr->num_lw = run <= a.max_entries ? run : 0u;  // over capacity: malformed
            a.hdr->lag_cur = a.hdr->lag;  // every block's atomicMax happened before its ticket
            a.hdr->lag = 0u;
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
}

template <int P, int THREADS>
__global__ void __launch_bounds__(THREADS) seg_plan_emit(SegArgs a) {
    __shared__ uint32_t list_seg[THREADS], list_pos[THREADS], list_span[THREADS];
    __shared__ uint32_t list_n;
    const int tid = threadIdx.x;
    const uint64_t S = seg_count(a);
    const uint64_t G = gridDim.x;
    const uint64_t R = (S + G - 1) / G;
    const uint64_t s0 = blockIdx.x * R, s1 = min(s0 + R, S);
    const uint32_t boff = a.blk_tot[blockIdx.x];
    for (uint64_t base = s0; base < s1; base += THREADS) {
        if (tid == 0) list_n = 0;
        __syncthreads();
        const uint64_t s = base + tid;
        if (s < s1) {
            const uint64_t a0 = a.offsets[s], a1 = a.offsets[s + 1];
            if (a1 >= a0 && a1 <= a.n && a1 - a0 > static_cast<uint64_t>(P)) {
                const uint32_t q = atomicAdd(&list_n, 1u);
                list_seg[q] = static_cast<uint32_t>(s);
                list_pos[q] = boff + a.span_loc[s];
                list_span[q] = static_cast<uint32_t>((a1 - 1) / P - a0 / P + 1);
            }
        }
        __syncthreads();
        const uint32_t cnt = list_n;
        for (uint32_t q = 0; q < cnt; q++) {  // the block emits each large segment's entries
            const uint32_t seg = list_seg[q], pos = list_pos[q], span = list_span[q];
            const uint64_t a0 = a.offsets[seg], a1 = a.offsets[seg + 1];
            const uint64_t w0 = a0 / P;
            if (static_cast<uint64_t>(pos) + span > a.max_entries) {  // malformed offsets
                if (tid == 0) atomicOr(&a.hdr->error, kErrSegments);
                continue;
            }
            for (uint32_t k = tid; k < span; k += THREADS) {
                const uint64_t w = w0 + k;
                LwEntry e;
                e.seg = seg;
                e.p0 = static_cast<uint32_t>(max(a0, w * P));
                e.p1 = static_cast<uint32_t>(min(a1, (w + 1) * P));
                e.jlast = pos + span - 1u;
                a.lw[pos + k] = e;
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------- main kernel --
template <class V, int M, int THREADS>
struct SegSmem {
    static constexpr int kItems = 64 / static_cast<int>(sizeof(V));
    static constexpr int kTile = THREADS * kItems;  // == P
    static constexpr uint32_t kAU = 16 / sizeof(V);
    static constexpr int kStageElems = kTile + static_cast<int>(kAU) * M;
    static constexpr size_t kStageBytes = static_cast<size_t>(kStageElems) * sizeof(V);
    static constexpr size_t kCntBytes = static_cast<size_t>(M) * THREADS * 2;
    static constexpr size_t kBytes = kStageBytes + kCntBytes + 64;
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

// One warp partitions one segment of length L <= P (two passes over it: the
// second finds it in L1/L2).  Lanes 0..M-1 also write the segment's sizes.
template <class V, class D, int M>
__device__ void seg_small_warp(const SegArgs& a, const D& d, uint64_t s, uint64_t a0, uint64_t L,
                               uint32_t* hist /* per-warp [M] */) {
    const int lane = threadIdx.x & 31;
    const V* in = static_cast<const V*>(a.in) + a0;
    V* out = static_cast<V*>(a.out) + a0;
    const uint32_t lt = lanemask_lt();
    for (int c = lane; c < M; c += 32) hist[c] = 0;
    __syncwarp();
    // pass 1: class counts
    for (uint64_t e0 = 0; e0 < L; e0 += 32) {
        const uint64_t e = e0 + lane;
        const bool live = e < L;
        const uint32_t c = live ? d(in[e]) : static_cast<uint32_t>(M);
        const uint32_t peers = __match_any_sync(0xffffffffu, c);
        if (live && (peers >> lane) == 1u) hist[c] += __popc(peers);
        __syncwarp();
    }
    // class offsets (exclusive scan over classes); lanes own classes lane, lane+32
    uint32_t off0 = 0, off1 = 0, tot0 = 0, tot1 = 0;
    {
        tot0 = lane < M ? hist[lane] : 0u;
        tot1 = lane + 32 < M ? hist[lane + 32] : 0u;
        const uint32_t i0 = warp_incl_scan(tot0);
        const uint32_t all0 = __shfl_sync(0xffffffffu, i0, 31);
        const uint32_t i1 = warp_incl_scan(tot1);
        off0 = i0 - tot0;
        off1 = all0 + i1 - tot1;
    }
    __syncwarp();
    if (lane < M) hist[lane] = off0;            // running destination per class
    if (lane + 32 < M) hist[lane + 32] = off1;
    if (a.seg_sizes != nullptr) {
        if (lane < M && static_cast<uint32_t>(lane) < a.m) a.seg_sizes[s * a.m + lane] = tot0;
        if (lane + 32 < M && static_cast<uint32_t>(lane + 32) < a.m)
            a.seg_sizes[s * a.m + lane + 32] = tot1;
    }
    if (a.headflags != nullptr) {
        if (lane < M && tot0 > 0) a.headflags[a0 + off0] = tot0;
        if (lane + 32 < M && tot1 > 0) a.headflags[a0 + off1] = tot1;
    }
    __syncwarp();
    // pass 2: ranks in input order, scatter into the segment's output
    for (uint64_t e0 = 0; e0 < L; e0 += 32) {
        const uint64_t e = e0 + lane;
        const bool live = e < L;
        V v = V();
        if (live) v = in[e];
        const uint32_t c = live ? d(v) : static_cast<uint32_t>(M);
        const uint32_t peers = __match_any_sync(0xffffffffu, c);
        const uint32_t before = live ? hist[c] : 0u;
        const uint32_t r = __popc(peers & lt);
        if (live) out[before + r] = v;
        __syncwarp();
        if (live && (peers >> lane) == 1u) hist[c] = before + r + 1u;
        __syncwarp();
    }
}

template <class V, class D, int M, int THREADS>
__global__ void __launch_bounds__(THREADS) seg_main(SegArgs a, D d) {
    using L = SegSmem<V, M, THREADS>;
    constexpr int ITEMS = L::kItems;
    constexpr int P = L::kTile;
    constexpr uint32_t AU = L::kAU;
    constexpr int W = THREADS / 32;
    constexpr int PER = THREADS / 32;
    constexpr uint32_t K = 32;  // segments per small-segment group
    static_assert(M <= 16 && M >= 2, "class bound");
    static_assert(M <= 2 * W, "each warp scans at most two rows");
    static_assert(PER == 8, "row scans load 8 entries per lane");
    static_assert(L::kStageElems < 65536, "16-bit stage slots");

    extern __shared__ __align__(128) unsigned char smem_raw[];
    V* stage = reinterpret_cast<V*>(smem_raw);
    uint16_t* cnt_sm = reinterpret_cast<uint16_t*>(smem_raw + L::kStageBytes);

    __shared__ uint32_t ticket_sh, next_seg_sh;
    __shared__ uint32_t hist[W][M];
    __shared__ uint32_t red[W][M];
    __shared__ uint32_t run_start[M], run_cnt[M], run_dst[M], rowtot[M];
    __shared__ uint32_t piece_base[M];  // class offset in segment + piece's exclusive prefix
    __shared__ int fail_sh;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const V* in = static_cast<const V*>(a.in);
    V* out = static_cast<V*>(a.out);
    const uint32_t out_phase =
        static_cast<uint32_t>(reinterpret_cast<uintptr_t>(out) / sizeof(V)) & (AU - 1u);
    const uint64_t S = seg_count(a);
    const uint32_t epoch = a.hdr->epoch;
    const uint32_t num_lw = a.hdr->num_lw;
    const uint32_t lag = min(max(a.hdr->lag_cur, 1u), max(num_lw, 1u));
    const uint32_t small_items = static_cast<uint32_t>((S + K - 1) / K);
    const uint32_t total = small_items + 2u * num_lw;
    uint16_t* my_cnt = cnt_sm + tid;
    const uint32_t e0 = tid * ITEMS;

    for (;;) {
        if (tid == 0) ticket_sh = atomicAdd(&a.hdr->ticket, 1u);
        __syncthreads();
        const uint32_t t = ticket_sh;
        if (t >= total) break;

        if (t < small_items) {
            // ---------------- small segments: one warp per segment ----------
            if (tid == 0) next_seg_sh = 0;
            __syncthreads();
            const uint64_t g0 = static_cast<uint64_t>(t) * K;
            for (;;) {
                uint32_t q = 0;
                if (lane == 0) q = atomicAdd(&next_seg_sh, 1u);
                q = __shfl_sync(0xffffffffu, q, 0);
                if (q >= K) break;
                const uint64_t s = g0 + q;
                if (s >= S) break;
                const uint64_t a0 = a.offsets[s], a1 = a.offsets[s + 1];
                if (a1 < a0 || a1 > a.n) continue;          // malformed: flagged by the planner
                if (a1 - a0 > static_cast<uint64_t>(P)) continue;  // large: window items
                seg_small_warp<V, D, M>(a, d, s, a0, a1 - a0, hist[warp]);
            }
            __syncthreads();
            continue;
        }

        // ---------------- large-segment window items ----------------
        const uint32_t u = t - small_items;
        uint32_t j;
        bool is_count;
        if (u < lag) {
            j = u;
            is_count = true;
        } else {
            const uint32_t v = u - lag;
            const uint32_t pairs = num_lw - lag;
            if (v < 2u * pairs) {
                is_count = (v & 1u) != 0u;
                j = is_count ? lag + (v >> 1) : (v >> 1);
            } else {
                is_count = false;
                j = pairs + (v - 2u * pairs);
                if (lag >= num_lw) j = num_lw - 1u - j;  // all counts first: walk back for L2 reuse
            }
        }
        const LwEntry ent = a.lw[j];
        const uint32_t wbase = (ent.p0 / P) * P;
        const uint32_t lo = ent.p0 - wbase, hi = ent.p1 - wbase;
        const bool first_piece = (ent.p0 == static_cast<uint32_t>(a.offsets[ent.seg]));
        const bool last_piece = (j == ent.jlast);

        // the piece's elements, blocked: thread t holds tile-local e0 .. e0+ITEMS-1
        V v[ITEMS];
        const bool whole = (e0 >= lo) && (e0 + ITEMS <= hi);
        if (whole) {
            const uint4* vp = reinterpret_cast<const uint4*>(in + wbase + e0);
            const bool al = ((reinterpret_cast<uintptr_t>(in) & 15u) == 0);
            if (al) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const uint4 r = __ldg(vp + q);
                    unpack16_to<V>(r, &v[q * AU]);
                }
            } else {
#pragma unroll
                for (int q = 0; q < ITEMS; q++) v[q] = in[wbase + e0 + q];
            }
        } else {
#pragma unroll
            for (int q = 0; q < ITEMS; q++)
                v[q] = (e0 + q >= lo && e0 + q < hi) ? in[wbase + e0 + q] : V();
        }

        if (is_count) {
            // ---------------- C(j): class counts of the piece + look-back ----
            NibbleCounts<M> nc;
            nc.init();
            uint32_t last_c = M;
#pragma unroll
            for (int q = 0; q < ITEMS; q++) {
                if (e0 + q >= lo && e0 + q < hi) {
                    const uint32_t c = d(v[q]);
                    if (q < 15) nc.inc(c); else last_c = c;
                }
            }
#pragma unroll
            for (int c = 0; c < M; c++) {
                const uint32_t x = warp_sum(nc.get(c) + (static_cast<uint32_t>(c) == last_c ? 1u : 0u));
                if (lane == 0) red[warp][c] = x;
            }
            __syncthreads();
            if (warp == 0) {
                const uint32_t c = lane;
                uint32_t agg = 0;
                if (c < static_cast<uint32_t>(M))
                    for (int w = 0; w < W; w++) agg += red[w][c];
                uint64_t* st = a.status + static_cast<uint64_t>(j) * M;
                uint32_t prefix = 0;
                bool ok = true;
                if (c < static_cast<uint32_t>(M)) {
                    if (first_piece) {
                        a.excl[static_cast<uint64_t>(j) * M + c] = 0u;
                        __threadfence();
                        st_release_u64(st + c, st_pack(epoch, kStInc, agg));
                    } else {
                        st_release_u64(st + c, st_pack(epoch, kStAgg, agg));
                        // decoupled look-back over this segment's earlier pieces
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
                if (last_piece) {
                    // segment totals -> sizes (tuple and head-flag forms)
                    const uint32_t tot = (c < static_cast<uint32_t>(M)) ? prefix + agg : 0u;
                    const uint32_t incl = warp_incl_scan(tot);
                    const uint64_t a0 = a.offsets[ent.seg];
                    if (c < static_cast<uint32_t>(M)) {
                        if (a.seg_sizes != nullptr && c < a.m) a.seg_sizes[static_cast<uint64_t>(ent.seg) * a.m + c] = tot;
                        if (a.headflags != nullptr && tot > 0) a.headflags[a0 + incl - tot] = tot;
                    }
                }
            }
            __syncthreads();
            continue;
        }

        // ---------------- S(j): scatter the piece ----------------
        // totals of the segment (its last entry) and this piece's prefix
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
                piece_base[c] = static_cast<uint32_t>(a.offsets[ent.seg]) + (incl - tot) + pre;
            const bool bad = __any_sync(0xffffffffu, !ok);
            if (lane == 0) {
                fail_sh = bad ? 1 : 0;
                if (bad) atomicOr(&a.hdr->error, kErrTimeout);
            }
        }
        // local ranks of the piece's elements (as in plain_scatter_tma_kernel)
        NibbleCounts<M> nc;
        nc.init();
        uint32_t lr[(ITEMS + 7) / 8];
#pragma unroll
        for (int q = 0; q < (ITEMS + 7) / 8; q++) lr[q] = 0;
        uint32_t last_c = M;
#pragma unroll
        for (int q = 0; q < ITEMS; q++) {
            if (e0 + q >= lo && e0 + q < hi) {
                const uint32_t c = d(v[q]);
                lr[q >> 3] += nc.get(c) << (4 * (q & 7));
                if (q < 15) nc.inc(c); else last_c = c;
            }
        }
#pragma unroll
        for (int c = 0; c < M; c++) my_cnt[c * THREADS] = static_cast<uint16_t>(nc.get(c));
        if (last_c < static_cast<uint32_t>(M)) my_cnt[last_c * THREADS] += 1;
        __syncthreads();
        if (fail_sh) {
            __syncthreads();
            continue;
        }
        uint32_t pre_r[2][PER];
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
                    pre_r[h][q] = run;
                    run += x[q];
                }
                if (lane == 31) rowtot[c] = incl;
            }
        }
        __syncthreads();
        {
            const uint32_t c = static_cast<uint32_t>(lane);
            const uint32_t cc = c < static_cast<uint32_t>(M) ? rowtot[c] : 0u;
            // the piece's class-c elements precede nothing else of the piece in
            // the output: its class-c run starts at piece_base[c]
            const uint32_t dst = c < static_cast<uint32_t>(M) ? piece_base[c] : 0u;
            const uint32_t room = cc + (c < static_cast<uint32_t>(M) ? AU : 0u);
            const uint32_t q0 = warp_incl_scan(room) - room;
            const uint32_t st = q0 + (((out_phase + dst) - q0) & (AU - 1u));
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int row = warp + h * W;
                if (row < M) {
                    const uint32_t add = __shfl_sync(0xffffffffu, st, row);
                    const uint32_t add2 = add | (add << 16);
                    *reinterpret_cast<uint4*>(cnt_sm + row * THREADS + lane * PER) =
                        make_uint4((pre_r[h][0] | (pre_r[h][1] << 16)) + add2,
                                   (pre_r[h][2] | (pre_r[h][3] << 16)) + add2,
                                   (pre_r[h][4] | (pre_r[h][5] << 16)) + add2,
                                   (pre_r[h][6] | (pre_r[h][7] << 16)) + add2);
                }
            }
            if (warp == 0 && c < static_cast<uint32_t>(M)) {
                run_start[c] = st;
                run_cnt[c] = cc;
                run_dst[c] = dst;
            }
        }
        if (tid < M) bulk_wait_read<0>();  // the stage's previous bulk stores
        __syncthreads();
#pragma unroll
        for (int q = 0; q < ITEMS; q++) {
            if (e0 + q >= lo && e0 + q < hi) {
                const uint32_t c = d(v[q]);
                const uint32_t slot = my_cnt[c * THREADS] + ((lr[q >> 3] >> (4 * (q & 7))) & 15u);
                stage[slot] = v[q];
            }
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (tid < M) {
            const uint32_t s = run_start[tid], cc = run_cnt[tid];
            uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
            if (head > cc) head = cc;
            const uint32_t body = ((cc - head) / AU) * AU;
            if (body > 0)
                bulk_store_s2g(out + run_dst[tid] + head, stage + s + head, body * sizeof(V));
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
            if (off != 0xffffffffu) out[run_dst[c] + off] = stage[s + off];
        }
        __syncthreads();
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
