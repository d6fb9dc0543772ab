// mdx_tile.cuh -- the per-tile rank / stage / write-out step shared by the
// plain scatter kernel and the segmented scatter items (m <= 16).
//
// A tile is THREADS * ITEMS elements (BPT = 64 or 32 contiguous bytes per
// thread: two tile geometries, chosen per call by the tuning table).  For
// the elements of tile-local range [lo, hi):
//  * pass 1: each thread ranks its own consecutive elements with 4-bit
//    counters in a register (local rank = number of its earlier elements of
//    the same class; the 16th element is kept aside so no lane can reach 16)
//    and publishes its per-class counts to a [class][thread] u16 matrix;
//  * row scans: warp w < m/2 scans rows w and w + m/2 of the matrix at once,
//    packed in u16 pairs (exclusive prefix over threads = stable order); those
//    warps derive the tile's class runs (lanes = classes) and fold each run's
//    stage slot into their rows;
//  * pass 2: element -> stage slot = row prefix + local rank;
//  * write-out: each class run sits in the stage at the same 16-byte phase as
//    its destination, so its aligned interior leaves by one bulk store
//    (cp.async.bulk shared -> global) and threads store the < 16-byte head and
//    tail.  Before the stage is rewritten the previous bulk stores must have
//    read it (cp.async.bulk.wait_group.read).
#pragma once

#include "mdx_device.cuh"

namespace mdx {

// Per-thread class counters in 4-bit lanes: one u32 holds 8 classes, two
// hold 16.
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
        } else {  // sixteen nibbles: one 64-bit shift
            const uint64_t x = (static_cast<uint64_t>(w[1]) << 32) | w[0];
            return static_cast<uint32_t>(x >> (c << 2)) & 15u;
        }
    }
    __device__ __forceinline__ void inc(uint32_t c) {
        if constexpr (NW == 1) {
            w[0] += 1u << (c << 2);
        } else {
            uint64_t x = (static_cast<uint64_t>(w[1]) << 32) | w[0];
            x += 1ull << (c << 2);
            w[0] = static_cast<uint32_t>(x);
            w[1] = static_cast<uint32_t>(x >> 32);
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
template <>
__device__ __forceinline__ void unpack16_to<Rec16>(const uint4& r, Rec16* e) {
    e[0].w[0] = r.x; e[0].w[1] = r.y; e[0].w[2] = r.z; e[0].w[3] = r.w;
}

template <class V, int THREADS, int M, int BPT = 64>
struct TileGeom {
    static_assert(BPT == 64 || BPT == 32, "64 or 32 bytes per thread");
    static constexpr int kItems = BPT / static_cast<int>(sizeof(V));  // BPT bytes per thread
    static constexpr int kTile = THREADS * kItems;
    static constexpr int kRows = kTile * static_cast<int>(sizeof(V)) / 128;  // 128-byte rows
    static constexpr uint32_t kAU = 16 / sizeof(V);                 // elements per 16 bytes
    // every class run gets kAU slots of slack for its 16-byte phase
    static constexpr int kStageElems = kTile + static_cast<int>(kAU) * M;
    static constexpr size_t kStageBytes = static_cast<size_t>(kStageElems) * sizeof(V);
    // m <= 16: [class][thread] u16 counts; more classes: [warp][class] u32
    // counts, then stage bases (tile_scatter_wide)
    static constexpr size_t kCntBytes = M <= 16 ? static_cast<size_t>(M) * THREADS * 2
                                                : static_cast<size_t>(THREADS / 32) * M * 4;
    static_assert(kStageElems < 65536, "stage slots are kept in 16 bits");
};

// Shared-memory state of the tile step.
template <int M>
struct TileShared {
    uint32_t cursor[2][M];  // ping-pong by tile parity
    uint32_t run_start[M], run_cnt[M], run_dst[M], rowtot[M];
};

// Where a tile's class runs go.  `idx` is an element's position in the whole
// output (< 2^32).
//
// OutFlat: one array.  phase = (out / sizeof(V)) mod (16 / sizeof(V)).
template <class V>
struct OutFlat {
    V* out;
    uint32_t phase_;
    __device__ __forceinline__ uint32_t phase() const { return phase_; }
    __device__ __forceinline__ V* at(uint32_t idx) const { return out + idx; }
    // End of the piece [idx, end) that lies in one buffer.
    __device__ __forceinline__ uint32_t piece_end(uint32_t, uint32_t end) const { return end; }
};

// OutSharded: the output is cut into R chunks that live in different buffers
// (one per rank, typically on other GPUs, reached through peer mappings):
// chunk q holds positions [q * chunk, (q + 1) * chunk) (trailing chunks may
// be short or empty), the last chunk everything from (R - 1) * chunk on.
// Every chunk pointer is 16-byte aligned and `chunk` is a multiple of
// 16 / sizeof(V) elements, so a position's 16-byte phase is the same in every
// chunk and a run that crosses a chunk boundary splits into pieces that each
// stay bulk-store aligned.
constexpr int kMaxRanks = 128;
template <class V>
struct OutSharded {
    V* chunks[kMaxRanks];
    uint32_t chunk;
    uint32_t R;
    __device__ __forceinline__ uint32_t phase() const { return 0u; }
    __device__ __forceinline__ V* at(uint32_t idx) const {
        const uint32_t q = min(idx / chunk, R - 1u);
        return chunks[q] + (idx - q * chunk);
    }
    __device__ __forceinline__ uint32_t piece_end(uint32_t idx, uint32_t end) const {
        const uint32_t q = idx / chunk;
        if (q + 1u >= R) return end;
        const uint64_t b = static_cast<uint64_t>(q + 1u) * chunk;
        return b < end ? static_cast<uint32_t>(b) : end;
    }
};

// Take a thread's ITEMS * sizeof(V) (64 or 32) bytes of a tile that TMA
// placed in shared memory with the 128-byte swizzle (16-byte chunk q of
// 128-byte row r sits at chunk q ^ (r & 7)).
template <class V, int ITEMS>
__device__ __forceinline__ void take_swizzled(const V* tile, V (&v)[ITEMS]) {
    constexpr uint32_t AU = 16 / sizeof(V);
    constexpr uint32_t BPT = ITEMS * sizeof(V);
    static_assert(BPT == 64 || BPT == 32, "64 or 32 bytes per thread");
    constexpr uint32_t TPR = 128 / BPT, CPT = BPT / 16;  // threads per row, chunks per thread
    const unsigned char* tb = reinterpret_cast<const unsigned char*>(tile);
    const uint32_t row = threadIdx.x / TPR;
#pragma unroll
    for (uint32_t q = 0; q < CPT; q++) {
        const uint32_t chunk = ((threadIdx.x % TPR) * CPT + q) ^ (row & 7u);
        const uint4 r = *reinterpret_cast<const uint4*>(tb + row * 128u + chunk * 16u);
        unpack16_to<V>(r, &v[q * AU]);
    }
}

// One tile: see the file comment.  `full` means lo == 0 and hi == TILE (no
// bounds checks).  FORWARD: run c of this tile starts at cursor[par][c] and
// the cursor advances; otherwise it ends there and the cursor moves back.
// `after_counts` runs right after the first barrier (the input ring slot is
// consumed by then).  Returns false, having written nothing, when `ok` is
// false on any thread.
template <class V, class D, int M, int THREADS, bool FORWARD, class OUT, class AfterCounts,
          int ITEMS>
__device__ __forceinline__ bool tile_scatter(const D& d, const V (&v)[ITEMS], uint32_t lo,
                                             uint32_t hi, bool full, V* stage, uint16_t* cnt_sm,
                                             TileShared<M>& sh, uint32_t par, const OUT& out,
                                             bool ok, AfterCounts after_counts) {
    using G = TileGeom<V, THREADS, M, ITEMS * static_cast<int>(sizeof(V))>;
    static_assert(G::kItems == ITEMS, "geometry");
    constexpr uint32_t AU = G::kAU;
    constexpr int W = THREADS / 32;
    constexpr int PER = THREADS / 32;
    constexpr int LR = (ITEMS + 7) / 8;
    static_assert(M <= 16 && M >= 2, "class bound");
    static_assert(M <= 2 * W, "each warp scans at most two rows");
    static_assert((M & (M - 1)) == 0, "rows paired as w and w + M/2");
    static_assert(ITEMS == 16 || ITEMS == 8 || ITEMS == 4 || ITEMS == 2, "thread elements");
    static_assert(PER == 8 || PER == 16, "row scans load 8 or 16 entries per lane");

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t e0 = tid * ITEMS;
    uint16_t* my_cnt = cnt_sm + tid;  // this thread's column: my_cnt[c * THREADS]

    // ---- pass 1
    NibbleCounts<M> nc;
    nc.init();
    uint32_t lr[LR];
#pragma unroll
    for (int q = 0; q < LR; q++) lr[q] = 0;
    uint32_t last_c = M;  // class of element 15 (kept out of the nibbles)
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
            if (e0 + j >= lo && e0 + j < hi) {
                const uint32_t c = d(v[j]);
                lr[j >> 3] += nc.get(c) << (4 * (j & 7));
                if (j < 15) nc.inc(c); else last_c = c;
            }
        }
    }
#pragma unroll
    for (int c = 0; c < M; c++) my_cnt[c * THREADS] = static_cast<uint16_t>(nc.get(c));
    if (last_c < static_cast<uint32_t>(M)) my_cnt[last_c * THREADS] += 1;
    if (__syncthreads_or(!ok)) return false;  // (A)
    after_counts();

    // ---- row scans: warp w < M/2 scans rows w and w + M/2 at once, the two
    // rows' u16 counts packed in one word (row w low, row w + M/2 high; a
    // row's sum is at most the tile, < 2^16); the other warps idle here.  A
    // lane holds PER consecutive threads' entries (8 at 256 threads, 16 at 512)
    constexpr int H = M / 2;
    constexpr int NV = PER / 8;  // 16-byte loads per row and lane
    const bool scans = warp < H;
    uint32_t pre[PER];  // packed exclusive prefixes of this lane's threads
    if (scans) {
        uint32_t x[PER];
#pragma unroll
        for (int u = 0; u < NV; u++) {
            const uint4 xa =
                *reinterpret_cast<const uint4*>(cnt_sm + warp * THREADS + lane * PER + 8 * u);
            const uint4 xb =
                *reinterpret_cast<const uint4*>(cnt_sm + (warp + H) * THREADS + lane * PER + 8 * u);
            x[8 * u + 0] = __byte_perm(xa.x, xb.x, 0x5410);
            x[8 * u + 1] = __byte_perm(xa.x, xb.x, 0x7632);
            x[8 * u + 2] = __byte_perm(xa.y, xb.y, 0x5410);
            x[8 * u + 3] = __byte_perm(xa.y, xb.y, 0x7632);
            x[8 * u + 4] = __byte_perm(xa.z, xb.z, 0x5410);
            x[8 * u + 5] = __byte_perm(xa.z, xb.z, 0x7632);
            x[8 * u + 6] = __byte_perm(xa.w, xb.w, 0x5410);
            x[8 * u + 7] = __byte_perm(xa.w, xb.w, 0x7632);
        }
        uint32_t tot = 0;
#pragma unroll
        for (int q = 0; q < PER; q++) tot += x[q];
        const uint32_t incl = warp_incl_scan(tot);
        uint32_t run = incl - tot;
#pragma unroll
        for (int q = 0; q < PER; q++) {
            pre[q] = run;
            run += x[q];
        }
        if (lane == 31) {
            sh.rowtot[warp] = incl & 0xffffu;
            sh.rowtot[warp + H] = incl >> 16;
        }
    }
    __syncthreads();  // (B)

    // ---- class runs (the scanning warps, lanes = classes): destination of
    // run c and its stage slot, at the destination's 16-byte phase within kAU
    // slots of slack per run; each scanning warp folds the slots into its rows
    if (scans) {
        const uint32_t c = static_cast<uint32_t>(lane);
        const bool cls = c < static_cast<uint32_t>(M);
        const uint32_t cc = cls ? sh.rowtot[c] : 0u;
        const uint32_t cur = cls ? sh.cursor[par][c] : 0u;
        const uint32_t dst = FORWARD ? cur : cur - cc;
        const uint32_t room = cc + (cls ? AU : 0u);
        const uint32_t q0 = warp_incl_scan(room) - room;
        const uint32_t st = q0 + (((out.phase() + dst) - q0) & (AU - 1u));
        // slots < kStageElems < 2^16: the two rows' slots stay packed
        const uint32_t add = __shfl_sync(0xffffffffu, st, warp) |
                             (__shfl_sync(0xffffffffu, st, warp + H) << 16);
#pragma unroll
        for (int u = 0; u < NV; u++) {
            uint32_t p[8];
#pragma unroll
            for (int q = 0; q < 8; q++) p[q] = pre[8 * u + q] + add;
            *reinterpret_cast<uint4*>(cnt_sm + warp * THREADS + lane * PER + 8 * u) =
                make_uint4(__byte_perm(p[0], p[1], 0x5410), __byte_perm(p[2], p[3], 0x5410),
                           __byte_perm(p[4], p[5], 0x5410), __byte_perm(p[6], p[7], 0x5410));
            *reinterpret_cast<uint4*>(cnt_sm + (warp + H) * THREADS + lane * PER + 8 * u) =
                make_uint4(__byte_perm(p[0], p[1], 0x7632), __byte_perm(p[2], p[3], 0x7632),
                           __byte_perm(p[4], p[5], 0x7632), __byte_perm(p[6], p[7], 0x7632));
        }
        if (warp == 0 && cls) {
            sh.cursor[par ^ 1u][c] = FORWARD ? cur + cc : dst;
            sh.run_start[c] = st;
            sh.run_cnt[c] = cc;
            sh.run_dst[c] = dst;
        }
    }
    // the stage is about to be rewritten: the previous tile's bulk stores
    // must have finished reading it
    if (tid < M) bulk_wait_read<0>();
    __syncthreads();  // (C)

    // ---- pass 2: scatter into the class-sorted stage
    if (full) {
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const uint32_t c = d(v[j]);
            stage[my_cnt[c * THREADS] + ((lr[j >> 3] >> (4 * (j & 7))) & 15u)] = v[j];
        }
    } else {
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            if (e0 + j >= lo && e0 + j < hi) {
                const uint32_t c = d(v[j]);
                stage[my_cnt[c * THREADS] + ((lr[j >> 3] >> (4 * (j & 7))) & 15u)] = v[j];
            }
        }
    }
    fence_proxy_async_smem();
    __syncthreads();  // (D)

    // ---- write-out: bulk store of each run's aligned interior; threads store
    // the unaligned head and tail elements
    if (tid < M) {
        const uint32_t s = sh.run_start[tid], cc = sh.run_cnt[tid];
        uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
        if (head > cc) head = cc;
        const uint32_t body = ((cc - head) / AU) * AU;
        uint32_t a0 = sh.run_dst[tid] + head, sl = s + head;
        const uint32_t a1 = a0 + body;
        while (a0 < a1) {  // one piece per destination buffer
            const uint32_t b = out.piece_end(a0, a1);
            bulk_store_s2g(out.at(a0), stage + sl, (b - a0) * sizeof(V));
            sl += b - a0;
            a0 = b;
        }
        bulk_commit();
    } else if (tid >= 32 && tid < 32 + M * 2 * static_cast<int>(AU)) {
        const uint32_t c = (tid - 32) / (2 * AU), q = (tid - 32) % (2 * AU);
        const uint32_t s = sh.run_start[c], cc = sh.run_cnt[c];
        uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
        if (head > cc) head = cc;
        const uint32_t body = ((cc - head) / AU) * AU;
        uint32_t off = 0xffffffffu;
        if (q < AU) {
            if (q < head) off = q;
        } else if (head + body + (q - AU) < cc) {
            off = head + body + (q - AU);
        }
        if (off != 0xffffffffu) *out.at(sh.run_dst[c] + off) = stage[s + off];
    }
    return true;
}

// -------------------------------------------------------------- 2 classes --
// The filter case (m = 2; Haskell reference haskell_code/ParFilter.hs:8-21
// splits a list by a predicate, stably).  Same thread-contiguous elements
// and write-out as tile_scatter, with the counting done by bit masks:
//  * pass 1: each thread builds a mask of its class-1 elements (one bit per
//    element) and of its valid ones; its class counts are two popcounts; one
//    warp scan of the packed pair (class 0 low 16 bits, class 1 high) gives
//    each thread's prefix within the warp, lane 31 publishes the warp total;
//  * warp 0 scans the warp totals and places the two class runs at the
//    destination's 16-byte phase;
//  * pass 2: element j of a thread goes to its class's stage base + thread
//    prefix + popc(class mask & bits below j).
// No [class][thread] count matrix and no row scans: three barriers per tile
// instead of four and about half the instructions of the nibble step.  The
// scatter is bound by memory at m = 2 either way (N = 2^28 u32, B200: scatter
// kernel 0.383 ms with either step, against 0.337 ms for a plain 1 GiB
// device copy); the whole call at m = 2 is 1.02x the count kernel plus that
// copy.
template <class V, class D, int THREADS, bool FORWARD, class OUT, class AfterCounts, int ITEMS>
__device__ __forceinline__ bool tile_filter(const D& d, const V (&v)[ITEMS], uint32_t lo,
                                            uint32_t hi, bool full, V* stage, uint32_t* scr,
                                            TileShared<2>& sh, uint32_t par, const OUT& out, bool ok,
                                            AfterCounts after_counts) {
    using G = TileGeom<V, THREADS, 2, ITEMS * static_cast<int>(sizeof(V))>;
    constexpr uint32_t AU = G::kAU;
    constexpr int W = THREADS / 32;
    static_assert(ITEMS <= 16 && W <= 32, "16-bit packed warp counts, one lane per warp");
    uint32_t* wsum = scr;      // [W] packed class totals of each warp
    uint32_t* wpre = scr + W;  // [W] packed class prefixes of each warp

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t e0 = tid * ITEMS;

    // ---- pass 1: class-1 and valid masks, thread counts, warp prefixes
    uint32_t m1 = 0, mv = 0;
    if (full) {
#pragma unroll
        for (int j = 0; j < ITEMS; j++) m1 |= (d(v[j]) & 1u) << j;
        mv = (1u << ITEMS) - 1u;
    } else {
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            if (e0 + j >= lo && e0 + j < hi) {
                m1 |= (d(v[j]) & 1u) << j;
                mv |= 1u << j;
            }
        }
    }
    const uint32_t n1 = static_cast<uint32_t>(__popc(m1));
    const uint32_t x = (static_cast<uint32_t>(__popc(mv)) - n1) | (n1 << 16);
    const uint32_t incl = warp_incl_scan(x);
    if (lane == 31) wsum[warp] = incl;
    if (__syncthreads_or(!ok)) return false;  // (A)
    after_counts();

    // ---- the two class runs (warp 0; lane c = class c), warp prefixes
    if (warp == 0) {
        const uint32_t wt = lane < W ? wsum[lane] : 0u;
        const uint32_t wi = warp_incl_scan(wt);
        if (lane < W) wpre[lane] = wi - wt;
        const uint32_t tot = __shfl_sync(0xffffffffu, wi, 31);
        if (lane < 2) {
            const uint32_t c = static_cast<uint32_t>(lane);
            const uint32_t cc = c ? (tot >> 16) : (tot & 0xffffu);
            const uint32_t cur = sh.cursor[par][c];
            const uint32_t dst = FORWARD ? cur : cur - cc;
            const uint32_t q0 = c ? (tot & 0xffffu) + AU : 0u;  // class 0's room comes first
            const uint32_t st = q0 + (((out.phase() + dst) - q0) & (AU - 1u));
            sh.cursor[par ^ 1u][c] = FORWARD ? cur + cc : dst;
            sh.run_start[c] = st;
            sh.run_cnt[c] = cc;
            sh.run_dst[c] = dst;
        }
    }
    // the stage is about to be rewritten: the previous tile's bulk stores
    // must have finished reading it
    if (tid < 2) bulk_wait_read<0>();
    __syncthreads();  // (B)

    // ---- pass 2: stage slot = class base + thread prefix + rank in the thread
    {
        const uint32_t pre = wpre[warp] + incl - x;
        const uint32_t b0 = sh.run_start[0] + (pre & 0xffffu);
        const uint32_t b1 = sh.run_start[1] + (pre >> 16);
        const uint32_t m0 = mv & ~m1;
#pragma unroll
        for (int j = 0; j < ITEMS; j++) {
            const uint32_t below = (1u << j) - 1u;
            const uint32_t slot = ((m1 >> j) & 1u) ? b1 + static_cast<uint32_t>(__popc(m1 & below))
                                                   : b0 + static_cast<uint32_t>(__popc(m0 & below));
            if ((mv >> j) & 1u) stage[slot] = v[j];
        }
    }
    fence_proxy_async_smem();
    __syncthreads();  // (C)

    // ---- write-out: as tile_scatter
    if (tid < 2) {
        const uint32_t s = sh.run_start[tid], cc = sh.run_cnt[tid];
        uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
        if (head > cc) head = cc;
        const uint32_t body = ((cc - head) / AU) * AU;
        uint32_t a0 = sh.run_dst[tid] + head, sl = s + head;
        const uint32_t a1 = a0 + body;
        while (a0 < a1) {  // one piece per destination buffer
            const uint32_t b = out.piece_end(a0, a1);
            bulk_store_s2g(out.at(a0), stage + sl, (b - a0) * sizeof(V));
            sl += b - a0;
            a0 = b;
        }
        bulk_commit();
    } else if (tid >= 32 && tid < 32 + 2 * 2 * static_cast<int>(AU)) {
        const uint32_t c = (tid - 32) / (2 * AU), q = (tid - 32) % (2 * AU);
        const uint32_t s = sh.run_start[c], cc = sh.run_cnt[c];
        uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
        if (head > cc) head = cc;
        const uint32_t body = ((cc - head) / AU) * AU;
        uint32_t off = 0xffffffffu;
        if (q < AU) {
            if (q < head) off = q;
        } else if (head + body + (q - AU) < cc) {
            off = head + body + (q - AU);
        }
        if (off != 0xffffffffu) *out.at(sh.run_dst[c] + off) = stage[s + off];
    }
    return true;
}

// ------------------------------------------------------------ 17..64 classes --
// With more than 16 classes the per-thread nibble counters no longer fit in a
// register pair, so ranks come from the warp instead (striped layout):
//  * in round j lane l of warp w holds tile element w*32*ITEMS + j*32 + l, so
//    (warp, round, lane) is input order; TMA places these tiles without
//    swizzle, so a round is one conflict-free shared load per lane;
//  * the lanes of a round that share a class are found from log2(M) ballots
//    of the class bits (peers = AND over bits of ballot or ~ballot), the rank
//    in the round is popc(peers & lanemask_lt);
//  * lane k keeps the warp's running count of class k (and k + 32 when M = 64)
//    in a register, read by one shuffle per element and advanced by a popcount
//    of the lanes of class k (the same AND over bits with k's own bits);
//  * warp 0 turns the [warp][class] counts into class runs at the
//    destination's 16-byte phase and stage bases per (warp, class), which pass
//    2 reads from shared memory; the write-out is that of tile_scatter.
// The step is bound by the ALU pipe (ncu, m = 64: 72 % of peak), so full
// tiles take a path without the bounds tests and selects.

// A warp's striped elements of a tile that TMA placed in shared memory
// without swizzle (element e at tile[e]).
template <class V, int ITEMS>
__device__ __forceinline__ void take_striped(const V* tile, V (&v)[ITEMS]) {
    const V* p = tile + (threadIdx.x >> 5) * 32u * ITEMS + (threadIdx.x & 31u);
#pragma unroll
    for (int j = 0; j < ITEMS; j++) v[j] = p[j * 32];
}

template <class V, class D, int M, int THREADS, bool FORWARD, bool FULL, class OUT,
          class AfterCounts, int ITEMS>
__device__ __forceinline__ bool tile_scatter_wide_impl(const D& d, const V (&v)[ITEMS],
                                                       uint32_t lo, uint32_t hi, V* stage,
                                                       uint32_t* wtab, TileShared<M>& sh,
                                                       uint32_t par, const OUT& out, bool ok,
                                                       AfterCounts after_counts) {
    using G = TileGeom<V, THREADS, M, ITEMS * static_cast<int>(sizeof(V))>;
    constexpr uint32_t AU = G::kAU;
    constexpr int W = THREADS / 32;
    constexpr int B = M == 32 ? 5 : 6;
    static_assert(M == 32 || M == 64, "17..64 classes (class bound 32 or 64)");
    static_assert(32 * ITEMS <= 512, "warp ranks < 512 fit the packed 16-bit slots");

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt = lanemask_lt();
    const uint32_t ew = static_cast<uint32_t>(warp) * 32u * ITEMS + static_cast<uint32_t>(lane);

    // ---- pass 1: warp ranks.  Lane k builds the mask of the lanes holding
    // class k (and k + 32): one LOP3 per class bit against its own bits; an
    // element's peers are then lane (c mod 32)'s mask, fetched by a shuffle.
    uint32_t inv[5];  // bit i of the lane id set: ballot as is, else its complement
#pragma unroll
    for (int i = 0; i < 5; i++) inv[i] = ((lane >> i) & 1) ? 0u : 0xffffffffu;
    uint32_t runs = 0;       // warp's running count of class lane (low 16 bits), lane + 32 (high)
    uint32_t rk[ITEMS / 2];  // ranks, two per word
#pragma unroll
    for (int q = 0; q < ITEMS / 2; q++) rk[q] = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        bool valid = true;
        if constexpr (!FULL) {
            const uint32_t e = ew + j * 32u;
            valid = e >= lo && e < hi;
        }
        const uint32_t c = valid ? d(v[j]) : 0u;
        uint32_t com = FULL ? 0xffffffffu : __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int i = 0; i < 5; i++) com &= __ballot_sync(0xffffffffu, (c >> i) & 1u) ^ inv[i];
        uint32_t peers, base;
        // a shuffle's source lane is taken mod 32: c selects lane c mod 32
        const uint32_t x = __shfl_sync(0xffffffffu, runs, c);
        if constexpr (B == 6) {
            const uint32_t hi = (c >> 5) & 1u;
            const uint32_t b5 = __ballot_sync(0xffffffffu, hi);
            const uint32_t com1 = com & b5;
            // lanes of class (c mod 32) with the same sixth bit as c
            const uint32_t p = __shfl_sync(0xffffffffu, com, c);
            peers = p & (b5 ^ (hi - 1u));
            base = __byte_perm(x, 0u, 0x4410u + hi * 0x22u);  // low or high 16 bits
            const uint32_t n1 = static_cast<uint32_t>(__popc(com1));
            runs += (static_cast<uint32_t>(__popc(com)) - n1) + (n1 << 16);
        } else {
            peers = __shfl_sync(0xffffffffu, com, c);
            base = x;
            runs += static_cast<uint32_t>(__popc(com));
        }
        const uint32_t r = base + __popc(peers & lt);
        rk[j >> 1] |= r << (16 * (j & 1));
    }
    wtab[warp * M + lane] = runs & 0xffffu;
    if constexpr (M == 64) wtab[warp * M + lane + 32] = runs >> 16;
    if (__syncthreads_or(!ok)) return false;  // (A)
    after_counts();

    // ---- class runs (warp 0, lane = classes lane and lane + 32): totals over
    // warps, runs at the destination's 16-byte phase, stage base per (warp, class)
    if (warp == 0) {
        constexpr int KL = M / 32;
        uint32_t st_prev = 0;  // end of the rooms of the classes scanned so far
#pragma unroll
        for (int h = 0; h < KL; h++) {
            const uint32_t c = static_cast<uint32_t>(lane + 32 * h);
            uint32_t pre[W];
            uint32_t cc = 0;
#pragma unroll
            for (int w = 0; w < W; w++) {
                pre[w] = cc;
                cc += wtab[w * M + c];
            }
            const uint32_t cur = sh.cursor[par][c];
            const uint32_t dst = FORWARD ? cur : cur - cc;
            const uint32_t room = cc + AU;
            const uint32_t incl = warp_incl_scan(room);
            const uint32_t q0 = st_prev + incl - room;
            st_prev += __shfl_sync(0xffffffffu, incl, 31);
            const uint32_t st = q0 + (((out.phase() + dst) - q0) & (AU - 1u));
#pragma unroll
            for (int w = 0; w < W; w++) wtab[w * M + c] = st + pre[w];
            sh.cursor[par ^ 1u][c] = FORWARD ? cur + cc : dst;
            sh.run_start[c] = st;
            sh.run_cnt[c] = cc;
            sh.run_dst[c] = dst;
        }
    }
    // the stage is about to be rewritten: the previous tile's bulk stores
    // must have finished reading it
    if (tid < M) bulk_wait_read<0>();
    __syncthreads();  // (B)

    // ---- pass 2: stage slot = base of (warp, class) + warp rank
    const uint32_t* wb = wtab + warp * M;
#pragma unroll
    for (int j = 0; j < ITEMS; j++) {
        bool valid = true;
        if constexpr (!FULL) {
            const uint32_t e = ew + j * 32u;
            valid = e >= lo && e < hi;
        }
        if (valid) stage[wb[d(v[j])] + ((rk[j >> 1] >> (16 * (j & 1))) & 0xffffu)] = v[j];
    }
    fence_proxy_async_smem();
    __syncthreads();  // (C)

    // ---- write-out: bulk store of each run's aligned interior; all threads
    // store the unaligned heads and tails
    if (tid < M) {
        const uint32_t s = sh.run_start[tid], cc = sh.run_cnt[tid];
        uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
        if (head > cc) head = cc;
        const uint32_t body = ((cc - head) / AU) * AU;
        uint32_t a0 = sh.run_dst[tid] + head, sl = s + head;
        const uint32_t a1 = a0 + body;
        while (a0 < a1) {
            const uint32_t b = out.piece_end(a0, a1);
            bulk_store_s2g(out.at(a0), stage + sl, (b - a0) * sizeof(V));
            sl += b - a0;
            a0 = b;
        }
        bulk_commit();
    }
    for (int t = tid; t < M * 2 * static_cast<int>(AU); t += THREADS) {
        const uint32_t c = static_cast<uint32_t>(t) / (2 * AU), q = static_cast<uint32_t>(t) % (2 * AU);
        const uint32_t s = sh.run_start[c], cc = sh.run_cnt[c];
        uint32_t head = (AU - (s & (AU - 1u))) & (AU - 1u);
        if (head > cc) head = cc;
        const uint32_t body = ((cc - head) / AU) * AU;
        uint32_t off = 0xffffffffu;
        if (q < AU) {
            if (q < head) off = q;
        } else if (head + body + (q - AU) < cc) {
            off = head + body + (q - AU);
        }
        if (off != 0xffffffffu) *out.at(sh.run_dst[c] + off) = stage[s + off];
    }
    return true;
}

template <class V, class D, int M, int THREADS, bool FORWARD, class OUT, class AfterCounts,
          int ITEMS>
__device__ __forceinline__ bool tile_scatter_wide(const D& d, const V (&v)[ITEMS],
                                                  uint32_t lo, uint32_t hi, bool full, V* stage,
                                                  uint32_t* wtab, TileShared<M>& sh, uint32_t par,
                                                  const OUT& out, bool ok,
                                                  AfterCounts after_counts) {
    if (full)
        return tile_scatter_wide_impl<V, D, M, THREADS, FORWARD, true>(d, v, lo, hi, stage, wtab, sh,
                                                                     par, out, ok, after_counts);
    return tile_scatter_wide_impl<V, D, M, THREADS, FORWARD, false>(d, v, lo, hi, stage, wtab, sh,
                                                                  par, out, ok, after_counts);
}

}  // namespace mdx
