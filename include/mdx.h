/*
 * mdx.h -- C ABI of the B200-native m-discriminator (stable m-way partition).
 *
 * The operation (reference spec haskell_code/Mdiscr.hs:9-54, CPU ground truth
 * cuda_code/SeqMdiscr.h:10-57): every element maps to a class in [0, m); the
 * output holds all class-0 elements, then all class-1 elements, ..., each class
 * in input order, plus the m class sizes.
 *
 * Every entry point is asynchronous on the given stream, never calls exit(),
 * never allocates device memory per call (the caller passes a workspace sized
 * by mdx_workspace_size and initialised once by mdx_workspace_init), and
 * returns an mdx_status.  Device-side failures (a bounded wait that ran out)
 * are latched in the workspace and read back by mdx_workspace_error.
 *
 * A workspace serves one call at a time: calls that share a workspace must be
 * ordered (same stream, or synchronised).
 */
#ifndef MDX_H
#define MDX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* mdx_stream_t; /* == cudaStream_t; NULL = legacy default stream */

typedef enum {
    MDX_OK = 0,
    MDX_ERR_INVALID = 1,     /* bad argument (null pointer, m out of range, n too large, ...) */
    MDX_ERR_WORKSPACE = 2,   /* workspace too small or misaligned */
    MDX_ERR_CUDA = 3,        /* a CUDA runtime call failed (launch, copy, attribute query) */
    MDX_ERR_TIMEOUT = 4,     /* a device-side bounded wait ran out (latched in the workspace) */
    MDX_ERR_UNSUPPORTED = 5, /* valid request this build does not handle */
    MDX_ERR_SEGMENTS = 6,    /* malformed segment description */
    MDX_ERR_CANCELLED = 7    /* a served request withdrawn before launch (mdx_server_cancel) */
} mdx_status;

/* Element layouts.  U32: one unsigned 32-bit value, class from the value
 * (InType = unsigned int of Mod4/Mod8/Mod<N>, HelpersCommon.h:587-596,840-849,
 * 1200-1210).  REC8: 8-byte record {u32 key; u32 payload}, class from the key
 * (ModArray<N,2>, MdiscrHost_arrays.cu.h:26-36 with LEN = 2).  REC16: 16-byte
 * record {u32 key; 12 bytes of payload}, 16-byte aligned (ModArray<N,4>);
 * plain partitions only (mdx_partition, mdx_partition_records): the
 * segmented, distributed and no-allocation entry points return
 * MDX_ERR_UNSUPPORTED for it. */
typedef enum { MDX_ELEM_U32 = 0, MDX_ELEM_REC8 = 1, MDX_ELEM_REC16 = 2 } mdx_elem;

/* Discriminator families.  MOD: class = key % m (Mod<N>::apply,
 * HelpersCommon.h:1207-1209).  MASK: class = key & (m-1), m a power of two
 * (Mod4::apply / Mod8::apply, HelpersCommon.h:593-595, 846-848). */
typedef enum { MDX_DISCR_MOD = 0, MDX_DISCR_MASK = 1 } mdx_discr_kind;

typedef struct {
    int32_t kind;    /* mdx_discr_kind */
    uint32_t m;      /* number of classes, 1 <= m <= MDX_MAX_CLASSES (TupleType::cardinal) */
} mdx_discr;

#define MDX_MAX_CLASSES 64u
#define MDX_MAX_ELEMS 0xFFFFFFFFull /* class sizes are u32, as the reference's TupleType */

/* Bytes of workspace mdx_partition needs for n elements of `elem` with m
 * classes.  Replaces the per-call cudaMalloc of d_tr_in / cond_res / inds_res
 * in mdiscr (cuda_code/MdiscrHost_optimized_clean.cu.h:43-45). */
size_t mdx_workspace_size(uint64_t n, mdx_elem elem, uint32_t m);

/* Bytes of workspace mdx_partition_segmented needs.  Replaces the nine
 * per-call N-sized cudaMallocs of mdiscrSegm (cuda_code/MdiscrSegmHost.cu.h:60-68). */
size_t mdx_segmented_workspace_size(uint64_t n, uint64_t num_segments, mdx_elem elem, uint32_t m);

/* Bytes of workspace mdx_mdiscr_segm (head-flag segment input) needs: the
 * segmented workspace for up to n segments plus room for the offsets. */
size_t mdx_mdiscr_segm_workspace_size(uint64_t n, mdx_elem elem, uint32_t m);

/* Zero a freshly allocated workspace (once, before its first use). */
mdx_status mdx_workspace_init(void* d_ws, size_t ws_bytes, mdx_stream_t stream);

/* Synchronise `stream`, return the latched device error of the workspace
 * (MDX_OK; MDX_ERR_TIMEOUT: a bounded wait ran out; MDX_ERR_SEGMENTS:
 * malformed segments; MDX_ERR_INVALID: inconsistent class counts handed to
 * mdx_dist_scatter) and clear it. */
mdx_status mdx_workspace_error(void* d_ws, mdx_stream_t stream);

/*
 * Plain stable partition of n elements.  Replaces
 *   template<class DISCR> DISCR::TupleType mdiscr(n, num_hwd_thds, d_in, d_out)
 *     (cuda_code/MdiscrHost_optimized_clean.cu.h:9-15)
 * and
 *   template<class DISCR> void mdiscr(n, in, out, int* sizes)
 *     (cuda_code/MdiscrHost_baseline.cu.h:23-28).
 *
 * d_in, d_out : device arrays of n elements (distinct, non-overlapping).
 * d_sizes     : device array of m u32 -- the class sizes (tuple form); may be NULL.
 * d_headflags : device array of n u32 -- sizes in the reference's head-flag form
 *               (count_c at offset_c for every non-empty class, 0 elsewhere,
 *               SeqMdiscr.h:44-49); may be NULL.
 */
mdx_status mdx_partition(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                         mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                         void* d_ws, size_t ws_bytes, mdx_stream_t stream);

/* mdx_partition that also records `ev_count_done` (a cudaEvent_t, may be
 * NULL) on the stream between its counting and its scattering kernel, so a
 * caller can time the two phases separately with CUDA events. */
mdx_status mdx_partition_timed(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                               mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                               void* d_ws, size_t ws_bytes, mdx_stream_t stream,
                               void* ev_count_done);

/*
 * Reference-shaped synchronous form of mdx_partition: returns the m class
 * sizes on the host in h_sizes, as mdiscr<DISCR> returns its TupleType by value
 * (MdiscrHost_optimized_clean.cu.h:149).  num_hwd_thds is accepted for
 * signature parity and ignored (it only shaped the reference's transposed
 * layout, MdiscrHost_optimized_clean.cu.h:24-26).
 */
mdx_status mdx_mdiscr(uint32_t n, uint32_t num_hwd_thds, const void* d_in, void* d_out,
                      mdx_elem elem, mdx_discr discr, uint32_t* h_sizes,
                      void* d_ws, size_t ws_bytes, mdx_stream_t stream);

/*
 * Segmented stable partition: each segment [d_offsets[s], d_offsets[s+1]) of
 * the n elements is partitioned independently (mdiscrSegm,
 * cuda_code/MdiscrSegmHost.cu.h:36-42; validated per segment against seqMdiscr
 * by MdiscrSegmTest.cu:8-41).
 *
 * d_offsets      : device u64[num_segments + 1], non-decreasing, [0] = 0, [S] = n.
 * d_seg_sizes    : device u32[num_segments * m], row s = class sizes of segment s; may be NULL.
 * d_headflags    : device u32[n] -- per-segment head-flag sizes relative to the
 *                  segment start, the form mdiscrSegm writes into new_sizes
 *                  (MdiscrSegmKernels.cu.h:89-114); may be NULL.
 * Segments that do not tile [0, n) exactly latch MDX_ERR_SEGMENTS in the
 * workspace (read it with mdx_workspace_error).  m <= 16 in this build.
 */
mdx_status mdx_partition_segmented(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                   mdx_discr discr, const uint64_t* d_offsets,
                                   uint64_t num_segments, uint32_t* d_seg_sizes,
                                   uint32_t* d_headflags, void* d_ws, size_t ws_bytes,
                                   mdx_stream_t stream);

/*
 * Segmented partition in which every segment has its own class count:
 * segment s uses class = key % d_seg_m[s], 1 <= d_seg_m[s] <= m_max <= 16
 * (no reference counterpart: mdiscrSegm fixes one DISCR per call,
 * MdiscrSegmHost.cu.h:36-42).  It lets independent requests with different m
 * share one batched launch.  Rows of d_seg_sizes are m_max wide (classes at
 * or above a segment's m count 0).  Workspace: mdx_segmented_workspace_size
 * with m = m_max.  A d_seg_m entry outside [1, m_max] latches
 * MDX_ERR_SEGMENTS (the kernel clamps it).
 */
mdx_status mdx_partition_segmented_multi(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                         const uint32_t* d_seg_m, uint32_t m_max,
                                         const uint64_t* d_offsets, uint64_t num_segments,
                                         uint32_t* d_seg_sizes, uint32_t* d_headflags,
                                         void* d_ws, size_t ws_bytes, mdx_stream_t stream);

/*
 * Reference-shaped segmented form with head-flag segment sizes in and out:
 *   template<class DISCR> void mdiscrSegm(n, in, int* segment_sizes, out, int* new_sizes)
 *     (cuda_code/MdiscrSegmHost.cu.h:36-42)
 * d_segment_sizes: device i32[n], length of the segment at each segment start,
 * 0 elsewhere.  d_new_sizes: device i32[n] (head-flag output).  Needs a
 * workspace of mdx_mdiscr_segm_workspace_size(n, elem, m) bytes (the segment
 * count is only known on the device).  Malformed flags latch
 * MDX_ERR_SEGMENTS in the workspace (read it with mdx_workspace_error).
 */
mdx_status mdx_mdiscr_segm(uint32_t n, const void* d_in, const int32_t* d_segment_sizes,
                           void* d_out, int32_t* d_new_sizes, mdx_elem elem, mdx_discr discr,
                           void* d_ws, size_t ws_bytes, mdx_stream_t stream);

/*
 * CUDA-graph capture and replay (no reference counterpart: the reference launches
 * every kernel from the host each call, cuda_code/MdiscrSegmHost.cu.h:70-158).
 * mdx_graph_partition / mdx_graph_partition_segmented record one call with
 * the given arguments into a CUDA graph (captured on a private stream of the
 * current device; nothing runs yet); mdx_graph_launch replays it on `stream`
 * (the pointers are fixed, their contents may change between replays; replays
 * sharing a workspace must not overlap); mdx_graph_destroy frees it.
 */
typedef struct mdx_graph_st* mdx_graph;

mdx_status mdx_graph_partition(mdx_graph* graph, const void* d_in, void* d_out, uint64_t n,
                               mdx_elem elem, mdx_discr discr, uint32_t* d_sizes,
                               uint32_t* d_headflags, void* d_ws, size_t ws_bytes);

mdx_status mdx_graph_partition_segmented(mdx_graph* graph, const void* d_in, void* d_out,
                                         uint64_t n, mdx_elem elem, mdx_discr discr,
                                         const uint64_t* d_offsets, uint64_t num_segments,
                                         uint32_t* d_seg_sizes, uint32_t* d_headflags,
                                         void* d_ws, size_t ws_bytes);

mdx_status mdx_graph_launch(mdx_graph graph, mdx_stream_t stream);

mdx_status mdx_graph_destroy(mdx_graph graph);

/*
 * mdx_partition for callers that cannot allocate device memory (no
 * counterpart in the reference): code running inside a device allocator or
 * memory-pool callback, a plugin whose host forbids device allocations after
 * start-up, or a loop that cannot afford cudaMalloc's device-wide
 * synchronisation, and that has no workspace to hand in.  Same arguments and
 * results as mdx_partition minus the workspace: the scratch is a fixed
 * 525,312-byte array inside the library, present on every GPU that loads it
 * until the process exits.
 *   - m <= 16 at any n < 2^32; m > 16 returns MDX_ERR_WORKSPACE (the request
 *     needs more scratch than the array holds) before anything is launched.
 *   - The first call on a device does a one-time set-up for that device
 *     (looks up the array's device address, sets kernel attributes): make it
 *     before any stream capture.
 *   - All calls share the array; each call clears what must start at zero on
 *     its stream.  Calls that may overlap on the GPU race: keep them in one
 *     stream or order them.
 *   - A device-side wait that runs out (a tile copy that never lands within a
 *     second) leaves that call's output incomplete and latches a bit in the
 *     array's error word, which later calls keep; mdx_partition_noalloc_error
 *     reports it.
 * Allocates nothing: no cudaMalloc, no cudaFree, no allocating library call.
 */
mdx_status mdx_partition_noalloc(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                 mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                                 mdx_stream_t stream);

/*
 * Device-side errors latched by mdx_partition_noalloc calls on the current
 * device since the last query (no counterpart in the reference): MDX_OK, or
 * MDX_ERR_TIMEOUT when a wait ran out.  Reads and clears the built-in array's
 * error word on `stream` and synchronizes that stream; allocates nothing.
 */
mdx_status mdx_partition_noalloc_error(mdx_stream_t stream);

/*
 * Wide elements.  Records of record_bytes (a multiple of 4) whose class comes
 * from their first u32 word: mdiscr<ModArray<N,LEN>, LEN> over arrays of LEN
 * unsigned ints (cuda_code/MdiscrHost_arrays.cu.h:26-36,250-430) is
 * mdx_partition_records with record_bytes = 4 * LEN.  Columns permuted
 * together (cuda_code/MdiscrHost_tuples.cu.h:262-429 partitions a u32, a u8 and
 * a bool array by a functor of the first): column 0 is the u32 key the class
 * comes from, the others (1, 2, 4 or 8 bytes per row, up to 8 columns in all)
 * follow its rows.  Both build {key, row} 8-byte records, partition them with
 * the 8-byte-record kernels and gather the rows (4- and 8-byte records take the
 * direct paths); workspaces from the two size functions (they hold the record
 * arrays: about 16 bytes per row).  Outputs must not overlap any input.
 */
size_t mdx_records_workspace_size(uint64_t n, uint32_t record_bytes, uint32_t m);
mdx_status mdx_partition_records(const void* d_in, void* d_out, uint64_t n, uint32_t record_bytes,
                                 mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                                 void* d_ws, size_t ws_bytes, mdx_stream_t stream);

typedef struct {
    const void* in;      /* device, n rows */
    void* out;           /* device, n rows */
    uint32_t elem_bytes; /* 1, 2, 4 or 8 (column 0: 4, the key) */
} mdx_column;

size_t mdx_columns_workspace_size(uint64_t n, uint32_t m);
mdx_status mdx_partition_columns(const mdx_column* cols, uint32_t num_cols, uint64_t n,
                                 mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                                 void* d_ws, size_t ws_bytes, mdx_stream_t stream);

/*
 * Distributed plain partition (no reference counterpart: the reference is
 * single-GPU; this is mdiscr<DISCR> of cuda_code/MdiscrHost_optimized_clean.cu.h:9-15
 * over one array spread across R ranks, one GPU each).  Rank r holds a
 * contiguous chunk of the global input; the global stable partition is written
 * into R output chunks: chunk q holds output positions
 * [q * out_chunk, (q + 1) * out_chunk) within [0, n_total) (so trailing chunks
 * may be short or empty), the last chunk every position from
 * (R - 1) * out_chunk on.
 *   1. mdx_dist_count: count this rank's chunk; its m class counts go to
 *      d_counts (device).
 *   2. the caller all-gathers the counts of every rank into d_all_counts
 *      ([R][m], rank-major; one tiny collective, e.g. an NCCL all-gather);
 *   3. mdx_dist_scatter (same workspace, same n_local): each element is stored
 *      straight into the chunk that owns its output position -- through
 *      out_chunks[q], a HOST array of R device pointers, peers' chunks mapped
 *      into this process (mdx_ipc_*) -- by the same kernel that ranks it; the
 *      global m sizes go to d_sizes (device, may be NULL).  A barrier across
 *      ranks (any collective after this call on the same stream) must precede
 *      reading an output chunk.
 * m <= 64; out_chunk a multiple of 16 bytes of elements; chunk pointers 16-byte aligned; n_total < 2^32.  Counts that do
 * not match this rank's own count or do not add up to n_total make the
 * scatter write nothing and latch an error (mdx_workspace_error:
 * MDX_ERR_INVALID).
 */
mdx_status mdx_dist_count(const void* d_in, uint64_t n_local, mdx_elem elem, mdx_discr discr,
                          uint32_t* d_counts, void* d_ws, size_t ws_bytes, mdx_stream_t stream);

mdx_status mdx_dist_scatter(const void* d_in, uint64_t n_local, mdx_elem elem, mdx_discr discr,
                            const uint32_t* d_all_counts, uint32_t num_ranks, uint32_t rank,
                            void* const* out_chunks, uint64_t out_chunk, uint64_t n_total,
                            uint32_t* d_sizes, void* d_ws, size_t ws_bytes, mdx_stream_t stream);

/*
 * Peer mappings for mdx_dist_scatter's output chunks (CUDA IPC, no multicast):
 * mdx_ipc_get_handle gives the 64-byte handle of the allocation holding d_ptr
 * and d_ptr's offset in it; another process on the same node opens it with
 * mdx_ipc_open (peer access enabled on demand) and releases it with
 * mdx_ipc_close(d_ptr, offset).
 */
mdx_status mdx_ipc_get_handle(const void* d_ptr, void* handle, uint64_t* offset);
mdx_status mdx_ipc_open(const void* handle, uint64_t offset, void** d_ptr);
mdx_status mdx_ipc_close(void* d_ptr, uint64_t offset);

/*
 * Serving loop (continuous batching; no reference counterpart -- the
 * reference has one synchronous call per array).  Requests are u32 arrays
 * with their own m (class = value % m, 1 <= m <= m_max <= 16); their buffers
 * are device memory or page-locked host memory (pageable memory is refused
 * with MDX_ERR_INVALID).  The server owns budget_bytes of device memory (an
 * input and an output ring), admits requests in FIFO order as ring space
 * allows, coalesces consecutive admitted requests into batched segmented
 * launches on up to num_streams streams at once (new requests are admitted
 * and launched while earlier batches run), and records every request's
 * latency from submit to completion.  Long requests in device memory
 * (direct_min_elems) still take their place in the pool but are partitioned
 * in place by the plain kernels, one launch each, without the pool's copies.
 * Batched (short) requests run on streams of the device's highest priority,
 * in-place (long) ones on its lowest, so short requests are not parked behind
 * long ones on the GPU.  A batch's stream is free again as soon as that batch
 * is done.
 */
typedef struct mdx_server_st* mdx_server;

typedef struct {
    uint64_t budget_bytes;        /* device memory for request data (both rings) */
    uint32_t num_streams;         /* batches in flight at once (0: 2) */
    uint32_t max_batch_requests;  /* requests per batched launch (0: 1024, <= 65535) */
    uint64_t max_batch_elems;     /* elements per batched launch (0: 2^24, at most the ring);
                                     also the longest request the pool takes */
    uint32_t m_max;               /* largest m a request may use (0: 16, <= 16) */
    uint64_t direct_min_elems;    /* requests at least this long whose buffers are device
                                     memory are partitioned in place, without the pool's
                                     copies (0: 2^20; UINT64_MAX: never) */
} mdx_server_config;

typedef struct {
    uint64_t submitted, completed, batches, elements;
    uint64_t waiting, inflight_batches;
    double p50_s, p99_s, mean_s;  /* latency of completed requests, submit to completion */
    double window_s;              /* from the last reset to the last completion */
    uint64_t direct;              /* requests partitioned in place */
    double queue_p50_s, queue_p99_s;  /* submit -> launch of the request's batch (or lane) */
    double exec_p50_s, exec_p99_s;    /* launch -> completion stamp */
    double launch_busy_s;             /* host time spent issuing launches since the reset */
} mdx_server_stats;

mdx_status mdx_server_create(mdx_server* server, const mdx_server_config* config);
/* in: n values; out: n values; sizes: m class sizes.  Returns immediately. */
mdx_status mdx_server_submit(mdx_server server, const uint32_t* in, uint32_t* out, uint32_t* sizes,
                             uint64_t n, uint32_t m, uint64_t* ticket);
/* Block until the request is done; its latency in seconds.  MDX_ERR_CANCELLED
 * for a request withdrawn by mdx_server_cancel (its outputs are untouched). */
mdx_status mdx_server_wait(mdx_server server, uint64_t ticket, double* latency_s);
/* Withdraw a request that has not been launched yet (still queued or
 * admitted): MDX_OK, and its wait returns MDX_ERR_CANCELLED; MDX_ERR_INVALID
 * when the ticket is unknown or the request is already on the GPU or done. */
mdx_status mdx_server_cancel(mdx_server server, uint64_t ticket);
mdx_status mdx_server_get_stats(mdx_server server, mdx_server_stats* stats);
mdx_status mdx_server_reset_stats(mdx_server server);
/* Finishes the work already submitted, then frees everything. */
mdx_status mdx_server_destroy(mdx_server server);

/*
 * Run-time knobs of the kernels (no reference counterpart; the reference fixes
 * its block shapes at compile time with -D macros swept by cuda_code/run.py).
 * Entries are kept per (element layout, class bound = smallest power of two
 * >= m, ceil(log2 n)); mdx_set_tuning sets every n bucket in
 * [log2_n_lo, log2_n_hi].  Zero fields keep the built-in default.
 */
typedef struct {
    uint32_t plain_ctas_per_sm;  /* plain path: CTAs per SM of the chunk grid (0: as many as fit) */
    uint32_t run_tiles;          /* segmented: tiles per run of a large segment (default 8) */
    uint32_t group_batch;        /* segmented: small-segment groups per work item (default 8, at most 32) */
    uint32_t plain_two_kernel;   /* plain path: 1 = count and scatter as two kernels; 0 (default) =
                                    one cooperative kernel where the input allows TMA */
    uint32_t pool_pct;           /* one-kernel plain path: % of every chunk's tiles that the CTAs
                                    share by ticket at the end of each phase (0: default 10;
                                    100: none) */
    uint32_t mid_tiles;          /* segmented: a segment of more than one tile spanning at most this
                                    many tiles (2, the most the medium-segment kernel holds) is read
                                    once, counted and scattered from shared memory; 0 (default) and
                                    1: none, every segment longer than a tile goes through count +
                                    scatter runs */
    uint32_t tile_bytes;         /* plain path: bytes of a tile per thread, 64 (default, 0) or 32
                                    (tiles half as long: more CTAs busy on short inputs; count +
                                    scatter as two kernels; 4- and 8-byte elements) */
    uint32_t tile_threads;       /* plain path: threads of a scatter CTA, 256 (default, 0) or 512
                                    (64-byte tiles twice as long, half the per-tile steps; count +
                                    scatter as two kernels; 4- and 8-byte elements, m <= 16;
                                    takes precedence over tile_bytes) */
} mdx_tuning;

mdx_status mdx_set_tuning(mdx_elem elem, uint32_t m, uint32_t log2_n_lo, uint32_t log2_n_hi,
                          const mdx_tuning* tuning);
mdx_status mdx_get_tuning(mdx_elem elem, uint32_t m, uint64_t n, mdx_tuning* tuning);

/* Human-readable text of a status. */
const char* mdx_strerror(mdx_status s);

/*
 * Fault injection for tests (no reference counterpart; the reference exits on
 * any CUDA error, HelpersHost.cu.h:11-19): the `nth` device or page-locked
 * host allocation that the serving loop's set-up (mdx_server_create) makes
 * from now on fails as if memory were exhausted; 0 turns it off.  Lets a test
 * check that every failing allocation is reported (MDX_ERR_CUDA) and that
 * what was already allocated is freed.  Host-side only: no GPU fault.
 */
void mdx_test_inject_alloc_failure(uint32_t nth);

/*
 * Makes a device-side wait run out, for tests (no reference counterpart):
 * the one-kernel plain partition's grid barrier expects `extra_arrivals` more
 * CTAs than its grid has, so no arrival completes it, and waits at most
 * `wait_limit_ns` (0: the normal 1 s).  The call then latches
 * MDX_ERR_TIMEOUT in its workspace (mdx_workspace_error) and writes no
 * output; nothing faults or hangs.  After a timeout re-initialise the
 * workspace (mdx_workspace_init).  extra_arrivals = 0 restores normal calls.
 */
void mdx_test_set_barrier_shortfall(uint32_t extra_arrivals, uint64_t wait_limit_ns);

/* Library version string, e.g. "mdx 0.1.0 sm_100a". */
const char* mdx_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MDX_H */
