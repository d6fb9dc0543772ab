// mdx_server.cu -- serving loop: continuous batching of partition requests.
//
// A request is one u32 array of n elements with its own class count m
// (class = value % m, 1 <= m <= m_max <= 16); its input, output and sizes live
// either in device memory or in page-locked host memory (both are reachable
// from kernels through unified addressing).  The server owns a device pool of
// `budget_bytes`: an input ring and an output ring of equal size.
//
//  * Admission: a submitted request waits in FIFO order until its n elements
//    fit in the rings; admitted requests hold consecutive ring slots, so any
//    run of them is one contiguous array.
//  * Scheduling: whenever admitted requests are waiting and one of the
//    `num_streams` batch slots is free, the scheduler thread takes the longest
//    contiguous run of them (up to max_batch_requests / max_batch_elems) and
//    issues, on that slot's stream: a gather kernel copying every request's
//    input into its ring slot, the per-segment-m segmented partition
//    (mdx_partition_segmented_multi: one segment per request), a scatter
//    kernel copying results and class sizes back to each request, and an
//    event whose completion the poller thread stamps.  Requests that arrive while
//    batches run are admitted as ring space frees and launched on another
//    stream: their work overlaps the batches already on the device.
//  * In place: a request of at least direct_min_elems whose buffers are all
//    device memory (and do not overlap) takes no ring space; it is admitted in
//    its FIFO turn and partitioned by the plain kernels straight on its own
//    buffers, queued on four lanes (a stream, a workspace and a launcher
//    thread each, up to four requests in stream order on each), so
//    the long requests that carry most elements skip the pool's two copies
//    and do not cut the runs of short requests that share a batch.
//  * Priorities: the batch streams (short requests) are created with the
//    device's highest stream priority and the in-place lanes with its lowest,
//    so the GPU schedules the blocks of a short request's kernels ahead of
//    the queued blocks of long ones instead of parking them behind.
//  * Completion: a batch slot is free again as soon as its own batch is
//    done; ring space is released in admission order (every allocation
//    carries a done mark, the ring's tail advances over finished ones);
//    waiters are woken; the latency of every request (submit to completion
//    stamp) goes into the p50 / p99 statistics.
//  * Cancellation: a request that has not been launched yet can be
//    withdrawn (mdx_server_cancel); its wait then returns MDX_ERR_CANCELLED.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/mdx.h"

namespace mdx {
// mdx_partition without the cooperative one-kernel path (mdx_capi.cu): the
// in-place lanes run next to the batches and to each other.
mdx_status partition_two_kernel(const void* d_in, void* d_out, uint64_t n, mdx_elem elem,
                                mdx_discr discr, uint32_t* d_sizes, uint32_t* d_headflags,
                                void* d_ws, size_t ws_bytes, mdx_stream_t stream);
namespace server {

constexpr int kCopyThreads = 256;
constexpr uint64_t kDefaultBatchElems = 1ull << 24;  // elements per batched launch (default)
constexpr uint32_t kCopyChunk = 8192;  // elements per copy CTA

struct CopyJob {            // one request in a batch
    const uint32_t* src;    // gather: request input;  scatter: ring output
    uint32_t* dst;          // gather: ring input;     scatter: request output
    uint64_t n;
    const uint32_t* sizes_src;  // scatter only: this segment's row of class sizes
    uint32_t* sizes_dst;        // scatter only: the request's m sizes
    uint32_t m;
    uint32_t first_chunk;       // index of this job's first chunk in the launch
};

// One CTA per chunk of kCopyChunk elements over all the jobs of a launch
// (jobs in order of first_chunk; every job has n >= 1).  8 independent loads
// in flight per thread; accesses are coalesced 4-byte words, so the source
// and destination need no common alignment.
constexpr int kCopyUnroll = 8;
__global__ void __launch_bounds__(kCopyThreads) copy_jobs(const CopyJob* jobs, uint32_t num_jobs) {
    __shared__ uint32_t js;
    const uint32_t bid = blockIdx.x;
    if (threadIdx.x == 0) {  // the last job whose first chunk is <= bid
        uint32_t lo = 0, hi = num_jobs;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (jobs[mid].first_chunk <= bid) lo = mid; else hi = mid;
        }
        js = lo;
    }
    __syncthreads();
    const CopyJob j = jobs[js];
    const uint64_t a = static_cast<uint64_t>(bid - j.first_chunk) * kCopyChunk;
    if (a == 0 && j.sizes_dst != nullptr && threadIdx.x < j.m)
        j.sizes_dst[threadIdx.x] = j.sizes_src[threadIdx.x];
    if (a >= j.n) return;
    const uint32_t cnt = static_cast<uint32_t>(min(static_cast<uint64_t>(kCopyChunk), j.n - a));
    const uint32_t* src = j.src + a;
    uint32_t* dst = j.dst + a;
    for (uint32_t base = 0; base < cnt; base += kCopyThreads * kCopyUnroll) {
        uint32_t v[kCopyUnroll];
#pragma unroll
        for (int u = 0; u < kCopyUnroll; u++) {
            const uint32_t e = base + u * kCopyThreads + threadIdx.x;
            if (e < cnt) v[u] = __ldg(src + e);
        }
#pragma unroll
        for (int u = 0; u < kCopyUnroll; u++) {
            const uint32_t e = base + u * kCopyThreads + threadIdx.x;
            if (e < cnt) dst[e] = v[u];
        }
    }
}

// True if p points into device memory (not host memory mapped for the device).
inline bool is_device_memory(const void* p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice;
}

// The device-side address of a buffer, or null when kernels cannot reach it
// (pageable host memory, unknown pointers).
template <class T>
T* device_view(T* p) {
    if (p == nullptr) return nullptr;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (attr.type == cudaMemoryTypeUnregistered) return nullptr;
    return static_cast<T*>(attr.devicePointer);
}

// Test fault injection (mdx_test_inject_alloc_failure): counts down the
// set-up's allocations; the one that brings the count to zero fails.
std::atomic<uint32_t> g_fail_countdown{0};
inline bool injected_failure() {
    uint32_t c = g_fail_countdown.load();
    while (c > 0)
        if (g_fail_countdown.compare_exchange_weak(c, c - 1)) return c == 1;
    return false;
}
template <class T>
cudaError_t dev_alloc(T** p, size_t bytes) {
    *p = nullptr;
    if (injected_failure()) return cudaErrorMemoryAllocation;
    return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}
template <class T>
cudaError_t pinned_alloc(T** p, size_t bytes) {
    *p = nullptr;
    if (injected_failure()) return cudaErrorMemoryAllocation;
    return cudaMallocHost(reinterpret_cast<void**>(p), bytes);
}

// A spin-wait hint to the core (lets its sibling hyperthread run).
inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
    __builtin_ia32_pause();
#elif defined(__aarch64__)
    asm volatile("yield" ::: "memory");
#endif
}

using Clock = std::chrono::steady_clock;
inline double now_s() {
    return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

struct Req {
    uint64_t id;
    uint64_t n;
    uint32_t m;
    const uint32_t* in;
    uint32_t* out;
    uint32_t* sizes;
    uint64_t off = 0;  // ring slot
    double t_submit = 0, t_launch = 0, t_done = 0;
    bool done = false;
    bool launched = false;
    bool direct = false;  // partitioned in place (long, device-resident): no ring copies
    mdx_status status = MDX_OK;  // MDX_ERR_CANCELLED when withdrawn before launch
    struct LiveEntry* ring = nullptr;  // its ring allocation (ring requests)
};

// One admitted ring allocation; `done` once its request finished or was
// cancelled.  The ring's tail advances over done entries in admission order.
struct LiveEntry {
    uint64_t off, n;
    bool done;
};

struct Batch;

// Completion of the work on one stream: the scheduler records an event after
// each unit of work (a batch, an in-place request) and queues it here with
// what to do when it is done.  One poller thread serves every stream's queue:
// it queries the front events (cudaEventQuery, without the server's lock),
// stamps the time and runs the actions under the lock.  Nothing is queued on
// the stream itself, so the stream never stalls on the host.  One polling
// thread, instead of a cudaEventSynchronize spinning per stream, keeps the
// server to one busy core however many streams it drives.
struct Waiter {
    std::deque<std::pair<cudaEvent_t, std::function<void(double)>>> q;  // under Server::mu
};

struct Slot {                   // one stream's worth of batch resources
    Waiter waiter;
    cudaStream_t stream = nullptr;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    uint32_t* d_seg_sizes = nullptr;  // [max_batch * m_max]
    // a batch's descriptors, packed: segment offsets [S + 1], per-segment m [S],
    // copy jobs [2 S] (gather then scatter); staged in pinned memory and
    // uploaded by one copy
    unsigned char* d_desc = nullptr;
    unsigned char* h_desc = nullptr;
    bool busy = false;
};

struct Server;

// Requests partitioned in place (long, in device memory): a stream and a
// workspace, up to kLaneDepth requests queued on it in stream order.  A call
// on ~10^6 elements fills well under half of the GPU, so several lanes run at
// once (served mix, every request at once: 2 lanes 187, 4 lanes 221, 8 lanes
// 224 Gelem/s).
constexpr uint32_t kLanes = 4;
constexpr uint32_t kLaneDepth = 4;
struct Lane {
    cudaStream_t stream = nullptr;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    uint32_t inflight = 0;      // queued for launch or on the GPU
    std::deque<Req*> todo;      // assigned by the scheduler, not launched yet (under Server::mu)
    std::condition_variable cv;
    bool stop = false;
    std::thread launcher;       // issues this lane's launches, off the scheduler thread
    Waiter waiter;
};

// Packed batch descriptors: byte offsets of the three parts for S requests.
struct DescLayout {
    size_t offsets, seg_m, jobs, total;
};
inline DescLayout desc_layout(uint32_t S) {
    DescLayout d;
    d.offsets = 0;
    d.seg_m = (sizeof(uint64_t) * (S + 1) + 15) & ~size_t{15};
    d.jobs = (d.seg_m + sizeof(uint32_t) * S + 15) & ~size_t{15};
    d.total = d.jobs + sizeof(CopyJob) * 2 * S;
    return d;
}

struct Batch {
    int slot;
    std::vector<uint64_t> ids;
    uint64_t ring_end;  // ring position after this batch's requests
    bool done = false;
    double t_done = 0;
    struct Server* server;
};

struct Server {
    mdx_server_config cfg{};
    int device = 0;
    uint32_t* d_in = nullptr;
    uint32_t* d_out = nullptr;
    uint64_t cap = 0;        // elements per ring
    uint64_t head = 0;       // next allocation
    std::deque<LiveEntry> live;  // admitted allocations, in order (references stay valid)
    std::vector<Slot> slots;

    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<Req*> waiting;   // submitted, not admitted
    std::deque<Req*> admitted;  // in the ring, not launched
    std::deque<Req*> admitted_direct;  // partitioned in place, not launched
    std::vector<Lane> lanes;
    std::vector<cudaEvent_t> free_events;
    std::unordered_map<uint64_t, Req*> reqs;  // every request not yet collected
    uint32_t inflight_batches = 0;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread sched;
    std::vector<Waiter*> waiters;  // every slot's and lane's completion queue
    std::condition_variable cv_poll;
    bool poll_stop = false;
    std::thread poller;
    mdx_status sticky = MDX_OK;   // first failure of a launch (reported by wait)

    // statistics
    uint64_t st_submitted = 0, st_completed = 0, st_batches = 0, st_elements = 0, st_direct = 0;
    double st_launch_s = 0;  // host time inside launch calls
    std::vector<double> latencies, queue_lat, exec_lat;
    double st_t0 = 0, st_t_last = 0;

    // ring: [off, off + n) for a new request, or false if it does not fit now.
    // Live allocations are consecutive in admission order; when the head wraps
    // to 0 the unused end [head, cap) is skipped until the tail passes it.
    LiveEntry* ring_alloc(uint64_t n) {
        if (n == 0 || n > cap) return nullptr;
        uint64_t o = 0;
        uint64_t* off = &o;
        if (live.empty()) {
            head = 0;
            *off = 0;
        } else {
            const uint64_t tail = live.front().off;
            if (head > tail) {  // not wrapped: free [head, cap) and [0, tail)
                if (head + n <= cap) *off = head;
                else if (n <= tail) *off = 0;
                else return nullptr;
            } else {  // wrapped: free [head, tail)
                if (head + n <= tail) *off = head;
                else return nullptr;
            }
        }
        head = *off + n;
        live.push_back(LiveEntry{*off, n, false});
        return &live.back();
    }
    // Advance the ring's tail over finished allocations.
    void ring_release() {
        while (!live.empty() && live.front().done) live.pop_front();
    }
};

// The poller: completes tracked work in each stream's order.  While anything
// is in flight it polls the front events (a pause of a few hundred
// nanoseconds between rounds that find nothing); with nothing in flight it
// sleeps until track() queues an event.
void poll_loop(Server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    std::vector<std::pair<Waiter*, cudaEvent_t>> fronts;
    std::vector<cudaError_t> res;
    for (;;) {
        fronts.clear();
        for (Waiter* w : s->waiters)
            if (!w->q.empty()) fronts.emplace_back(w, w->q.front().first);
        if (fronts.empty()) {
            if (s->poll_stop) break;
            s->cv_poll.wait(lk);
            continue;
        }
        lk.unlock();
        res.resize(fronts.size());
        bool any = false;
        for (size_t i = 0; i < fronts.size(); i++) {
            res[i] = cudaEventQuery(fronts[i].second);
            any = any || res[i] != cudaErrorNotReady;
        }
        if (!any) {
            for (int k = 0; k < 64; k++) cpu_relax();
            lk.lock();
            continue;
        }
        const double t = now_s();
        lk.lock();
        for (size_t i = 0; i < fronts.size(); i++) {
            if (res[i] == cudaErrorNotReady) continue;
            if (res[i] != cudaSuccess && s->sticky == MDX_OK) s->sticky = MDX_ERR_CUDA;
            Waiter* w = fronts[i].first;  // only this thread pops: the front is unchanged
            auto done = std::move(w->q.front().second);
            w->q.pop_front();
            done(t);
            s->free_events.push_back(fronts[i].second);
        }
        s->cv_sched.notify_all();
    }
}

// Record an event on `st` and hand `done` to its waiter.  Caller holds the lock.
bool track(Server* s, Waiter& w, cudaStream_t st, std::function<void(double)> done) {
    cudaEvent_t ev = nullptr;
    if (!s->free_events.empty()) {
        ev = s->free_events.back();
        s->free_events.pop_back();
    } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        return false;
    }
    if (cudaEventRecord(ev, st) != cudaSuccess) {
        s->free_events.push_back(ev);
        return false;
    }
    w.q.emplace_back(ev, std::move(done));
    s->cv_poll.notify_one();
    return true;
}

// Admit waiting requests (FIFO) while they fit.  In-place requests need no
// ring space.  Caller holds the lock.
void admit(Server* s) {
    while (!s->waiting.empty()) {
        Req* r = s->waiting.front();
        if (r->direct) {
            s->admitted_direct.push_back(r);
        } else {
            LiveEntry* e = s->ring_alloc(r->n);
            if (e == nullptr) break;
            r->ring = e;
            r->off = e->off;
            s->admitted.push_back(r);
        }
        s->waiting.pop_front();
    }
}

void complete(Server* s, Req* r, double t_done) {  // caller holds the lock
    r->t_done = t_done;
    r->done = true;
    s->st_completed++;
    s->st_elements += r->n;
    s->latencies.push_back(r->t_done - r->t_submit);
    s->queue_lat.push_back(r->t_launch - r->t_submit);
    s->exec_lat.push_back(r->t_done - r->t_launch);
    s->st_t_last = r->t_done;
}

// A batch finished: complete its requests, free its slot at once and
// release ring space in admission order.  Caller holds the lock.
void finish_batch(Server* s, Batch* b, double t_done) {
    for (uint64_t id : b->ids) {
        Req* r = s->reqs[id];
        complete(s, r, t_done);
        if (r->ring != nullptr) r->ring->done = true;
    }
    s->slots[b->slot].busy = false;
    s->inflight_batches--;
    delete b;
    s->ring_release();
    s->cv_done.notify_all();
}

mdx_status launch_batch(Server* s, Slot& sl, const std::vector<Req*>& batch) {
    const uint64_t base = batch.front()->off;
    const uint32_t S = static_cast<uint32_t>(batch.size());
    const DescLayout dl = desc_layout(S);
    uint64_t* h_offsets = reinterpret_cast<uint64_t*>(sl.h_desc + dl.offsets);
    uint32_t* h_seg_m = reinterpret_cast<uint32_t*>(sl.h_desc + dl.seg_m);
    CopyJob* h_jobs = reinterpret_cast<CopyJob*>(sl.h_desc + dl.jobs);
    uint64_t acc = 0;
    uint32_t chunks = 0;
    for (uint32_t i = 0; i < S; i++) {
        Req* r = batch[i];
        h_offsets[i] = acc;
        h_seg_m[i] = r->m;
        h_jobs[i] = CopyJob{r->in, s->d_in + r->off, r->n, nullptr, nullptr, 0, chunks};
        h_jobs[S + i] = CopyJob{s->d_out + r->off, r->out, r->n,
                                sl.d_seg_sizes + static_cast<uint64_t>(i) * s->cfg.m_max,
                                r->sizes, r->m, chunks};
        chunks += static_cast<uint32_t>((r->n + kCopyChunk - 1) / kCopyChunk);
        acc += r->n;
    }
    h_offsets[S] = acc;
    cudaStream_t st = sl.stream;
    if (cudaMemcpyAsync(sl.d_desc, sl.h_desc, dl.total, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return MDX_ERR_CUDA;
    const uint64_t* d_offsets = reinterpret_cast<const uint64_t*>(sl.d_desc + dl.offsets);
    const uint32_t* d_seg_m = reinterpret_cast<const uint32_t*>(sl.d_desc + dl.seg_m);
    const CopyJob* d_jobs = reinterpret_cast<const CopyJob*>(sl.d_desc + dl.jobs);
    copy_jobs<<<chunks, kCopyThreads, 0, st>>>(d_jobs, S);
    mdx_status r = mdx_partition_segmented_multi(
        s->d_in + base, s->d_out + base, acc, MDX_ELEM_U32, d_seg_m, s->cfg.m_max,
        d_offsets, S, sl.d_seg_sizes, nullptr, sl.ws, sl.ws_bytes,
        reinterpret_cast<mdx_stream_t>(st));
    if (r != MDX_OK) return r;
    copy_jobs<<<chunks, kCopyThreads, 0, st>>>(d_jobs + S, S);
    return cudaGetLastError() == cudaSuccess ? MDX_OK : MDX_ERR_CUDA;
}

// A lane's launcher: issues the in-place requests the scheduler assigned to
// the lane, in order, so their host-side launch cost runs beside the
// scheduler's batch launches instead of behind them.
void lane_loop(Server* s, Lane* l) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        while (l->todo.empty() && !l->stop) l->cv.wait(lk);
        if (l->todo.empty()) break;  // stopped with nothing assigned
        Req* r = l->todo.front();
        l->todo.pop_front();
        r->t_launch = now_s();
        lk.unlock();
        const mdx_discr dc = {MDX_DISCR_MOD, r->m};
        const double tl0 = now_s();
        mdx_status st = partition_two_kernel(r->in, r->out, r->n, MDX_ELEM_U32, dc, r->sizes, nullptr,
                                             l->ws, l->ws_bytes,
                                             reinterpret_cast<mdx_stream_t>(l->stream));
        const double tl1 = now_s();
        lk.lock();
        s->st_launch_s += tl1 - tl0;
        auto done = [s, l, r](double t) {
            complete(s, r, t);
            l->inflight--;
            s->cv_done.notify_all();
        };
        if (st != MDX_OK || !track(s, l->waiter, l->stream, done)) {
            // nothing will complete this request: finish it now
            if (s->sticky == MDX_OK) s->sticky = st != MDX_OK ? st : MDX_ERR_CUDA;
            done(now_s());
            s->cv_sched.notify_all();
        }
    }
}

void scheduler(Server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        admit(s);
        // long requests in device memory: the plain kernels straight on their
        // buffers, queued on the least loaded lane up to its depth
        while (!s->admitted_direct.empty()) {
            Lane* l = nullptr;
            for (Lane& c : s->lanes)
                if (c.inflight < kLaneDepth && (l == nullptr || c.inflight < l->inflight)) l = &c;
            if (l == nullptr) break;
            Req* r = s->admitted_direct.front();
            s->admitted_direct.pop_front();
            l->inflight++;
            r->launched = true;
            s->st_direct++;
            l->todo.push_back(r);  // the lane's own thread issues it
            l->cv.notify_one();
        }
        int free_slot = -1;
        for (size_t k = 0; k < s->slots.size(); k++)
            if (!s->slots[k].busy) { free_slot = static_cast<int>(k); break; }
        bool lanes_busy = false, lane_free = false;
        for (const Lane& l : s->lanes) {
            lanes_busy = lanes_busy || l.inflight > 0;
            lane_free = lane_free || l.inflight < kLaneDepth;
        }
        if (s->stop && s->admitted.empty() && s->admitted_direct.empty() && s->waiting.empty() &&
            s->inflight_batches == 0 && !lanes_busy)
            break;
        const bool can_batch = free_slot >= 0 && !s->admitted.empty();
        const bool can_direct = lane_free && !s->admitted_direct.empty();
        if (!can_batch) {
            if (!can_direct) s->cv_sched.wait(lk);
            continue;
        }
        // the longest contiguous run of admitted ring requests, within the caps
        std::vector<Req*> batch;
        uint64_t elems = 0, end = 0;
        while (!s->admitted.empty() && batch.size() < s->cfg.max_batch_requests) {
            Req* r = s->admitted.front();
            if (!batch.empty() && (r->off != end || elems + r->n > s->cfg.max_batch_elems)) break;
            batch.push_back(r);
            elems += r->n;
            end = r->off + r->n;
            s->admitted.pop_front();
        }
        Slot& sl = s->slots[free_slot];
        sl.busy = true;
        Batch* b = new Batch{free_slot, {}, end, false, 0, s};
        const double t_launch = now_s();
        for (Req* r : batch) {
            b->ids.push_back(r->id);
            r->t_launch = t_launch;
            r->launched = true;
        }
        s->inflight_batches++;
        s->st_batches++;
        lk.unlock();
        const double tl0 = now_s();
        mdx_status st = launch_batch(s, sl, batch);
        const double tl1 = now_s();
        lk.lock();
        s->st_launch_s += tl1 - tl0;
        auto done = [s, b](double t) { finish_batch(s, b, t); };
        if (st != MDX_OK || !track(s, sl.waiter, sl.stream, done)) {
            // nothing will complete this batch: finish it now
            if (s->sticky == MDX_OK) s->sticky = st != MDX_OK ? st : MDX_ERR_CUDA;
            done(now_s());
        }
    }
}

}  // namespace server
}  // namespace mdx

struct mdx_server_st {
    mdx::server::Server s;
};

using namespace mdx::server;

extern "C" {

mdx_status mdx_server_create(mdx_server* out, const mdx_server_config* cfg_in) {
    if (out == nullptr || cfg_in == nullptr) return MDX_ERR_INVALID;
    *out = nullptr;
    mdx_server_config cfg = *cfg_in;
    if (cfg.num_streams == 0) cfg.num_streams = 2;
    if (cfg.max_batch_requests == 0) cfg.max_batch_requests = 1024;
    if (cfg.max_batch_requests > 65535) cfg.max_batch_requests = 65535;
    if (cfg.m_max == 0) cfg.m_max = 16;
    if (cfg.direct_min_elems == 0) cfg.direct_min_elems = 1ull << 20;
    if (cfg.m_max > 16 || cfg.budget_bytes < 8 * 4096) return MDX_ERR_INVALID;
    auto* h = new mdx_server_st();
    Server& s = h->s;
    s.cfg = cfg;
    s.cap = cfg.budget_bytes / 8;  // u32 input ring + u32 output ring
    if (s.cap > MDX_MAX_ELEMS) s.cap = MDX_MAX_ELEMS;
    // a batch runs at the batch streams' high priority: capped so that one
    // batch cannot hold the GPU for long while in-place requests wait (without
    // a cap, 50k requests/s queued long requests for ~14 ms at p99; 2^24: 0.24 ms)
    if (cfg.max_batch_elems == 0) s.cfg.max_batch_elems = kDefaultBatchElems;
    if (s.cfg.max_batch_elems > s.cap) s.cfg.max_batch_elems = s.cap;
    bool ok = cudaGetDevice(&s.device) == cudaSuccess &&
              dev_alloc(&s.d_in, s.cap * 4) == cudaSuccess &&
              dev_alloc(&s.d_out, s.cap * 4) == cudaSuccess;
    const uint32_t B = s.cfg.max_batch_requests;
    int prio_low = 0, prio_high = 0;  // numerically lower = higher priority
    if (ok) ok = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) == cudaSuccess;
    s.slots = std::vector<Slot>(cfg.num_streams);  // sized once: completions hold pointers
    for (auto& sl : s.slots) {
        if (!ok) break;
        sl.ws_bytes = mdx_segmented_workspace_size(s.cfg.max_batch_elems, B, MDX_ELEM_U32, cfg.m_max);
        ok = cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, prio_high) == cudaSuccess &&
             dev_alloc(&sl.ws, sl.ws_bytes) == cudaSuccess &&
             mdx_workspace_init(sl.ws, sl.ws_bytes, reinterpret_cast<mdx_stream_t>(sl.stream)) == MDX_OK &&
             dev_alloc(&sl.d_desc, desc_layout(B).total) == cudaSuccess &&
             dev_alloc(&sl.d_seg_sizes, sizeof(uint32_t) * B * cfg.m_max) == cudaSuccess &&
             pinned_alloc(&sl.h_desc, desc_layout(B).total) == cudaSuccess;
    }
    s.lanes = std::vector<Lane>(kLanes);  // sized once: completions hold Lane pointers
    for (auto& l : s.lanes) {
        if (!ok) break;
        l.ws_bytes = mdx_workspace_size(s.cfg.max_batch_elems, MDX_ELEM_U32, cfg.m_max);
        ok = cudaStreamCreateWithPriority(&l.stream, cudaStreamNonBlocking, prio_low) == cudaSuccess &&
             dev_alloc(&l.ws, l.ws_bytes) == cudaSuccess &&
             mdx_workspace_init(l.ws, l.ws_bytes, reinterpret_cast<mdx_stream_t>(l.stream)) == MDX_OK;
    }
    if (!ok || cudaDeviceSynchronize() != cudaSuccess) {
        mdx_server_destroy(h);
        return MDX_ERR_CUDA;
    }
    s.st_t0 = now_s();
    for (auto& sl : s.slots) s.waiters.push_back(&sl.waiter);
    for (auto& l : s.lanes) s.waiters.push_back(&l.waiter);
    s.poller = std::thread(poll_loop, &s);
    for (auto& l : s.lanes) l.launcher = std::thread(lane_loop, &s, &l);
    s.sched = std::thread(scheduler, &s);
    *out = h;
    return MDX_OK;
}

void mdx_test_inject_alloc_failure(uint32_t nth) { g_fail_countdown.store(nth); }

mdx_status mdx_server_submit(mdx_server h, const uint32_t* in, uint32_t* out, uint32_t* sizes,
                             uint64_t n, uint32_t m, uint64_t* ticket) {
    if (h == nullptr || ticket == nullptr) return MDX_ERR_INVALID;
    Server& s = h->s;
    if (m < 1 || m > s.cfg.m_max || n == 0 || n > MDX_MAX_ELEMS) return MDX_ERR_INVALID;
    // every buffer must be reachable from kernels: device memory, or
    // page-locked host memory mapped into the device's address space
    const uint32_t* d_in = device_view(in);
    uint32_t* d_out = device_view(out);
    uint32_t* d_sizes = device_view(sizes);
    if (d_in == nullptr || d_out == nullptr || d_sizes == nullptr) return MDX_ERR_INVALID;
    Req* r = new Req();
    r->n = n;
    r->m = m;
    r->in = d_in;
    r->out = d_out;
    r->sizes = d_sizes;
    if (n >= s.cfg.direct_min_elems && is_device_memory(in) && is_device_memory(out) &&
        is_device_memory(sizes)) {
        const char* ib = reinterpret_cast<const char*>(d_in);
        const char* ob = reinterpret_cast<const char*>(d_out);
        r->direct = !(ib < ob + n * 4 && ob < ib + n * 4);  // overlapping buffers go through the ring
    }
    // a request through the pool must fit one batch and the ring
    if (!r->direct && (n > s.cap || n > s.cfg.max_batch_elems)) {
        delete r;
        return MDX_ERR_INVALID;
    }
    {
        std::lock_guard<std::mutex> lk(s.mu);
        r->id = s.next_id++;
        r->t_submit = now_s();
        s.reqs[r->id] = r;
        s.waiting.push_back(r);
        s.st_submitted++;
        *ticket = r->id;
    }
    s.cv_sched.notify_all();
    return MDX_OK;
}

mdx_status mdx_server_wait(mdx_server h, uint64_t ticket, double* latency_s) {
    if (h == nullptr) return MDX_ERR_INVALID;
    Server& s = h->s;
    std::unique_lock<std::mutex> lk(s.mu);
    auto it = s.reqs.find(ticket);
    if (it == s.reqs.end()) return MDX_ERR_INVALID;
    Req* r = it->second;
    s.cv_done.wait(lk, [&] { return r->done; });
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    const mdx_status st = r->status != MDX_OK ? r->status : s.sticky;
    s.reqs.erase(it);
    delete r;
    return st;
}

mdx_status mdx_server_cancel(mdx_server h, uint64_t ticket) {
    if (h == nullptr) return MDX_ERR_INVALID;
    Server& s = h->s;
    {
        std::lock_guard<std::mutex> lk(s.mu);
        auto it = s.reqs.find(ticket);
        if (it == s.reqs.end()) return MDX_ERR_INVALID;
        Req* r = it->second;
        if (r->launched || r->done) return MDX_ERR_INVALID;  // too late
        auto drop = [r](std::deque<Req*>& q) {
            auto qi = std::find(q.begin(), q.end(), r);
            if (qi == q.end()) return false;
            q.erase(qi);
            return true;
        };
        if (!drop(s.waiting) && !drop(s.admitted) && !drop(s.admitted_direct))
            return MDX_ERR_INVALID;
        if (r->ring != nullptr) {
            r->ring->done = true;  // its ring slot is released in admission order
            s.ring_release();
        }
        r->status = MDX_ERR_CANCELLED;
        r->done = true;
        r->t_done = now_s();
    }
    s.cv_done.notify_all();
    s.cv_sched.notify_all();
    return MDX_OK;
}

mdx_status mdx_server_get_stats(mdx_server h, mdx_server_stats* out) {
    if (h == nullptr || out == nullptr) return MDX_ERR_INVALID;
    Server& s = h->s;
    std::lock_guard<std::mutex> lk(s.mu);
    out->submitted = s.st_submitted;
    out->completed = s.st_completed;
    out->batches = s.st_batches;
    out->elements = s.st_elements;
    out->waiting = s.waiting.size();
    out->inflight_batches = s.inflight_batches;
    auto pct = [](std::vector<double> v, double q) {
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        return v[std::min(v.size() - 1, static_cast<size_t>(q * (v.size() - 1) + 0.5))];
    };
    out->p50_s = out->p99_s = out->mean_s = 0;
    if (!s.latencies.empty()) {
        out->p50_s = pct(s.latencies, 0.5);
        out->p99_s = pct(s.latencies, 0.99);
        double sum = 0;
        for (double x : s.latencies) sum += x;
        out->mean_s = sum / s.latencies.size();
    }
    out->queue_p50_s = pct(s.queue_lat, 0.5);
    out->queue_p99_s = pct(s.queue_lat, 0.99);
    out->exec_p50_s = pct(s.exec_lat, 0.5);
    out->exec_p99_s = pct(s.exec_lat, 0.99);
    out->window_s = s.st_t_last > s.st_t0 ? s.st_t_last - s.st_t0 : 0.0;
    out->direct = s.st_direct;
    out->launch_busy_s = s.st_launch_s;
    return MDX_OK;
}

mdx_status mdx_server_reset_stats(mdx_server h) {
    if (h == nullptr) return MDX_ERR_INVALID;
    Server& s = h->s;
    std::lock_guard<std::mutex> lk(s.mu);
    s.st_submitted = s.st_completed = s.st_batches = s.st_elements = s.st_direct = 0;
    s.st_launch_s = 0;
    s.latencies.clear();
    s.queue_lat.clear();
    s.exec_lat.clear();
    s.st_t0 = now_s();
    s.st_t_last = s.st_t0;
    return MDX_OK;
}

mdx_status mdx_server_destroy(mdx_server h) {
    if (h == nullptr) return MDX_OK;
    Server& s = h->s;
    if (s.sched.joinable()) {
        {
            std::lock_guard<std::mutex> lk(s.mu);
            s.stop = true;
        }
        s.cv_sched.notify_all();
        s.sched.join();
    }
    {  // the scheduler left with nothing in flight: launchers and waiters have no work left
        std::lock_guard<std::mutex> lk(s.mu);
        for (auto& l : s.lanes) l.stop = true;
    }
    for (auto& l : s.lanes) {
        l.cv.notify_all();
        if (l.launcher.joinable()) l.launcher.join();
    }
    {
        std::lock_guard<std::mutex> lk(s.mu);
        s.poll_stop = true;
    }
    s.cv_poll.notify_all();
    if (s.poller.joinable()) s.poller.join();
    for (cudaEvent_t ev : s.free_events) cudaEventDestroy(ev);
    for (auto& sl : s.slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        cudaFree(sl.ws);
        cudaFree(sl.d_desc);
        cudaFree(sl.d_seg_sizes);
        cudaFreeHost(sl.h_desc);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    for (auto& l : s.lanes) {
        if (l.stream) cudaStreamSynchronize(l.stream);
        cudaFree(l.ws);
        if (l.stream) cudaStreamDestroy(l.stream);
    }
    cudaFree(s.d_in);
    cudaFree(s.d_out);
    for (auto& kv : s.reqs) delete kv.second;
    delete h;
    return MDX_OK;
}

}  // extern "C"
