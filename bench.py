"""Benchmark of the plain stable m-way partition on B200.

Workload (one "step" = one partition of one synthetic batch resident in HBM):
plain mdiscr, N = 2^28 int32 values uniform over [0, 2^31) from a seeded
generator (mdiscriminator_b200.workloads, seed "c2a"), m = 8, class = value
mod 8 (Mod8: value & 7), stable; outputs the permuted array and the 8 class
sizes.  Inputs (1 GiB) and outputs (1 GiB) are larger than the 126 MB L2, so
no flush is needed between steps.

Printed JSON (rank 0, one line):
  value      elements/s over all ranks, kernels only, inputs resident in HBM
  e2e        the same metric through the public API with pinned host buffers:
             host->device copy of the input, the partition, device->host copy
             of the output and sizes, all inside the timed region
  roofline   the partition call against the HBM roofline of reading and
             writing each element once (2*N*4 + 4*m bytes), and each of its
             two kernels against its own algorithmic bytes
  configs    every other plain configuration of the benchmark list, each on
             its own seeded input: N=2^20 m=4 (L2 flushed between reps), the
             Zipf-skewed N=2^28 m=8, and N=2^27 8-byte records at m in
             {2,4,16,32,64}, random and pre-sorted by class
  batched    100,000 log-normal segments, offsets form and head-flag form
  served     Poisson request arrivals through the serving loop
  cpu_baseline  the reference's OpenmpMdiscr (compiled from its sources,
             oracle/_ref) on the same input as the GPU (the whole array when
             host memory allows), on this host's cores; its seqMdiscr on one
             core on a prefix of that input

--impl reference runs the reference's own CPU implementation (OpenmpMdiscr)
instead, on rank 0 only, with every host thread, on the same seeded input.

Multi-GPU (torchrun, one process per GPU): every rank partitions its own
N = 2^28 array (independent units, no data-path collective; weak scaling);
the step time is the max over ranks.  The same run then partitions the
ranks' arrays as ONE array spread over them (count all-gather + scatter into
peer chunks) and reports it under "distributed"; --distributed runs only
that.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_DEFAULT = 1 << 28
M_DEFAULT = 8
WORKLOAD = "plain mdiscr int32 N=2^28 uniform[0,2^31) m=8 (class = v mod 8)"
METRIC = "Gelem/s & % HBM roofline (N=2^28, m=8)"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, copy burst)"
    return 6650.0, "fallback 6.65 TB/s"


def traffic_from_profiles():
    """DRAM bytes per call of the two kernels from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "plain_partition_n2p28_m8_traffic.txt")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            if ":" in line and line.split(":")[0].strip() in ("count_kernel_bytes",
                                                              "scatter_kernel_bytes"):
                k, v = line.split(":", 1)
                try:
                    out[k.strip()] = float(v.split()[0])
                except ValueError:
                    pass
    return out


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML (read
    only) by a background thread during the timed region."""
    REASONS = {  # nvmlClocksEventReason* bits
        "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
        "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, gpu_index: int, period_s: float = 0.002):
        self.gpu = gpu_index
        self.period = period_s
        self.samples = []
        self.reasons = 0
        self._stop = threading.Event()
        self._t = None
        self.nv = None
        self.max_mhz = None

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = self.gpu
            if vis:
                ids = [v.strip() for v in vis.split(",") if v.strip()]
                if ids and ids[0].isdigit():
                    idx = int(ids[self.gpu])
            self.h = nv.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.nv = nv
        except Exception:  # NVML missing: no clock record
            self.nv = None
            return
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        nv = self.nv
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons")
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                self.reasons |= int(get_reasons(self.h))
            except Exception:
                pass
            time.sleep(self.period)

    def stop(self):
        if self.nv is None:
            return None
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(k for k, b in self.REASONS.items() if self.reasons & b),
                "samples": len(self.samples), "source": "NVML, every 2 ms in the timed region"}


def make_input(torch, n, seed, device):
    """n int32 values uniform over [0, 2^31): the splitmix64 stream of
    mdiscriminator_b200.workloads, generated on the device."""
    from mdiscriminator_b200 import workloads as W
    return W.uniform_u32_torch(torch, n, seed, device)


def batched_measurement(torch, mdx, dev, peak, steps=10, warmup=3, sample_segments=2000,
                        num_segments=100_000, keep="all", with_plain=True, with_flags=True):
    """Batched segmented partition: 100,000 segments, lengths
    LogNormal(ln 1024, 1.5) clamped to [1, 2^22] (~3e8 int32), m = 4,
    class = v mod 4, as one segmented call replayed from a CUDA graph, against
    one plain partition per segment (a CUDA graph of per-segment calls over a
    sample of consecutive segments).  The same segments are also given in the
    reference's head-flag form (mdiscrSegm: i32 length at every segment start,
    head-flag class sizes out), timed the same way.  ``keep`` = "large" /
    "small" keeps only the segments longer than / at most one 4096-element
    tile (for profiling the two halves of the kernel)."""
    import numpy as np

    from mdiscriminator_b200 import workloads as W
    m = 4
    lengths = W.lognormal_lengths(num_segments, W.SEEDS["c4"])
    if keep == "large":
        lengths = lengths[lengths > 4096]
    elif keep == "small":
        lengths = lengths[lengths <= 4096]
    S = len(lengths)
    offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
    n = int(offs[-1])
    d_in = make_input(torch, n, W.SEEDS["c4"], dev)
    d_out = torch.empty_like(d_in)
    d_offs = torch.from_numpy(offs).to(dev)
    seg_sizes = torch.empty((S, m), dtype=torch.uint32, device=dev)
    ws = mdx.new_workspace(mdx.segmented_workspace_size(n, S, mdx.ELEM_U32, m), dev)
    stream = torch.cuda.Stream(device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def graph_time(issue, reps):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                issue()
            stream.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream):
                issue()
            g.replay()
            stream.synchronize()
            e0.record(stream)
            for _ in range(reps):
                g.replay()
            e1.record(stream)
            stream.synchronize()
        del g
        return e0.elapsed_time(e1) * 1e-3 / reps

    t_b = graph_time(lambda: mdx.partition_segmented(d_in, d_offs, ("mod", m), out=d_out,
                                                     seg_sizes=seg_sizes, ws=ws), steps)
    if ws.error() != mdx.MDX_OK:
        raise SystemExit("device error in the batched measurement")
    alg = 2 * n * 4 + 8 * (S + 1) + 4 * m * S
    workload = (f"{S:,} segments, LogNormal(ln 1024, 1.5) clamped [1, 2^22]"
                + ("" if keep == "all" else f" (only the {keep} ones of {num_segments:,})")
                + ", int32, m=4, segment offsets, one segmented launch sequence replayed from a "
                  "CUDA graph")
    res = {"workload": workload, "n": n, "segments": S, "value": n / t_b / 1e9, "unit": "Gelem/s",
           "ms": t_b * 1e3,
           "roofline": {"bound": "hbm", "achieved": alg / t_b / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / t_b / 1e9 / peak, "alg_bytes": "2*N*4 + 8*(S+1) + 4*m*S"}}
    if with_flags:
        # the reference's own form: head-flag segment sizes in, head-flag class
        # sizes out (mdiscrSegm, MdiscrSegmHost.cu.h:36-42)
        flags = torch.zeros(n, dtype=torch.int32, device=dev)
        flags[d_offs[:-1]] = torch.from_numpy(lengths.astype(np.int32)).to(dev)
        new_sizes = torch.empty(n, dtype=torch.int32, device=dev)
        fws = mdx.new_workspace(int(mdx.lib().mdx_mdiscr_segm_workspace_size(n, mdx.ELEM_U32, m)),
                                dev)
        t_f = graph_time(lambda: mdx.mdiscr_segm(d_in, flags, ("mod", m), d_out=d_out,
                                                 d_new_sizes=new_sizes, ws=fws), steps)
        if fws.error() != mdx.MDX_OK:
            raise SystemExit("device error in the head-flag batched measurement")
        alg_f = 2 * n * 4 + 4 * n + 4 * n
        res["head_flag_form"] = {
            "value": n / t_f / 1e9, "unit": "Gelem/s", "ms": t_f * 1e3,
            "roofline": {"achieved": alg_f / t_f / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg_f / t_f / 1e9 / peak,
                         "alg_bytes": "2*N*4 + 4*N (flags in) + 4*N (head-flag sizes out)"},
            "what": "mdx_mdiscr_segm: i32 segment lengths at segment starts in, i32 head-flag "
                    "class sizes per segment out, one CUDA graph replay per step"}
        del flags, new_sizes, fws
    if not with_plain:
        return res
    # one plain launch per segment, on a sample of consecutive segments
    s0 = S // 2
    s1 = s0 + sample_segments
    a0, a1 = int(offs[s0]), int(offs[s1])
    pws = mdx.new_workspace(max(mdx.workspace_size(int(lengths[s0:s1].max()), mdx.ELEM_U32, m), 1 << 20), dev)
    sizes = torch.empty(m, dtype=torch.uint32, device=dev)
    views = [(int(offs[s]), int(offs[s + 1])) for s in range(s0, s1)]

    def per_segment():
        for a, b in views:
            mdx.partition(d_in[a:b], ("mod", m), out=d_out[a:b], sizes=sizes, ws=pws)
    t_p = graph_time(per_segment, 3)
    v_p = (a1 - a0) / t_p / 1e9
    res["per_segment_plain"] = {"value": v_p, "unit": "Gelem/s",
                                "sample": f"segments {s0}..{s1 - 1} ({a1 - a0} elements), one "
                                          "mdx_partition per segment, CUDA graph of the calls"}
    res["speedup_vs_per_segment"] = res["value"] / v_p
    return res


def sort_measurement(torch, d_in, d_out, m, reps=3):
    """The sort-based alternative on the same GPU and input (the reference's
    SortTest.cu:130-154 uses thrust::stable_sort_by_key): a stable library
    radix sort of the class keys (torch.sort, stable) and a gather of the
    values by the sorted indices.  Library code, timed as a reference point;
    its result is checked against mdx's."""
    keys = d_in % m if (m & (m - 1)) else d_in & (m - 1)
    _, idx = torch.sort(keys, stable=True)
    same = bool(torch.equal(d_in[idx], d_out))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        k = d_in % m if (m & (m - 1)) else d_in & (m - 1)
        _, idx = torch.sort(k, stable=True)
        out = d_in[idx]
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del keys, idx, out
    return {"value": d_in.numel() / ms / 1e6, "unit": "Gelem/s", "ms": ms,
            "equal_to_mdx": same,
            "what": "torch.sort(class keys, stable=True) + gather by the indices, same input, "
                    "CUDA events (library code, reference point)"}


def served_measurement(torch, mdx, dev, peak, loads=(1000, 5000, 20000, 50000), duration_s=1.0):
    """Served partition requests: open-loop Poisson arrivals at each offered
    load; lengths log-uniform over [2^10, 2^24], values uniform over [0, 2^31),
    m uniform over {2, 4, 8, 16}, class = v mod m; a 16 GiB device budget for
    the server's request pool; requests' data in device memory (views of a
    resident array, outputs to distinct slices).  p50 / p99 latency (submit to
    completion) and elements/s per load, against one plain partition per
    request issued back to back on one stream.

    The load generator runs with Python's garbage collector off (one
    collection before each load): a generation-2 collection inside the submit
    loop paused submission for 63 ms at 50k requests/s, after which the next
    ~3,000 requests went in as one burst above the server's capacity and their
    queueing, not the server's, set the p99.  `max_lag_ms` reports how far
    the submissions ran behind their Poisson schedule."""
    import gc
    import math

    import numpy as np
    rng = np.random.default_rng(17)
    src_n = 1 << 28
    from mdiscriminator_b200 import workloads as W
    src = make_input(torch, src_n, W.SEEDS["c5"], dev)
    out_pool = torch.empty(1 << 30, dtype=torch.int32, device=dev)
    sizes_pool = torch.empty((1 << 16, 16), dtype=torch.int32, device=dev)
    res = []
    srv = mdx.Server(budget_bytes=16 << 30, num_streams=4, max_batch_requests=1024)

    def make_requests(k):
        n = np.exp(rng.uniform(math.log(1 << 10), math.log(1 << 24), size=k)).astype(np.int64)
        m = rng.choice([2, 4, 8, 16], size=k)
        st = rng.integers(0, src_n - (1 << 24), size=k)
        reqs, pos = [], 0
        for i in range(k):
            if pos + n[i] > out_pool.numel():
                pos = 0
            reqs.append((src[st[i]:st[i] + n[i]], out_pool[pos:pos + n[i]],
                         sizes_pool[i % sizes_pool.shape[0]], int(m[i]), int(n[i])))
            pos += int(n[i])
        return reqs

    # warm-up (set-up of every kernel family)
    for d_in, d_out, sz, m, _ in make_requests(64):
        srv.wait(srv.submit(d_in, d_out, sz, m))
    for load in loads:
        k = max(int(load * duration_s), 200)
        reqs = make_requests(k)
        arrivals = np.cumsum(rng.exponential(1.0 / load, size=k))
        gc.collect()
        gc.disable()
        srv.reset_stats()
        tickets = []
        lag = 0.0
        t0 = time.perf_counter()
        for (d_in, d_out, sz, m, _), ta in zip(reqs, arrivals):
            while time.perf_counter() - t0 < ta:
                pass
            lag = max(lag, time.perf_counter() - t0 - ta)
            tickets.append(srv.submit(d_in, d_out, sz, m))
        t_sub = time.perf_counter() - t0
        gc.enable()
        for t in tickets:
            srv.wait(t)
        st = srv.stats()
        elems = sum(r[4] for r in reqs)
        res.append({"offered_req_per_s": load, "achieved_submit_rate": k / t_sub,
                    "max_lag_ms": lag * 1e3, "requests": k, "p50_ms": st["p50_s"] * 1e3, "p99_ms": st["p99_s"] * 1e3,
                    "queue_p99_ms": st["queue_p99_s"] * 1e3, "exec_p99_ms": st["exec_p99_s"] * 1e3,
                    "direct": st["direct"],
                    "gelem_per_s": elems / st["window_s"] / 1e9 if st["window_s"] > 0 else None,
                    "batches": st["batches"], "mean_request_elems": elems / k})
    # capacity: every request of a closed batch submitted at once
    reqs = make_requests(2000)
    gc.collect()
    gc.disable()
    srv.reset_stats()
    t0 = time.perf_counter()
    tickets = [srv.submit(d_in, d_out, sz, m) for d_in, d_out, sz, m, _ in reqs]
    for t in tickets:
        srv.wait(t)
    t_all = time.perf_counter() - t0
    gc.enable()
    st = srv.stats()
    elems = sum(r[4] for r in reqs)
    saturated = {"requests": len(reqs), "gelem_per_s": elems / t_all / 1e9,
                 "req_per_s": len(reqs) / t_all, "batches": st["batches"],
                 "p50_ms": st["p50_s"] * 1e3, "p99_ms": st["p99_s"] * 1e3,
                 "sample": "2000 requests of the same mix submitted at once (host wall clock "
                           "from the first submit to the last completion)"}
    srv.close()
    # one plain launch per request, back to back, on the same request mix
    reqs = make_requests(400)
    ws = mdx.new_workspace(mdx.workspace_size(1 << 24, mdx.ELEM_U32, 16), dev)
    sizes = torch.empty(16, dtype=torch.uint32, device=dev)
    for d_in, d_out, _, m, _ in reqs[:10]:
        mdx.partition(d_in, ("mod", m), out=d_out, sizes=sizes[:m], ws=ws)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for d_in, d_out, _, m, _ in reqs:
        mdx.partition(d_in, ("mod", m), out=d_out, sizes=sizes[:m], ws=ws)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    plain = sum(r[4] for r in reqs) / t_plain / 1e9
    return {"workload": "served requests: Poisson arrivals, n log-uniform [2^10, 2^24] int32, "
                        "m uniform {2,4,8,16}, 16 GiB budget, device-resident request data",
            "loads": res,
            "saturated": saturated,
            "per_request_plain": {"value": plain, "unit": "Gelem/s",
                                  "sample": "400 requests of the same mix, one mdx_partition each, "
                                            "back to back on one stream (host wall clock)"}}


def time_calls(torch, fn, reps, warmup, flush=None):
    """Median and mean device time (ms) of ``fn`` over ``reps`` calls, CUDA
    events around each call on the current stream; ``flush`` (a tensor larger
    than L2) is rewritten before every call."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(reps)]
    for a, b in evs:
        if flush is not None:
            flush.fill_(7)
        a.record()
        fn()
        b.record()
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in evs]
    return statistics.median(ms), statistics.mean(ms)


def configs_measurement(torch, mdx, dev, peak, reps=20, warmup=3):
    """The plain configurations of the benchmark list other than the headline,
    each on its own seeded input generated on the device
    (mdiscriminator_b200.workloads), timed call by call with CUDA events."""
    from mdiscriminator_b200 import workloads as W
    out = []

    def entry(name, d_in, m, what, flush=None):
        n = d_in.numel()
        w = d_in.element_size()
        d_out = torch.empty_like(d_in)
        sizes = torch.empty(m, dtype=torch.uint32, device=dev)
        ws = mdx.new_workspace(mdx.workspace_size(n, mdx.ELEM_U32 if w == 4 else mdx.ELEM_REC8, m),
                               dev)
        discr = ("mask", m) if (m & (m - 1)) == 0 else ("mod", m)
        med, mean = time_calls(torch, lambda: mdx.partition(d_in, discr, out=d_out, sizes=sizes,
                                                            ws=ws), reps, warmup, flush)
        if ws.error() != mdx.MDX_OK:
            raise SystemExit(f"device error in config {name}")
        t = med * 1e-3
        alg = 2 * n * w + 4 * m
        out.append({"config": name, "what": what, "n": n, "elem_bytes": w, "m": m,
                    "ms": med, "ms_mean": mean, "gelem_per_s": n / t / 1e9,
                    "roofline_frac": alg / t / 1e9 / peak,
                    "frac_of_two_pass_bound": (3 * n * w + 4 * m) / t / 1e9 / peak})
        del d_out, sizes, ws

    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    d = make_input(torch, 1 << 20, W.SEEDS["c1"], dev)
    entry("c1", d, 4, "N=2^20 int32 uniform, m=4 (class = v mod 4); L2 flushed (512 MB write) "
                      "before every call", flush)
    del d, flush
    d = W.zipf8_torch(torch, 1 << 28, W.SEEDS["c2b"], dev)
    entry("c2b", d, 8, "N=2^28 int32, class ~ Zipf(1.1) over 8 classes, v = 8*U[0,2^28) + class, "
                       "m=8 (v & 7)")
    del d
    d = make_input(torch, 1 << 28, W.SEEDS["c2a"], dev)
    for m in (2, 16, 32, 64):
        entry(f"c2a_m{m}", d, m, f"N=2^28 int32 uniform [0,2^31) (the headline input), m={m} "
                                 f"(v & {m - 1})")
    del d
    for presorted in (False, True):
        for m in (2, 4, 16, 32, 64):
            d = W.records_torch(torch, 1 << 27, W.SEEDS["c3"], m, presorted, dev)
            entry(f"c3_m{m}" + ("_presorted" if presorted else ""), d, m,
                  f"N=2^27 8-byte records {{key uniform [0,2^31), payload = index}}, class = "
                  f"key & {m - 1}" + (", keys pre-sorted by class" if presorted else ""))
            del d
    torch.cuda.empty_cache()
    return out


def host_mem_available() -> int:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def openmp_sample_size(n: int, m: int) -> int:
    """Largest prefix of the n-element input (n itself when it fits) whose
    openmpMdiscr run fits in ~60% of the available host memory: input,
    output, head flags, the per-element classes and two N x m tuple arrays
    (cuda_code/OpenmpMdiscr.h:18-22)."""
    per_elem = 4 + 4 + 4 + 4 + 2 * 4 * m
    fit = int(0.6 * host_mem_available()) // per_elem
    k = n
    while k > fit and k > (1 << 20):
        k //= 2
    return k


def cpu_baseline(x, m: int, reps: int, seq_sample: int = 1 << 25):
    """The reference's openmpMdiscr on the GPU arm's own input ``x`` (the
    whole array, or its largest prefix that host memory allows), every host
    thread; and its seqMdiscr (Mod8 / Mod4 for m = 8 / 4, else Mod<m>) on one
    core on a prefix of the same input.  Rank 0, N = 1 only."""
    import oracle
    if not oracle.ref_available():
        return None, "oracle/_ref not built"
    n = x.shape[0]
    k = openmp_sample_size(n, m)
    xs = x[:k]
    threads = os.cpu_count() or 1
    best = None
    for _ in range(reps):
        _, _, us = oracle.ref_openmp(xs, m, threads=threads)
        if us > 0 and (best is None or us < best):
            best = us
    if best is None:
        return None, "reference run failed"
    ks = min(seq_sample, n)
    _, _, seq_us = oracle.ref_seq(x[:ks], m, specialized=m in (4, 8), measure=True)
    res = {"value": k / (best * 1e-6) / 1e9, "unit": "Gelem/s", "cores": threads,
           "kind": "reference", "same_input": True,
           "sample": (f"openmpMdiscr (cuda_code/OpenmpMdiscr.h) on the GPU arm's own input "
                      + ("(the whole array)" if k == n else
                         f"(its first {k} elements: the whole array needs more host memory)")
                      + f", m={m}, best of {reps}, its own gettimeofday timer, OMP threads={threads}")}
    if seq_us and seq_us > 0:
        res["seq_single_core"] = {
            "value": ks / (seq_us * 1e-6) / 1e9, "unit": "Gelem/s", "cores": 1,
            "sample": f"seqMdiscr<{'Mod%d' % m if m in (4, 8) else 'Mod<%d>' % m}, true> "
                      f"(cuda_code/SeqMdiscr.h:10-57) on the first {ks} elements of the same "
                      "input, its own timer, one run"}
    return res, None


def distributed_leg(args, torch, dist, dev, world, x, m, discr):
    """With more than one rank: the ranks' arrays taken as ONE array of
    world * N elements (rank r holds chunk r) and partitioned across them by
    mdiscriminator_b200.distributed (class counts, an all-gather of the
    counts over NCCL, the scatter kernel storing into every rank's output
    chunk through IPC peer mappings) -- the exchange step of the sharded
    path, next to the independent arrays of the headline.  The first call
    checks the device error status; device time by CUDA events, max over
    ranks.  Every rank takes the same collective steps; an error is reported
    in the line instead of ending the run."""
    from mdiscriminator_b200 import distributed as D
    try:
        out, _ = D.partition_distributed(x, discr, out=None)
        for _ in range(2):
            out, _ = D.partition_distributed(x, discr, out=out, check=False)
        torch.cuda.synchronize()
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            out, _ = D.partition_distributed(x, discr, out=out, check=False)
        e1.record()
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1) / args.steps], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        res = {"metric": "Gelem/s, one array over the ranks (distributed partition)",
               "value": world * x.numel() / ms / 1e6, "unit": "Gelem/s", "ms_per_step": ms,
               "workload": f"one array of {world} x {x.numel()} int32 (rank r holds chunk r), "
                           f"m={m}; output in balanced chunks across the ranks",
               "transport": "count all-gather (NCCL) + scatter into peer chunks (CUDA IPC)"}
    except Exception as e:  # noqa: BLE001 -- reported, not fatal to the headline line
        res = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    finally:
        try:
            D.close_peer_maps()
        except Exception:  # noqa: BLE001
            pass
    return res


def distributed_main(args, torch, dist, mdx, dev, world, rank):
    """--distributed: one array of world * N elements, rank r holding the r-th
    chunk of N (weak scaling), partitioned by the "p2p" transport of
    mdiscriminator_b200.distributed (count, all-gather of the counts, the
    scatter kernel storing into every rank's output chunk through IPC
    mappings, completion barrier).  Device time by CUDA events, max over
    ranks."""
    import socket

    from mdiscriminator_b200 import distributed as D
    if world == 1:
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                                world_size=1, device_id=dev)
    n, m = args.n, args.m
    discr = ("mask", m) if (m & (m - 1)) == 0 else ("mod", m)
    from mdiscriminator_b200 import workloads as W
    x = make_input(torch, n, W.SEEDS["c2a"] + rank, dev)
    out = None
    for _ in range(args.warmup):
        out, _ = D.partition_distributed(x, discr, out=out)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        out, _ = D.partition_distributed(x, discr, out=out, check=False)
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1) / args.steps], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    if rank == 0:
        print(json.dumps({
            "metric": "Gelem/s, one array over the ranks (distributed partition)",
            "value": world * n / ms / 1e6, "unit": "Gelem/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": f"stable partition of {world} x {n} int32, m={m}, rank r holds "
                                   "chunk r; output in balanced chunks across the ranks",
                       "n_per_rank": n, "m": m, "parallelism": f"p2p over {world} ranks"},
            "gpu_launches": 3 * args.steps}))
    D.close_peer_maps()
    dist.destroy_process_group()


def run_reference(args):
    """--impl reference: the reference's CPU implementation (openmpMdiscr,
    compiled from its sources into oracle/_ref) on rank 0 only, every host
    thread, on the GPU arm's own seeded input: the whole array when host
    memory and the run's time allow, else its largest prefix that does."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    from mdiscriminator_b200 import workloads as W
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's "
                          "OpenmpMdiscr build) is missing"}))
        return 0
    threads = os.cpu_count() or 1
    x = W.uniform_u32(args.n, W.SEEDS["c2a"])
    k = openmp_sample_size(args.n, args.m)
    # keep the whole run within a few minutes: probe one step, halve the
    # prefix while (warm-up + timed steps) would take longer than budget_s
    budget_s = 150.0
    while True:
        _, _, us = oracle.ref_openmp(x[:k], args.m, threads=threads)
        if us <= 0:
            print(json.dumps({"impl": "reference", "unavailable": "openmpMdiscr run failed"}))
            return 0
        if (args.steps + args.warmup) * us * 1e-6 <= budget_s or k <= (1 << 20):
            break
        k //= 2
    xs = x[:k]
    for _ in range(max(args.warmup - 1, 0)):
        oracle.ref_openmp(xs, args.m, threads=threads)
    times = []
    for _ in range(args.steps):
        _, _, us = oracle.ref_openmp(xs, args.m, threads=threads)
        times.append(us * 1e-6)
    t = statistics.mean(times)
    value = k / t / 1e9
    sample = ("the whole input" if k == args.n else
              f"the first {k} elements of the same input (the whole array would need more host "
              "memory or time)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gelem/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": args.n, "m": args.m,
                   "seed": W.SEEDS["c2a"], "sample_per_step": k, "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "Gelem/s", "cores": threads, "kind": "reference",
                         "same_input": True,
                         "sample": f"openmpMdiscr (cuda_code/OpenmpMdiscr.h) on {sample}, its own "
                                   "gettimeofday timer"},
        "e2e": {"value": value, "unit": "Gelem/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mdx", choices=["mdx", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--m", type=int, default=M_DEFAULT)
    ap.add_argument("--e2e-steps", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other plain configurations")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched segmented measurement")
    ap.add_argument("--no-served", action="store_true",
                    help="skip the served-requests measurement")
    ap.add_argument("--no-sort", action="store_true",
                    help="skip the sort-based reference point")
    ap.add_argument("--distributed", action="store_true",
                    help="partition one array spread over the ranks (p2p transport)")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the batched segmented measurement and print its JSON")
    ap.add_argument("--batched-segments", type=int, default=100_000)
    ap.add_argument("--batched-keep", default="all", choices=["all", "large", "small"])
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    import mdiscriminator_b200 as mdx

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    if args.distributed:
        return distributed_main(args, torch, dist, mdx, dev, world, rank)

    if args.batched_only:
        peak, _ = peaks()
        res = batched_measurement(torch, mdx, dev, peak, steps=args.steps, warmup=args.warmup,
                                  num_segments=args.batched_segments, keep=args.batched_keep,
                                  with_plain=False)
        print(json.dumps(res))
        return

    n, m = args.n, args.m
    discr = ("mask", m) if (m & (m - 1)) == 0 else ("mod", m)
    from mdiscriminator_b200 import workloads as W
    d_in = make_input(torch, n, W.SEEDS["c2a"] + rank, dev)
    d_out = torch.empty_like(d_in)
    sizes = torch.empty(m, dtype=torch.uint32, device=dev)
    ws = mdx.new_workspace(mdx.workspace_size(n, mdx.ELEM_U32, m), dev)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up
    for _ in range(args.warmup):
        mdx.partition(d_in, discr, out=d_out, sizes=sizes, ws=ws)
    barrier()

    # timed region: K partitions on the path the tuning table picks for this
    # size (one cooperative kernel, or count + scatter with programmatic
    # dependent launch), events on the launching stream
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        mdx.partition(d_in, discr, out=d_out, sizes=sizes, ws=ws)
        ev[i][1].record(stream)
    t_end.record(stream)
    barrier()
    clk = clocks.stop()
    total_s = t_start.elapsed_time(t_end) * 1e-3
    if world > 1:
        tt = torch.tensor([total_s], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_s = float(tt.item())
    err = ws.error()
    if err != mdx.MDX_OK:
        raise SystemExit(f"device error during the timed region: {mdx.strerror(err)}")
    step_s = total_s / args.steps
    call_ms = [a.elapsed_time(b) for a, b in ev]
    value = world * n / step_s / 1e9
    # the two kernels apart (after the timed region): count and scatter as two
    # launches with an event between them (no dependent launch across it)
    kev = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(3)) for _ in range(10)]
    for _, mid, _ in kev:  # torch creates the CUDA event on its first record
        mid.record(stream)
    barrier()
    for a0, mid, a1 in kev:
        a0.record(stream)
        mdx.partition(d_in, discr, out=d_out, sizes=sizes, ws=ws, count_done_event=mid)
        a1.record(stream)
    barrier()
    count_ms = [a.elapsed_time(b) for a, b, _ in kev[2:]]
    scat_ms = [b.elapsed_time(c) for _, b, c in kev[2:]]
    split_call_ms = [a.elapsed_time(c) for a, _, c in kev[2:]]

    # end to end through the public API: every step copies its input from
    # pinned host memory, partitions it and copies the result and the sizes
    # back.  Three streams (host-to-device copies, partitions, device-to-host
    # copies) and two buffer sets, ordered by events, so that in steady state
    # one step's input and an earlier step's result cross PCIe at the same
    # time in the two directions while the partition runs in between.
    e2e_sets = []
    for k in range(2):
        h_in = torch.empty(n, dtype=torch.int32, pin_memory=True)
        h_in.copy_(d_in)
        e2e_sets.append({
            "h_in": h_in, "h_out": torch.empty(n, dtype=torch.int32, pin_memory=True),
            "h_sizes": torch.empty(m, dtype=torch.uint32, pin_memory=True),
            "d_in": torch.empty_like(d_in), "d_out": torch.empty_like(d_in),
            "sizes": torch.empty(m, dtype=torch.uint32, device=dev),
            "ws": mdx.new_workspace(mdx.workspace_size(n, mdx.ELEM_U32, m), dev),
            "in_ready": torch.cuda.Event(), "part_done": torch.cuda.Event(),
            "out_done": torch.cuda.Event()})
    s_h2d, s_cmp, s_d2h = (torch.cuda.Stream(device=dev) for _ in range(3))

    def e2e_step(i):
        b = e2e_sets[i % 2]
        if i >= 2:  # d_in of this set is free once step i - 2's partition read it
            s_h2d.wait_event(b["part_done"])
        with torch.cuda.stream(s_h2d):
            b["d_in"].copy_(b["h_in"], non_blocking=True)
            b["in_ready"].record(s_h2d)
        s_cmp.wait_event(b["in_ready"])
        if i >= 2:  # d_out of this set is free once step i - 2's result left
            s_cmp.wait_event(b["out_done"])
        mdx.partition(b["d_in"], discr, out=b["d_out"], sizes=b["sizes"], ws=b["ws"],
                      stream=s_cmp)
        b["part_done"].record(s_cmp)
        s_d2h.wait_event(b["part_done"])
        with torch.cuda.stream(s_d2h):
            b["h_out"].copy_(b["d_out"], non_blocking=True)
            b["h_sizes"].copy_(b["sizes"], non_blocking=True)
            b["out_done"].record(s_d2h)

    for i in range(2):
        e2e_step(i)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for st in (s_h2d, s_cmp, s_d2h):
        st.wait_event(e0)
    for i in range(args.e2e_steps):
        e2e_step(i)
    for st in (s_h2d, s_cmp, s_d2h):
        stream.wait_stream(st)
    e1.record(stream)
    barrier()
    e2e_s = e0.elapsed_time(e1) * 1e-3
    if world > 1:
        tt = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e_value = world * n * args.e2e_steps / e2e_s / 1e9
    # sanity: the last result equals the device result of the same input
    assert torch.equal(e2e_sets[(args.e2e_steps - 1) % 2]["h_out"].to(dev), d_out)
    # the bound of the e2e leg: the same copies alone, no partition -- as many
    # steps, the host-to-device copies on one stream and the device-to-host
    # copies on the other, both directions busy at once (pinned memory)
    a, b = e2e_sets
    c0 = torch.cuda.Event(enable_timing=True)
    c1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    c0.record(stream)
    s_h2d.wait_event(c0)
    s_d2h.wait_event(c0)
    for i in range(args.e2e_steps):
        with torch.cuda.stream(s_h2d):
            e2e_sets[i % 2]["d_in"].copy_(e2e_sets[i % 2]["h_in"], non_blocking=True)
        with torch.cuda.stream(s_d2h):
            e2e_sets[(i + 1) % 2]["h_out"].copy_(e2e_sets[(i + 1) % 2]["d_out"], non_blocking=True)
    stream.wait_stream(s_h2d)
    stream.wait_stream(s_d2h)
    c1.record(stream)
    torch.cuda.synchronize()
    copy_s = c0.elapsed_time(c1) * 1e-3 / args.e2e_steps
    pcie_gbs = n * 4 / copy_s / 1e9        # per direction, both directions busy
    e2e_bound = world * n / copy_s / 1e9   # elements/s if the copies were all a step cost
    del e2e_sets, a, b
    dist_leg = distributed_leg(args, torch, dist, dev, world, d_in, m, discr) if world > 1 else None

    if rank == 0:
        peak, peak_src = peaks()
        call_s = statistics.mean(call_ms) * 1e-3
        alg = 2 * n * 4 + 4 * m
        achieved = alg / call_s / 1e9
        cnt_s = statistics.mean(count_ms) * 1e-3
        sct_s = statistics.mean(scat_ms) * 1e-3
        tr = traffic_from_profiles()
        traffic = (tr["count_kernel_bytes"] + tr["scatter_kernel_bytes"]) if len(tr) == 2 else None
        roofline = {
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "peak_source": peak_src,
            "what": "one partition call on the tuned path against 2*N*4 + 4*m bytes",
            "path": ("count + scatter kernels, dependent launch"
                     if mdx.get_tuning(mdx.ELEM_U32, m, n)["plain_two_kernel"]
                     else "one cooperative kernel"),
            "frac_of_two_pass_bound": (3 * n * 4 + 4 * m) / call_s / 1e9 / peak,
            "kernels": {
                "count": {"ms": cnt_s * 1e3, "alg_bytes": n * 4,
                          "achieved_gbs": n * 4 / cnt_s / 1e9,
                          "frac": n * 4 / cnt_s / 1e9 / peak,
                          "traffic": tr.get("count_kernel_bytes")},
                "scatter": {"ms": sct_s * 1e3, "alg_bytes": 2 * n * 4,
                            "achieved_gbs": 2 * n * 4 / sct_s / 1e9,
                            "frac": 2 * n * 4 / sct_s / 1e9 / peak,
                            "traffic": tr.get("scatter_kernel_bytes")},
                "split_call_ms": statistics.mean(split_call_ms),
                "note": "kernels timed apart: 8 calls as two launches with an event "
                        "between count and scatter, after the timed region",
            },
        }
        configs = None
        if world == 1 and not args.no_configs:
            configs = configs_measurement(torch, mdx, dev, peak)
        batched = None
        if world == 1 and not args.no_batched:
            batched = batched_measurement(torch, mdx, dev, peak)
        sort_ref = None
        if world == 1 and not args.no_sort:
            sort_ref = sort_measurement(torch, d_in, d_out, m)
        served = None
        if world == 1 and not args.no_served:
            served = served_measurement(torch, mdx, dev, peak)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            import numpy as np
            x_host = d_in.cpu().numpy().view(np.uint32)
            del d_in, d_out
            torch.cuda.empty_cache()
            cpu, why = cpu_baseline(x_host, m, reps=2)
            del x_host
            if cpu is None:
                cpu = {"value": None, "unavailable": why}
        line = {
            "metric": METRIC, "value": value, "unit": "Gelem/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": n, "m": m, "discr": f"{discr[0]} {m}",
                       "seed": W.SEEDS["c2a"],
                       "l2": "inputs and outputs (1 GiB each) larger than L2; no flush",
                       "parallelism": f"independent arrays per rank x{world}" if world > 1
                       else "single GPU"},
            "e2e": {"value": e2e_value, "unit": "Gelem/s", "h2d_bytes_per_step": n * 4,
                    "d2h_bytes_per_step": n * 4 + m * 4,
                    "pcie_duplex_gbs": pcie_gbs, "copy_bound": e2e_bound,
                    "frac_of_copy_bound": e2e_value / e2e_bound,
                    "note": "copy_bound: the same number of steps of 1 GiB host-to-device and "
                            "1 GiB device-to-host copies, the two directions at once on the same "
                            "copy streams, no partition (CUDA events)"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "configs": configs,
            "batched": batched,
            "served": served,
            "sort_baseline": sort_ref,
            "clocks": clk,
            # kernels of this repository per timed step: count + scatter, or
            # the one cooperative kernel
            "gpu_launches": (2 if mdx.get_tuning(mdx.ELEM_U32, m, n)["plain_two_kernel"] else 1)
            * args.steps,
        }
        if dist_leg is not None:
            line["distributed"] = dist_leg
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
