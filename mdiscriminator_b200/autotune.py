"""Autotuner: times the kernels' run-time knobs on this GPU and writes the
table mdiscriminator_b200 loads at import (tuning.json).

Keys: element layout (4-byte values / 8-byte records), class bound (the
smallest power of two >= m) and a range of ceil(log2 n).  Knobs:

* plain path: count and scatter as two kernels against one cooperative
  kernel (`plain_two_kernel`), CTAs per SM of the chunk grid
  (`plain_ctas_per_sm`), the tile geometry (`tile_bytes`: 64 or 32 bytes of
  a tile per thread, 256 threads; two-kernel path) and, for the one-kernel
  path, the share of every chunk drained by ticket (`pool_pct`);
* segmented path: tiles per run of a large segment (`run_tiles`),
  small-segment groups per work item (`group_batch`) and whether segments of
  two tiles are read once by the medium-segment kernel (`mid_tiles`).

The reference picked its block shapes by recompiling with -D macros and
timing them (cuda_code/run.py:12-96); here the choice is made at run time.

Usage (on the GPU):  python -m mdiscriminator_b200.autotune [--out PATH] [--quick]
"""
from __future__ import annotations

import argparse
import itertools
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))

import mdiscriminator_b200 as mdx  # noqa: E402

# n buckets: (timed n of 4-byte values, ceil(log2 n) range the winner is
# installed for); 8-byte records are timed at half the count (same bytes)
BUCKETS = [(1 << 20, (0, 21)), (1 << 24, (22, 25)), (1 << 28, (26, 33))]

# plain-path candidates: (plain_two_kernel, plain_ctas_per_sm, pool_pct, tile_bytes,
# tile_threads)
PLAIN_CANDIDATES = [(1, 4, 0, 64, 256), (1, 3, 0, 64, 256), (1, 0, 0, 64, 256),
                    (1, 4, 0, 32, 256), (1, 0, 0, 32, 256), (1, 0, 0, 64, 512),
                    (0, 4, 100, 64, 256), (0, 4, 10, 64, 256), (0, 4, 20, 64, 256),
                    (0, 4, 33, 64, 256), (0, 3, 10, 64, 256)]


def timeit(fn, torch, reps=20, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def lognormal_offsets(n_target, seed):
    rng = np.random.default_rng(seed)
    lengths = []
    total = 0
    while total < n_target:
        L = int(np.clip(np.rint(rng.lognormal(math.log(1024), 1.5)), 1, 1 << 22))
        L = min(L, n_target - total)
        lengths.append(L)
        total += L
    return np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=mdx.TUNING_PATH)
    ap.add_argument("--quick", action="store_true", help="fewer candidates and sizes")
    args = ap.parse_args(argv)
    import torch
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(1)
    entries = []
    bounds = [2, 4, 8, 16] if args.quick else [2, 4, 8, 16, 32, 64]
    buckets = BUCKETS[1:] if args.quick else BUCKETS
    t0 = time.time()
    for elem in (mdx.ELEM_U32, mdx.ELEM_REC8):
        ename = "u32" if elem == mdx.ELEM_U32 else "rec8"
        dtype = torch.int32 if elem == mdx.ELEM_U32 else torch.int64
        for n4, (lo, hi) in buckets:
            n = n4 if elem == mdx.ELEM_U32 else n4 // 2
            d = torch.randint(0, 1 << 31, (n,), device=dev, dtype=torch.int64, generator=g).to(dtype)
            out = torch.empty_like(d)
            ws = mdx.new_workspace(mdx.workspace_size(n, elem, 64), dev)
            for M in bounds:
                sizes = torch.empty(M, dtype=torch.uint32, device=dev)
                best = None
                for two, k, pool, tb, tt in PLAIN_CANDIDATES:
                    if tt == 512 and M > 16:  # 512-thread tiles serve m <= 16 only
                        continue
                    mdx.set_tuning(elem, M, lo, hi, plain_ctas_per_sm=k, plain_two_kernel=two,
                                   pool_pct=pool, tile_bytes=tb, tile_threads=tt)
                    ms = timeit(lambda: mdx.partition(d, ("mask", M), out=out, sizes=sizes, ws=ws),
                                torch)
                    if ws.error() != mdx.MDX_OK:
                        raise SystemExit(f"device error while tuning {ename} m={M}")
                    if best is None or ms < best[0]:
                        best = (ms, k, two, pool, tb, tt)
                entries.append({"elem": ename, "m": M, "log2_n": [lo, hi], "path": "plain",
                                "plain_ctas_per_sm": best[1], "plain_two_kernel": best[2],
                                "pool_pct": best[3], "tile_bytes": best[4],
                                "tile_threads": best[5], "ms": best[0]})
                mdx.set_tuning(elem, M, lo, hi, plain_ctas_per_sm=best[1],
                               plain_two_kernel=best[2], pool_pct=best[3], tile_bytes=best[4],
                               tile_threads=best[5])
            del d, out, ws
        seg_bounds = [2, 4, 8, 16]
        for n4, (lo, hi) in buckets:
            n_target = min(n4 if elem == mdx.ELEM_U32 else n4 // 2, 1 << 27)
            offs = lognormal_offsets(n_target, 3)
            n = int(offs[-1])
            S = len(offs) - 1
            d = torch.randint(0, 1 << 31, (n,), device=dev, dtype=torch.int64, generator=g).to(dtype)
            out = torch.empty_like(d)
            do = torch.from_numpy(offs).to(dev)
            ws = mdx.new_workspace(mdx.segmented_workspace_size(n, S, elem, 16), dev)
            cands = list(itertools.product((2, 4, 8, 16), (2, 4, 8, 16)))
            if args.quick:
                cands = list(itertools.product((4, 8, 16), (8,)))
            for M in seg_bounds:
                ss = torch.empty((S, M), dtype=torch.uint32, device=dev)
                pe = next(e for e in entries
                          if e["elem"] == ename and e["m"] == M and e["path"] == "plain"
                          and e["log2_n"] == [lo, hi])
                plain_k, plain_two, pool = pe["plain_ctas_per_sm"], pe["plain_two_kernel"], pe["pool_pct"]
                tb, tt = pe["tile_bytes"], pe["tile_threads"]
                best = None
                # (run_tiles, group_batch) without medium segments, then the
                # winner with the medium-segment kernel on
                for cand in [(rt, gb, 1) for rt, gb in cands] + [None]:
                    rt, gb, mid = cand if cand is not None else (best[1], best[2], 2)
                    mdx.set_tuning(elem, M, lo, hi, plain_ctas_per_sm=plain_k,
                                   plain_two_kernel=plain_two, pool_pct=pool, tile_bytes=tb,
                                   tile_threads=tt, run_tiles=rt, group_batch=gb, mid_tiles=mid)
                    ms = timeit(lambda: mdx.partition_segmented(d, do, ("mask", M), out=out,
                                                                seg_sizes=ss, ws=ws), torch)
                    if best is None or ms < best[0]:
                        best = (ms, rt, gb, mid)
                entries.append({"elem": ename, "m": M, "log2_n": [lo, hi], "path": "segmented",
                                "plain_ctas_per_sm": plain_k, "plain_two_kernel": plain_two,
                                "pool_pct": pool, "tile_bytes": tb, "tile_threads": tt,
                                "run_tiles": best[1],
                                "group_batch": best[2], "mid_tiles": best[3], "ms": best[0]})
                mdx.set_tuning(elem, M, lo, hi, plain_ctas_per_sm=plain_k,
                               plain_two_kernel=plain_two, pool_pct=pool, tile_bytes=tb,
                               tile_threads=tt, run_tiles=best[1], group_batch=best[2],
                               mid_tiles=best[3])
            del d, out, ws
    # one entry per key: the segmented entry (it carries the plain knob too)
    merged = {}
    for e in entries:
        key = (e["elem"], e["m"], tuple(e["log2_n"]))
        if key not in merged or e["path"] == "segmented":
            merged[key] = e
    table = {"device": torch.cuda.get_device_name(0), "tuned_in_s": round(time.time() - t0, 1),
             "entries": list(merged.values()), "timings": entries}
    with open(args.out, "w") as f:
        json.dump(table, f, indent=1)
    print(f"wrote {len(merged)} entries to {args.out} in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
