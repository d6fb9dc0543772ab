"""Distributed plain partition (mdiscriminator_b200.distributed).

CPU: the output layout and the exchange plan against the oracle's global
partition (pure numpy), and the whole "nccl" transport on world-size-2/3
gloo process groups with CPU tensors (local partitions done by the oracle, as
the checker stands in for each rank's GPU).  GPU: the fused sharded scatter
(mdx_dist_count + mdx_dist_scatter) with R ranks emulated in one process --
R output chunks in R buffers of one GPU, each rank's kernels launched in turn
(no kernel waits on another) -- and the "p2p" transport end to end on a
world-size-1 NCCL group.
"""
import os
import socket

import numpy as np
import pytest

import oracle
from mdiscriminator_b200 import distributed as D


def _split(n_total, R, rng):
    cuts = np.sort(rng.integers(0, n_total + 1, size=R - 1))
    return np.diff(np.concatenate([[0], cuts, [n_total]])).astype(np.int64)


def _global_case(seed, R, n_total, m, rng):
    x = oracle.fill_uniform_u32(n_total, seed)
    lens = _split(n_total, R, rng)
    starts = np.concatenate([[0], np.cumsum(lens)])
    return x, [x[starts[r]:starts[r + 1]] for r in range(R)]


@pytest.mark.parametrize("R", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("m", [1, 2, 3, 5, 8, 16])
def test_exchange_plan_places_every_element(R, m):
    rng = np.random.default_rng(100 * R + m)
    for n_total in (0, 1, 7, 100, 4099, 50_000):
        x, xs = _global_case(R + m + n_total, R, n_total, m, rng)
        loc = [oracle.partition(xr, m) for xr in xs]
        all_counts = np.stack([np.asarray(s, dtype=np.int64) for _, s in loc]) if R else None
        C = D.out_chunk_elems(n_total, R, 4)
        assert C % 4 == 0 and C > 0
        ranges = [D.chunk_range(q, R, C, n_total) for q in range(R)]
        assert ranges[0][0] == 0 and ranges[-1][1] == n_total
        assert all(ranges[q][1] == ranges[q + 1][0] for q in range(R - 1))
        outs = [np.full(b - a, 0xDEADBEEF, dtype=np.uint32) for a, b in ranges]
        for (src, dst, _c, soff, doff, ln) in D.exchange_plan(all_counts, C, n_total):
            outs[dst][doff:doff + ln] = loc[src][0][soff:soff + ln]
        eo, es = oracle.partition(x, m)
        assert np.array_equal(np.concatenate(outs) if outs else eo, eo)
        assert np.array_equal(all_counts.sum(axis=0), es)


def test_class_bases_match_the_definition():
    cnt = np.array([[3, 0, 2], [1, 4, 0], [0, 2, 5]])
    b = D.class_bases(cnt)
    # class 0: ranks 0,1,2 at 0,3,4; class 1 starts at 4: ranks at 4,4,8; class 2 at 10: 10,12,12
    assert b.tolist() == [[0, 4, 10], [3, 4, 12], [4, 8, 12]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, n_total, m, seed, q):
    import torch
    import torch.distributed as dist
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                world_size=world)
        rng = np.random.default_rng(seed)
        x, xs = _global_case(seed, world, n_total, m, rng)
        xr = torch.from_numpy(xs[rank].view(np.int32).copy())

        def local(t, mm):  # the oracle stands in for the rank's GPU partition
            o, s = oracle.partition(t.numpy().view(np.uint32), mm)
            return torch.from_numpy(o.view(np.int32).copy()), np.asarray(s, dtype=np.int64)

        out, sizes = D.partition_distributed(xr, ("mod", m), transport="nccl",
                                             local_partition=local)
        eo, es = oracle.partition(x, m)
        C = D.out_chunk_elems(n_total, world, 4)
        a, b = D.chunk_range(rank, world, C, n_total)
        ok = np.array_equal(out.numpy().view(np.uint32), eo[a:b]) and np.array_equal(sizes, es)
        dist.destroy_process_group()
        q.put((rank, bool(ok), ""))
    except Exception as e:  # reported to the parent
        q.put((rank, False, repr(e)))


@pytest.mark.parametrize("world,n_total,m", [(2, 30_011, 5), (3, 10_000, 8), (2, 5, 3)])
def test_gloo_ranks_exchange_runs(world, n_total, m):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, n_total, m, 7 + world, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(ok for _, ok, _ in res), res


# ---------------------------------------------------------------------- GPU --
def _emulate(torch, mdx, x, lens, discr, m, elem_dtype):
    """Every rank's count + sharded scatter on one GPU; returns the output chunks."""
    R = len(lens)
    starts = np.concatenate([[0], np.cumsum(lens)])
    n_total = int(starts[-1])
    w = np.dtype(elem_dtype).itemsize
    xd = [torch.from_numpy(x[starts[r]:starts[r + 1]].copy()).cuda() for r in range(R)]
    elem = mdx.ELEM_REC8 if w == 8 else mdx.ELEM_U32
    wss = [mdx.new_workspace(max(mdx.workspace_size(max(int(lens[r]), 1), elem, m), 256))
           for r in range(R)]
    counts = [mdx.dist_count(xd[r], discr, wss[r]) for r in range(R)]
    all_counts = torch.stack(counts)
    C = D.out_chunk_elems(n_total, R, w)
    rngs = [D.chunk_range(q, R, C, n_total) for q in range(R)]
    outs = [torch.full((b - a,), -1, dtype=xd[0].dtype, device="cuda") for a, b in rngs]
    sizes = [mdx.dist_scatter(xd[r], discr, all_counts, r, [o.data_ptr() for o in outs], C,
                              n_total, wss[r]) for r in range(R)]
    torch.cuda.synchronize()
    return outs, sizes, wss, all_counts, xd, C


@pytest.mark.gpu
@pytest.mark.parametrize("R", [1, 2, 3, 4, 7])
@pytest.mark.parametrize("m", [2, 5, 8, 16, 40])
def test_sharded_scatter_equals_global_partition(cuda_ready, R, m):
    torch = cuda_ready
    import mdiscriminator_b200 as mdx
    rng = np.random.default_rng(R * 31 + m)
    for n_total in (3, 4096 * 3 + 17, 1_000_003):
        x = oracle.fill_uniform_u32(n_total, R + m)
        lens = _split(n_total, R, rng)
        outs, sizes, wss, _, _, _ = _emulate(torch, mdx, x.view(np.int32), lens, ("mod", m), m,
                                             np.int32)
        eo, es = oracle.partition(x, m)
        got = torch.cat(outs).cpu().numpy().view(np.uint32)
        assert np.array_equal(got, eo), (R, m, n_total)
        for s in sizes:
            assert np.array_equal(s.cpu().numpy(), es)
        assert all(ws.error() == mdx.MDX_OK for ws in wss)


@pytest.mark.gpu
def test_sharded_scatter_records(cuda_ready):
    torch = cuda_ready
    import mdiscriminator_b200 as mdx
    n_total, R, m = 600_001, 3, 16
    keys = oracle.fill_uniform_u32(n_total, 3)
    rec = (keys.astype(np.uint64) | (np.arange(n_total, dtype=np.uint64) << 32)).view(np.int64)
    lens = np.array([200_000, 1, n_total - 200_001])
    outs, _, _, _, _, _ = _emulate(torch, mdx, rec, lens, ("mask", m), m, np.int64)
    got = torch.cat(outs).cpu().numpy().view(np.uint64)
    eo, _ = oracle.partition(rec.view(np.uint64), m, kind=oracle.DISCR_MASK)
    assert np.array_equal(got, eo)


@pytest.mark.gpu
def test_inconsistent_counts_write_nothing(cuda_ready):
    torch = cuda_ready
    import mdiscriminator_b200 as mdx
    n_total, R, m = 100_000, 2, 4
    x = oracle.fill_uniform_u32(n_total, 5).view(np.int32)
    lens = np.array([50_000, 50_000])
    outs, _, wss, all_counts, xd, C = _emulate(torch, mdx, x, lens, ("mod", m), m, np.int32)
    for o in outs:
        o.fill_(-1)
    ptrs = [o.data_ptr() for o in outs]
    # Each rank checks what it can: its own row of the table against its own
    # count, and the table's total against n_total.  A rank that fails either
    # check writes nothing (a rank that passes both stays inside [0, n_total)).
    bad_np = all_counts.cpu().numpy().copy()
    bad_np[1, 0] += 1  # rank 1's row disagrees with its own count (total adjusted)
    bad = torch.from_numpy(bad_np).cuda()
    torch.cuda.synchronize()
    mdx.dist_scatter(xd[1], ("mod", m), bad, 1, ptrs, C, n_total + 1, wss[1])
    torch.cuda.synchronize()
    assert all(bool((o == -1).all()) for o in outs)
    assert wss[1].error() == mdx.MDX_ERR_INVALID
    # rank 0: its row is right but the total is not
    mdx.dist_scatter(xd[0], ("mod", m), all_counts, 0, ptrs, C, n_total + 5, wss[0])
    torch.cuda.synchronize()
    assert all(bool((o == -1).all()) for o in outs)
    assert wss[0].error() == mdx.MDX_ERR_INVALID
    # and the same workspaces work again with consistent counts
    for r in range(R):
        mdx.dist_scatter(xd[r], ("mod", m), all_counts, r, ptrs, C, n_total, wss[r])
    torch.cuda.synchronize()
    eo, _ = oracle.partition(x.view(np.uint32), m)
    assert np.array_equal(torch.cat(outs).cpu().numpy().view(np.uint32), eo)
    with pytest.raises(mdx.MdxError):  # misaligned chunk size
        mdx.dist_scatter(xd[0], ("mod", m), all_counts, 0, [o.data_ptr() for o in outs], C + 1,
                         n_total, wss[0])


@pytest.mark.gpu
def test_p2p_transport_on_one_rank(cuda_ready):
    torch = cuda_ready
    import torch.distributed as dist
    os.environ.setdefault("NCCL_NVLS_ENABLE", "0")
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1, device_id=torch.device("cuda", 0))
    try:
        x = oracle.fill_uniform_u32(777_777, 11)
        out, sizes = D.partition_distributed(torch.from_numpy(x.view(np.int32)).cuda(), ("mod", 6),
                                             transport="p2p")
        eo, es = oracle.partition(x, 6)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), eo)
        assert np.array_equal(sizes, es)
    finally:
        dist.destroy_process_group()
        D.close_peer_maps()
