"""One array partitioned across the ranks of a process group.

The reference partitions one array on one GPU (mdiscr<DISCR>,
cuda_code/MdiscrHost_optimized_clean.cu.h:9-15).  Here rank r of a process
group holds a contiguous chunk of a global input of N elements (chunks in rank
order); the result is the global stable partition -- exactly what one
mdiscr<DISCR> over the concatenated input returns -- cut into balanced output
chunks, plus the m global class sizes:

    output chunk q = positions [q * C, (q + 1) * C) within [0, N), the last
    rank every position from (R - 1) * C on, with C = A * ceil(N / (R * A))
    and A = 16 bytes of elements (so every chunk starts 16-byte aligned).

Where rank r's class-c elements go: base[r][c] = (elements of classes < c on
all ranks) + (elements of class c on ranks < r), then in input order.  So the
only exchange step is the all-gather of the R x m class counts, after which
every rank knows where each of its elements lands.

Transports:

``"p2p"`` (CUDA tensors, NCCL process group; the B200 path)
    mdx_dist_count counts the local chunk; one all-gather of the counts;
    mdx_dist_scatter ranks every element and stores it straight into the
    output chunk that owns its position -- the peers' chunks mapped into this
    process by CUDA IPC (no multicast), written over NVLink by the scatter
    kernel itself (bulk stores split at chunk boundaries); an all-reduce on
    the same stream is the completion barrier.  Data crosses NVLink once and
    HBM is read twice and written once per element, as on one GPU.

``"nccl"`` (any backend with send/recv; the baseline)
    A local partition (mdx.partition, or an injected function), the same
    count all-gather, then every class run is sent to the rank(s) owning its
    output positions with point-to-point send/recv straight into the
    receivers' chunks (:func:`exchange_plan`).  With gloo and CPU tensors it
    runs without a GPU, which is how the exchange logic is tested.
"""
from __future__ import annotations

import math
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from . import (ELEM_REC8, MdxError, MDX_ERR_INVALID, dist_count, dist_scatter, ipc_close,
               ipc_handle, ipc_open, make_discr, new_workspace, partition, workspace_size)


# ------------------------------------------------------------------ layout --
def out_chunk_elems(n_total: int, num_ranks: int, elem_bytes: int) -> int:
    """C: elements per output chunk (a multiple of 16 bytes of elements)."""
    a = 16 // elem_bytes
    return a * max(1, math.ceil(n_total / (num_ranks * a)))


def chunk_range(q: int, num_ranks: int, chunk: int, n_total: int) -> Tuple[int, int]:
    """[start, end) of output chunk q."""
    start = min(q * chunk, n_total)
    end = n_total if q == num_ranks - 1 else min((q + 1) * chunk, n_total)
    return start, max(start, end)


def class_bases(all_counts: np.ndarray) -> np.ndarray:
    """base[r][c] = (elements of classes < c on every rank) + (class c on ranks < r)."""
    cnt = np.asarray(all_counts, dtype=np.int64)
    tot = cnt.sum(axis=0)
    below_c = np.concatenate([[0], np.cumsum(tot)[:-1]])
    below_r = np.cumsum(cnt, axis=0) - cnt
    return below_c[None, :] + below_r


def exchange_plan(all_counts: np.ndarray, chunk: int, n_total: int) -> List[Tuple[int, int, int, int, int, int]]:
    """Pieces (src rank, dst rank, class, offset in src's locally partitioned
    array, offset in dst's output chunk, length) that move every element to its
    output position, ordered by (src, dst, class, position) -- the order in
    which both ends post their sends and receives."""
    cnt = np.asarray(all_counts, dtype=np.int64)
    R, m = cnt.shape
    base = class_bases(cnt)
    local_start = np.cumsum(cnt, axis=1) - cnt  # class c's run in a rank's local partition
    pieces = []
    for r in range(R):
        for c in range(m):
            g0, n = int(base[r, c]), int(cnt[r, c])
            done = 0
            while done < n:
                g = g0 + done
                q = min(g // chunk, R - 1)
                _, qend = chunk_range(q, R, chunk, n_total)
                take = min(n - done, qend - g)
                qstart, _ = chunk_range(q, R, chunk, n_total)
                pieces.append((r, q, c, int(local_start[r, c]) + done, g - qstart, take))
                done += take
    pieces.sort(key=lambda p: (p[0], p[1], p[2], p[3]))
    return pieces


# --------------------------------------------------------------- transports --
_peer_maps: Dict[bytes, int] = {}   # IPC handle -> base address of the mapping in this process
_workspaces: Dict[Tuple[int, int], object] = {}


def close_peer_maps() -> None:
    """Release every peer mapping opened by the "p2p" transport."""
    for h, p in list(_peer_maps.items()):
        try:
            ipc_close(p, 0)
        finally:
            _peer_maps.pop(h, None)


def _workspace(nbytes: int, device):
    key = (device.index or 0, nbytes)
    ws = _workspaces.get(key)
    if ws is None:
        ws = new_workspace(nbytes, device)
        _workspaces[key] = ws
    return ws


def _gather_counts(counts_i64, group, R):
    import torch
    import torch.distributed as dist
    parts = [torch.empty_like(counts_i64) for _ in range(R)]
    dist.all_gather(parts, counts_i64, group=group)
    return torch.stack(parts)


def _handle_row(out):
    """(offset, 8 handle words) of a tensor's allocation; zeros for none."""
    if out is not None and out.numel() > 0:
        h, off = ipc_handle(out)
        return [off] + [int(w) for w in np.frombuffer(h, dtype=np.int64)]
    return [0] * 9


def _peer_ptrs(rows, rank, out):
    """Device addresses of every rank's output chunk in this process (a
    handle seen before reuses its mapping)."""
    ptrs = []
    for q, v in enumerate(rows):
        hq = np.asarray(v[1:], dtype=np.int64).tobytes()
        if q == rank:
            ptrs.append(out.data_ptr())
        elif not any(hq):
            ptrs.append(0)
        else:
            if hq not in _peer_maps:
                _peer_maps[hq] = ipc_open(hq, 0)
            ptrs.append(_peer_maps[hq] + int(v[0]))
    return ptrs


def _partition_p2p(x_local, discr, m, group, R, rank, out, check):
    """The "p2p" transport: count, one all-gather of a row per rank (its m
    counts, its length, and -- when ``out`` is given -- its output chunk's
    allocation handle and offset), one read of the gathered table on the host
    (the call's only wait), the sharded scatter into the mapped chunks, and an
    all-reduce as the completion barrier."""
    import torch
    import torch.distributed as dist
    dev = x_local.device
    ebytes = x_local.element_size()
    n_local = x_local.numel()
    ws = _workspace(max(workspace_size(max(n_local, 1), ELEM_REC8 if ebytes == 8 else 0, m), 256),
                    dev)
    counts = dist_count(x_local, discr, ws)
    tail = torch.tensor([n_local] + _handle_row(out), dtype=torch.int64).pin_memory()
    row = torch.cat([counts.to(torch.int64), tail.to(dev, non_blocking=True)])
    parts = [torch.empty_like(row) for _ in range(R)]
    dist.all_gather(parts, row, group=group)
    table_dev = torch.stack(parts)
    table = table_dev.cpu().numpy()
    n_total = int(table[:, m].sum())
    chunk = out_chunk_elems(n_total, R, ebytes)
    a, b = chunk_range(rank, R, chunk, n_total)
    rows = table[:, m + 1:]
    if out is None:  # first call: the chunk exists only now, its handle goes round once more
        out = torch.empty(b - a, dtype=x_local.dtype, device=dev)
        mine = torch.tensor(_handle_row(out), dtype=torch.int64, device=dev)
        hparts = [torch.empty_like(mine) for _ in range(R)]
        dist.all_gather(hparts, mine, group=group)
        rows = torch.stack(hparts).cpu().numpy()
    elif out.numel() != b - a or out.dtype != x_local.dtype:
        raise MdxError(MDX_ERR_INVALID, "partition_distributed: out has the wrong shape or type")
    ptrs = _peer_ptrs(rows, rank, out)
    dist_scatter(x_local, discr, table_dev[:, :m].to(torch.uint32), rank, ptrs, chunk, n_total, ws)
    # completion barrier: no rank reads its chunk before every rank's stores
    # into it have finished
    flag = torch.zeros(1, dtype=torch.int64, device=dev)
    dist.all_reduce(flag, group=group)
    if check:
        err = ws.error()
        if err != 0:
            raise MdxError(err, "partition_distributed")
    return out, table[:, :m].sum(axis=0)


def partition_distributed(x_local, discr, group=None, transport: str = "auto", out=None,
                          local_partition: Optional[Callable] = None, check: bool = True):
    """Stable partition of the array whose rank-ordered chunks the ranks of
    ``group`` hold (``x_local``: this rank's chunk, 1-D int32/uint32 or
    int64/uint64 records).  Returns ``(out_chunk, sizes)``: this rank's output
    chunk of the layout in the module docstring and the m global class sizes
    (int64, host).  Every rank must call it with the same ``discr``.

    ``local_partition(x, m) -> (partitioned x, counts)`` replaces the local
    mdx.partition in the "nccl" transport (tests use it to run the exchange
    on CPU tensors).
    """
    import torch
    import torch.distributed as dist

    R = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dc = make_discr(discr)
    m = dc.m
    if transport == "auto":
        transport = "p2p" if x_local.is_cuda else "nccl"
    if transport == "p2p":
        return _partition_p2p(x_local, discr, m, group, R, rank, out, check)
    ebytes = x_local.element_size()
    n_local = x_local.numel()
    n_all = torch.tensor([n_local], dtype=torch.int64, device=x_local.device)
    parts = [torch.empty_like(n_all) for _ in range(R)]
    dist.all_gather(parts, n_all, group=group)
    n_total = int(sum(int(p.item()) for p in parts))
    chunk = out_chunk_elems(n_total, R, ebytes)
    a, b = chunk_range(rank, R, chunk, n_total)
    if out is None:
        out = torch.empty(b - a, dtype=x_local.dtype, device=x_local.device)
    elif out.numel() != b - a or out.dtype != x_local.dtype:
        raise MdxError(MDX_ERR_INVALID, "partition_distributed: out has the wrong shape or type")

    if transport != "nccl":
        raise MdxError(MDX_ERR_INVALID, f"unknown transport {transport!r}")
    if local_partition is None:
        loc, cnt = partition(x_local, discr)
        cnt = cnt.to(torch.int64)
    else:
        loc, cnt = local_partition(x_local, m)
        cnt = torch.as_tensor(cnt, dtype=torch.int64, device=x_local.device)
    all_counts = _gather_counts(cnt, group, R).cpu().numpy()
    ops = []
    for (src, dst, _c, soff, doff, ln) in exchange_plan(all_counts, chunk, n_total):
        if src == rank and dst == rank:
            out[doff:doff + ln].copy_(loc[soff:soff + ln])
        elif src == rank:
            ops.append(dist.P2POp(dist.isend, loc[soff:soff + ln].contiguous(),
                                  dist.get_global_rank(group, dst) if group is not None else dst,
                                  group))
        elif dst == rank:
            ops.append(dist.P2POp(dist.irecv, out[doff:doff + ln],
                                  dist.get_global_rank(group, src) if group is not None else src,
                                  group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    return out, all_counts.sum(axis=0)
