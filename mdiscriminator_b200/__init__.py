"""mdiscriminator_b200 -- B200-native stable m-way partition (m-discriminator).

The Python layer mirrors the reference's host entry points and forwards to the
C ABI of ``libmdx.so`` (``include/mdx.h``); torch tensors only carry device
memory and streams.  There is no CPU fallback: if the CUDA library is missing
or a tensor is not on a CUDA device, the call raises.

Reference entry points and their counterparts here:

* ``mdiscr<DISCR>(n, num_hwd_thds, d_in, d_out) -> TupleType``
  (cuda_code/MdiscrHost_optimized_clean.cu.h:9-15)  ->  :func:`mdiscr`
* ``mdiscr<DISCR>(n, in, out, int* sizes)`` with head-flag sizes
  (cuda_code/MdiscrHost_baseline.cu.h:23-28)        ->  :func:`partition` (``headflags=True``)
* ``mdiscrSegm<DISCR>(n, in, segment_sizes, out, new_sizes)``
  (cuda_code/MdiscrSegmHost.cu.h:36-42)             ->  :func:`mdiscr_segm`,
  and the offsets form :func:`partition_segmented`.

A discriminator is ``("mod", m)`` -- ``Mod<N>::apply = x % N``
(HelpersCommon.h:1200-1210) -- or ``("mask", m)`` -- ``Mod4``/``Mod8``
``apply = x & (m-1)`` (HelpersCommon.h:587-596, 840-849).  4-byte elements
are u32 values; 8-byte elements are ``{u32 key, u32 payload}`` records whose
class comes from the key (``ModArray<N,2>``, MdiscrHost_arrays.cu.h:26-36).
"""
from __future__ import annotations

import ctypes
import os
import threading
from dataclasses import dataclass
from typing import Optional, Tuple

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdx.so")

MDX_OK = 0
MDX_ERR_INVALID = 1
MDX_ERR_WORKSPACE = 2
MDX_ERR_CUDA = 3
MDX_ERR_TIMEOUT = 4
MDX_ERR_UNSUPPORTED = 5
MDX_ERR_SEGMENTS = 6
MDX_ERR_CANCELLED = 7

ELEM_U32 = 0
ELEM_REC8 = 1
ELEM_REC16 = 2  # 16-byte records, plain partitions only
DISCR_MOD = 0
DISCR_MASK = 1
MAX_CLASSES = 64


class MdxError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {strerror(status)} (status {status})" if what else strerror(status))


class Discr(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("m", ctypes.c_uint32)]


class Column(ctypes.Structure):
    _fields_ = [("inp", ctypes.c_void_p), ("out", ctypes.c_void_p), ("elem_bytes", ctypes.c_uint32)]


class Tuning(ctypes.Structure):
    _fields_ = [("plain_ctas_per_sm", ctypes.c_uint32), ("run_tiles", ctypes.c_uint32),
                ("group_batch", ctypes.c_uint32), ("plain_two_kernel", ctypes.c_uint32),
                ("pool_pct", ctypes.c_uint32), ("mid_tiles", ctypes.c_uint32),
                ("tile_bytes", ctypes.c_uint32), ("tile_threads", ctypes.c_uint32)]


TUNING_PATH = os.path.join(HERE, "tuning.json")


def set_tuning(elem: int, m: int, log2_n_lo: int, log2_n_hi: int, **knobs) -> None:
    """Install run-time knobs for (element layout, class bound of m, n buckets)."""
    t = Tuning(**{k: int(v) for k, v in knobs.items() if k in dict(Tuning._fields_)})
    _check(lib().mdx_set_tuning(elem, m, log2_n_lo, log2_n_hi, ctypes.byref(t)), "mdx_set_tuning")


def get_tuning(elem: int, m: int, n: int) -> dict:
    t = Tuning()
    _check(lib().mdx_get_tuning(elem, m, n, ctypes.byref(t)), "mdx_get_tuning")
    return {name: getattr(t, name) for name, _ in Tuning._fields_}


def load_tuning(path: str, missing_ok: bool = False) -> int:
    """Install the autotuner's table (mdiscriminator_b200/autotune.py output)."""
    import json
    if not os.path.exists(path):
        if missing_ok:
            return 0
        raise FileNotFoundError(path)
    with open(path) as f:
        table = json.load(f)
    k = 0
    for e in table.get("entries", []):
        elem = ELEM_REC8 if e["elem"] == "rec8" else ELEM_U32
        lo, hi = e["log2_n"]
        set_tuning(elem, e["m"], lo, hi, **{x: e[x] for x in ("plain_ctas_per_sm", "run_tiles",
                                                             "group_batch", "plain_two_kernel",
                                                             "pool_pct", "mid_tiles",
                                                             "tile_bytes", "tile_threads")
                                                  if x in e})
        k += 1
    return k


_lib = None
_lib_lock = threading.Lock()


def lib() -> ctypes.CDLL:
    """Load libmdx.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"{LIB_PATH} is missing: run mdiscriminator_b200.build.build()")
            L = ctypes.CDLL(LIB_PATH)
            vp, u64, u32, sz = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_size_t
            st = ctypes.c_int
            L.mdx_workspace_size.argtypes = [u64, ctypes.c_int, u32]
            L.mdx_workspace_size.restype = sz
            L.mdx_segmented_workspace_size.argtypes = [u64, u64, ctypes.c_int, u32]
            L.mdx_segmented_workspace_size.restype = sz
            L.mdx_mdiscr_segm_workspace_size.argtypes = [u64, ctypes.c_int, u32]
            L.mdx_mdiscr_segm_workspace_size.restype = sz
            L.mdx_workspace_init.argtypes = [vp, sz, vp]
            L.mdx_workspace_init.restype = st
            L.mdx_workspace_error.argtypes = [vp, vp]
            L.mdx_workspace_error.restype = st
            L.mdx_partition.argtypes = [vp, vp, u64, ctypes.c_int, Discr, vp, vp, vp, sz, vp]
            L.mdx_partition.restype = st
            L.mdx_partition_timed.argtypes = [vp, vp, u64, ctypes.c_int, Discr, vp, vp, vp, sz, vp,
                                              vp]
            L.mdx_partition_timed.restype = st
            L.mdx_mdiscr.argtypes = [u32, u32, vp, vp, ctypes.c_int, Discr, vp, vp, sz, vp]
            L.mdx_mdiscr.restype = st
            L.mdx_partition_segmented.argtypes = [vp, vp, u64, ctypes.c_int, Discr, vp, u64, vp,
                                                  vp, vp, sz, vp]
            L.mdx_partition_segmented.restype = st
            L.mdx_partition_segmented_multi.argtypes = [vp, vp, u64, ctypes.c_int, vp, u32, vp, u64,
                                                        vp, vp, vp, sz, vp]
            L.mdx_partition_segmented_multi.restype = st
            L.mdx_mdiscr_segm.argtypes = [u32, vp, vp, vp, vp, ctypes.c_int, Discr, vp, sz, vp]
            L.mdx_mdiscr_segm.restype = st
            L.mdx_graph_partition.argtypes = [ctypes.POINTER(vp), vp, vp, u64, ctypes.c_int, Discr,
                                              vp, vp, vp, sz]
            L.mdx_graph_partition.restype = st
            L.mdx_graph_partition_segmented.argtypes = [ctypes.POINTER(vp), vp, vp, u64, ctypes.c_int,
                                                        Discr, vp, u64, vp, vp, vp, sz]
            L.mdx_graph_partition_segmented.restype = st
            L.mdx_graph_launch.argtypes = [vp, vp]
            L.mdx_graph_launch.restype = st
            L.mdx_graph_destroy.argtypes = [vp]
            L.mdx_graph_destroy.restype = st
            L.mdx_set_tuning.argtypes = [ctypes.c_int, u32, u32, u32, ctypes.POINTER(Tuning)]
            L.mdx_set_tuning.restype = st
            L.mdx_get_tuning.argtypes = [ctypes.c_int, u32, u64, ctypes.POINTER(Tuning)]
            L.mdx_get_tuning.restype = st
            L.mdx_records_workspace_size.argtypes = [u64, u32, u32]
            L.mdx_records_workspace_size.restype = sz
            L.mdx_partition_records.argtypes = [vp, vp, u64, u32, Discr, vp, vp, vp, sz, vp]
            L.mdx_partition_records.restype = st
            L.mdx_columns_workspace_size.argtypes = [u64, u32]
            L.mdx_columns_workspace_size.restype = sz
            L.mdx_partition_columns.argtypes = [ctypes.POINTER(Column), u32, u64, Discr, vp, vp, vp,
                                                sz, vp]
            L.mdx_partition_columns.restype = st
            L.mdx_dist_count.argtypes = [vp, u64, ctypes.c_int, Discr, vp, vp, sz, vp]
            L.mdx_dist_count.restype = st
            L.mdx_dist_scatter.argtypes = [vp, u64, ctypes.c_int, Discr, vp, u32, u32,
                                           ctypes.POINTER(vp), u64, u64, vp, vp, sz, vp]
            L.mdx_dist_scatter.restype = st
            L.mdx_ipc_get_handle.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(u64)]
            L.mdx_ipc_get_handle.restype = st
            L.mdx_ipc_open.argtypes = [ctypes.c_char_p, u64, ctypes.POINTER(vp)]
            L.mdx_ipc_open.restype = st
            L.mdx_ipc_close.argtypes = [vp, u64]
            L.mdx_ipc_close.restype = st
            L.mdx_strerror.argtypes = [st]
            L.mdx_strerror.restype = ctypes.c_char_p
            L.mdx_version.argtypes = []
            L.mdx_version.restype = ctypes.c_char_p
            _lib = L
            load_tuning(TUNING_PATH, missing_ok=True)
    return _lib


def strerror(status: int) -> str:
    try:
        return lib().mdx_strerror(status).decode()
    except ImportError:
        return f"status {status}"


def version() -> str:
    return lib().mdx_version().decode()


def _check(status: int, what: str) -> None:
    if status != MDX_OK:
        raise MdxError(status, what)


def make_discr(discr) -> Discr:
    """``("mod", m)`` / ``("mask", m)`` / ``m`` (= mod) -> the C struct."""
    if isinstance(discr, Discr):
        return discr
    if isinstance(discr, int):
        return Discr(DISCR_MOD, discr)
    kind, m = discr
    k = {"mod": DISCR_MOD, "mask": DISCR_MASK}.get(kind, kind)
    return Discr(int(k), int(m))


# --------------------------------------------------------------- workspaces --
@dataclass
class Workspace:
    """A device workspace for the C ABI, zero-initialised once (mdx_workspace_init)."""
    tensor: object
    nbytes: int

    @property
    def ptr(self) -> int:
        return self.tensor.data_ptr()

    def error(self, stream=None) -> int:
        """Synchronise and return (and clear) the latched device error status."""
        return lib().mdx_workspace_error(ctypes.c_void_p(self.ptr), _stream_ptr(stream))


_ws_cache = {}
_ws_lock = threading.Lock()


def _torch():
    import torch  # plumbing: device memory and streams
    return torch


def _stream_ptr(stream) -> ctypes.c_void_p:
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def workspace(nbytes: int, device=None, stream=None) -> Workspace:
    """The cached workspace of at least ``nbytes`` on ``device`` (grown on demand).

    A cached workspace serves one call at a time; calls on different streams
    that run concurrently need their own (:func:`new_workspace`).
    """
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else
                       torch.device(device).index or 0)
    with _ws_lock:
        ws = _ws_cache.get(dev.index)
        if ws is None or ws.nbytes < nbytes:
            ws = new_workspace(max(nbytes, 1 << 20), dev, stream)
            _ws_cache[dev.index] = ws
        return ws


def new_workspace(nbytes: int, device=None, stream=None) -> Workspace:
    torch = _torch()
    t = torch.empty(int(nbytes), dtype=torch.uint8, device=device or "cuda")
    _check(lib().mdx_workspace_init(ctypes.c_void_p(t.data_ptr()), int(nbytes),
                                    _stream_ptr(stream)), "mdx_workspace_init")
    return Workspace(t, int(nbytes))


def _elem_of(t) -> int:
    es = t.element_size()
    if es == 4:
        return ELEM_U32
    if es == 8:
        return ELEM_REC8
    raise TypeError(f"unsupported element size {es} (4-byte values or 8-byte records)")


def _require_cuda(*tensors) -> None:
    for t in tensors:
        if t is None:
            continue
        if not t.is_cuda:
            raise ValueError("mdiscriminator_b200 operates on CUDA tensors only (no CPU path)")
        if not t.is_contiguous():
            raise ValueError("tensors must be contiguous")


# --------------------------------------------------------------- plain path --
def workspace_size(n: int, elem: int, m: int) -> int:
    return int(lib().mdx_workspace_size(int(n), int(elem), int(m)))


def partition(d_in, discr, out=None, sizes=None, headflags=False, ws: Optional[Workspace] = None,
              stream=None, count_done_event=None):
    """Stable partition of a 1-D CUDA tensor (async on the current stream).

    Returns ``(out, sizes)`` with ``sizes`` a device u32 tensor of m class
    sizes, plus the head-flag array when ``headflags`` is true (a tensor, or
    True to allocate one).  ``count_done_event`` (a ``torch.cuda.Event``) is
    recorded between the counting and the scattering kernel.
    """
    torch = _torch()
    _require_cuda(d_in)
    dc = make_discr(discr)
    n = d_in.numel()
    elem = _elem_of(d_in)
    if out is None:
        out = torch.empty_like(d_in)
    if sizes is None:
        sizes = torch.empty(dc.m, dtype=torch.uint32, device=d_in.device)
    hf = None
    if headflags is True:
        hf = torch.empty(n, dtype=torch.uint32, device=d_in.device)
    elif headflags is not False and headflags is not None:
        hf = headflags
    _require_cuda(out, sizes, hf)
    need = workspace_size(n, elem, dc.m)
    if need == 0:
        raise MdxError(MDX_ERR_INVALID, "mdx_workspace_size")
    ws = ws or workspace(need, d_in.device, stream)
    ev = ctypes.c_void_p(count_done_event.cuda_event if count_done_event is not None else 0)
    st = lib().mdx_partition_timed(ctypes.c_void_p(d_in.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), n, elem, dc,
                                   ctypes.c_void_p(sizes.data_ptr()),
                                   ctypes.c_void_p(hf.data_ptr() if hf is not None else 0),
                                   ctypes.c_void_p(ws.ptr), ws.nbytes, _stream_ptr(stream), ev)
    _check(st, "mdx_partition")
    return (out, sizes, hf) if hf is not None else (out, sizes)


# ------------------------------------------------------------ wide elements --
def partition_records(d_in, record_bytes: int, discr, out=None, sizes=None, headflags=False,
                      ws: Optional[Workspace] = None, stream=None):
    """Stable partition of n records of ``record_bytes`` (a multiple of 4) held
    in the byte view of ``d_in`` (any dtype, n * record_bytes bytes); the class
    comes from each record's first u32 word (mdx_partition_records).  Returns
    ``(out, sizes)`` [, head flags]."""
    torch = _torch()
    _require_cuda(d_in)
    dc = make_discr(discr)
    nbytes = d_in.numel() * d_in.element_size()
    if record_bytes < 4 or record_bytes % 4 or nbytes % record_bytes:
        raise MdxError(MDX_ERR_INVALID, "partition_records: bad record size")
    n = nbytes // record_bytes
    if out is None:
        out = torch.empty_like(d_in)
    if sizes is None:
        sizes = torch.empty(dc.m, dtype=torch.uint32, device=d_in.device)
    hf = torch.empty(n, dtype=torch.uint32, device=d_in.device) if headflags is True else (
        headflags if headflags not in (False, None) else None)
    need = int(lib().mdx_records_workspace_size(n, record_bytes, dc.m))
    ws = ws or workspace(need, d_in.device, stream)
    _check(lib().mdx_partition_records(ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                       n, record_bytes, dc, ctypes.c_void_p(sizes.data_ptr()),
                                       ctypes.c_void_p(hf.data_ptr() if hf is not None else 0),
                                       ctypes.c_void_p(ws.ptr), ws.nbytes, _stream_ptr(stream)),
           "mdx_partition_records")
    return (out, sizes, hf) if hf is not None else (out, sizes)


def partition_columns(columns, discr, outs=None, sizes=None, headflags=False,
                      ws: Optional[Workspace] = None, stream=None):
    """Stable partition of rows held in several 1-D CUDA tensors of equal
    length (``columns[0]``: the u32/i32 key the class comes from; the others
    of 1, 2, 4 or 8 bytes per element follow its rows; mdx_partition_columns).
    Returns ``(outs, sizes)`` [, head flags]."""
    torch = _torch()
    _require_cuda(*columns)
    dc = make_discr(discr)
    n = columns[0].numel()
    if any(c.numel() != n for c in columns) or columns[0].element_size() != 4:
        raise MdxError(MDX_ERR_INVALID, "partition_columns: columns of one length, a 4-byte key")
    outs = outs or [torch.empty_like(c) for c in columns]
    if sizes is None:
        sizes = torch.empty(dc.m, dtype=torch.uint32, device=columns[0].device)
    hf = torch.empty(n, dtype=torch.uint32, device=columns[0].device) if headflags is True else (
        headflags if headflags not in (False, None) else None)
    arr = (Column * len(columns))(*[Column(c.data_ptr(), o.data_ptr(), c.element_size())
                                    for c, o in zip(columns, outs)])
    need = int(lib().mdx_columns_workspace_size(n, dc.m))
    ws = ws or workspace(need, columns[0].device, stream)
    _check(lib().mdx_partition_columns(arr, len(columns), n, dc, ctypes.c_void_p(sizes.data_ptr()),
                                       ctypes.c_void_p(hf.data_ptr() if hf is not None else 0),
                                       ctypes.c_void_p(ws.ptr), ws.nbytes, _stream_ptr(stream)),
           "mdx_partition_columns")
    return (outs, sizes, hf) if hf is not None else (outs, sizes)


# ------------------------------------------------- distributed plain path --
def dist_count(d_in, discr, ws: Workspace, counts=None, stream=None):
    """Step 1 of the distributed partition (mdx_dist_count): this rank's m
    class counts (device u32 tensor).  Step 2 must use the same workspace."""
    torch = _torch()
    _require_cuda(d_in)
    dc = make_discr(discr)
    if counts is None:
        counts = torch.empty(dc.m, dtype=torch.uint32, device=d_in.device)
    _require_cuda(counts)
    _check(lib().mdx_dist_count(ctypes.c_void_p(d_in.data_ptr()), d_in.numel(), _elem_of(d_in), dc,
                                ctypes.c_void_p(counts.data_ptr()), ctypes.c_void_p(ws.ptr),
                                ws.nbytes, _stream_ptr(stream)), "mdx_dist_count")
    return counts


def dist_scatter(d_in, discr, all_counts, rank: int, out_chunk_ptrs, out_chunk: int, n_total: int,
                 ws: Workspace, sizes=None, stream=None):
    """Step 3 of the distributed partition (mdx_dist_scatter): store this
    rank's elements into the output chunks of every rank.  ``all_counts`` is
    the [R, m] device u32 tensor of every rank's counts, ``out_chunk_ptrs``
    the R device addresses (ints) of the output chunks.  Returns the global
    class sizes (device u32 tensor)."""
    torch = _torch()
    _require_cuda(d_in, all_counts)
    dc = make_discr(discr)
    R = len(out_chunk_ptrs)
    if sizes is None:
        sizes = torch.empty(dc.m, dtype=torch.uint32, device=d_in.device)
    ptrs = (ctypes.c_void_p * R)(*[ctypes.c_void_p(int(p)) for p in out_chunk_ptrs])
    _check(lib().mdx_dist_scatter(ctypes.c_void_p(d_in.data_ptr()), d_in.numel(), _elem_of(d_in),
                                  dc, ctypes.c_void_p(all_counts.data_ptr()), R, int(rank),
                                  ptrs, int(out_chunk), int(n_total),
                                  ctypes.c_void_p(sizes.data_ptr()), ctypes.c_void_p(ws.ptr),
                                  ws.nbytes, _stream_ptr(stream)), "mdx_dist_scatter")
    return sizes


def ipc_handle(t) -> Tuple[bytes, int]:
    """(64-byte CUDA IPC handle of the allocation holding tensor t, t's offset in it)."""
    buf = ctypes.create_string_buffer(64)
    off = ctypes.c_uint64(0)
    _check(lib().mdx_ipc_get_handle(ctypes.c_void_p(t.data_ptr()), buf, ctypes.byref(off)),
           "mdx_ipc_get_handle")
    return buf.raw, int(off.value)


def ipc_open(handle: bytes, offset: int) -> int:
    """Map another process's allocation; the device address at `offset` in it."""
    p = ctypes.c_void_p(0)
    _check(lib().mdx_ipc_open(handle, int(offset), ctypes.byref(p)), "mdx_ipc_open")
    return int(p.value)


def ipc_close(ptr: int, offset: int) -> None:
    _check(lib().mdx_ipc_close(ctypes.c_void_p(int(ptr)), int(offset)), "mdx_ipc_close")


def mdiscr(d_in, discr, d_out=None, num_hwd_thds: int = 1 << 16, ws: Optional[Workspace] = None,
           stream=None) -> Tuple[object, list]:
    """Reference-shaped ``mdiscr``: partitions into ``d_out`` and returns the
    m class sizes on the host (synchronous), as ``mdiscr<DISCR>`` returns its
    ``TupleType`` (MdiscrHost_optimized_clean.cu.h:149).  Raises
    :class:`MdxError` where the reference's ``gpuErrchk`` would exit."""
    torch = _torch()
    _require_cuda(d_in)
    dc = make_discr(discr)
    n = d_in.numel()
    elem = _elem_of(d_in)
    if d_out is None:
        d_out = torch.empty_like(d_in)
    _require_cuda(d_out)
    need = workspace_size(n, elem, dc.m)
    ws = ws or workspace(need, d_in.device, stream)
    h_sizes = (ctypes.c_uint32 * dc.m)()
    st = lib().mdx_mdiscr(n, num_hwd_thds, ctypes.c_void_p(d_in.data_ptr()),
                          ctypes.c_void_p(d_out.data_ptr()), elem, dc,
                          ctypes.cast(h_sizes, ctypes.c_void_p), ctypes.c_void_p(ws.ptr),
                          ws.nbytes, _stream_ptr(stream))
    _check(st, "mdx_mdiscr")
    return d_out, list(h_sizes)


# ----------------------------------------------------------- segmented path --
def segmented_workspace_size(n: int, num_segments: int, elem: int, m: int) -> int:
    return int(lib().mdx_segmented_workspace_size(int(n), int(num_segments), int(elem), int(m)))


def partition_segmented(d_in, d_offsets, discr, out=None, seg_sizes=None, headflags=False,
                        ws: Optional[Workspace] = None, stream=None):
    """Per-segment stable partition; ``d_offsets`` is a CUDA u64/i64 tensor of
    S+1 non-decreasing offsets (0 first, n last).  Returns ``(out, seg_sizes)``
    with seg_sizes of shape (S, m) [, head flags]."""
    torch = _torch()
    _require_cuda(d_in, d_offsets)
    if d_offsets.element_size() != 8:
        raise TypeError("segment offsets are 64-bit")
    dc = make_discr(discr)
    n = d_in.numel()
    S = d_offsets.numel() - 1
    if S < 0:
        raise ValueError("offsets need at least one entry")
    elem = _elem_of(d_in)
    if out is None:
        out = torch.empty_like(d_in)
    if seg_sizes is None:
        seg_sizes = torch.empty((S, dc.m), dtype=torch.uint32, device=d_in.device)
    hf = None
    if headflags is True:
        hf = torch.empty(n, dtype=torch.uint32, device=d_in.device)
    elif headflags is not False and headflags is not None:
        hf = headflags
    _require_cuda(out, seg_sizes, hf)
    need = segmented_workspace_size(n, S, elem, dc.m)
    if need == 0:
        raise MdxError(MDX_ERR_INVALID, "mdx_segmented_workspace_size")
    ws = ws or workspace(need, d_in.device, stream)
    st = lib().mdx_partition_segmented(
        ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(out.data_ptr()), n, elem, dc,
        ctypes.c_void_p(d_offsets.data_ptr()), S, ctypes.c_void_p(seg_sizes.data_ptr()),
        ctypes.c_void_p(hf.data_ptr() if hf is not None else 0), ctypes.c_void_p(ws.ptr),
        ws.nbytes, _stream_ptr(stream))
    _check(st, "mdx_partition_segmented")
    return (out, seg_sizes, hf) if hf is not None else (out, seg_sizes)


def partition_segmented_multi(d_in, d_offsets, d_seg_m, m_max: int, out=None, seg_sizes=None,
                              headflags=False, ws: Optional[Workspace] = None, stream=None):
    """Segmented partition with a class count per segment (class = key % m_s);
    ``d_seg_m`` is a CUDA u32/i32 tensor of S entries in [1, m_max], m_max <= 16.
    Returns ``(out, seg_sizes[S, m_max])`` [, head flags]."""
    torch = _torch()
    _require_cuda(d_in, d_offsets, d_seg_m)
    n = d_in.numel()
    S = d_offsets.numel() - 1
    elem = _elem_of(d_in)
    if out is None:
        out = torch.empty_like(d_in)
    if seg_sizes is None:
        seg_sizes = torch.empty((S, m_max), dtype=torch.uint32, device=d_in.device)
    hf = None
    if headflags is True:
        hf = torch.empty(n, dtype=torch.uint32, device=d_in.device)
    elif headflags is not False and headflags is not None:
        hf = headflags
    need = segmented_workspace_size(n, S, elem, m_max)
    ws = ws or workspace(need, d_in.device, stream)
    st = lib().mdx_partition_segmented_multi(
        ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(out.data_ptr()), n, elem,
        ctypes.c_void_p(d_seg_m.data_ptr()), m_max, ctypes.c_void_p(d_offsets.data_ptr()), S,
        ctypes.c_void_p(seg_sizes.data_ptr()),
        ctypes.c_void_p(hf.data_ptr() if hf is not None else 0), ctypes.c_void_p(ws.ptr),
        ws.nbytes, _stream_ptr(stream))
    _check(st, "mdx_partition_segmented_multi")
    return (out, seg_sizes, hf) if hf is not None else (out, seg_sizes)


def mdiscr_segm(d_in, d_segment_sizes, discr, d_out=None, d_new_sizes=None,
                ws: Optional[Workspace] = None, stream=None):
    """Reference-shaped ``mdiscrSegm``: head-flag segment sizes in (i32, the
    length at each segment start, 0 elsewhere), per-segment head-flag class
    sizes out (i32 ``new_sizes``).  Returns ``(d_out, d_new_sizes)``."""
    torch = _torch()
    _require_cuda(d_in, d_segment_sizes)
    dc = make_discr(discr)
    n = d_in.numel()
    elem = _elem_of(d_in)
    if d_out is None:
        d_out = torch.empty_like(d_in)
    if d_new_sizes is None:
        d_new_sizes = torch.empty(n, dtype=torch.int32, device=d_in.device)
    _require_cuda(d_out, d_new_sizes)
    need = int(lib().mdx_mdiscr_segm_workspace_size(n, elem, dc.m))
    if need == 0:
        raise MdxError(MDX_ERR_INVALID, "mdx_mdiscr_segm_workspace_size")
    ws = ws or workspace(need, d_in.device, stream)
    st = lib().mdx_mdiscr_segm(n, ctypes.c_void_p(d_in.data_ptr()),
                               ctypes.c_void_p(d_segment_sizes.data_ptr()),
                               ctypes.c_void_p(d_out.data_ptr()),
                               ctypes.c_void_p(d_new_sizes.data_ptr()), elem, dc,
                               ctypes.c_void_p(ws.ptr), ws.nbytes, _stream_ptr(stream))
    _check(st, "mdx_mdiscr_segm")
    return d_out, d_new_sizes


# ------------------------------------------------------------- CUDA graphs --
class Graph:
    """One captured partition call (mdx_graph_*): replay with :meth:`launch`.

    The captured pointers are fixed; their contents may change between
    replays.  Keeps the tensors it was captured with alive."""

    def __init__(self, handle, keep):
        self._h = handle
        self._keep = keep

    def launch(self, stream=None):
        _check(lib().mdx_graph_launch(self._h, _stream_ptr(stream)), "mdx_graph_launch")

    def close(self):
        if self._h:
            lib().mdx_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def capture_partition(d_in, discr, out, sizes, headflags=None, ws: Optional[Workspace] = None):
    """Capture mdx_partition(d_in -> out, sizes[, headflags]) into a Graph."""
    _require_cuda(d_in, out, sizes, headflags)
    dc = make_discr(discr)
    n = d_in.numel()
    elem = _elem_of(d_in)
    ws = ws or new_workspace(workspace_size(n, elem, dc.m), d_in.device)
    h = ctypes.c_void_p()
    st = lib().mdx_graph_partition(ctypes.byref(h), ctypes.c_void_p(d_in.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr()), n, elem, dc,
                                   ctypes.c_void_p(sizes.data_ptr()),
                                   ctypes.c_void_p(headflags.data_ptr() if headflags is not None else 0),
                                   ctypes.c_void_p(ws.ptr), ws.nbytes)
    _check(st, "mdx_graph_partition")
    return Graph(h, (d_in, out, sizes, headflags, ws))


def capture_partition_segmented(d_in, d_offsets, discr, out, seg_sizes, headflags=None,
                                ws: Optional[Workspace] = None):
    """Capture mdx_partition_segmented into a Graph."""
    _require_cuda(d_in, d_offsets, out, seg_sizes, headflags)
    dc = make_discr(discr)
    n = d_in.numel()
    S = d_offsets.numel() - 1
    elem = _elem_of(d_in)
    ws = ws or new_workspace(segmented_workspace_size(n, S, elem, dc.m), d_in.device)
    h = ctypes.c_void_p()
    st = lib().mdx_graph_partition_segmented(
        ctypes.byref(h), ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(out.data_ptr()), n, elem,
        dc, ctypes.c_void_p(d_offsets.data_ptr()), S, ctypes.c_void_p(seg_sizes.data_ptr()),
        ctypes.c_void_p(headflags.data_ptr() if headflags is not None else 0),
        ctypes.c_void_p(ws.ptr), ws.nbytes)
    _check(st, "mdx_graph_partition_segmented")
    return Graph(h, (d_in, d_offsets, out, seg_sizes, headflags, ws))


# ------------------------------------------------------------ serving loop --
class ServerConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_uint64), ("num_streams", ctypes.c_uint32),
                ("max_batch_requests", ctypes.c_uint32), ("max_batch_elems", ctypes.c_uint64),
                ("m_max", ctypes.c_uint32), ("direct_min_elems", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("batches", ctypes.c_uint64), ("elements", ctypes.c_uint64),
                ("waiting", ctypes.c_uint64), ("inflight_batches", ctypes.c_uint64),
                ("p50_s", ctypes.c_double), ("p99_s", ctypes.c_double), ("mean_s", ctypes.c_double),
                ("window_s", ctypes.c_double), ("direct", ctypes.c_uint64),
                ("queue_p50_s", ctypes.c_double), ("queue_p99_s", ctypes.c_double),
                ("exec_p50_s", ctypes.c_double), ("exec_p99_s", ctypes.c_double),
                ("launch_busy_s", ctypes.c_double)]


def _bind_server(L):
    if getattr(L, "_server_bound", False):
        return L
    vp = ctypes.c_void_p
    L.mdx_server_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ServerConfig)]
    L.mdx_server_create.restype = ctypes.c_int
    L.mdx_server_submit.argtypes = [vp, vp, vp, vp, ctypes.c_uint64, ctypes.c_uint32,
                                    ctypes.POINTER(ctypes.c_uint64)]
    L.mdx_server_submit.restype = ctypes.c_int
    L.mdx_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]
    L.mdx_server_wait.restype = ctypes.c_int
    L.mdx_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.mdx_server_get_stats.restype = ctypes.c_int
    L.mdx_server_reset_stats.argtypes = [vp]
    L.mdx_server_reset_stats.restype = ctypes.c_int
    L.mdx_server_destroy.argtypes = [vp]
    L.mdx_server_destroy.restype = ctypes.c_int
    L.mdx_server_cancel.argtypes = [vp, ctypes.c_uint64]
    L.mdx_server_cancel.restype = ctypes.c_int
    L.mdx_test_inject_alloc_failure.argtypes = [ctypes.c_uint32]
    L.mdx_test_inject_alloc_failure.restype = None
    L._server_bound = True
    return L


class Server:
    """Continuous-batching partition server (mdx_server_*): u32 requests with
    their own m, in device or page-locked host tensors; FIFO admission into a
    device pool of ``budget_bytes``; consecutive admitted requests share one
    batched segmented launch; up to ``num_streams`` batches run at once."""

    def __init__(self, budget_bytes: int, num_streams: int = 2, max_batch_requests: int = 1024,
                 max_batch_elems: int = 0, m_max: int = 16, direct_min_elems: int = 0):
        L = _bind_server(lib())
        cfg = ServerConfig(budget_bytes, num_streams, max_batch_requests, max_batch_elems, m_max,
                           direct_min_elems)
        h = ctypes.c_void_p()
        _check(L.mdx_server_create(ctypes.byref(h), ctypes.byref(cfg)), "mdx_server_create")
        self._h = h
        self._L = L
        self._keep = {}

    def submit(self, d_in, d_out, sizes, m: int) -> int:
        """Queue one request; the tensors must stay alive until wait()."""
        for x in (d_in, d_out, sizes):
            if not x.is_contiguous() or x.element_size() != 4:
                raise ValueError("requests are contiguous 4-byte arrays")
        if d_out.numel() < d_in.numel() or sizes.numel() < m:
            raise ValueError("output needs n entries and sizes m entries")
        t = ctypes.c_uint64()
        _check(self._L.mdx_server_submit(self._h, ctypes.c_void_p(d_in.data_ptr()),
                                         ctypes.c_void_p(d_out.data_ptr()),
                                         ctypes.c_void_p(sizes.data_ptr()), d_in.numel(), m,
                                         ctypes.byref(t)), "mdx_server_submit")
        self._keep[t.value] = (d_in, d_out, sizes)
        return t.value

    def wait(self, ticket: int) -> float:
        lat = ctypes.c_double()
        st = self._L.mdx_server_wait(self._h, ticket, ctypes.byref(lat))
        self._keep.pop(ticket, None)
        _check(st, "mdx_server_wait")
        return lat.value

    def cancel(self, ticket: int) -> bool:
        """Withdraw a request not yet launched; True if it was withdrawn (its
        wait() then raises MdxError with MDX_ERR_CANCELLED), False if it is
        already on the GPU or done."""
        return self._L.mdx_server_cancel(self._h, ticket) == MDX_OK

    def stats(self) -> dict:
        s = ServerStats()
        _check(self._L.mdx_server_get_stats(self._h, ctypes.byref(s)), "mdx_server_get_stats")
        return {name: getattr(s, name) for name, _ in ServerStats._fields_}

    def reset_stats(self) -> None:
        _check(self._L.mdx_server_reset_stats(self._h), "mdx_server_reset_stats")

    def close(self) -> None:
        if self._h:
            self._L.mdx_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
