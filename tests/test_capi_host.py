"""The C-ABI library on the host (no GPU): it loads, exports every symbol
include/*.h declares, and rejects bad arguments before touching the device."""
import ctypes
import os
import re

import pytest

import mdiscriminator_b200 as mdx
from mdiscriminator_b200 import build as mdx_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    mdx_build.build()
    return mdx.lib()


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for root, _, files in os.walk(inc):
        for f in files:
            if not f.endswith(".h"):
                continue
            text = open(os.path.join(root, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(mdx_\w+)\s*\(", text, re.M):
                names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ("mdx_partition", "mdx_mdiscr", "mdx_partition_segmented", "mdx_mdiscr_segm",
                     "mdx_workspace_size", "mdx_workspace_init", "mdx_strerror"):
        assert required in names


def test_library_exports_every_declared_symbol(L):
    for name in declared_symbols():
        assert hasattr(L, name), f"libmdx.so does not export {name}"


def test_version_and_strerror(L):
    assert "sm_100a" in mdx.version()
    for s in range(8):
        assert mdx.strerror(s)
    assert mdx.strerror(mdx.MDX_ERR_TIMEOUT).startswith("device-side")


def test_workspace_size_rules(L):
    assert mdx.workspace_size(1 << 28, mdx.ELEM_U32, 8) > 0
    assert mdx.workspace_size(1 << 20, mdx.ELEM_U32, 0) == 0
    assert mdx.workspace_size(1 << 20, mdx.ELEM_U32, 65) == 0
    assert mdx.workspace_size(1 << 20, 7, 4) == 0
    # grows with m and n, bounded by the chunk cap
    assert mdx.workspace_size(1 << 28, mdx.ELEM_U32, 64) >= mdx.workspace_size(1 << 28, mdx.ELEM_U32, 8)
    # past the chunk cap only the one-kernel path's per-tile tables grow:
    # 2 x m u32 per 4096-element tile, well under 1 % of the input
    big, small = mdx.workspace_size(1 << 30, mdx.ELEM_U32, 8), mdx.workspace_size(1 << 28, mdx.ELEM_U32, 8)
    assert small < big <= small + 2 * 8 * 4 * ((1 << 30) - (1 << 28)) // 4096
    assert big < (1 << 30) * 4 // 100


def _call_partition(L, n, elem, discr, ws=0, ws_bytes=0, inp=1 << 20, out=1 << 30):
    return L.mdx_partition(ctypes.c_void_p(inp), ctypes.c_void_p(out), n, elem, discr, None, None,
                           ctypes.c_void_p(ws), ws_bytes, None)


def test_argument_validation_happens_before_any_device_work(L):
    D = mdx.Discr
    # bad class counts / kinds / element layouts
    assert _call_partition(L, 10, mdx.ELEM_U32, D(mdx.DISCR_MOD, 0)) == mdx.MDX_ERR_INVALID
    assert _call_partition(L, 10, mdx.ELEM_U32, D(mdx.DISCR_MOD, 65)) == mdx.MDX_ERR_INVALID
    assert _call_partition(L, 10, mdx.ELEM_U32, D(mdx.DISCR_MASK, 3)) == mdx.MDX_ERR_INVALID
    assert _call_partition(L, 10, mdx.ELEM_U32, D(9, 4)) == mdx.MDX_ERR_INVALID
    assert _call_partition(L, 10, 5, D(mdx.DISCR_MOD, 4)) == mdx.MDX_ERR_INVALID
    # n beyond u32 class sizes
    assert _call_partition(L, 1 << 32, mdx.ELEM_U32, D(mdx.DISCR_MOD, 4)) == mdx.MDX_ERR_INVALID
    # overlapping input and output
    assert _call_partition(L, 100, mdx.ELEM_U32, D(mdx.DISCR_MOD, 4), inp=4096,
                           out=4096 + 64) == mdx.MDX_ERR_INVALID
    # null arrays
    assert _call_partition(L, 100, mdx.ELEM_U32, D(mdx.DISCR_MOD, 4), inp=0) == mdx.MDX_ERR_INVALID
    # workspace missing / too small / misaligned
    assert _call_partition(L, 100, mdx.ELEM_U32, D(mdx.DISCR_MOD, 4)) == mdx.MDX_ERR_WORKSPACE
    assert _call_partition(L, 100, mdx.ELEM_U32, D(mdx.DISCR_MOD, 4), ws=1 << 24,
                           ws_bytes=16) == mdx.MDX_ERR_WORKSPACE
    need = mdx.workspace_size(100, mdx.ELEM_U32, 4)
    assert _call_partition(L, 100, mdx.ELEM_U32, D(mdx.DISCR_MOD, 4), ws=(1 << 24) + 8,
                           ws_bytes=need) == mdx.MDX_ERR_WORKSPACE
    # n == 0 with no outputs is a no-op
    assert _call_partition(L, 0, mdx.ELEM_U32, D(mdx.DISCR_MOD, 4)) == mdx.MDX_OK


def test_no_cpu_fallback_for_host_tensors():
    torch = pytest.importorskip("torch")
    x = torch.zeros(16, dtype=torch.int32)
    with pytest.raises(ValueError, match="CUDA tensors only"):
        mdx.partition(x, ("mod", 4))


def test_distributed_entry_points_validate_before_device_work(L):
    """mdx_dist_count / mdx_dist_scatter / mdx_ipc_* refuse bad arguments on the
    host: rank counts, ranks, chunk sizes that break the 16-byte rule, null or
    misaligned chunk pointers, counts larger than the total."""
    d = mdx.make_discr(("mod", 5))
    vp = ctypes.c_void_p
    fake = vp(0x100000)  # never dereferenced: every call below fails its checks first
    two = (vp * 2)(vp(0x200000), vp(0x300000))
    E = mdx.MDX_ERR_INVALID
    assert L.mdx_dist_count(fake, 10, mdx.ELEM_U32, d, None, None, 0, None) == E  # no counts
    assert L.mdx_dist_count(fake, 10, 9, d, fake, None, 0, None) == E  # element layout
    bad_m = mdx.Discr(mdx.DISCR_MOD, 65)
    assert L.mdx_dist_count(fake, 10, mdx.ELEM_U32, bad_m, fake, None, 0, None) == E
    args = lambda R, rank, ptrs, chunk, total, n=10: (fake, n, mdx.ELEM_U32, d, fake, R, rank, ptrs,
                                                      chunk, total, None, fake, 1 << 20, None)
    assert L.mdx_dist_scatter(*args(0, 0, two, 8, 16)) == E       # no ranks
    assert L.mdx_dist_scatter(*args(2, 2, two, 8, 16)) == E       # rank out of range
    assert L.mdx_dist_scatter(*args(129, 0, two, 8, 16)) == E     # more ranks than supported
    assert L.mdx_dist_scatter(*args(2, 0, two, 6, 16)) == E       # chunk not 16 bytes of elements
    assert L.mdx_dist_scatter(*args(2, 0, two, 0, 16)) == E       # empty chunk
    assert L.mdx_dist_scatter(*args(2, 0, two, 8, 9, n=10)) == E  # more local rows than the total
    misaligned = (vp * 2)(vp(0x200004), vp(0x300000))
    assert L.mdx_dist_scatter(*args(2, 0, misaligned, 8, 16)) == E
    nulls = (vp * 2)(vp(0x200000), vp(0))
    assert L.mdx_dist_scatter(*args(2, 0, nulls, 8, 16)) == E     # rank 1's chunk is not empty
    assert L.mdx_ipc_get_handle(None, None, None) == E
    assert L.mdx_ipc_open(None, 0, None) == E
    assert L.mdx_ipc_close(None, 0) == E
