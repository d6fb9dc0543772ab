"""mdx_partition_noalloc: the plain partition for callers that cannot
allocate device memory (an allocator or memory-pool callback, a plugin host
that forbids device allocations after start-up, a loop that cannot take
cudaMalloc's device-wide synchronisation) and hold no workspace of their own.

Its scratch is a fixed array inside libmdx.so shared by every call, so the
test makes two calls in a row on different inputs (the second one finds the
first one's leftovers in the array) and checks each against the workspace
entry point mdx_partition: bit-exact, the tolerance of every partition test
here (integer results).  This file is collected last so a stopping run has
already executed every other test; it also passes alone in a fresh process
(its first call performs the one-time per-device set-up).
"""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


def _bind(mdx):
    L = mdx.lib()
    vp = ctypes.c_void_p
    L.mdx_partition_noalloc.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_int, mdx.Discr, vp, vp, vp]
    L.mdx_partition_noalloc.restype = ctypes.c_int
    return L


def _call(L, mdx, torch, x, discr, elem):
    n = x.numel()
    out = torch.empty_like(x)
    sizes = torch.empty(discr.m, dtype=torch.uint32, device=x.device)
    flags = torch.empty(n, dtype=torch.uint32, device=x.device)
    st = L.mdx_partition_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), n,
                                 elem, discr, ctypes.c_void_p(sizes.data_ptr()),
                                 ctypes.c_void_p(flags.data_ptr()),
                                 ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st, out, sizes, flags


def test_noalloc_matches_workspace_entry_point_two_calls(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    L = _bind(mdx)
    g = torch.Generator(device="cuda").manual_seed(11)
    cases = [  # two calls in a row: different n, m, element layout
        (torch.randint(0, 1 << 31, (3_000_017,), device="cuda", dtype=torch.int64,
                       generator=g).to(torch.int32), mdx.Discr(mdx.DISCR_MOD, 8), mdx.ELEM_U32),
        (torch.randint(0, 1 << 62, (1_234_567,), device="cuda", dtype=torch.int64,
                       generator=g), mdx.Discr(mdx.DISCR_MOD, 5), mdx.ELEM_REC8),
    ]
    for x, discr, elem in cases:
        st, out, sizes, flags = _call(L, mdx, torch, x, discr, elem)
        assert st == mdx.MDX_OK, mdx.strerror(st)
        eout, esizes, eflags = mdx.partition(x, discr, headflags=True)
        torch.cuda.synchronize()
        assert torch.equal(out, eout)
        assert torch.equal(sizes.to(torch.int64), esizes.to(torch.int64))
        assert torch.equal(flags.to(torch.int64), eflags.to(torch.int64))


def test_noalloc_rejects_requests_beyond_its_scratch(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    L = _bind(mdx)
    x = torch.zeros(1000, dtype=torch.int32, device="cuda")
    st, *_ = _call(L, mdx, torch, x, mdx.Discr(mdx.DISCR_MOD, 17), mdx.ELEM_U32)
    assert st == mdx.MDX_ERR_WORKSPACE
