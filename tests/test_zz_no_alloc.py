"""mdx_partition_noalloc: the plain partition for callers that cannot
allocate device memory (an allocator or memory-pool callback, a plugin host
that forbids device allocations after start-up, a loop that cannot take
cudaMalloc's device-wide synchronisation) and hold no workspace of their own.

Its scratch is a fixed array inside libmdx.so shared by every call, so each
case makes two calls in a row on different inputs (the second one finds the
first one's leftovers in the array) and checks both against the CPU oracle
(the C restatement of SeqMdiscr) and against the workspace entry point
mdx_partition: bit-exact, the tolerance of every partition test here
(integer results).  The cases cover m = 1 (which runs the two-class kernels
here but a copy in mdx_partition), m = 2, 5, 8 and 16 (16 is the largest m
the array holds), MOD and MASK discriminators, 4-byte values and 8-byte
records.  A further test checks that calls after the first on a device
allocate no device memory, and that the latched-error query reports nothing
after good calls.  This file is collected last so a stopping run has already
executed every other test; it also passes alone in a fresh process (its first
call performs the one-time per-device set-up).
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _bind(mdx):
    L = mdx.lib()
    vp = ctypes.c_void_p
    L.mdx_partition_noalloc.argtypes = [vp, vp, ctypes.c_uint64, ctypes.c_int, mdx.Discr, vp, vp, vp]
    L.mdx_partition_noalloc.restype = ctypes.c_int
    L.mdx_partition_noalloc_error.argtypes = [vp]
    L.mdx_partition_noalloc_error.restype = ctypes.c_int
    return L


def _stream(torch):
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _call(L, torch, x, discr, elem, out, sizes, flags):
    return L.mdx_partition_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                   x.numel(), elem, discr, ctypes.c_void_p(sizes.data_ptr()),
                                   ctypes.c_void_p(flags.data_ptr()), _stream(torch))


def _inputs(n, seed, rec):
    v = oracle.fill_uniform_u32(n, seed)
    if not rec:
        return v
    hi = oracle.fill_uniform_u32(n, seed + 1).astype(np.uint64) << np.uint64(32)
    return v.astype(np.uint64) | hi


# pairs of calls made back to back: (n, m, kind, records)
PAIRS = [
    [(3_000_017, 8, "mod", False), (1_234_567, 5, "mod", True)],
    [(2_000_003, 16, "mask", False), (777_777, 16, "mod", True)],
    [(1_500_001, 1, "mod", False), (999_999, 2, "mask", False)],
    [(65_537, 2, "mod", True), (4_097, 16, "mod", False)],
]


def _pair_id(p):
    return "+".join(f"n{n}m{m}{k}{'rec' if r else 'u32'}" for n, m, k, r in p)


@pytest.mark.parametrize("pair", PAIRS, ids=_pair_id)
def test_noalloc_matches_oracle_and_workspace_entry_point_two_calls(cuda_ready, pair):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    L = _bind(mdx)
    for i, (n, m, kind, rec) in enumerate(pair):
        x = _inputs(n, 100 + 7 * i + n % 97, rec)
        d = torch.from_numpy(x.view(np.int64) if rec else x.view(np.int32)).cuda()
        discr = mdx.Discr(mdx.DISCR_MASK if kind == "mask" else mdx.DISCR_MOD, m)
        out = torch.empty_like(d)
        sizes = torch.empty(m, dtype=torch.int32, device="cuda")
        flags = torch.empty(n, dtype=torch.int32, device="cuda")
        st = _call(L, torch, d, discr, mdx.ELEM_REC8 if rec else mdx.ELEM_U32, out, sizes, flags)
        assert st == mdx.MDX_OK, mdx.strerror(st)
        torch.cuda.synchronize()
        got_out = out.cpu().numpy().view(x.dtype)
        got_sizes = sizes.cpu().numpy().view(np.uint32)
        got_flags = flags.cpu().numpy().view(np.uint32)
        eo, es, ef = oracle.partition(x, m, kind=oracle.DISCR_MASK if kind == "mask" else
                                      oracle.DISCR_MOD, headflags=True)
        assert np.array_equal(got_sizes, es), f"sizes differ from the oracle (call {i})"
        assert np.array_equal(got_out, eo), f"permutation differs from the oracle (call {i})"
        assert np.array_equal(got_flags, ef), f"head flags differ from the oracle (call {i})"
        wo, ws, wf = mdx.partition(d, discr, headflags=True)
        torch.cuda.synchronize()
        assert torch.equal(out, wo)
        assert np.array_equal(ws.cpu().numpy().view(np.uint32), got_sizes)
        assert np.array_equal(wf.cpu().numpy().view(np.uint32), got_flags)
    assert L.mdx_partition_noalloc_error(_stream(torch)) == mdx.MDX_OK


def test_noalloc_allocates_nothing_after_set_up(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    L = _bind(mdx)
    cases = [(1 << 20, 8, False), (1 << 22, 16, True), (12_345, 3, False)]
    bufs = []
    for n, m, rec in cases:  # every tensor exists before the measurement
        x = _inputs(n, n, rec)
        d = torch.from_numpy(x.view(np.int64) if rec else x.view(np.int32)).cuda()
        bufs.append((d, mdx.Discr(mdx.DISCR_MOD, m), mdx.ELEM_REC8 if rec else mdx.ELEM_U32,
                     torch.empty_like(d), torch.empty(m, dtype=torch.int32, device="cuda"),
                     torch.empty(n, dtype=torch.int32, device="cuda")))
    for b in bufs:  # set-up of every kernel family used below
        assert _call(L, torch, *b) == mdx.MDX_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        for b in bufs:
            assert _call(L, torch, *b) == mdx.MDX_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device memory changed by {free0 - free1} bytes"
    assert L.mdx_partition_noalloc_error(_stream(torch)) == mdx.MDX_OK


def test_noalloc_rejects_requests_beyond_its_scratch(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    L = _bind(mdx)
    x = torch.zeros(1000, dtype=torch.int32, device="cuda")
    out = torch.empty_like(x)
    sizes = torch.empty(17, dtype=torch.int32, device="cuda")
    flags = torch.empty(1000, dtype=torch.int32, device="cuda")
    st = _call(L, torch, x, mdx.Discr(mdx.DISCR_MOD, 17), mdx.ELEM_U32, out, sizes, flags)
    assert st == mdx.MDX_ERR_WORKSPACE
