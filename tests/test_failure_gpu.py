"""Device-side failure paths that can be driven without a GPU fault.

The one-kernel plain partition waits at a grid barrier; a test setting makes
that barrier expect one CTA more than its grid has, so the bounded wait runs
out after a short limit (20 ms here).  The call must latch MDX_ERR_TIMEOUT in
its workspace, leave the output untouched, and the workspace must serve a
correct call again once re-initialised.  The flag that never arrives is the
whole fault: nothing traps, faults or hangs.
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_grid_barrier_wait_runs_out_and_is_reported(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    L = mdx.lib()
    L.mdx_test_set_barrier_shortfall.argtypes = [ctypes.c_uint32, ctypes.c_uint64]
    L.mdx_test_set_barrier_shortfall.restype = None
    n, m = (1 << 22) + 5, 8
    x = oracle.fill_uniform_u32(n, 61)
    d = torch.from_numpy(x).cuda()
    ws = mdx.new_workspace(mdx.workspace_size(n, mdx.ELEM_U32, m))
    out = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    sizes = torch.empty(m, dtype=torch.uint32, device="cuda")
    # the one-kernel path whatever the tuning table picks for this size
    mdx.set_tuning(mdx.ELEM_U32, m, 0, 33, plain_two_kernel=0)
    L.mdx_test_set_barrier_shortfall(1, 20_000_000)
    try:
        mdx.partition(d, ("mod", m), out=out, sizes=sizes, ws=ws)
        torch.cuda.synchronize()
    finally:
        L.mdx_test_set_barrier_shortfall(0, 0)
        mdx.set_tuning(mdx.ELEM_U32, m, 0, 33)
        mdx.load_tuning(mdx.TUNING_PATH, missing_ok=True)
    assert ws.error() == mdx.MDX_ERR_TIMEOUT
    assert bool((out == -1).all())  # no CTA scattered from an incomplete count
    mdx._check(L.mdx_workspace_init(ctypes.c_void_p(ws.ptr), ws.nbytes, None), "mdx_workspace_init")
    mdx.partition(d, ("mod", m), out=out, sizes=sizes, ws=ws)
    torch.cuda.synchronize()
    assert ws.error() == mdx.MDX_OK
    eo, es = oracle.partition(x, m)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), eo)
    assert np.array_equal(sizes.cpu().numpy(), es)
