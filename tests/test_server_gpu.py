"""The serving loop (mdx_server_*): continuous batching of partition requests
with their own m.  Every request must equal the oracle, and a request's result
must be the same when it runs alone and when it runs in a mix of concurrent
requests (tolerance 0: integer results)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _request(torch, n, seed, pinned=False):
    x = oracle.fill_uniform_u32(n, seed)
    t = torch.from_numpy(x)
    if pinned:
        d = t.pin_memory()
        out = torch.empty(n, dtype=torch.uint32).pin_memory()
    else:
        d = t.cuda()
        out = torch.empty(n, dtype=torch.uint32, device="cuda")
    return x, d, out


def _sizes(torch, m, pinned=False):
    if pinned:
        return torch.empty(m, dtype=torch.uint32).pin_memory()
    return torch.empty(m, dtype=torch.uint32, device="cuda")


def test_result_alone_equals_result_in_the_mix(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    with mdx.Server(budget_bytes=1 << 30, num_streams=3) as srv:
        xr, dr, outr = _request(torch, 300_007, 1)
        sr = _sizes(torch, 8)
        srv.wait(srv.submit(dr, outr, sr, 8))
        alone_out, alone_sizes = outr.cpu().numpy().copy(), sr.cpu().numpy().copy()
        eo, es = oracle.partition(xr, 8)
        assert np.array_equal(alone_out, eo) and np.array_equal(alone_sizes, es)

        rng = np.random.default_rng(2)
        reqs = []
        for i in range(240):
            if i % 40 == 17:  # the same request, several times inside the mix
                o, s = torch.empty_like(outr), _sizes(torch, 8)
                reqs.append((xr, dr, o, s, 8, True))
                continue
            n = int(np.exp(rng.uniform(np.log(1 << 10), np.log(1 << 20))))
            m = int(rng.choice([2, 4, 8, 16]))
            x, d, o = _request(torch, n, 100 + i)
            reqs.append((x, d, o, _sizes(torch, m), m, False))
        tickets = [srv.submit(d, o, s, m) for (_, d, o, s, m, _) in reqs]  # all in flight at once
        for t in tickets:
            srv.wait(t)
        st = srv.stats()
        assert st["batches"] < len(reqs) + 1  # requests were coalesced
        for k, (x, d, o, s, m, same) in enumerate(reqs):
            got_o, got_s = o.cpu().numpy(), s.cpu().numpy()
            if same:
                assert np.array_equal(got_o, alone_out) and np.array_equal(got_s, alone_sizes)
            elif k % 7 == 0:
                eo, es = oracle.partition(x, m)
                assert np.array_equal(got_o, eo) and np.array_equal(got_s, es), f"request {k}"
        assert 0 < st["p50_s"] <= st["p99_s"]
        assert st["completed"] == st["submitted"] == len(reqs) + 1


def test_pinned_host_requests(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    with mdx.Server(budget_bytes=256 << 20) as srv:
        reqs = []
        for i, (n, m) in enumerate([(5000, 3), (70_001, 16), (1 << 18, 5)]):
            x, d, o = _request(torch, n, 50 + i, pinned=True)
            s = _sizes(torch, m, pinned=True)
            reqs.append((x, o, s, m, srv.submit(d, o, s, m)))
        for x, o, s, m, t in reqs:
            srv.wait(t)
            eo, es = oracle.partition(x, m)
            assert np.array_equal(o.numpy(), eo) and np.array_equal(s.numpy(), es)


def test_pageable_memory_is_refused(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    with mdx.Server(budget_bytes=64 << 20) as srv:
        x = torch.zeros(1000, dtype=torch.uint32)  # pageable host memory
        with pytest.raises(mdx.MdxError) as e:
            srv.submit(x, torch.empty_like(x), torch.empty(4, dtype=torch.uint32), 4)
        assert e.value.status == mdx.MDX_ERR_INVALID


def test_admission_waits_for_budget(cuda_ready):
    """Requests totalling 8x the ring are admitted as earlier ones finish."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    budget = 8 << 20  # 1 Mi elements per ring
    with mdx.Server(budget_bytes=budget, num_streams=2, max_batch_requests=16) as srv:
        reqs = []
        for i in range(32):
            n = 200_000 + 1000 * i
            x, d, o = _request(torch, n, 300 + i)
            s = _sizes(torch, 4)
            reqs.append((x, o, s, srv.submit(d, o, s, 4)))
        for x, o, s, t in reqs:
            srv.wait(t)
            eo, es = oracle.partition(x, 4)
            assert np.array_equal(o.cpu().numpy(), eo) and np.array_equal(s.cpu().numpy(), es)
        assert srv.stats()["batches"] > 1


def test_long_device_requests_are_partitioned_in_place(cuda_ready):
    """Requests of at least direct_min_elems in device memory skip the pool's
    copies (plain kernels on their own buffers); mixed with short ones, their
    results equal the oracle and the same requests served with that path
    switched off."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    rng = np.random.default_rng(11)
    specs = []
    for i in range(24):
        n = int(rng.choice([3000, 70_000, 1 << 20, 3_000_017, 5 << 20]))
        specs.append((n, int(rng.choice([2, 5, 8, 16])), 500 + i))
    results = {}
    for direct_min in (0, 2**64 - 1):  # default threshold (2^20), then never
        with mdx.Server(budget_bytes=1 << 30, num_streams=3, direct_min_elems=direct_min) as srv:
            reqs = []
            for n, m, seed in specs:
                x, d, o = _request(torch, n, seed)
                reqs.append((x, d, o, _sizes(torch, m), m))
            tickets = [srv.submit(d, o, s, m) for (_, d, o, s, m) in reqs]
            for t in tickets:
                srv.wait(t)
            st = srv.stats()
            long_ones = sum(1 for n, _, _ in specs if n >= (1 << 20))
            assert st["direct"] == (long_ones if direct_min == 0 else 0)
            results[direct_min] = [(o.cpu().numpy(), s.cpu().numpy()) for (_, _, o, s, _) in reqs]
            for k, (x, _, _, _, m) in enumerate(reqs):
                if k % 3 == 0:
                    eo, es = oracle.partition(x, m)
                    assert np.array_equal(results[direct_min][k][0], eo), f"request {k}"
                    assert np.array_equal(results[direct_min][k][1], es), f"request {k}"
    for (a_o, a_s), (b_o, b_s) in zip(results[0], results[2**64 - 1]):
        assert np.array_equal(a_o, b_o) and np.array_equal(a_s, b_s)


def test_server_set_up_reports_each_failed_allocation_and_frees_the_rest(cuda_ready):
    """Host-side fault injection: the k-th allocation of mdx_server_create
    fails (as if memory were exhausted), for every k until creation needs no
    more.  Each failure is reported as MDX_ERR_CUDA, no server is returned and
    the device memory already allocated is freed again."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    L = mdx._bind_server(mdx.lib())
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    failures = 0
    try:
        for k in range(1, 200):
            L.mdx_test_inject_alloc_failure(k)
            try:
                srv = mdx.Server(budget_bytes=64 << 20, num_streams=2)
            except mdx.MdxError as e:
                assert e.status == mdx.MDX_ERR_CUDA
                failures += 1
                continue
            srv.close()  # k is past the last allocation: created normally
            break
    finally:
        L.mdx_test_inject_alloc_failure(0)
    assert failures >= 10  # rings, per-stream workspaces and tables, lanes
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert abs(free1 - free0) < (2 << 20), f"{free0 - free1} bytes not freed"


def test_cancel_before_launch(cuda_ready):
    """Requests queued behind a long batch are withdrawn before launch: their
    wait reports MDX_ERR_CANCELLED and their outputs stay untouched; the
    others complete and equal the oracle."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    with mdx.Server(budget_bytes=1 << 30, num_streams=1, direct_min_elems=1 << 40,
                    max_batch_elems=1 << 26) as srv:
        xa, da, oa = _request(torch, 1 << 26, 5)
        sa = _sizes(torch, 4)
        ta = srv.submit(da, oa, sa, 4)  # keeps the only batch stream busy
        reqs = []
        for i in range(24):
            x, d, o = _request(torch, 5000 + 17 * i, 300 + i)
            o.view(torch.int32).fill_(-559038737)  # 0xDEADBEEF
            s = _sizes(torch, 8)
            t = srv.submit(d, o, s, 8)
            cancelled = srv.cancel(t) if i % 2 == 0 else False
            reqs.append((x, o, s, t, cancelled))
        srv.wait(ta)
        n_cancelled = 0
        for x, o, s, t, cancelled in reqs:
            if cancelled:
                n_cancelled += 1
                with pytest.raises(mdx.MdxError) as ei:
                    srv.wait(t)
                assert ei.value.status == mdx.MDX_ERR_CANCELLED
                assert bool((o.cpu().numpy() == 0xDEADBEEF).all())
                assert not srv.cancel(t)  # unknown once collected
            else:
                srv.wait(t)
                eo, es = oracle.partition(x, 8)
                assert np.array_equal(o.cpu().numpy(), eo) and np.array_equal(s.cpu().numpy(), es)
        assert n_cancelled >= 1
        eo, es = oracle.partition(xa, 4)
        assert np.array_equal(oa.cpu().numpy(), eo)
