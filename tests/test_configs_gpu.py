"""Parity at the benchmark configurations, on the benchmark's own inputs.

Every configuration the bench times is partitioned here from the same seeded
generator (``mdiscriminator_b200.workloads``, generated on the device exactly
as bench.py does) and compared bit-exactly with the CPU oracle (the C
restatement of SeqMdiscr, cuda_code/SeqMdiscr.h:10-57) on the whole permuted
array, the m class sizes and, for the headline configuration, the head-flag
sizes:

* N = 2^20 u32, m = 4 (class = v mod 4)
* N = 2^28 u32, m = 8, uniform and Zipf(1.1)-skewed classes
* the uniform N = 2^28 u32 input at m in {2, 16, 32, 64}
* N = 2^27 8-byte records {key, payload = index}, class = key & (m - 1),
  m in {2, 4, 16, 32, 64}, random keys and keys pre-sorted by class.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _gpu_partition(torch, d, m, kind, headflags=False):
    import mdiscriminator_b200 as mdx
    res = mdx.partition(d, (kind, m), headflags=headflags)
    torch.cuda.synchronize()
    ws_err = mdx.workspace(0, d.device).error()
    assert ws_err == mdx.MDX_OK, mdx.strerror(ws_err)
    return [r.cpu().numpy() for r in res]


def _compare(got, exp, what):
    if not np.array_equal(got, exp):
        bad = np.nonzero(got != exp)[0]
        raise AssertionError(f"{what}: differs at {bad.size} positions, first {bad[:8]}")


def test_device_generators_equal_host_generators(cuda_ready):
    torch = cuda_ready
    from mdiscriminator_b200 import workloads as W
    n = (1 << 22) + 3
    got = W.uniform_u32_torch(torch, n, 77, "cuda").cpu().numpy().view(np.uint32)
    _compare(got, W.uniform_u32(n, 77), "uniform")
    _compare(got, oracle.fill_uniform_u32(n, 77), "uniform vs the oracle's generator")
    got = W.zipf8_torch(torch, n, 78, "cuda").cpu().numpy().view(np.uint32)
    _compare(got, W.zipf8(n, 78), "zipf")
    for m, pre in [(4, False), (32, True)]:
        got = W.records_torch(torch, n, 79, m, pre, "cuda").cpu().numpy().view(np.uint64)
        _compare(got, W.records(n, 79, m, pre), f"records m={m} presorted={pre}")


def test_c1_n2p20_m4(cuda_ready):
    torch = cuda_ready
    from mdiscriminator_b200 import workloads as W
    d = W.uniform_u32_torch(torch, 1 << 20, W.SEEDS["c1"], "cuda")
    x = d.cpu().numpy().view(np.uint32)
    go, gs, gf = _gpu_partition(torch, d, 4, "mod", headflags=True)
    eo, es, ef = oracle.partition(x, 4, kind=oracle.DISCR_MOD, headflags=True)
    _compare(gs, es, "sizes")
    _compare(go.view(np.uint32), eo, "permutation")
    _compare(gf, ef, "head flags")


@pytest.mark.parametrize("dist", ["uniform", "zipf"])
def test_c2_n2p28_m8_bench_input(cuda_ready, dist):
    torch = cuda_ready
    from mdiscriminator_b200 import workloads as W
    n = 1 << 28
    if dist == "uniform":
        d = W.uniform_u32_torch(torch, n, W.SEEDS["c2a"], "cuda")
    else:
        d = W.zipf8_torch(torch, n, W.SEEDS["c2b"], "cuda")
    x = d.cpu().numpy().view(np.uint32)
    hf = dist == "uniform"
    res = _gpu_partition(torch, d, 8, "mask", headflags=hf)
    del d
    exp = oracle.partition(x, 8, kind=oracle.DISCR_MASK, headflags=hf)
    _compare(res[1], exp[1], "sizes")
    _compare(res[0].view(np.uint32), exp[0], "permutation")
    if hf:
        _compare(res[2], exp[2], "head flags")
    torch.cuda.empty_cache()


@pytest.mark.parametrize("m", [2, 16, 32, 64])
def test_c2a_other_class_counts(cuda_ready, m):
    """The headline input (N = 2^28 u32, the bench's seed) at the other class
    counts the bench times, against the oracle."""
    torch = cuda_ready
    from mdiscriminator_b200 import workloads as W
    d = W.uniform_u32_torch(torch, 1 << 28, W.SEEDS["c2a"], "cuda")
    x = d.cpu().numpy().view(np.uint32)
    go, gs = _gpu_partition(torch, d, m, "mask")
    del d
    eo, es = oracle.partition(x, m, kind=oracle.DISCR_MASK)
    _compare(gs, es, "sizes")
    _compare(go.view(np.uint32), eo, "permutation")
    torch.cuda.empty_cache()


@pytest.mark.parametrize("presorted", [False, True])
@pytest.mark.parametrize("m", [2, 4, 16, 32, 64])
def test_c3_records_n2p27(cuda_ready, m, presorted):
    torch = cuda_ready
    from mdiscriminator_b200 import workloads as W
    n = 1 << 27
    d = W.records_torch(torch, n, W.SEEDS["c3"], m, presorted, "cuda")
    x = d.cpu().numpy().view(np.uint64)
    go, gs = _gpu_partition(torch, d, m, "mask")
    del d
    eo, es = oracle.partition(x, m, kind=oracle.DISCR_MASK)
    _compare(gs, es, "sizes")
    _compare(go.view(np.uint64), eo, "permutation")
    torch.cuda.empty_cache()
