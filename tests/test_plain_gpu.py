"""Parity of the plain CUDA partition (through the C ABI) with the CPU oracle.

Bit-exact on the permuted array, the class sizes (tuple form) and the
head-flag sizes.  Full-size configurations are checked through properties
(class sizes vs a device bincount, stable order against an independent
torch stable argsort, and for records the payload = index permutation proof).
"""
import json
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def records(n, seed):
    keys = oracle.fill_uniform_u32(n, seed).astype(np.uint64)
    return keys | (np.arange(n, dtype=np.uint64) << np.uint64(32))


def run_gpu(torch, x, m, kind="mod", headflags=True):
    import mdiscriminator_b200 as mdx
    d = torch.from_numpy(x).cuda()
    res = mdx.partition(d, (kind, m), headflags=headflags)
    torch.cuda.synchronize()
    return [r.cpu().numpy() for r in res]


def check(torch, x, m, kind="mod"):
    k = oracle.DISCR_MASK if kind == "mask" else oracle.DISCR_MOD
    eo, es, ef = oracle.partition(x, m, kind=k, headflags=True)
    go, gs, gf = run_gpu(torch, x, m, kind)
    assert np.array_equal(gs, es), f"sizes differ (n={len(x)}, m={m}, {kind})"
    if not np.array_equal(go, eo):
        bad = np.nonzero(go != eo)[0]
        raise AssertionError(f"output differs at {bad.size} positions, first {bad[:8]} "
                             f"(n={len(x)}, m={m}, {kind})")
    assert np.array_equal(gf, ef), f"head flags differ (n={len(x)}, m={m}, {kind})"


def test_known_answers(cuda_ready):
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        ka = json.load(f)["plain"]
    x = np.array(ka["in"], dtype=np.uint32)
    for case in ka["cases"]:
        go, gs, gf = run_gpu(cuda_ready, x, case["m"])
        assert go.tolist() == case["out"]
        assert gf.tolist() == case["flags"]


@pytest.mark.parametrize("m", [1, 2, 3, 4, 5, 8, 16, 32, 64])
def test_small_sizes_exhaustive(cuda_ready, m):
    sizes = list(range(0, 300)) + [511, 512, 513, 1023, 1024, 1025, 4095, 4096, 4097, 8191,
                                    8192, 8193, 12287, 12289]
    for n in sizes:
        check(cuda_ready, oracle.fill_uniform_u32(n, 1000 + n), m)


@pytest.mark.parametrize("kind", ["mod", "mask"])
@pytest.mark.parametrize("m", [2, 4, 8, 16, 32, 64])
def test_random_sizes_u32(cuda_ready, kind, m):
    rng = np.random.default_rng(m)
    for n in [int(v) for v in rng.integers(1, 1 << 21, size=4)] + [1 << 20, (1 << 22) + 17]:
        check(cuda_ready, oracle.fill_uniform_u32(n, n ^ m), m, kind)


@pytest.mark.parametrize("m", [3, 5, 6, 7, 9, 13, 33, 63])
def test_non_power_of_two_mod(cuda_ready, m):
    for n in (777, 100000, 1 << 20):
        check(cuda_ready, oracle.fill_uniform_u32(n, 7 * m + n), m)


@pytest.mark.parametrize("m", [2, 4, 16, 32, 64])
def test_records(cuda_ready, m):
    for n in (1, 2047, 2048, 2049, 99999, 1 << 20):
        check(cuda_ready, records(n, 31 * m + n), m, "mask")


def test_adversarial_inputs(cuda_ready):
    n = (1 << 20) + 5
    base = oracle.fill_uniform_u32(n, 77)
    for m in (2, 8, 64):
        cls = base % m
        # one class only, the highest class only, pre-sorted by class, reverse-sorted
        check(cuda_ready, np.full(n, 3 * m, dtype=np.uint32), m)
        check(cuda_ready, np.full(n, m - 1, dtype=np.uint32), m)
        check(cuda_ready, base[np.argsort(cls, kind="stable")], m)
        check(cuda_ready, base[np.argsort(-cls.astype(np.int64), kind="stable")], m)
        # only a few classes present (many empty classes)
        check(cuda_ready, (base // m) * m + (base % 2) * (m - 1), m)


def test_zipf_skew(cuda_ready):
    n = 1 << 22
    rng = np.random.default_rng(5)
    p = (np.arange(1, 9, dtype=np.float64)) ** -1.1
    k = rng.choice(8, size=n, p=p / p.sum()).astype(np.uint32)
    v = (rng.integers(0, 1 << 28, size=n, dtype=np.uint32) * 8 + k).astype(np.uint32)
    check(cuda_ready, v, 8, "mask")


def test_reference_shaped_mdiscr_returns_host_tuple(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    x = oracle.fill_uniform_u32(1 << 20, 1)  # config: N = 2^20, m = 4, Mod4
    out, sizes = mdx.mdiscr(torch.from_numpy(x).cuda(), ("mask", 4))
    eo, es = oracle.partition(x, 4, kind=oracle.DISCR_MASK)
    assert sizes == es.tolist()
    assert np.array_equal(out.cpu().numpy(), eo)


def test_unaligned_input_pointer(cuda_ready):
    # a view starting one element into a buffer: the kernels drop the TMA path
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    x = oracle.fill_uniform_u32(100001, 3)
    d = torch.from_numpy(x).cuda()[1:]
    out, sizes = mdx.partition(d, ("mod", 8))
    eo, es = oracle.partition(x[1:], 8)
    assert np.array_equal(out.cpu().numpy(), eo)
    assert np.array_equal(sizes.cpu().numpy(), es)


def test_repeat_calls_are_deterministic(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    d = torch.from_numpy(oracle.fill_uniform_u32(3 << 20, 11)).cuda()
    a, sa = mdx.partition(d, ("mod", 8))
    a = a.clone()
    for _ in range(3):
        b, sb = mdx.partition(d, ("mod", 8))
        assert torch.equal(a, b) and torch.equal(sa, sb)
    ws = mdx.workspace(0)
    assert ws.error() == mdx.MDX_OK


def _stable_reference(torch, d, m):
    cls = (d.to(torch.int64) & 0xFFFFFFFF) % m
    order = torch.argsort(cls, stable=True)
    return d[order], torch.bincount(cls, minlength=m)


@pytest.mark.parametrize("dist", ["uniform", "zipf"])
def test_full_size_2pow28_m8(cuda_ready, dist):
    """N = 2^28 int32, m = 8: the headline configuration, checked against an
    independent torch stable argsort on the device (bit-exact)."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    n = 1 << 28
    g = torch.Generator(device="cuda").manual_seed(2)
    if dist == "uniform":
        d = torch.randint(0, 1 << 31, (n,), device="cuda", dtype=torch.int64, generator=g)
    else:
        p = torch.arange(1, 9, device="cuda", dtype=torch.float64) ** -1.1
        k = torch.multinomial(p / p.sum(), n, replacement=True, generator=g)
        d = torch.randint(0, 1 << 28, (n,), device="cuda", dtype=torch.int64, generator=g) * 8 + k
    d = d.to(torch.int32)  # values < 2^31: int32 carries the same bits
    out, sizes, hf = mdx.partition(d, ("mask", 8), headflags=True)
    ref, counts = _stable_reference(torch, d, 8)
    assert torch.equal(sizes.to(torch.int64), counts)
    assert torch.equal(out, ref)
    starts = torch.cumsum(counts, 0) - counts
    nz = counts > 0
    expect = torch.zeros(n, dtype=torch.int64, device="cuda")
    expect[starts[nz]] = counts[nz]
    assert torch.equal(hf.to(torch.int64), expect)


def test_full_size_records_permutation_proof(cuda_ready):
    """N = 2^27 records {key, payload = index}, m = 64: within every class run
    the payloads strictly increase and each record equals in[payload], which
    proves the output is the stable partition."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    n = 1 << 27
    m = 64
    g = torch.Generator(device="cuda").manual_seed(3)
    keys = torch.randint(0, 1 << 31, (n,), device="cuda", dtype=torch.int64, generator=g)
    rec = keys | (torch.arange(n, device="cuda", dtype=torch.int64) << 32)
    out, sizes = mdx.partition(rec, ("mask", m))
    o = out
    payload = o >> 32
    okeys = o & 0xFFFFFFFF
    cls = okeys & (m - 1)
    counts = torch.bincount(keys & (m - 1), minlength=m)
    assert torch.equal(sizes.to(torch.int64), counts)
    assert bool((cls[1:] >= cls[:-1]).all())
    same = cls[1:] == cls[:-1]
    assert bool((payload[1:][same] > payload[:-1][same]).all())
    assert torch.equal(okeys, keys[payload])


def test_single_class_is_a_copy(cuda_ready):
    """m = 1 takes the copy path: output = input, one class of size n, head
    flag n at 0 -- for values and records, through both plain entry points."""
    torch = cuda_ready
    import mdiscriminator_b200 as mdx
    for n in (1, 4097, 1 << 20):
        check(torch, oracle.fill_uniform_u32(n, n), 1)
        check(torch, records(n, n + 1), 1, "mod")
        out, sizes = mdx.mdiscr(torch.from_numpy(oracle.fill_uniform_u32(n, 5)).cuda(), ("mod", 1))
        assert list(sizes) == [n]
        assert np.array_equal(out.cpu().numpy(), oracle.fill_uniform_u32(n, 5))


@pytest.mark.parametrize("m", [2, 5, 8, 16, 32, 64])
def test_one_kernel_and_two_kernel_paths_agree_with_oracle(cuda_ready, m):
    """The three launch forms of the plain call against the oracle: one
    cooperative kernel (count, grid barrier, scatter), count + scatter with
    programmatic dependent launch, and count + scatter with an event recorded
    between them; for values and records, at sizes with one tile per CTA,
    many tiles per CTA and a ragged last tile."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    forms = [("one_kernel", 0, False), ("dependent_launch", 1, False), ("event", 1, True)]
    try:
        for n in (4096, 300_001, 5 << 20, (1 << 24) + 13):
            for rec in (False, True):
                x = records(n, n + m) if rec else oracle.fill_uniform_u32(n, n + m)
                d = torch.from_numpy(x).cuda()
                eo, es, ef = oracle.partition(x, m, kind=oracle.DISCR_MOD, headflags=True)
                for form, two, with_event in forms:
                    mdx.set_tuning(mdx.ELEM_REC8 if rec else mdx.ELEM_U32, m, 0, 33,
                                   plain_two_kernel=two)
                    ev = torch.cuda.Event() if with_event else None
                    out, sizes, hf = mdx.partition(d, ("mod", m), headflags=True,
                                                   count_done_event=ev)
                    torch.cuda.synchronize()
                    what = f"n={n} m={m} rec={rec} form={form}"
                    assert np.array_equal(sizes.cpu().numpy(), es), what
                    assert np.array_equal(out.cpu().numpy(), eo), what
                    assert np.array_equal(hf.cpu().numpy(), ef), what
        assert mdx.workspace(0).error() == mdx.MDX_OK
    finally:
        for elem in (mdx.ELEM_U32, mdx.ELEM_REC8):
            mdx.set_tuning(elem, m, 0, 33)
        mdx.load_tuning(mdx.TUNING_PATH, missing_ok=True)
