"""Parity of the segmented CUDA partition with the CPU oracle (seqMdiscr per
segment, as the reference's MdiscrSegmTest.cu:8-41 validates mdiscrSegm).

Bit-exact on the permuted array, the per-segment class sizes (S x m) and the
per-segment head-flag sizes, for the offsets form and the reference's
head-flag form.  Windows are 4096 elements for u32 and 2048 for records, so
the lengths below straddle the small/large boundary on purpose.
"""
import json
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
P_U32 = 4096


def offsets_from_lengths(lengths):
    return np.concatenate([[0], np.cumsum(np.asarray(lengths, dtype=np.uint64))]).astype(np.uint64)


def lognormal_lengths(S, seed, mu=np.log(1024), sigma=1.5, hi=1 << 22):
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(rng.lognormal(mu, sigma, size=S)), 1, hi).astype(np.int64)


def run_offsets(torch, x, offs, m, kind="mod"):
    import mdiscriminator_b200 as mdx
    d = torch.from_numpy(x).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    out, seg_sizes, hf = mdx.partition_segmented(d, do, (kind, m), headflags=True)
    torch.cuda.synchronize()
    err = mdx.workspace(0).error()
    return out.cpu().numpy(), seg_sizes.cpu().numpy(), hf.cpu().numpy(), err


def check(torch, x, offs, m, kind="mod"):
    import mdiscriminator_b200 as mdx
    k = oracle.DISCR_MASK if kind == "mask" else oracle.DISCR_MOD
    eo, es, ef = oracle.partition_segmented(x, offs, m, kind=k, headflags=True)
    go, gs, gf, err = run_offsets(torch, x, offs, m, kind)
    assert err == mdx.MDX_OK, mdx.strerror(err)
    assert np.array_equal(gs, es), "segment class sizes differ"
    if not np.array_equal(go, eo):
        bad = np.nonzero(go != eo)[0]
        seg = np.searchsorted(offs, bad[0], side="right") - 1
        raise AssertionError(f"output differs at {bad.size} positions, first {bad[:6]} "
                             f"(segment {seg}, length {int(offs[seg + 1] - offs[seg])})")
    assert np.array_equal(gf, ef), "head flags differ"


def test_known_answer_head_flag_form(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        ka = json.load(f)["segmented"]
    x = torch.tensor(ka["in"], dtype=torch.int32, device="cuda")
    flags = torch.tensor(ka["segment_sizes"], dtype=torch.int32, device="cuda")
    out, new_sizes = mdx.mdiscr_segm(x, flags, ("mod", ka["m"]))
    torch.cuda.synchronize()
    assert out.cpu().tolist() == ka["out"]
    assert new_sizes.cpu().tolist() == ka["new_sizes"]


@pytest.mark.parametrize("m", [1, 2, 3, 4, 8, 16])
def test_lognormal_batch(cuda_ready, m):
    lengths = lognormal_lengths(1500, 10 + m)
    offs = offsets_from_lengths(lengths)
    x = oracle.fill_uniform_u32(int(offs[-1]), 20 + m)
    check(cuda_ready, x, offs, m)


@pytest.mark.parametrize("m", [2, 4, 8, 16])
def test_window_edges(cuda_ready, m):
    P = P_U32
    lengths = [1, P - 1, P, P + 1, 2 * P, 2 * P + 1, 3, 5 * P + 7, 31, 32, 33, P, 1, 7 * P - 3,
               2, P + 2, 64, 10 * P, 1, 1, 1, 3 * P + 1]
    offs = offsets_from_lengths(lengths)
    x = oracle.fill_uniform_u32(int(offs[-1]), 77 + m)
    check(cuda_ready, x, offs, m, "mask")
    # the same lengths shifted by one element, so every window boundary moves
    offs2 = offsets_from_lengths([1] + lengths)
    x2 = oracle.fill_uniform_u32(int(offs2[-1]), 78 + m)
    check(cuda_ready, x2, offs2, m, "mask")


def test_empty_and_tiny_segments(cuda_ready):
    rng = np.random.default_rng(3)
    lengths = rng.integers(0, 6, size=20000)  # includes zero-length segments
    offs = offsets_from_lengths(lengths)
    x = oracle.fill_uniform_u32(int(offs[-1]), 5)
    for m in (2, 3, 4):
        check(cuda_ready, x, offs, m)


@pytest.mark.parametrize("m", [3, 16])
def test_group_partition_edges(cuda_ready, m):
    """Small segments are partitioned by a whole CTA per group, each thread
    owning k consecutive elements (k odd, at most 33 for u32): lengths at and
    around those per-thread spans, around the group window and the
    small-segment bound (both 4096), runs of empty segments, and groups cut
    after 128 segments."""
    rng = np.random.default_rng(40 + m)
    pool = [0, 0, 0, 1, 2, 7, 9, 21, 23, 31, 32, 33, 34, 65, 66, 67, 99, 1535, 2048, 3000, 4095,
            4096]
    lengths = rng.choice(pool, size=6000)
    lengths[1000:1400] = 1  # 400 one-element segments in a row
    offs = offsets_from_lengths(lengths)
    x = oracle.fill_uniform_u32(int(offs[-1]), 41 + m)
    check(cuda_ready, x, offs, m)


@pytest.mark.parametrize("m", [4, 16])
def test_unaligned_buffers(cuda_ready, m):
    """Input and output views off their 16-byte alignment: the group copies,
    run counts and run scatter fall back from bulk copies, 16-byte loads and
    TMA to element loads and stores; the result must not change."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    lengths = np.concatenate([lognormal_lengths(400, 60 + m), [20000, 3, 70000, 1, 4097]])
    offs = offsets_from_lengths(lengths)
    n = int(offs[-1])
    x = oracle.fill_uniform_u32(n, 61 + m)
    eo, es, ef = oracle.partition_segmented(x, offs, m, kind=oracle.DISCR_MOD, headflags=True)
    for din, dout in ((1, 0), (0, 3), (3, 1)):
        base_in = torch.zeros(n + 4, dtype=torch.int32, device="cuda")
        base_in[din:din + n] = torch.from_numpy(x.view(np.int32)).cuda()
        base_out = torch.zeros(n + 4, dtype=torch.int32, device="cuda")
        d_in, d_out = base_in[din:din + n], base_out[dout:dout + n]
        out, seg_sizes, hf = mdx.partition_segmented(
            d_in, torch.from_numpy(offs.view(np.int64)).cuda(), ("mod", m), out=d_out,
            headflags=True)
        torch.cuda.synchronize()
        assert mdx.workspace(0).error() == mdx.MDX_OK
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), eo), (din, dout)
        assert np.array_equal(seg_sizes.cpu().numpy(), es)
        assert np.array_equal(hf.cpu().numpy(), ef)


def test_single_huge_segment_equals_plain(cuda_ready):
    n = (1 << 22) + 123
    x = oracle.fill_uniform_u32(n, 9)
    offs = np.array([0, n], dtype=np.uint64)
    check(cuda_ready, x, offs, 8, "mask")


def test_mixed_large_and_small(cuda_ready):
    rng = np.random.default_rng(4)
    lengths = []
    for _ in range(300):
        r = rng.random()
        lengths.append(int(rng.integers(1, 200)) if r < 0.6 else
                       int(rng.integers(200, 5000)) if r < 0.9 else int(rng.integers(5000, 60000)))
    offs = offsets_from_lengths(lengths)
    x = oracle.fill_uniform_u32(int(offs[-1]), 6)
    for m, kind in ((4, "mod"), (5, "mod"), (16, "mask")):
        check(cuda_ready, x, offs, m, kind)


def _medium_lengths(P, seed):
    """Segments around the medium-segment bounds (more than one tile, at most
    mid_tiles row-aligned tiles), at varied 128-byte-row phases (the small
    segments between them shift each start), ending with a medium segment
    whose last elements lie past the input's last whole 128-byte row."""
    rng = np.random.default_rng(seed)
    edges = [P + 1, P + 40, 2 * P - 64, 2 * P - 33, 2 * P - 32, 2 * P - 1, 2 * P, 2 * P + 1,
             3 * P - 5, 4 * P + 1, 9 * P]
    lengths = []
    for _ in range(3):
        for L in edges:
            lengths.append(int(L))
            lengths.append(int(rng.integers(1, 40)))
    row = P // 128  # elements per 128-byte row
    a0 = sum(lengths)
    lengths.append(2 * P - a0 % row - row + 7)  # two tiles; the input ends 7 elements into a row
    return lengths


@pytest.mark.parametrize("rec", [False, True])
@pytest.mark.parametrize("mid_tiles", [1, 2])
def test_medium_segments(cuda_ready, mid_tiles, rec):
    """Medium segments are read once by seg_mid (both tiles in shared memory,
    count pass, then the tile scatter); mid_tiles = 1 sends them through
    the run kernels instead.  Both must give the oracle's result."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    P = P_U32 // 2 if rec else P_U32
    elem = mdx.ELEM_REC8 if rec else mdx.ELEM_U32
    lengths = _medium_lengths(P, 70 + mid_tiles)
    offs = offsets_from_lengths(lengths)
    n = int(offs[-1])
    assert n % (P // 128) == 7
    x = oracle.fill_uniform_u32(n, 71 + mid_tiles)
    if rec:
        x = x.astype(np.uint64) | (np.arange(n, dtype=np.uint64) << np.uint64(32))
    saved = {m: mdx.get_tuning(elem, m, n) for m in (3, 16)}
    try:
        for m, kind in ((3, "mod"), (16, "mask")):
            t = dict(saved[m])
            t["mid_tiles"] = mid_tiles
            mdx.set_tuning(elem, m, 0, 33, **t)
            assert mdx.get_tuning(elem, m, n)["mid_tiles"] == mid_tiles
            check(torch, x, offs, m, kind)
    finally:
        for m, t in saved.items():
            mdx.set_tuning(elem, m, 0, 33, **t)
        mdx.load_tuning(mdx.TUNING_PATH, missing_ok=True)


@pytest.mark.parametrize("m", [2, 4, 16])
def test_records(cuda_ready, m):
    lengths = lognormal_lengths(800, 30 + m, mu=np.log(700))
    offs = offsets_from_lengths(lengths)
    n = int(offs[-1])
    keys = oracle.fill_uniform_u32(n, 40 + m).astype(np.uint64)
    x = keys | (np.arange(n, dtype=np.uint64) << np.uint64(32))
    check(cuda_ready, x, offs, m, "mask")


def test_head_flag_form_matches_offsets_form(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    lengths = lognormal_lengths(2000, 55)
    offs = offsets_from_lengths(lengths)
    n = int(offs[-1])
    x = oracle.fill_uniform_u32(n, 56)
    flags = np.zeros(n, dtype=np.int32)
    flags[offs[:-1].astype(np.int64)] = lengths
    out, new_sizes = mdx.mdiscr_segm(torch.from_numpy(x).cuda(), torch.from_numpy(flags).cuda(),
                                     ("mod", 4))
    torch.cuda.synchronize()
    assert mdx.workspace(0).error() == mdx.MDX_OK
    eo, es, ef = oracle.partition_segmented(x, offs, 4, headflags=True)
    assert np.array_equal(out.cpu().numpy(), eo)
    assert np.array_equal(new_sizes.cpu().numpy().astype(np.uint32), ef)


def test_repeated_calls_reuse_workspace(cuda_ready):
    # back-to-back calls on one workspace: every ticket, count and list the
    # planner resets must be reset (nothing is cleared between calls)
    lengths = lognormal_lengths(400, 61)
    offs = offsets_from_lengths(lengths)
    x = oracle.fill_uniform_u32(int(offs[-1]), 62)
    for _ in range(4):
        check(cuda_ready, x, offs, 4)


def test_malformed_offsets_are_reported(cuda_ready):
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    x = torch.zeros(1000, dtype=torch.int32, device="cuda")
    bad = torch.tensor([0, 500, 400, 1000], dtype=torch.int64, device="cuda")  # decreasing
    mdx.partition_segmented(x, bad, ("mod", 4))
    assert mdx.workspace(0).error() == mdx.MDX_ERR_SEGMENTS
    short = torch.tensor([0, 500, 900], dtype=torch.int64, device="cuda")  # does not reach n
    mdx.partition_segmented(x, short, ("mod", 4))
    assert mdx.workspace(0).error() == mdx.MDX_ERR_SEGMENTS
    flags = torch.zeros(1000, dtype=torch.int32, device="cuda")
    flags[0] = 600  # next start at 600 expected, found at 500
    flags[500] = 500
    mdx.mdiscr_segm(x, flags, ("mod", 4))
    assert mdx.workspace(0).error() == mdx.MDX_ERR_SEGMENTS
    # and a good call afterwards is clean
    lengths = lognormal_lengths(50, 1)
    offs = offsets_from_lengths(lengths)
    check(torch, oracle.fill_uniform_u32(int(offs[-1]), 2), offs, 4)


def test_full_size_100k_lognormal_segments(cuda_ready):
    """100,000 segments, lengths LogNormal(ln 1024, 1.5) clamped to [1, 2^22],
    m = 4: checked against a segment-aware torch stable argsort (bit-exact)."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    lengths = lognormal_lengths(100_000, 2024)
    offs = offsets_from_lengths(lengths)
    n = int(offs[-1])
    g = torch.Generator(device="cuda").manual_seed(7)
    d = torch.randint(0, 1 << 31, (n,), device="cuda", dtype=torch.int64, generator=g)
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    out, seg_sizes = mdx.partition_segmented(d.to(torch.int32), do, ("mod", 4))
    assert mdx.workspace(0).error() == mdx.MDX_OK
    seg_id = torch.repeat_interleave(torch.arange(len(lengths), device="cuda"),
                                     torch.from_numpy(lengths).cuda())
    key = seg_id * 4 + (d % 4)
    order = torch.argsort(key, stable=True)
    assert torch.equal(out, d.to(torch.int32)[order])
    counts = torch.bincount(key, minlength=len(lengths) * 4).view(-1, 4)
    assert torch.equal(seg_sizes.to(torch.int64), counts)


def test_one_workspace_serves_plain_and_segmented_calls(cuda_ready):
    """Plain and segmented calls alternate on the cached workspace: each path
    keeps its own counters, so neither leaves state the other misreads."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    lengths = lognormal_lengths(300, 71)
    offs = offsets_from_lengths(lengths)
    x = oracle.fill_uniform_u32(int(offs[-1]), 72)
    d = torch.from_numpy(x).cuda()
    do = torch.from_numpy(offs.view(np.int64)).cuda()
    eo, es = oracle.partition(x, 8)
    so, ss = oracle.partition_segmented(x, offs, 4)
    for _ in range(2):
        out, seg_sizes = mdx.partition_segmented(d, do, ("mod", 4))
        assert np.array_equal(out.cpu().numpy(), so) and np.array_equal(seg_sizes.cpu().numpy(), ss)
        out, sizes = mdx.partition(d, ("mod", 8))
        assert np.array_equal(out.cpu().numpy(), eo) and np.array_equal(sizes.cpu().numpy(), es)
    assert mdx.workspace(0).error() == mdx.MDX_OK


@pytest.mark.parametrize("m_max", [4, 16])
@pytest.mark.parametrize("short", [False, True])
def test_per_segment_class_counts(cuda_ready, m_max, short):
    """One launch, a class count per segment (class = v % m_s): each segment
    equals the oracle run with its own m.  ``short``: segments of 0..59
    elements, so one thread's elements span segments of different m."""
    import mdiscriminator_b200 as mdx
    torch = cuda_ready
    rng = np.random.default_rng(90 + m_max)
    lengths = rng.integers(0, 60, size=3000) if short else lognormal_lengths(1200, 91 + m_max)
    offs = offsets_from_lengths(lengths)
    seg_m = rng.integers(1, m_max + 1, size=len(lengths)).astype(np.int32)
    x = oracle.fill_uniform_u32(int(offs[-1]), 92)
    out, seg_sizes, hf = mdx.partition_segmented_multi(
        torch.from_numpy(x).cuda(), torch.from_numpy(offs.view(np.int64)).cuda(),
        torch.from_numpy(seg_m).cuda(), m_max, headflags=True)
    torch.cuda.synchronize()
    assert mdx.workspace(0).error() == mdx.MDX_OK
    go, gs, gf = out.cpu().numpy(), seg_sizes.cpu().numpy(), hf.cpu().numpy()
    for s in range(len(lengths)):
        a, b = int(offs[s]), int(offs[s + 1])
        eo, es, ef = oracle.partition(x[a:b], int(seg_m[s]), headflags=True)
        assert np.array_equal(go[a:b], eo), f"segment {s}"
        assert np.array_equal(gs[s, :seg_m[s]], es) and not gs[s, seg_m[s]:].any()
        assert np.array_equal(gf[a:b], ef)
