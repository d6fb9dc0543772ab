"""Wide elements (mdx_partition_records / mdx_partition_columns) against the
oracle: the expected order of the rows is the oracle's stable partition of
{key, row index} records (the class comes from the key), applied to the rows;
sizes and head flags come from the same oracle call."""
import numpy as np
import pytest

import oracle


def expected_perm(keys, m, kind):
    k = oracle.DISCR_MASK if kind == "mask" else oracle.DISCR_MOD
    rec = keys.astype(np.uint64) | (np.arange(len(keys), dtype=np.uint64) << np.uint64(32))
    out, sizes, flags = oracle.partition(rec, m, kind=k, headflags=True)
    return (out >> np.uint64(32)).astype(np.int64), sizes, flags


@pytest.mark.gpu
@pytest.mark.parametrize("record_bytes", [12, 16, 20, 32])
@pytest.mark.parametrize("m,kind", [(2, "mask"), (5, "mod"), (16, "mask"), (64, "mod")])
def test_records_match_oracle(cuda_ready, record_bytes, m, kind):
    torch = cuda_ready
    import mdiscriminator_b200 as mdx
    words = record_bytes // 4
    for n in (1, 1000, 100_003, 1 << 20):
        rng = np.random.default_rng(n + record_bytes + m)
        recs = rng.integers(0, 2**32, size=(n, words), dtype=np.uint64).astype(np.uint32)
        recs[:, 0] = oracle.fill_uniform_u32(n, n + m)
        perm, es, ef = expected_perm(recs[:, 0], m, kind)
        d = torch.from_numpy(recs.reshape(-1).view(np.int32)).cuda()
        out, sizes, flags = mdx.partition_records(d, record_bytes, (kind, m), headflags=True)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32).reshape(n, words)
        assert np.array_equal(got, recs[perm]), (record_bytes, m, n)
        assert np.array_equal(sizes.cpu().numpy(), es)
        assert np.array_equal(flags.cpu().numpy(), ef)


@pytest.mark.gpu
def test_small_records_take_the_direct_paths(cuda_ready):
    torch = cuda_ready
    import mdiscriminator_b200 as mdx
    n = 50_001
    keys = oracle.fill_uniform_u32(n, 3)
    d = torch.from_numpy(keys.view(np.int32)).cuda()
    out, sizes = mdx.partition_records(d, 4, ("mod", 7))
    eo, es = oracle.partition(keys, 7)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), eo)
    rec = keys.astype(np.uint64) | (np.arange(n, dtype=np.uint64) << np.uint64(32))
    out, sizes = mdx.partition_records(torch.from_numpy(rec.view(np.int64)).cuda(), 8, ("mod", 7))
    eo, es = oracle.partition(rec, 7)
    assert np.array_equal(out.cpu().numpy().view(np.uint64), eo)


@pytest.mark.gpu
@pytest.mark.parametrize("m", [3, 16, 64])
def test_16_byte_records_aligned_and_not(cuda_ready, m):
    """16-byte records at a 16-byte aligned address take the 16-byte record
    kernels; 4 bytes off that alignment they take the gathered route.  Both
    must give the oracle's order."""
    torch = cuda_ready
    import mdiscriminator_b200 as mdx
    for n in (5, 4097, 1 << 19):
        rng = np.random.default_rng(n * m)
        recs = rng.integers(0, 2**32, size=(n, 4), dtype=np.uint64).astype(np.uint32)
        recs[:, 0] = oracle.fill_uniform_u32(n, n + 7 * m)
        perm, es, _ = expected_perm(recs[:, 0], m, "mod")
        flat = torch.from_numpy(
            np.concatenate([np.zeros(1, np.uint32), recs.reshape(-1)]).view(np.int32)).cuda()
        for d in (flat[1:].clone(), flat[1:]):
            out, sizes = mdx.partition_records(d, 16, ("mod", m))
            got = out.cpu().numpy().view(np.uint32).reshape(n, 4)
            assert np.array_equal(got, recs[perm]), (n, d.data_ptr() % 16)
            assert np.array_equal(sizes.cpu().numpy(), es)


@pytest.mark.gpu
@pytest.mark.parametrize("m", [4, 13])
def test_columns_follow_the_key(cuda_ready, m):
    """The reference's tuple layout (a u32, a u8 and a bool array) plus a
    2-byte and an 8-byte column, permuted by the class of the u32 key."""
    torch = cuda_ready
    import mdiscriminator_b200 as mdx
    for n in (1, 777, 300_001):
        rng = np.random.default_rng(n * m)
        keys = oracle.fill_uniform_u32(n, n ^ m)
        c8 = rng.integers(0, 256, size=n, dtype=np.uint8)
        cb = rng.integers(0, 2, size=n).astype(np.bool_)
        c16 = rng.integers(0, 2**16, size=n, dtype=np.uint16)
        c64 = rng.integers(0, 2**63, size=n, dtype=np.int64)
        cols = [torch.from_numpy(keys.view(np.int32)).cuda(), torch.from_numpy(c8).cuda(),
                torch.from_numpy(cb).cuda(), torch.from_numpy(c16.view(np.int16)).cuda(),
                torch.from_numpy(c64).cuda()]
        outs, sizes, flags = mdx.partition_columns(cols, ("mod", m), headflags=True)
        torch.cuda.synchronize()
        perm, es, ef = expected_perm(keys, m, "mod")
        assert np.array_equal(outs[0].cpu().numpy().view(np.uint32), keys[perm])
        assert np.array_equal(outs[1].cpu().numpy(), c8[perm])
        assert np.array_equal(outs[2].cpu().numpy(), cb[perm])
        assert np.array_equal(outs[3].cpu().numpy().view(np.uint16), c16[perm])
        assert np.array_equal(outs[4].cpu().numpy(), c64[perm])
        assert np.array_equal(sizes.cpu().numpy(), es)
        assert np.array_equal(flags.cpu().numpy(), ef)


def test_wide_workspace_sizes_and_validation():
    """Host-side checks (no GPU): workspace sizes and refused arguments."""
    import ctypes
    import mdiscriminator_b200 as mdx
    L = mdx.lib()
    assert L.mdx_records_workspace_size(1000, 16, 5) > 16 * 1000
    assert L.mdx_records_workspace_size(1000, 4, 5) == mdx.workspace_size(1000, mdx.ELEM_U32, 5)
    assert L.mdx_records_workspace_size(1000, 6, 5) == 0  # not a multiple of 4
    assert L.mdx_records_workspace_size(1000, 16, 65) == 0
    # 16-byte records: plain partitions only
    assert mdx.workspace_size(1000, mdx.ELEM_REC16, 5) > 0
    assert L.mdx_segmented_workspace_size(1000, 10, mdx.ELEM_REC16, 5) == 0
    assert L.mdx_mdiscr_segm_workspace_size(1000, mdx.ELEM_REC16, 5) == 0
    assert L.mdx_columns_workspace_size(1000, 0) == 0
    d = mdx.make_discr(("mod", 3))
    assert L.mdx_partition_records(None, None, 10, 6, d, None, None, None, 0, None) == mdx.MDX_ERR_INVALID
    cols = (mdx.Column * 1)(mdx.Column(0, 0, 2))  # the key column must be 4 bytes wide
    assert L.mdx_partition_columns(cols, 1, 10, d, None, None, None, 0, None) == mdx.MDX_ERR_INVALID
    assert L.mdx_partition_columns(cols, 9, 10, d, None, None, None, 0, None) == mdx.MDX_ERR_INVALID
