"""Run-time knobs (mdx_set_tuning / mdx_get_tuning): host-side table checks
on the CPU, and bit-exact results under non-default knobs on the GPU."""
import json
import os

import numpy as np
import pytest

import mdiscriminator_b200 as mdx
import oracle
from mdiscriminator_b200 import build as mdx_build


def test_tuning_table_roundtrip_and_validation():
    mdx_build.build()
    other_bucket = mdx.get_tuning(mdx.ELEM_U32, 7, 1 << 20)
    other_layout = mdx.get_tuning(mdx.ELEM_REC8, 7, 3000)
    mdx.set_tuning(mdx.ELEM_U32, 5, 10, 12, run_tiles=4, group_batch=16, plain_two_kernel=1,
                   plain_ctas_per_sm=2)
    t = mdx.get_tuning(mdx.ELEM_U32, 7, 3000)  # m=7 -> class bound 8, log2 3000 -> 12
    assert t == {"plain_ctas_per_sm": 2, "run_tiles": 4, "group_batch": 16, "plain_two_kernel": 1,
                 "pool_pct": 10, "mid_tiles": 1, "tile_bytes": 64, "tile_threads": 256}
    assert mdx.get_tuning(mdx.ELEM_U32, 7, 1 << 20) == other_bucket   # other bucket untouched
    assert mdx.get_tuning(mdx.ELEM_REC8, 7, 3000) == other_layout     # other element layout
    with pytest.raises(mdx.MdxError):
        mdx.set_tuning(mdx.ELEM_U32, 4, 5, 3, run_tiles=8)   # empty range
    with pytest.raises(mdx.MdxError):
        mdx.set_tuning(mdx.ELEM_U32, 4, 0, 40, run_tiles=8)  # past the last bucket
    with pytest.raises(mdx.MdxError):
        mdx.set_tuning(mdx.ELEM_U32, 4, 0, 10, run_tiles=1000)
    with pytest.raises(mdx.MdxError):
        mdx.set_tuning(mdx.ELEM_U32, 4, 0, 10, plain_two_kernel=2)
    with pytest.raises(mdx.MdxError):
        mdx.set_tuning(mdx.ELEM_U32, 4, 0, 10, mid_tiles=3)  # more than seg_mid's slab holds
    with pytest.raises(mdx.MdxError):
        mdx.set_tuning(mdx.ELEM_U32, 4, 0, 10, tile_bytes=48)  # no such tile geometry
    with pytest.raises(mdx.MdxError):
        mdx.set_tuning(mdx.ELEM_U32, 4, 0, 10, tile_threads=384)
    mdx.set_tuning(mdx.ELEM_U32, 5, 10, 12)  # back to the defaults
    mdx.load_tuning(mdx.TUNING_PATH, missing_ok=True)


def test_committed_table_is_well_formed():
    if not os.path.exists(mdx.TUNING_PATH):
        pytest.skip("no tuning table committed")
    with open(mdx.TUNING_PATH) as f:
        table = json.load(f)
    for e in table["entries"]:
        assert e["elem"] in ("u32", "rec8") and 1 <= e["m"] <= 64
        lo, hi = e["log2_n"]
        assert 0 <= lo <= hi <= 33


@pytest.mark.gpu
@pytest.mark.parametrize("knobs", [dict(run_tiles=1, group_batch=1, plain_two_kernel=1, plain_ctas_per_sm=1,
                                        mid_tiles=1),
                                   dict(run_tiles=16, group_batch=32, plain_two_kernel=0,
                                        plain_ctas_per_sm=2, mid_tiles=2)])
def test_results_do_not_depend_on_knobs(cuda_ready, knobs):
    torch = cuda_ready
    rng = np.random.default_rng(4)
    lengths = np.clip(np.rint(rng.lognormal(np.log(1024), 1.5, size=1500)), 1, 1 << 22).astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(lengths)]).astype(np.uint64)
    n = int(offs[-1])
    x = oracle.fill_uniform_u32(n, 9)
    mdx.set_tuning(mdx.ELEM_U32, 4, 0, 33, **knobs)
    try:
        d = torch.from_numpy(x).cuda()
        out, seg_sizes = mdx.partition_segmented(d, torch.from_numpy(offs.view(np.int64)).cuda(),
                                                 ("mod", 4))
        pout, psizes = mdx.partition(d, ("mod", 4))
        torch.cuda.synchronize()
        eo, es = oracle.partition_segmented(x, offs, 4)
        assert np.array_equal(out.cpu().numpy(), eo) and np.array_equal(seg_sizes.cpu().numpy(), es)
        po, ps = oracle.partition(x, 4)
        assert np.array_equal(pout.cpu().numpy(), po) and np.array_equal(psizes.cpu().numpy(), ps)
    finally:
        mdx.set_tuning(mdx.ELEM_U32, 4, 0, 33)
        mdx.load_tuning(mdx.TUNING_PATH, missing_ok=True)


@pytest.mark.gpu
@pytest.mark.parametrize("rec", [False, True])
@pytest.mark.parametrize("tile_bytes,tile_threads", [(32, 256), (64, 256), (64, 512)])
def test_tile_geometries_match_oracle(cuda_ready, tile_bytes, tile_threads, rec):
    """Every tile geometry of the plain path (64 or 32 bytes of a tile per
    thread at 256 threads, 64 bytes at 512 threads) gives the oracle's
    permutation, sizes and head flags: every class
    bound (m = 2 filter step, nibble steps, warp-rank steps up to 64), one
    tile and less, a partial last tile, an unaligned input view and a length
    whose tail is not a whole 128-byte row."""
    torch = cuda_ready
    elem = mdx.ELEM_REC8 if rec else mdx.ELEM_U32
    saved = {}
    try:
        for m in (2, 3, 8, 13, 16, 32, 64):
            saved[m] = mdx.get_tuning(elem, m, 1 << 20)
            mdx.set_tuning(elem, m, 0, 33, plain_two_kernel=1, tile_bytes=tile_bytes,
                           tile_threads=tile_threads)
            got = mdx.get_tuning(elem, m, 1 << 20)
            assert got["tile_bytes"] == tile_bytes and got["tile_threads"] == tile_threads
            for n, off in ((1000, 0), (2048 + 7, 0), ((1 << 20) + 5, 0), ((1 << 18) + 3, 1)):
                x = oracle.fill_uniform_u32(n + off, 1000 * m + n)
                if rec:
                    x = x.astype(np.uint64) | (np.arange(n + off, dtype=np.uint64) << np.uint64(32))
                base = torch.from_numpy(x.view(np.int64) if rec else x.view(np.int32)).cuda()
                d = base[off:]
                kind = "mask" if (m & (m - 1)) == 0 else "mod"
                out, sizes, hf = mdx.partition(d, (kind, m), headflags=True)
                torch.cuda.synchronize()
                eo, es, ef = oracle.partition(x[off:], m, kind=oracle.DISCR_MASK if kind == "mask"
                                              else oracle.DISCR_MOD, headflags=True)
                got = out.cpu().numpy().view(np.uint64 if rec else np.uint32)
                assert np.array_equal(sizes.cpu().numpy().view(np.uint32), es), (m, n, off)
                assert np.array_equal(got, eo), (m, n, off)
                assert np.array_equal(hf.cpu().numpy().view(np.uint32), ef), (m, n, off)
    finally:
        for m in saved:
            mdx.set_tuning(elem, m, 0, 33)
        mdx.load_tuning(mdx.TUNING_PATH, missing_ok=True)
