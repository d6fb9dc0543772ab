"""The CPU oracle pinned against the reference (CPU only, no GPU).

* known answers of the reference's fixed fixtures (haskell_code/tests.hs,
  testsSegm.hs), as the reference's seqMdiscr computes them;
* golden digests produced by the reference's own seqMdiscr build
  (tests/golden/make_golden.py);
* where oracle/_ref is built, direct comparisons with the reference's
  seqMdiscr and openmpMdiscr on fresh seeded inputs.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def records(n, seed):
    keys = oracle.fill_uniform_u32(n, seed).astype(np.uint64)
    return keys | (np.arange(n, dtype=np.uint64) << np.uint64(32))


def test_known_answers_plain():
    ka = load("known_answers.json")["plain"]
    x = np.array(ka["in"], dtype=np.uint32)
    for case in ka["cases"]:
        out, sizes, flags = oracle.partition(x, case["m"], headflags=True)
        assert out.tolist() == case["out"]
        assert flags.tolist() == case["flags"]
        assert sizes.sum() == len(x)


def test_known_answers_segmented():
    ka = load("known_answers.json")["segmented"]
    x = np.array(ka["in"], dtype=np.uint32)
    offs = oracle.flags_to_offsets(np.array(ka["segment_sizes"], dtype=np.int32))
    out, seg_sizes, flags = oracle.partition_segmented(x, offs, ka["m"], headflags=True)
    assert out.tolist() == ka["out"]
    assert flags.tolist() == ka["new_sizes"]
    assert seg_sizes.sum(axis=1).tolist() == np.diff(offs).tolist()


def _segments_from_seed(n, seed, lo=25, hi=75):
    r = oracle.fill_uniform_u32(n, seed ^ 0x5EED)
    offs = [0]
    i = 0
    while offs[-1] < n:
        offs.append(min(n, offs[-1] + lo + int(r[i % n]) % (hi - lo)))
        i += 1
    return np.array(offs, dtype=np.uint64)


@pytest.mark.parametrize("case", load("ref_seq_golden.json")["cases"],
                         ids=lambda c: f"{c['kind']}-m{c['m']}-n{c['n']}"
                         + ("-segm" if "segments" in c else ""))
def test_oracle_matches_reference_golden(case):
    n, m = case["n"], case["m"]
    if case["kind"] == "u32":
        x = oracle.fill_uniform_u32(n, case["seed"])
    else:
        x = records(n, case["seed"])
    if "in" in case:
        assert x.tolist() == case["in"], "generator drifted from the golden input"
    if "segments" in case:
        offs = _segments_from_seed(n, case["seed"])
        assert digest(offs) == case["offsets_sha256"]
        out, _, flags = oracle.partition_segmented(x, offs, m, headflags=True)
    else:
        out, sizes, flags = oracle.partition(x, m, headflags=True)
        assert sizes.tolist() == case["sizes"]
    assert digest(out) == case["out_sha256"]
    assert digest(flags) == case["flags_sha256"]
    if "out" in case:
        assert out.tolist() == case["out"]
        assert flags.tolist() == case["flags"]


def test_mask_equals_mod_for_powers_of_two():
    x = oracle.fill_uniform_u32(5000, 99)
    for m in (1, 2, 4, 8, 16, 32, 64):
        a = oracle.partition(x, m, kind=oracle.DISCR_MOD, headflags=True)
        b = oracle.partition(x, m, kind=oracle.DISCR_MASK, headflags=True)
        for u, v in zip(a, b):
            assert np.array_equal(u, v)


def test_oracle_rejects_bad_arguments():
    x = np.zeros(4, dtype=np.uint32)
    with pytest.raises(ValueError):
        oracle.partition(x, 3, kind=oracle.DISCR_MASK)   # mask needs a power of two
    with pytest.raises(ValueError):
        oracle.partition(x, 0)
    with pytest.raises(ValueError):
        oracle.flags_to_offsets(np.array([3, 0, 5, 0], dtype=np.int32))  # overruns n


def test_tuple_to_headflags_matches_partition_flags():
    x = oracle.fill_uniform_u32(3000, 5)
    for m in (1, 3, 8, 64):
        _, sizes, flags = oracle.partition(x, m, headflags=True)
        assert np.array_equal(oracle.tuple_to_headflags(sizes, len(x)), flags)


def test_empty_and_single_class_edges():
    for m in (1, 2, 7, 64):
        out, sizes, flags = oracle.partition(np.zeros(0, dtype=np.uint32), m, headflags=True)
        assert out.size == 0 and sizes.tolist() == [0] * m
    x = np.full(100, 6, dtype=np.uint32)  # every element in class 6 of 7
    out, sizes, flags = oracle.partition(x, 7, headflags=True)
    assert sizes.tolist() == [0] * 6 + [100]
    assert flags[0] == 100 and flags[1:].sum() == 0


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("m", [1, 2, 3, 4, 5, 8, 16, 32, 64])
def test_oracle_vs_reference_seq_random(m):
    rng = np.random.default_rng(m)
    for n in (0, 1, 31, 32, 33, 4096, 12345):
        x = rng.integers(0, 1 << 31, size=n, dtype=np.uint32)
        out, _, flags = oracle.partition(x, m, headflags=True)
        rout, rflags, _ = oracle.ref_seq(x, m)
        assert np.array_equal(out, rout)
        assert np.array_equal(flags, rflags)


@needs_ref
@pytest.mark.parametrize("m", [2, 4, 16, 64])
def test_oracle_vs_reference_seq_records(m):
    x = records(20000, 7 + m)
    out, _, flags = oracle.partition(x, m, headflags=True)
    rout, rflags, _ = oracle.ref_seq(x, m)
    assert np.array_equal(out, rout)
    assert np.array_equal(flags, rflags)


@needs_ref
@pytest.mark.parametrize("m", [2, 4, 8])
def test_reference_openmp_matches_seq(m):
    x = oracle.fill_uniform_u32(1 << 16, 40 + m)
    out, flags, us = oracle.ref_openmp(x, m, threads=2)
    rout, rflags, _ = oracle.ref_seq(x, m)
    assert np.array_equal(out, rout)
    assert np.array_equal(flags.astype(np.uint32), rflags)
    assert us >= 0
