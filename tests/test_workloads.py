"""The seeded input generators (CPU): numpy and torch give the same values,
and the uniform stream is the oracle's splitmix64 generator."""
import numpy as np
import pytest

import oracle
from mdiscriminator_b200 import workloads as W


@pytest.mark.parametrize("n,seed", [(0, 1), (1, 1), (1000, 7), (1 << 20, 2), (300_001, 2**63 + 5)])
def test_generators_agree(n, seed):
    import torch
    a = W.uniform_u32(n, seed)
    assert np.array_equal(a, oracle.fill_uniform_u32(n, seed))
    assert np.array_equal(a, W.uniform_u32_torch(torch, n, seed, "cpu").numpy().view(np.uint32))
    z = W.zipf8(n, seed)
    assert np.array_equal(z, W.zipf8_torch(torch, n, seed, "cpu").numpy().view(np.uint32))
    for m, pre in [(2, False), (16, True), (64, True)]:
        r = W.records(n, seed, m, pre)
        rt = W.records_torch(torch, n, seed, m, pre, "cpu").numpy().view(np.uint64)
        assert np.array_equal(r, rt)


def test_distributions():
    x = W.uniform_u32(1 << 20, 3)
    assert x.max() < (1 << 31) and abs(x.mean() / (1 << 30) - 1) < 0.01
    z = W.zipf8(1 << 21, 3)
    p = np.arange(1, 9, dtype=np.float64) ** -1.1
    assert np.allclose(np.bincount(z & 7, minlength=8) / z.size, p / p.sum(), atol=2e-3)
    r = W.records(1 << 16, 4, 16, presorted=True)
    k = (r & np.uint64(15)).astype(np.int64)
    assert np.all(np.diff(k) >= 0)  # one contiguous run per class
    assert np.array_equal(r >> np.uint64(32), np.arange(1 << 16, dtype=np.uint64))
