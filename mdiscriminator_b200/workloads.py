"""Seeded synthetic inputs of the benchmark configurations.

The reference publishes no dataset; every configuration is synthetic.  One
generator serves the bench (both arms) and the parity tests, so they all
partition the very same values:

* ``uniform_u32(n, seed)``: value i = splitmix64(seed + (i + 1) * golden) >> 33,
  i.e. the i-th output of a splitmix64 stream started at ``seed`` (uniform over
  [0, 2^31)).  The stream is counter-based, so the same values come from numpy
  on the host and from torch integer arithmetic on the device.
* ``zipf8(n, seed)``: class k ~ Zipf(s = 1.1) over 8 classes (p_k proportional
  to (k + 1)^-1.1), value = 8 * U[0, 2^28) + k.
* ``records(n, seed, m, presorted)``: 8-byte records {u32 key uniform over
  [0, 2^31), u32 payload = index}; ``presorted`` orders the keys by class
  key & (m - 1) first (stable), so each class is one contiguous run.
* ``lognormal_lengths``: segment lengths LogNormal(mu, sigma), rounded, clamped.

Seeds of the configurations: ``SEEDS``.
"""
from __future__ import annotations

import math

import numpy as np

GOLDEN = 0x9E3779B97F4A7C15
MIX1 = 0xBF58476D1CE4E5B9
MIX2 = 0x94D049BB133111EB
SEED2_XOR = 0xD1B54A32D192ED03  # second, independent stream of the same seed

# plain N=2^20 m=4 (c1), plain N=2^28 m=8 uniform (c2a) and Zipf (c2b),
# 8-byte records N=2^27 (c3), batched segments (c4), served requests (c5)
SEEDS = {"c1": 1, "c2a": 2, "c2b": 3, "c3": 4, "c4": 5, "c5": 6}

ZIPF_S = 1.1


def _zipf_thresholds(m: int = 8, s: float = ZIPF_S) -> np.ndarray:
    """53-bit integer CDF thresholds: class = number of thresholds <= u53."""
    p = np.arange(1, m + 1, dtype=np.float64) ** -s
    cdf = np.cumsum(p / p.sum())[:-1]
    return np.floor(cdf * float(1 << 53)).astype(np.int64)


# ------------------------------------------------------------------- numpy --
def _mix_np(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * np.uint64(MIX1)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(MIX2)
    return z ^ (z >> np.uint64(31))


def _stream_np(n: int, seed: int, chunk: int = 1 << 22):
    """splitmix64 outputs 0..n-1 of the stream started at ``seed``, by chunks."""
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        with np.errstate(over="ignore"):
            z = np.uint64(seed) + (np.arange(a + 1, b + 1, dtype=np.uint64) * np.uint64(GOLDEN))
            yield a, b, _mix_np(z)


def uniform_u32(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint32)
    for a, b, z in _stream_np(n, seed):
        out[a:b] = (z >> np.uint64(33)).astype(np.uint32)
    return out


def zipf8(n: int, seed: int) -> np.ndarray:
    thr = _zipf_thresholds()
    out = np.empty(n, dtype=np.uint32)
    s2 = seed ^ SEED2_XOR
    for (a, b, z), (_, _, z2) in zip(_stream_np(n, seed), _stream_np(n, s2)):
        k = np.searchsorted(thr, (z >> np.uint64(11)).astype(np.int64), side="right")
        out[a:b] = ((z2 >> np.uint64(36)).astype(np.uint32) << np.uint32(3)) | k.astype(np.uint32)
    return out


def records(n: int, seed: int, m: int = 2, presorted: bool = False) -> np.ndarray:
    keys = uniform_u32(n, seed)
    if presorted:
        keys = keys[np.argsort(keys & np.uint32(m - 1), kind="stable")]
    return keys.astype(np.uint64) | (np.arange(n, dtype=np.uint64) << np.uint64(32))


def lognormal_lengths(S: int, seed: int, mu: float = math.log(1024), sigma: float = 1.5,
                      hi: int = 1 << 22) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(rng.lognormal(mu, sigma, size=S)), 1, hi).astype(np.int64)


# --------------------------------------------------------- torch (device) --
def _s64(c: int) -> int:
    c &= (1 << 64) - 1
    return c - (1 << 64) if c >= 1 << 63 else c


def _srl(x, k: int):
    """Logical right shift of int64 values (torch shifts int64 arithmetically)."""
    return (x >> k) & ((1 << (64 - k)) - 1)


def _stream_torch(torch, a: int, b: int, seed: int, device):
    # int64 products and sums wrap modulo 2^64 on the device as in numpy's uint64
    z = torch.arange(a + 1, b + 1, dtype=torch.int64, device=device) * _s64(GOLDEN) + _s64(seed)
    z = (z ^ _srl(z, 30)) * _s64(MIX1)
    z = (z ^ _srl(z, 27)) * _s64(MIX2)
    return z ^ _srl(z, 31)


def uniform_u32_torch(torch, n: int, seed: int, device, chunk: int = 1 << 26):
    """``uniform_u32`` generated on the device, as an int32 tensor (same bits)."""
    out = torch.empty(n, dtype=torch.int32, device=device)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        out[a:b] = _srl(_stream_torch(torch, a, b, seed, device), 33).to(torch.int32)
    return out


def zipf8_torch(torch, n: int, seed: int, device, chunk: int = 1 << 26):
    thr = torch.from_numpy(_zipf_thresholds()).to(device)
    out = torch.empty(n, dtype=torch.int32, device=device)
    s2 = seed ^ SEED2_XOR
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        z = _stream_torch(torch, a, b, seed, device)
        k = torch.bucketize(_srl(z, 11), thr, right=True)
        hi = _srl(_stream_torch(torch, a, b, s2, device), 36)
        out[a:b] = ((hi << 3) | k).to(torch.int32)  # < 2^31
    return out


def records_torch(torch, n: int, seed: int, m: int = 2, presorted: bool = False, device=None):
    """``records`` on the device, as an int64 tensor (key in the low word)."""
    keys = _srl(_stream_torch(torch, 0, n, seed, device), 33)
    if presorted:
        _, idx = torch.sort(keys & (m - 1), stable=True)
        keys = keys[idx]
        del idx
    return keys | (torch.arange(n, dtype=torch.int64, device=device) << 32)
