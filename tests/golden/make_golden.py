"""Generate the golden vectors in this directory from the REFERENCE's own code.

Runs the reference's ``seqMdiscr`` (cuda_code/SeqMdiscr.h:10-57), compiled from
its sources by ``oracle/Makefile`` into ``oracle/_ref/libref_mdiscr.so``, on
seeded inputs and records what it produced.  Needs the reference sources to
build ``oracle/_ref`` (this script is run where they are present; the JSON it
writes is committed and is all the tests read).

Inputs are regenerated from their seeds by the splitmix64 generator
(``oracle.fill_uniform_u32``), so only seeds, sizes, class sizes and SHA-256
digests of the outputs are stored, plus full arrays for the smallest cases.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def records(n: int, seed: int) -> np.ndarray:
    keys = oracle.fill_uniform_u32(n, seed).astype(np.uint64)
    return keys | (np.arange(n, dtype=np.uint64) << np.uint64(32))


def segments_from_seed(n: int, seed: int, lo: int = 25, hi: int = 75) -> np.ndarray:
    """Segment lengths in [lo, hi) from splitmix(seed), like populateSizesArray's
    rand() % 50 + 25 (HelpersCommon.h:105-151); returns S+1 offsets."""
    r = oracle.fill_uniform_u32(n, seed ^ 0x5EED)
    offs = [0]
    i = 0
    while offs[-1] < n:
        L = lo + int(r[i % n]) % (hi - lo)
        offs.append(min(n, offs[-1] + L))
        i += 1
    return np.array(offs, dtype=np.uint64)


def main() -> None:
    oracle.build()
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built: the reference sources are needed")
    cases = []
    # Plain u32: Mod<m> (and Mod4/Mod8 for m = 4/8), sizes across tile edges.
    for m in (1, 2, 3, 4, 5, 7, 8, 16, 32, 64):
        for n, seed in ((0, 1), (1, 2), (13, 3), (1000, 4), (4095, 5), (4097, 6), (65537, 7),
                        (1 << 20, 8)):
            if n == 0 and m > 8:
                continue
            x = oracle.fill_uniform_u32(n, seed)
            spec = m in (4, 8)
            out, flags, _ = oracle.ref_seq(x, m, specialized=spec)
            sizes = np.bincount(x % m, minlength=m).astype(np.uint32) if n else np.zeros(m, np.uint32)
            c = {"kind": "u32", "discr": "mod", "m": m, "n": n, "seed": seed,
                 "ref_functor": ("Mod4" if m == 4 else "Mod8") if spec else f"Mod<{m}>",
                 "sizes": sizes.tolist(), "out_sha256": digest(out), "flags_sha256": digest(flags)}
            if n <= 1000:
                c["in"] = x.tolist()
                c["out"] = out.tolist()
                c["flags"] = flags.tolist()
            cases.append(c)
    # 8-byte records {key, payload = index}, class = key % m.
    for m in (2, 4, 16, 32, 64):
        for n, seed in ((777, 11), (50000, 12)):
            x = records(n, seed)
            out, flags, _ = oracle.ref_seq(x, m)
            cases.append({"kind": "rec8", "discr": "mod", "m": m, "n": n, "seed": seed,
                          "ref_functor": f"RecMod<{m}> (ModArray<{m},2> semantics)",
                          "sizes": np.bincount((x & np.uint64(0xFFFFFFFF)) % np.uint64(m),
                                               minlength=m).astype(np.uint32).tolist(),
                          "out_sha256": digest(out), "flags_sha256": digest(flags)})
    # Segmented: the reference validates mdiscrSegm per segment with seqMdiscr
    # (MdiscrSegmTest.cu:8-41), so the golden output is seqMdiscr per segment.
    for m, n, seed in ((4, 5000, 21), (3, 20000, 22), (8, 100000, 23)):
        x = oracle.fill_uniform_u32(n, seed)
        offs = segments_from_seed(n, seed)
        out = np.empty_like(x)
        flags = np.zeros(n, dtype=np.uint32)
        for s in range(len(offs) - 1):
            a, b = int(offs[s]), int(offs[s + 1])
            o, f, _ = oracle.ref_seq(x[a:b], m)
            out[a:b] = o
            flags[a:b] = f
        cases.append({"kind": "u32", "discr": "mod", "m": m, "n": n, "seed": seed,
                      "segments": "splitmix lengths in [25, 75)", "num_segments": len(offs) - 1,
                      "offsets_sha256": digest(offs), "out_sha256": digest(out),
                      "flags_sha256": digest(flags), "ref_functor": f"Mod<{m}> per segment"})
    path = os.path.join(HERE, "ref_seq_golden.json")
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "reference": "cuda_code/SeqMdiscr.h seqMdiscr via oracle/_ref/libref_mdiscr.so",
                   "input": "splitmix64(seed) >> 33 (uniform in [0, 2^31))",
                   "cases": cases}, f, indent=0)
    print(f"wrote {len(cases)} cases to {path}")


if __name__ == "__main__":
    main()
