"""The fine-bucket refinement of the bucketed sort-reduce, as a plain-Python model.

After counting, a fine bucket over the 2,048-item capacity whose code range
holds more than one code gets one more splitter from its own samples: their
median, or the next sampled code above the range's first code when the median
is that code, or the first code + 1 when there is none, or the middle of the
range when no sample falls in it.  Up to 32 buckets are split per round: the
splitters are rewritten in place from the back, each item of a split bucket
is searched again, and every other item's bucket id moves up by the number of
splitters inserted below it.  The model checks the invariants the device code
relies on: the new splitter lies strictly inside the bucket's range, the
splitters stay strictly increasing, and the shifted ids equal a fresh search.
"""

from __future__ import annotations

import bisect

import numpy as np
import pytest

CAP = 2048
TOP = 2**64 - 1


def bucket_range(fs, j):
    lo = fs[j - 1] if j > 0 else 0
    if j < len(fs):
        if fs[j] == 0:
            return None
        hi = fs[j] - 1
    else:
        hi = TOP
    return (lo, hi) if lo <= hi else None


def refine_splitter(samp, lo, hi):
    a, b = bisect.bisect_left(samp, lo), bisect.bisect_right(samp, hi)
    if a >= b:
        return lo + (hi - lo) // 2 + 1
    m = samp[a + (b - a) // 2]
    if m > lo:
        return m
    c = a + bisect.bisect_right(samp[a:b], lo)
    return samp[c] if c < b else lo + 1


def refine(codes, samp, fs, slots, rounds=4, per_round=32):
    fid = [bisect.bisect_right(fs, c) for c in codes]
    split = 0
    for _ in range(rounds):
        cnt = np.bincount(fid, minlength=len(fs) + 1)
        fix = [f for f in range(len(fs) + 1)
               if cnt[f] > CAP and (r := bucket_range(fs, f)) is not None and r[0] < r[1]]
        m = min(len(fix), per_round, slots - 1 - len(fs))
        if m <= 0:
            break
        fix = sorted(fix)[:m]
        split += m
        vs = []
        for f in fix:
            lo, hi = bucket_range(fs, f)
            v = refine_splitter(samp, lo, hi)
            assert lo < v <= hi
            vs.append(v)
        # in place from the back, as the device does it
        ns = len(fs)
        out = fs + [None] * m
        shift = [None] * (ns + 1)
        w, q = ns + m - 1, m - 1
        for b in range(ns, -1, -1):
            if b < ns:
                out[w] = out[b]
                w -= 1
            sp = q >= 0 and fix[q] == b
            if sp:
                out[w] = vs[q]
                w -= 1
                q -= 1
            shift[b] = (q + 1, sp)
        fs = out
        assert all(fs[i] < fs[i + 1] for i in range(len(fs) - 1))
        fid = [bisect.bisect_right(fs, c) if shift[f][1] else f + shift[f][0] for c, f in zip(codes, fid)]
        assert fid == [bisect.bisect_right(fs, c) for c in codes]
    return fs, fid, split


@pytest.mark.parametrize("target,clusters,seed,must_split",
                         [(768, 2, 1, False), (1400, 4, 2, False), (1950, 3, 3, True), (2000, 1, 4, True)])
def test_refinement_splits_oversized_buckets(target, clusters, seed, must_split):
    rng = np.random.default_rng(20261204 + seed)
    n = 60000
    parts = [rng.integers(0, 2**63, size=n // 2, dtype=np.uint64)]
    for _ in range(clusters):
        c0 = int(rng.integers(0, 2**62))
        parts.append(np.uint64(c0) + rng.integers(0, 3000, size=n // (2 * clusters), dtype=np.uint64))
    codes = [int(v) for v in np.concatenate(parts)]
    samp = sorted(codes[i] for i in rng.integers(0, len(codes), 8192))
    t = max(1, -(-len(codes) // target))
    slots = t + t // 4 + 8
    share = max(1, len(samp) // t)
    fs, prev = [], None
    for i, v in enumerate(samp):
        if i > 0 and v != samp[i - 1] and (prev is None or i // share != prev // share):
            fs.append(v)
        if i == 0 or v != samp[i - 1]:
            prev = i
    fs = fs[: slots - 1]
    fs, fid, split = refine(codes, samp, fs, slots)
    assert split > 0 or not must_split
    cnt = np.bincount(fid, minlength=len(fs) + 1)
    over = [f for f in range(len(fs) + 1) if cnt[f] > CAP and (r := bucket_range(fs, f)) and r[0] < r[1]]
    assert not over
