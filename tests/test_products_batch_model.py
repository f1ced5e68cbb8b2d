"""The prepared product batch's split into a symbolic and a numeric pass, as a
plain-Python model (CPU), checked against the oracle.

wg_batch.cu computes, once per batch, every product's key (pair, x, z) and
code (pair-local index << 2 | phase exponent), sorts stably by key and cuts
the sorted products into segments of equal key; every run then only forms
coefficients from the codes, sums each segment left to right, culls and
compacts.  This model does the same with numpy and Python floats (whose
complex multiply and abs() round as the reference's g++ -O2 build and glibc
hypot do) and must equal the oracle's matmul + simplify bit for bit, for
fresh coefficients on the same symbolic pass.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.conftest import random_operator

I_POW = [1, 1j, -1, -1j]


def popcount(a: np.ndarray) -> np.ndarray:
    a = a.astype(np.uint64)
    return np.unpackbits(a.view(np.uint8)).reshape(*a.shape, 64).sum(axis=-1)


def symbolic(pairs, w):
    """Sorted segments of every pair: (pair, key words, [codes in nested-loop order])."""
    segs = []
    for p, (A, B) in enumerate(pairs):
        nl, nr = len(A[3]), len(B[3])
        if nl * nr == 0:
            continue
        l = np.repeat(np.arange(nl), nr)
        r = np.tile(np.arange(nr), nl)
        ax, az, bx, bz = A[1][l], A[2][l], B[1][r], B[2][r]
        px, pz = ax ^ bx, az ^ bz
        e = (popcount(px & pz) - popcount(ax & az) - popcount(bx & bz) + 2 * popcount(ax & bz)).sum(axis=1)
        e = (e % 4).astype(np.int64)  # unsigned wrap-around keeps the residue mod 4
        codes = (np.arange(nl * nr) << 2) | e
        # canonical key order: x0, z0, x1, z1, ... (word 0 most significant); stable
        cols = []
        for k in range(w):
            cols += [px[:, k], pz[:, k]]
        order = np.lexsort(tuple(reversed(cols)), axis=0) if cols else np.arange(nl * nr)
        keys = np.stack(cols, axis=1)[order] if cols else np.zeros((nl * nr, 0), np.uint64)
        codes = codes[order]
        start = 0
        for i in range(1, nl * nr + 1):
            if i == nl * nr or not np.array_equal(keys[i], keys[start]):
                segs.append((p, keys[start], codes[start:i]))
                start = i
    return segs


def numeric(segs, pairs, w, atol=1e-12):
    """Every pair's simplified product from the segments and current coefficients."""
    out = {p: ([], [], []) for p in range(len(pairs))}
    for p, key, codes in segs:
        A, B = pairs[p]
        nr = len(B[3])
        acc = 0j
        for code in codes:
            q, e = int(code) >> 2, int(code) & 3
            prod = complex(A[3][q // nr]) * complex(B[3][q % nr])
            acc += prod * I_POW[e]  # the rotation by i^e is exact
        if abs(acc) > atol:
            out[p][0].append(key[0::2])
            out[p][1].append(key[1::2])
            out[p][2].append(acc)
    res = []
    for p in range(len(pairs)):
        x, z, c = out[p]
        res.append((np.array(x, np.uint64).reshape(-1, w), np.array(z, np.uint64).reshape(-1, w),
                    np.array(c, np.complex128)))
    return res


@pytest.mark.parametrize("n,pool", [(6, None), (10, 12), (70, 20)])
def test_batch_model_equals_oracle_for_fresh_coefficients(oracle, n, pool):
    rng = np.random.default_rng(n)
    w = (n + 63) // 64
    pairs = [(random_operator(rng, n, int(rng.integers(1, 25)), 0.3, pool),
              random_operator(rng, n, int(rng.integers(1, 25)), 0.3, pool)) for _ in range(6)]
    pairs.append((random_operator(rng, n, 0, 0.3), random_operator(rng, n, 5, 0.3)))  # an empty pair
    segs = symbolic(pairs, w)
    for trial in range(2):  # the same symbolic pass serves new coefficients
        if trial:
            pairs = [((a[0], a[1], a[2], rng.normal(size=len(a[3])) + 1j * rng.normal(size=len(a[3]))),
                      (b[0], b[1], b[2], rng.normal(size=len(b[3])) + 1j * rng.normal(size=len(b[3]))))
                     for a, b in pairs]
        got = numeric(segs, pairs, w)
        for (A, B), g in zip(pairs, got):
            raw = oracle.matmul(n, A[1:], B[1:], simplify=False)
            want = oracle.simplify(n, *raw, 1e-12, 0.0)
            for a, b in zip(g, want):
                assert np.ascontiguousarray(a).tobytes() == np.ascontiguousarray(b).tobytes()
