"""Pins the scalar oracle to the reference's own C++ core (oracle/_ref).

Every oracle function is compared bit-for-bit (masks, order, coefficient bits,
groups) with the reference library compiled from its sources, on seeded inputs
that exercise each reference code path: sort and hash simplify paths, the fused
hash matmul path, multi-word keys, tolerance culls, the all-diagonal
expectation path and complex64 states.
"""

from __future__ import annotations

import zlib

import numpy as np
import pytest

from tests.conftest import random_operator


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def assert_same_sum(got, want):
    gx, gz, gc = got
    wx, wz, wc = want
    assert same_bits(gx, wx)
    assert same_bits(gz, wz)
    assert same_bits(gc, wc)


SIMPLIFY_CASES = [
    # (n, T, p, pool, atol, rtol)
    (1, 50, 0.5, 4, 0.0, 0.0),
    (5, 300, 0.3, None, 1e-12, 0.0),
    (20, 5000, 0.25, 600, 1e-12, 0.0),      # >= 4096 terms, duplicate-heavy: reference hash path
    (20, 5000, 0.25, None, 1e-12, 0.0),     # >= 4096 terms, few duplicates: sort path
    (64, 2000, 0.1, 300, 0.5, 0.0),         # cull by atol
    (65, 4500, 0.05, 500, 1e-12, 0.01),     # 2 words, hash path, rtol
    (100, 3000, 0.04, None, 0.0, 0.0),
    (130, 700, 0.05, 90, 0.0, 0.0),         # 3 words: generic path
    (0, 40, 0.0, None, 0.0, 0.0),           # zero qubits: every term is the identity
]


@pytest.mark.parametrize("case", SIMPLIFY_CASES)
def test_simplify_matches_reference(oracle, reference, case):
    n, T, p, pool, atol, rtol = case
    rng = np.random.default_rng(zlib.crc32(repr(case).encode()))
    _, x, z, c = random_operator(rng, n, T, p, pool)
    assert_same_sum(oracle.simplify(n, x, z, c, atol, rtol), reference.simplify(n, x, z, c, atol, rtol))


MATMUL_CASES = [
    # (n, nl, nr, p, pool_l, pool_r, simplify)
    (3, 8, 9, 0.5, None, None, False),
    (3, 8, 9, 0.5, None, None, True),
    (12, 200, 150, 0.3, None, None, True),
    (12, 300, 200, 0.3, 40, None, True),    # duplicate-heavy lhs: fused hash path (1 word)
    (20, 256, 256, 0.25, None, None, True),
    (70, 200, 180, 0.05, 30, None, True),   # fused path, 2 words
    (70, 120, 110, 0.05, None, None, True),
    (150, 60, 70, 0.03, None, None, True),  # 3 words
]


@pytest.mark.parametrize("case", MATMUL_CASES)
def test_matmul_matches_reference(oracle, reference, case):
    n, nl, nr, p, pl, pr, simp = case
    rng = np.random.default_rng(zlib.crc32(repr(case).encode()))
    A = random_operator(rng, n, nl, p, pl)
    B = random_operator(rng, n, nr, p, pr)
    got = oracle.matmul(n, A[1:], B[1:], simplify=simp)
    want = reference.matmul(n, A[1:], B[1:], simplify=simp)
    assert_same_sum(got, want)


def test_fused_path_detection(oracle):
    rng = np.random.default_rng(7)
    A = random_operator(rng, 12, 300, 0.3, 40)
    B = random_operator(rng, 12, 200, 0.3)
    assert oracle.matmul_uses_fused_path(12, A[1:], B[1:])
    assert not oracle.matmul_uses_fused_path(12, B[1:], B[1:])
    assert not oracle.matmul_uses_fused_path(12, A[1:], B[1:], simplify=False)


@pytest.mark.parametrize("n,nl,nr", [(1, 4, 4), (20, 100, 77), (64, 50, 33), (65, 40, 41), (128, 60, 61), (200, 10, 12)])
def test_commutes_matches_reference(oracle, reference, n, nl, nr):
    rng = np.random.default_rng(n * 1000 + nl)
    A = random_operator(rng, n, nl, 0.2)
    B = random_operator(rng, n, nr, 0.2)
    assert np.array_equal(oracle.commutes(n, A[1:], B[1:]), reference.commutes(n, A[1:], B[1:]))


@pytest.mark.parametrize("mode", ["qwc", "full"])
@pytest.mark.parametrize("n,T,p,pool", [(4, 30, 0.5, None), (10, 300, 0.2, None), (70, 400, 0.05, 250), (128, 500, 0.05, None)])
def test_group_commuting_matches_reference(oracle, reference, mode, n, T, p, pool):
    rng = np.random.default_rng(T + n)
    _, x, z, c = random_operator(rng, n, T, p, pool)
    groups = oracle.group_commuting(n, x, z, mode)
    want = reference.group_commuting(n, x, z, c, mode)
    assert len(groups) == len(want)
    for g, (wx, wz, wc) in zip(groups, want):
        assert same_bits(x[g], wx)
        assert same_bits(z[g], wz)
        assert same_bits(c[g], wc)


@pytest.mark.parametrize("n,T,p,diag", [(1, 3, 0.5, False), (6, 20, 0.5, False), (10, 100, 0.3, False),
                                        (8, 80, 0.4, True), (8, 30, 0.4, True), (12, 300, 0.2, False)])
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_expectation_matches_reference(oracle, reference, n, T, p, diag, dtype):
    rng = np.random.default_rng(n * 31 + T)
    _, x, z, c = random_operator(rng, n, T, p)
    if diag:
        x[:] = 0
    psi = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)).astype(dtype)
    assert oracle.expectation(n, x, z, c, psi) == reference.expectation(n, x, z, c, psi)


def test_expectation_zero_qubits(oracle, reference):
    x = np.zeros((2, 0), np.uint64)
    c = np.array([2.5 - 0.75j, 1.0], np.complex128)
    psi = np.array([1.0 + 0.0j])
    assert oracle.expectation(0, x, x, c, psi) == reference.expectation(0, x, x, c, psi) == 3.5 - 0.75j


def test_term_expectations_and_hpsi_are_consistent(oracle):
    """sum_k c_k e_k == E and <psi|H psi> == E (FP64 oracle self-consistency)."""
    rng = np.random.default_rng(5)
    n, x, z, c = random_operator(rng, 9, 60, 0.3)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    e = oracle.term_expectations(n, x, z, psi)
    E = oracle.expectation(n, x, z, c, psi)
    assert abs(np.dot(c, e) - E) < 1e-11
    hp = oracle.hpsi(n, x, z, c, psi)
    assert abs(np.vdot(psi, hp) - E) < 1e-11


@pytest.mark.parametrize("n,T,rows", [(1, 2, 3), (7, 40, 100), (64, 30, 257), (65, 25, 90), (130, 12, 40)])
def test_z_counts_match_reference(oracle, reference, n, T, rows):
    """expectation_z_counts (src/expectation.cpp:219-247): the oracle takes the
    bitstrings packed, the reference as strings (first character = qubit n-1);
    the shim converts between them."""
    rng = np.random.default_rng(1000 + n * 7 + rows)
    _, x, z, c = random_operator(rng, n, T, 0.3)
    x[:] = 0
    w = (n + 63) // 64
    packed = rng.integers(0, 2**63, size=(rows, w), dtype=np.uint64)
    if n % 64:
        packed[:, -1] &= np.uint64((1 << (n % 64)) - 1)
    counts = rng.integers(0, 20, size=rows).astype(np.float64)
    counts[0] += 1.0  # a positive total
    assert oracle.expectation_z_counts(n, x, z, c, packed, counts) == reference.expectation_z_counts(
        n, x, z, c, packed, counts)


def test_z_counts_errors_match_reference(oracle, reference):
    from oracle import OracleError

    rng = np.random.default_rng(3)
    n, x, z, c = random_operator(rng, 6, 5, 0.5)
    packed = np.zeros((2, 1), np.uint64)
    for bad_x, counts, msg in [(True, np.array([1.0, 2.0]), "diagonal"), (False, np.array([-1.0, 2.0]), "non-negative"),
                               (False, np.array([0.0, 0.0]), "positive"), (False, np.array([np.inf, 1.0]), "finite")]:
        xx = x.copy() if bad_x else np.zeros_like(x)
        if bad_x:
            xx[0, 0] |= np.uint64(1)
        with pytest.raises(OracleError, match=msg):
            oracle.expectation_z_counts(n, xx, z, c, packed, counts)
        with pytest.raises(OracleError, match=msg):
            reference.expectation_z_counts(n, xx, z, c, packed, counts)


@pytest.mark.parametrize("n,nl,nr,pool,special", [(12, 120, 90, None, None), (70, 200, 150, 40, None),
                                                 (20, 60, 50, None, "inf"), (20, 60, 50, None, "nan"),
                                                 (10, 80, 70, None, "huge")])
def test_matmul_keyranges_tile_the_full_product(oracle, reference, n, nl, nr, pool, special):
    """or_matmul_keyrange over consecutive key ranges (cut at keys of the full
    result, plus an empty range before it and one after it) reproduces the
    reference's matmul + simplify, bit for bit; this is how the full-size
    product workload is checked range by range.  Non-finite and huge
    coefficients take the oracle's path that forms every product's magnitude."""
    rng = np.random.default_rng(zlib.crc32(repr((n, nl, nr, special)).encode()))
    A = random_operator(rng, n, nl, 0.2, pool)
    B = random_operator(rng, n, nr, 0.2, pool)
    if special == "inf":
        A[3][3] = complex(np.inf, 0.5)
    elif special == "nan":
        B[3][5] = complex(np.nan, 1.0)
    elif special == "huge":
        A[3][:] *= 1e200
        B[3][:] *= 1e200
    raw = reference.matmul(n, A[1:], B[1:], simplify=False)
    want = reference.simplify(n, *raw, 1e-12, 0.0)
    w = (n + 63) // 64
    U = len(want[2])

    def key(i):
        k = np.zeros(2 * w, np.uint64)
        k[0::2], k[1::2] = want[0][i], want[1][i]
        return k

    lo_all = np.zeros(2 * w, np.uint64)
    hi_all = np.full(2 * w, np.iinfo(np.uint64).max, np.uint64)
    cuts = [lo_all] + [key(i) for i in range(0, U, max(1, U // 5))] + [hi_all]
    got = [oracle.matmul_keyrange(n, A[1:], B[1:], lo, hi, cap=nl * nr) for lo, hi in zip(cuts[:-1], cuts[1:])]
    for k in range(3):
        assert same_bits(np.concatenate([g[k] for g in got]), want[k])


def test_hpsi_at_equals_full_hpsi(oracle):
    """or_hpsi_at (H psi at listed amplitudes) is the full or_hpsi, element for element."""
    rng = np.random.default_rng(8)
    n, x, z, c = random_operator(rng, 11, 90, 0.3)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    full = oracle.hpsi(n, x, z, c, psi)
    idx = rng.integers(0, 1 << n, size=200, dtype=np.uint64)
    assert same_bits(oracle.hpsi_at(n, x, z, c, psi, idx), full[idx.astype(np.int64)])
