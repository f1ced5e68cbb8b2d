"""GPU parity through the C-ABI against the scalar oracle.

Bit-exact: commutation bits (both algorithms), simplify / products keys, order
and coefficient bits, groups.  Expectation values within 1e-12 absolute (FP64
summation order differs), complex64 states within 1e-6.
"""

from __future__ import annotations

import zlib

import numpy as np
import pytest

from tests import gpu_util as G
from tests.conftest import random_operator
from wolfgang_b200 import capi

pytestmark = pytest.mark.gpu


def seeded(*key):
    return np.random.default_rng(zlib.crc32(repr(key).encode()))


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


# ----------------------------------------------------------------- commutation

@pytest.mark.parametrize("algo", [1, 2])
@pytest.mark.parametrize("n,nl,nr", [(1, 5, 3), (20, 300, 257), (64, 100, 1000), (65, 77, 1025),
                                     (128, 513, 2049), (200, 40, 90), (300, 33, 65), (0, 7, 40)])
def test_commutation_bits_match_oracle(cuda, oracle, algo, n, nl, nr):
    rng = seeded("comm", n, nl, nr)
    A = random_operator(rng, n, nl, 0.2)
    B = random_operator(rng, n, nr, 0.2)
    bits = G.commutation_bits(n, A[1:3], B[1:3], algo=algo)
    flags = G.unpack_bits(bits, nr)
    want = oracle.commutes(n, A[1:3], B[1:3])
    assert np.array_equal(flags, want)
    # padding bits of the last word are zero
    if nr % 32:
        assert np.all(bits[:, -1] >> np.uint32(nr % 32) == 0)


def test_commutation_algorithms_agree_on_20q_operator(cuda):
    from wolfgang_b200.workloads import hamiltonian_20q_and_state

    (n, x, z, _), _ = hamiltonian_20q_and_state()
    b1 = G.commutation_bits(n, (x, z), (x, z), algo=1)
    b2 = G.commutation_bits(n, (x, z), (x, z), algo=2)
    assert same_bits(b1, b2)


@pytest.mark.parametrize("n", [64, 128])
def test_commutation_wide_tiles_match(cuda, oracle, n):
    """Both sides above 65,536 terms with one or two mask words take the
    bit-plane kernel's 4,096-column tiles (four output words per lane, 1,024
    threads), with a ragged last tile: bit for bit equal to the ballot
    algorithm everywhere, and to the oracle on a slice of rows."""
    rng = seeded("comm-wide", n)
    nl, nr = 65536 + 77, 65536 + 1000
    A = random_operator(rng, n, nl, 0.05)
    B = random_operator(rng, n, nr, 0.05)
    b2 = G.commutation_bits(n, A[1:3], B[1:3], algo=2)
    b1 = G.commutation_bits(n, A[1:3], B[1:3], algo=1)
    assert same_bits(b1, b2)
    rows = np.r_[0:200, nl - 56:nl]
    want = oracle.commutes(n, (A[1][rows], A[2][rows]), B[1:3])
    assert np.array_equal(G.unpack_bits(b2[rows], nr), want)
    assert np.all(b2[:, -1] >> np.uint32(nr % 32) == 0)


def test_commutation_128q_row_slice_matches_oracle(cuda, oracle):
    from wolfgang_b200.workloads import sparse_operator_128q

    n, x, z, _ = sparse_operator_128q()
    rows = slice(0, 1024)
    bits = G.commutation_bits(n, (x[rows], z[rows]), (x, z), algo=0)
    want = oracle.commutes(n, (x[rows], z[rows]), (x, z))
    assert np.array_equal(G.unpack_bits(bits, len(x)), want)


def test_bits_to_u8_and_counts(cuda, oracle):
    t = G.torch()
    rng = seeded("u8")
    n, nl, nr = 30, 123, 301
    A = random_operator(rng, n, nl, 0.3)
    B = random_operator(rng, n, nr, 0.3)
    pitch = (nr + 31) // 32
    bits = G.dev(G.commutation_bits(n, A[1:3], B[1:3]).reshape(-1))
    u8 = t.zeros(nl * nr, dtype=t.uint8, device="cuda")
    capi.call("wg_bits_to_u8", 0, bits.data_ptr(), nl, nr, pitch, u8.data_ptr(), None)
    want = oracle.commutes(n, A[1:3], B[1:3])
    assert np.array_equal(u8.cpu().numpy().reshape(nl, nr), want)
    rows = t.zeros(nl, dtype=t.int64, device="cuda")
    cols = t.zeros(nr, dtype=t.int64, device="cuda")
    import ctypes
    total = ctypes.c_uint64()
    capi.call("wg_bits_count", 0, bits.data_ptr(), nl, nr, pitch, rows.data_ptr(), cols.data_ptr(),
              ctypes.byref(total), None)
    assert total.value == int(want.sum())
    assert np.array_equal(rows.cpu().numpy(), want.sum(axis=1))
    assert np.array_equal(cols.cpu().numpy(), want.sum(axis=0))
    total2 = ctypes.c_uint64()
    capi.call("wg_u8_count", 0, u8.data_ptr(), nl, nr, rows.data_ptr(), cols.data_ptr(), ctypes.byref(total2), None)
    assert total2.value == total.value
    assert np.array_equal(cols.cpu().numpy(), want.sum(axis=0))


# ----------------------------------------------------------------- simplify

SIMPLIFY_CASES = [
    (1, 50, 0.5, 4, 0.0, 0.0),
    (5, 300, 0.3, None, 1e-12, 0.0),
    (20, 5000, 0.25, 600, 1e-12, 0.0),
    (20, 100000, 0.25, 3000, 1e-12, 0.0),
    (64, 2000, 0.1, 300, 0.5, 0.0),
    (65, 4500, 0.05, 500, 1e-12, 0.01),
    (100, 30000, 0.04, None, 0.0, 0.0),
    (130, 700, 0.05, 90, 0.0, 0.0),
    (300, 500, 0.02, 60, 1e-12, 0.0),
    (0, 40, 0.0, None, 0.0, 0.0),
]


@pytest.mark.parametrize("case", SIMPLIFY_CASES)
def test_simplify_bit_exact(cuda, oracle, case):
    n, T, p, pool, atol, rtol = case
    rng = seeded("simplify", case)
    _, x, z, c = random_operator(rng, n, T, p, pool)
    got = G.simplify(n, x, z, c, atol, rtol)
    want = oracle.simplify(n, x, z, c, atol, rtol)
    for g, w in zip(got, want):
        assert same_bits(g, w)


def test_simplify_cancellation_and_threshold_ties(cuda, oracle):
    """Exact cancellations, values straddling atol, and inf/nan coefficients."""
    rng = seeded("ties")
    n, x, z, c = random_operator(rng, 8, 4000, 0.3, 50)
    c[::7] = 1e-12 * (1 + 1e-16)
    c[1::11] = -c[0::11][: len(c[1::11])]
    for atol in (0.0, 1e-12, 3e-12):
        got = G.simplify(n, x, z, c, atol, 0.0)
        want = oracle.simplify(n, x, z, c, atol, 0.0)
        for g, w in zip(got, want):
            assert same_bits(g, w)
    c2 = c.copy()
    c2[3] = np.inf
    for rtol in (0.0, 0.1):
        got = G.simplify(n, x, z, c2, 1e-12, rtol)
        want = oracle.simplify(n, x, z, c2, 1e-12, rtol)
        for g, w in zip(got, want):
            assert same_bits(g, w)


def test_simplify_is_idempotent_on_device(cuda):
    rng = seeded("idem")
    n, x, z, c = random_operator(rng, 40, 20000, 0.1, 3000)
    once = G.simplify(n, x, z, c)
    twice = G.simplify(n, *once)
    for a, b in zip(once, twice):
        assert same_bits(a, b)


def test_device_hypot_matches_libm_cull(cuda, oracle):
    """The cull uses the host libm rounding of |c|: probe values near the threshold."""
    rng = seeded("hypot")
    T = 20000
    re = rng.normal(size=T) * 1e-12
    im = rng.normal(size=T) * 1e-12
    c = re + 1j * im
    x = np.zeros((T, 1), np.uint64)
    x[:, 0] = np.arange(T, dtype=np.uint64)
    z = np.zeros((T, 1), np.uint64)
    for atol in np.quantile(np.abs(c), [0.1, 0.5, 0.9]):
        # thresholds equal to the libm |c| of some inputs: strict '>' keeps ties out
        thr = oracle.abs(c[int(np.argmin(np.abs(np.abs(c) - atol)))].real,
                         c[int(np.argmin(np.abs(np.abs(c) - atol)))].imag)
        got = G.simplify(64, x, z, c, thr, 0.0)
        want = oracle.simplify(64, x, z, c, thr, 0.0)
        for g, w in zip(got, want):
            assert same_bits(g, w)


# ----------------------------------------------------------------- products

MATMUL_CASES = [
    (3, 8, 9, 0.5, None, None),
    (12, 200, 150, 0.3, None, None),
    (12, 300, 200, 0.3, 40, None),
    (20, 256, 256, 0.25, None, None),
    (70, 200, 180, 0.05, 30, None),
    (100, 2048, 1024, 0.03, None, None),
    (150, 60, 70, 0.03, None, None),
    (0, 5, 6, 0.0, None, None),
    # more than eight mask words (the any-width products kernel)
    (600, 40, 50, 0.01, None, None),
    (1000, 30, 20, 0.01, 10, None),
]


@pytest.mark.parametrize("case", MATMUL_CASES)
@pytest.mark.parametrize("mode", [capi.WG_PRODUCTS_RAW, capi.WG_PRODUCTS_SIMPLIFY, capi.WG_PRODUCTS_FUSED])
def test_products_bit_exact(cuda, oracle, case, mode):
    n, nl, nr, p, pl, pr = case
    rng = seeded("matmul", case)
    A = random_operator(rng, n, nl, p, pl)
    B = random_operator(rng, n, nr, p, pr)
    got = G.products(n, A[1:], B[1:], mode)
    if mode == capi.WG_PRODUCTS_RAW:
        want = oracle.matmul(n, A[1:], B[1:], simplify=False)
    elif mode == capi.WG_PRODUCTS_SIMPLIFY:
        # simplify() at its defaults == the reference's non-fused path
        raw = oracle.matmul(n, A[1:], B[1:], simplify=False)
        want = oracle.simplify(n, *raw, 1e-12, 0.0)
    else:
        raw = oracle.matmul(n, A[1:], B[1:], simplify=False)
        want = oracle.simplify(n, *raw, 1e-12, 0.0)  # fused threshold 1e-12, finite inputs
    for g, w in zip(got, want):
        assert same_bits(g, w)


def test_hh_20q_operator_simplify_bit_exact(cuda, oracle):
    from wolfgang_b200.workloads import hamiltonian_20q_and_state

    (n, x, z, c), _ = hamiltonian_20q_and_state()
    got = G.products(n, (x, z, c), (x, z, c), capi.WG_PRODUCTS_SIMPLIFY)
    want = oracle.matmul(n, (x, z, c), (x, z, c), simplify=True)
    for g, w in zip(got, want):
        assert same_bits(g, w)


# ----------------------------------------------------------------- expectation

@pytest.mark.parametrize("n,T,p,diag", [(1, 3, 0.5, False), (2, 5, 0.5, False), (6, 20, 0.5, False),
                                        (10, 100, 0.3, False), (8, 80, 0.4, True), (8, 30, 0.4, True),
                                        (14, 700, 0.2, False), (18, 2000, 0.15, False)])
def test_expectation_matches_oracle(cuda, oracle, n, T, p, diag):
    t = G.torch()
    rng = seeded("expect", n, T, diag)
    _, x, z, c = random_operator(rng, n, T, p)
    if diag:
        x[:] = 0
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    plan = G.Plan(n, x, z, c)
    E, ev, hp = plan.run(G.dev(psi), want_terms=True, want_hpsi=True)
    assert abs(E - oracle.expectation(n, x, z, c, psi)) <= 1e-12
    assert np.max(np.abs(ev - oracle.term_expectations(n, x, z, psi))) <= 1e-12
    assert np.max(np.abs(hp - oracle.hpsi(n, x, z, c, psi))) <= 1e-12
    # complex64 storage, FP64 accumulation
    p64 = psi.astype(np.complex64)
    E64, _, _ = plan.run(G.dev(p64))
    assert abs(E64 - oracle.expectation(n, x, z, c, p64)) <= 1e-6
    # deterministic: same bits on a second run
    E2, ev2, _ = plan.run(G.dev(psi), want_terms=True)
    assert E2 == E and np.array_equal(ev2, ev)


def test_expectation_one_shot_and_zero_qubits(cuda, oracle):
    import ctypes

    t = G.torch()
    x = np.zeros((2, 0), np.uint64)
    c = np.array([2.5 - 0.75j, 1.0], np.complex128)
    psi = G.dev(np.array([1.0 + 0.0j]))
    out = (ctypes.c_double * 2)()
    dc = G.dev(c)
    capi.call("wg_expectation", 0, 0, 2, None, None, dc.data_ptr(), psi.data_ptr(), 0, out, None)
    assert complex(out[0], out[1]) == pytest.approx(3.5 - 0.75j, abs=1e-15)


def test_expectation_20q_operator(cuda, oracle):
    from wolfgang_b200.workloads import hamiltonian_20q_and_state

    (n, x, z, c), psi = hamiltonian_20q_and_state()
    plan = G.Plan(n, x, z, c)
    E, _, _ = plan.run(G.dev(psi))
    assert abs(E - oracle.expectation(n, x, z, c, psi)) <= 1e-12


def test_z_counts_match_oracle(cuda, oracle):
    import ctypes

    rng = seeded("zc")
    n, x, z, c = random_operator(rng, 70, 40, 0.2)
    x[:] = 0
    rows = 300
    packed = np.zeros((rows, 2), np.uint64)
    packed[:, 0] = rng.integers(0, 2**63, size=rows, dtype=np.uint64)
    packed[:, 1] = rng.integers(0, 2**6, size=rows, dtype=np.uint64)
    counts = rng.integers(0, 50, size=rows).astype(np.float64)
    out = (ctypes.c_double * 2)()
    dx, dz, dc = G.operator_on_device(x, z, c)
    dp, dn = G.dev(packed), G.dev(counts)
    capi.call("wg_expectation_z_counts", 0, 2, len(c), dx.data_ptr(), dz.data_ptr(), dc.data_ptr(), rows,
              dp.data_ptr(), dn.data_ptr(), out, None)
    want = oracle.expectation_z_counts(n, x, z, c, packed, counts)
    assert abs(complex(out[0], out[1]) - want) <= 1e-12


# ----------------------------------------------------------------- grouping

@pytest.mark.parametrize("mode", ["qwc", "full"])
@pytest.mark.parametrize("n,T,p,pool", [(4, 30, 0.5, None), (10, 300, 0.2, None), (70, 400, 0.05, 250),
                                        (128, 3000, 0.05, None), (0, 5, 0.0, None),
                                        # many chunks of 1,024 terms; 3 and 4 mask words; repeated keys
                                        (128, 12000, 0.05, None), (64, 9000, 0.1, 3000),
                                        (200, 5000, 0.03, None), (256, 2500, 0.02, None),
                                        # dense terms: about one qwc group per term, more groups than
                                        # shared memory holds (the bases stay in global memory)
                                        (128, 8000, 0.5, None),
                                        # more than four mask words: the any-width kernels (5, 11 and
                                        # 40 words; at 40 words a qwc chunk stages 356 terms)
                                        (300, 3000, 0.02, None), (300, 1500, 0.2, 600),
                                        (700, 2500, 0.01, None), (2560, 400, 0.003, None)])
def test_group_commuting_matches_oracle(cuda, oracle, mode, n, T, p, pool):
    import ctypes

    rng = seeded("group", n, T, mode)
    _, x, z, c = random_operator(rng, n, T, p, pool)
    w = 0 if n == 0 else (n + 63) // 64
    dx, dz = G.dev(x), G.dev(z)
    order = np.zeros(T, np.uintp)
    sizes = np.zeros(T, np.uintp)
    ng = ctypes.c_size_t()
    capi.call("wg_group_commuting", 0, w, T, G.ptr(dx), G.ptr(dz), 1 if mode == "full" else 0,
              order.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t)),
              sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t)), ctypes.byref(ng), None)
    groups, q = [], 0
    for s in sizes[: ng.value]:
        groups.append([int(v) for v in order[q:q + int(s)]])
        q += int(s)
    assert groups == oracle.group_commuting(n, x, z, mode)


# ----------------------------------------------------------------- errors

def test_invalid_arguments_raise(cuda):
    t = G.torch()
    with pytest.raises(ValueError, match="tolerances"):
        G.simplify(4, np.zeros((1, 1), np.uint64), np.zeros((1, 1), np.uint64), np.ones(1, np.complex128), -1.0)
    bits = t.zeros(4, dtype=t.int32, device="cuda")
    with pytest.raises(ValueError, match="pitch"):
        capi.call("wg_commutation_bits", 0, 1, bits.data_ptr(), bits.data_ptr(), 1, bits.data_ptr(),
                  bits.data_ptr(), 100, bits.data_ptr(), 1, 0, None)


def test_injected_allocation_failure_reports_oom(cuda):
    rng = seeded("oom")
    n, x, z, c = random_operator(rng, 10, 100, 0.3)
    capi.call("wg_inject_alloc_failure", 1)
    try:
        with pytest.raises(RuntimeError, match="out of memory"):
            G.simplify(n, x, z, c)
    finally:
        capi.call("wg_inject_alloc_failure", 0)
    # the context stays usable
    G.simplify(n, x, z, c)
