"""Bucketed sort-reduce (WG_SORT_BUCKET) against the oracle and the LSD path.

Both algorithms must give the same bits: keys, order and coefficients.  Cases
cover dense codes (at most 64 significant bits left in a bucket), position
codes with tie runs, long runs of one key, fine buckets over capacity (which
fall back to the LSD path), more than 255 significant bits (not eligible),
and infinite / NaN coefficients with both threshold modes.
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


def same(a, b):
    return all(np.ascontiguousarray(x).tobytes() == np.ascontiguousarray(y).tobytes() and x.shape == y.shape
               for x, y in zip(a, b))


def eligible(*xz):
    """1 to 255 significant key bits: the bucketed path's precondition."""
    total = 0
    for a in xz:
        a = np.asarray(a, np.uint64).reshape(len(a), -1)
        for w in range(a.shape[1]):
            total += bin(int(np.bitwise_or.reduce(a[:, w]) if len(a) else 0)).count("1")
    return 1 <= total <= 255


@pytest.fixture
def algo():
    """Sets the sort algorithm for one test and restores WG_SORT_AUTO after it."""
    def set_(a):
        capi.set_sort_algorithm(a)
    yield set_
    capi.set_sort_algorithm(capi.WG_SORT_AUTO)


def klocal(rng, n, T, weights=(2, 3, 4)):
    from wolfgang_b200.workloads import klocal_operator

    return klocal_operator(rng, n, T, weights)


SIMPLIFY_CASES = [
    (1, 50, 0.5, 4, 0.0, 0.0),
    (5, 300, 0.3, None, 1e-12, 0.0),
    (20, 5000, 0.25, 600, 1e-12, 0.0),
    (20, 100000, 0.25, 3000, 1e-12, 0.0),
    (64, 2000, 0.1, 300, 0.5, 0.0),
    (65, 4500, 0.05, 500, 1e-12, 0.01),
    (100, 30000, 0.04, None, 0.0, 0.0),
    (100, 60000, 0.08, 7000, 1e-12, 0.0),
    (127, 20000, 0.03, 2000, 1e-12, 0.5),
]


@pytest.mark.parametrize("case", SIMPLIFY_CASES)
def test_bucket_simplify_bit_exact(cuda, oracle, algo, case):
    n, T, p, pool, atol, rtol = case
    rng = seeded("bucket-simplify", case)
    _, x, z, c = random_operator(rng, n, T, p, pool)
    algo(capi.WG_SORT_BUCKET)
    got = G.simplify(n, x, z, c, atol, rtol)
    if eligible(x, z):
        assert capi.last_sort_algorithm() == capi.WG_SORT_BUCKET
    assert same(got, oracle.simplify(n, x, z, c, atol, rtol))
    algo(capi.WG_SORT_LSD)
    assert same(got, G.simplify(n, x, z, c, atol, rtol))
    assert capi.last_sort_algorithm() == capi.WG_SORT_LSD


MATMUL_CASES = [
    (3, 8, 9, 0.5, None, None),
    (12, 200, 150, 0.3, None, None),
    (12, 300, 200, 0.3, 40, None),
    (20, 256, 256, 0.25, None, None),
    (70, 200, 180, 0.05, 30, None),
    (100, 2048, 1024, 0.03, None, None),
    (128, 300, 400, 0.04, None, 50),
]


@pytest.mark.parametrize("case", MATMUL_CASES)
@pytest.mark.parametrize("mode", [capi.WG_PRODUCTS_SIMPLIFY, capi.WG_PRODUCTS_FUSED])
def test_bucket_products_bit_exact(cuda, oracle, algo, case, mode):
    n, nl, nr, p, pl, pr = case
    rng = seeded("bucket-matmul", case)
    A = random_operator(rng, n, nl, p, pl)
    B = random_operator(rng, n, nr, p, pr)
    algo(capi.WG_SORT_BUCKET)
    got = G.products(n, A[1:], B[1:], mode)
    if eligible(A[1], A[2], B[1], B[2]):
        assert capi.last_sort_algorithm() == capi.WG_SORT_BUCKET
    raw = oracle.matmul(n, A[1:], B[1:], simplify=False)
    assert same(got, oracle.simplify(n, *raw, 1e-12, 0.0))


def test_bucket_klocal_products_match_lsd(cuda, oracle, algo):
    """A scaled-down config-2 product (100 qubits, k-local terms): position codes."""
    rng = seeded("bucket-klocal")
    A = klocal(rng, 100, 2048)
    B = klocal(rng, 100, 1024)
    algo(capi.WG_SORT_BUCKET)
    got = G.products(100, A[1:], B[1:])
    assert capi.last_sort_algorithm() == capi.WG_SORT_BUCKET
    algo(capi.WG_SORT_LSD)
    assert same(got, G.products(100, A[1:], B[1:]))
    raw = oracle.matmul(100, A[1:], B[1:], simplify=False)
    assert same(got, oracle.simplify(100, *raw, 1e-12, 0.0))


def test_auto_sort_choice_by_key_width(cuda, oracle, algo):
    """WG_SORT_AUTO: H@H of the 4,096-term 20-qubit operator (2^24 products;
    keys vary in 6 of their 8-bit digits) takes the LSD pipeline, a 100-qubit
    k-local product of 2^21 items (keys vary in most digits) the bucketed
    path; both are bit-exact, and the other algorithm gives the same bits."""
    from wolfgang_b200.workloads import hamiltonian_20q_and_state

    (n, x, z, c), _ = hamiltonian_20q_and_state()
    algo(capi.WG_SORT_AUTO)
    got = G.products(n, (x, z, c), (x, z, c), capi.WG_PRODUCTS_SIMPLIFY)
    assert capi.last_sort_algorithm() == capi.WG_SORT_LSD
    assert same(got, oracle.matmul(n, (x, z, c), (x, z, c), simplify=True))
    algo(capi.WG_SORT_BUCKET)
    assert same(got, G.products(n, (x, z, c), (x, z, c), capi.WG_PRODUCTS_SIMPLIFY))
    assert capi.last_sort_algorithm() == capi.WG_SORT_BUCKET
    rng = seeded("auto-wide")
    A = klocal(rng, 100, 2048)
    B = klocal(rng, 100, 1024)
    algo(capi.WG_SORT_AUTO)
    got = G.products(100, A[1:], B[1:])
    assert capi.last_sort_algorithm() == capi.WG_SORT_BUCKET
    raw = oracle.matmul(100, A[1:], B[1:], simplify=False)
    assert same(got, oracle.simplify(100, *raw, 1e-12, 0.0))


def test_bucket_tie_heavy_position_codes(cuda, oracle, algo):
    """High-weight terms over 120 qubits: many keys share their first eight set
    bits, so position codes tie; results stay exact (bucketed or fallen back)."""
    rng = seeded("bucket-ties")
    A = random_operator(rng, 120, 400, 0.15)
    B = random_operator(rng, 120, 300, 0.15)
    algo(capi.WG_SORT_BUCKET)
    got = G.products(120, A[1:], B[1:])
    raw = oracle.matmul(120, A[1:], B[1:], simplify=False)
    assert same(got, oracle.simplify(120, *raw, 1e-12, 0.0))


@pytest.mark.parametrize("target", [1800, 1200])
def test_bucket_fine_buckets_split_again(cuda, oracle, algo, monkeypatch, capfd, target):
    """A fine-bucket target near the 2048-item capacity puts about one fine
    bucket in eight over it; each is split again from its own samples, so the
    bucketed path finishes without falling back and gives the oracle's bits.
    At 1200 items no bucket needs it."""
    import re

    rng = seeded("bucket-refine", target)
    _, x, z, c = random_operator(rng, 40, 400_000, 0.25, 150_000)
    algo(capi.WG_SORT_BUCKET)
    monkeypatch.setenv("WG_BUCKET_TRACE", "1")
    capi.set_bucket_fine_target(target)
    try:
        got = G.simplify(40, x, z, c)
        algo_used = capi.last_sort_algorithm()
    finally:
        capi.set_bucket_fine_target(0)
    err = capfd.readouterr().err
    refined = [int(v) for v in re.findall(r"refined=(\d+)", err)]
    assert algo_used == capi.WG_SORT_BUCKET
    assert refined and (refined[-1] > 0) == (target == 1800)
    assert same(got, oracle.simplify(40, x, z, c))


@pytest.mark.parametrize("one_pass", [True, False])
@pytest.mark.parametrize("case", ["klocal100", "dup40", "refine"])
def test_bucket_fine_layouts_identical(cuda, oracle, algo, monkeypatch, capfd, one_pass, case):
    """The fine partition written in one pass (every fine bucket owns 2048
    record slots) and in two passes (count, then pack) give the oracle's bits:
    k-local products, a duplicate-heavy simplify, and a fine target near
    capacity whose overfull fine buckets send their coarse buckets to the
    packed second pass and to refinement."""
    import re

    rng = seeded("fine-layout", case)
    algo(capi.WG_SORT_BUCKET)
    capi.set_bucket_one_pass(one_pass)
    try:
        if case == "klocal100":
            A, B = klocal(rng, 100, 2048), klocal(rng, 100, 1024)
            got = G.products(100, A[1:], B[1:])
            want = oracle.simplify(100, *oracle.matmul(100, A[1:], B[1:], simplify=False), 1e-12, 0.0)
        elif case == "dup40":
            _, x, z, c = random_operator(rng, 40, 1_200_000, 0.25, 300_000)
            got = G.simplify(40, x, z, c)
            want = oracle.simplify(40, x, z, c)
        else:
            _, x, z, c = random_operator(rng, 40, 400_000, 0.25, 150_000)
            monkeypatch.setenv("WG_BUCKET_TRACE", "1")
            capi.set_bucket_fine_target(1800)
            try:
                got = G.simplify(40, x, z, c)
            finally:
                capi.set_bucket_fine_target(0)
            refined = [int(v) for v in re.findall(r"refined=(\d+)", capfd.readouterr().err)]
            assert refined and refined[-1] > 0
            want = oracle.simplify(40, x, z, c)
        assert capi.last_sort_algorithm() == capi.WG_SORT_BUCKET
    finally:
        capi.set_bucket_one_pass(True)
    assert same(got, want)


def test_bucket_fine_target_rejects_out_of_range(cuda):
    for bad in (1, 31, 2049):
        with pytest.raises(capi.WGInvalid):
            capi.set_bucket_fine_target(bad)
    capi.set_bucket_fine_target(0)


@pytest.mark.parametrize("copies,bucketed", [(1500, True), (3500, True), (5000, True)])
def test_bucket_one_key_runs(cuda, oracle, algo, copies, bucketed):
    """One key of 14 set bits repeated: its eight-digit code does not fix the
    key, so the run's fine bucket is checked key by key; up to 2048 items it is
    sorted in shared memory, above that its indices are sorted in global
    memory and summed in order."""
    rng = seeded("bucket-run", copies)
    n = 40
    x = np.zeros((copies + 300, 1), np.uint64)
    z = np.zeros((copies + 300, 1), np.uint64)
    x[:copies, 0] = np.uint64(0x5A5A5)
    z[:copies, 0] = np.uint64(0x33)
    x[copies:, 0] = rng.integers(0, 1 << 40, size=300, dtype=np.uint64)
    c = rng.normal(size=copies + 300) + 1j * rng.normal(size=copies + 300)
    perm = rng.permutation(copies + 300)
    x, z, c = x[perm], z[perm], c[perm]
    algo(capi.WG_SORT_BUCKET)
    got = G.simplify(n, x, z, c)
    assert capi.last_sort_algorithm() == (capi.WG_SORT_BUCKET if bucketed else capi.WG_SORT_LSD)
    assert same(got, oracle.simplify(n, x, z, c))


def test_bucket_not_eligible_above_255_bits(cuda, oracle, algo):
    rng = seeded("bucket-256")
    n, x, z, c = random_operator(rng, 128, 3000, 0.5)
    algo(capi.WG_SORT_BUCKET)
    got = G.simplify(n, x, z, c)
    assert capi.last_sort_algorithm() == capi.WG_SORT_LSD
    assert same(got, oracle.simplify(n, x, z, c))


@pytest.mark.parametrize("rtol", [0.0, 0.25])
def test_bucket_nonfinite_and_cancellation(cuda, oracle, algo, rtol):
    rng = seeded("bucket-nonfinite", rtol)
    n, x, z, c = random_operator(rng, 30, 6000, 0.2, 400)
    c[1::11] = -c[0::11][: len(c[1::11])]
    c[::13] = 1e-12
    algo(capi.WG_SORT_BUCKET)
    for bad in (None, np.inf, np.nan, complex(1e308, 1e308)):
        cc = c.copy()
        if bad is not None:
            cc[17] = bad
        got = G.simplify(n, x, z, cc, 1e-12, rtol)
        assert same(got, oracle.simplify(n, x, z, cc, 1e-12, rtol))
        A = (x[:90], z[:90], cc[:90])
        B = (x[90:190], z[90:190], cc[90:190].copy())
        gotp = G.products(n, A, B, capi.WG_PRODUCTS_SIMPLIFY, 1e-12, rtol)
        raw = oracle.matmul(n, A, B, simplify=False)
        assert same(gotp, oracle.simplify(n, *raw, 1e-12, rtol))


def test_bucket_everything_cancels(cuda, oracle, algo):
    rng = seeded("bucket-cancel")
    _, x, z, c = random_operator(rng, 50, 3000, 0.1)
    x2, z2, c2 = np.concatenate([x, x]), np.concatenate([z, z]), np.concatenate([c, -c])
    algo(capi.WG_SORT_BUCKET)
    got = G.simplify(50, x2, z2, c2)
    assert capi.last_sort_algorithm() == capi.WG_SORT_BUCKET
    assert len(got[2]) == 0
    assert same(got, oracle.simplify(50, x2, z2, c2))


def test_sort_algorithm_rejects_unknown(cuda):
    with pytest.raises(ValueError):
        capi.set_sort_algorithm(7)


@pytest.mark.parametrize("nl,nr", [(2048, 1024), (4096, 2048)])
def test_public_matmul_large_host_result(cuda, algo, nl, nr):
    """PauliSum.matmul through the public API with a host result above 64 MiB
    (result vectors grown by appending the downloaded chunks behind fault-ahead
    helpers; the larger case spans many 8 MiB chunks per vector) equals the device-side
    products of the C-ABI, downloaded directly."""
    import wolfgang_quantum as wq

    rng = seeded("public-large", nl, nr)
    A = klocal(rng, 100, nl)
    B = klocal(rng, 100, nr)
    hA = wq.PauliSum._from_packed(100, A[1], A[2], A[3])
    hB = wq.PauliSum._from_packed(100, B[1], B[2], B[3])
    r = hA.matmul(hB, max_intermediate_terms=nl * nr)
    x, z, c = r._packed()
    assert x.nbytes + z.nbytes + c.nbytes >= 64 << 20
    gx, gz, gc = G.products(100, A[1:], B[1:], capi.WG_PRODUCTS_FUSED)
    assert np.array_equal(x, gx) and np.array_equal(z, gz)
    assert np.array_equal(c.view(np.uint64), gc.view(np.uint64))
