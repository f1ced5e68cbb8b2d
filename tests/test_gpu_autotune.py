"""The autotuner on the device: every candidate gives identical bits, and a
search caches a choice per shape class.

Each tuned operation is run with each of its candidates forced through an
imported cache line, and with a search, and compared with the untuned call
(WG_TUNE_OFF) and with the oracle: commutation bits, products + simplify
(bucketed path: keys, order and coefficient bits), grouping (groups and their
order).
"""

from __future__ import annotations

import ctypes
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


def lg(n):
    return int(np.ceil(np.log2(n))) if n > 1 else 0


@pytest.fixture()
def tuner(cuda):
    mode = capi.autotune_mode()
    capi.autotune_clear()
    yield capi
    capi.autotune_clear()
    capi.autotune_mode(mode)


@pytest.mark.parametrize("n,nl,nr", [(20, 700, 1500), (100, 3000, 2600), (150, 300, 900)])
def test_commutation_candidates_identical(tuner, oracle, n, nl, nr):
    rng = seeded("tune-comm", n, nl, nr)
    A = random_operator(rng, n, nl, 0.05)
    B = random_operator(rng, n, nr, 0.05)
    w = (n + 63) // 64
    tuner.autotune_mode(capi.WG_TUNE_OFF)
    base = G.commutation_bits(n, A[1:3], B[1:3], algo=0)
    assert np.array_equal(G.unpack_bits(base, nr), oracle.commutes(n, A[1:3], B[1:3]))
    tuner.autotune_mode(capi.WG_TUNE_CACHED)
    for c in range(5):  # candidate 2 and 4 serve 1-2 words only; others fall back to the default
        tuner.autotune_clear()
        tuner.autotune_import(f"commute {w} {lg(nl)} {lg(nr)} {c}\n")
        assert same_bits(G.commutation_bits(n, A[1:3], B[1:3], algo=0), base)
    tuner.autotune_clear()
    tuner.autotune_mode(capi.WG_TUNE_SEARCH)
    assert same_bits(G.commutation_bits(n, A[1:3], B[1:3], algo=0), base)  # the searching call
    assert same_bits(G.commutation_bits(n, A[1:3], B[1:3], algo=0), base)  # served from the cache
    lines = tuner.autotune_export().splitlines()
    assert len(lines) == 1 and lines[0].startswith(f"commute {w} {lg(nl)} {lg(nr)} ")


def test_bucket_fine_target_candidates_identical(tuner, oracle):
    rng = seeded("tune-bucket")
    n = 100
    from wolfgang_b200.workloads import klocal_operator

    A = klocal_operator(rng, n, 1024, np.array([2, 3, 4]))
    B = klocal_operator(rng, n, 1100, np.array([2, 3, 4]))  # 1.1e6 products: the bucketed path
    P = 1024 * 1100
    prev = capi.set_sort_algorithm(capi.WG_SORT_BUCKET)
    try:
        tuner.autotune_mode(capi.WG_TUNE_OFF)
        base = G.products(n, A[1:], B[1:], capi.WG_PRODUCTS_SIMPLIFY)
        assert capi.last_sort_algorithm() == capi.WG_SORT_BUCKET
        raw = oracle.matmul(n, A[1:], B[1:], simplify=False)
        for a, b in zip(base, oracle.simplify(n, *raw, 1e-12, 0.0)):
            assert same_bits(a, b)
        tuner.autotune_mode(capi.WG_TUNE_CACHED)
        for c in range(5):
            tuner.autotune_clear()
            tuner.autotune_import(f"bucket 2 {lg(P)} 0 {c}\n")
            for a, b in zip(G.products(n, A[1:], B[1:], capi.WG_PRODUCTS_SIMPLIFY), base):
                assert same_bits(a, b)
        tuner.autotune_clear()
        tuner.autotune_mode(capi.WG_TUNE_SEARCH)
        for _ in range(2):  # the searching call, then the cached one
            for a, b in zip(G.products(n, A[1:], B[1:], capi.WG_PRODUCTS_SIMPLIFY), base):
                assert same_bits(a, b)
        assert tuner.autotune_export().startswith(f"bucket 2 {lg(P)} 0 ")
    finally:
        capi.set_sort_algorithm(prev)


def _groups(n, x, z, mode):
    w = 0 if n == 0 else (n + 63) // 64
    T = len(x)
    dx, dz = G.dev(x), G.dev(z)
    order = np.zeros(T, np.uintp)
    sizes = np.zeros(T, np.uintp)
    ng = ctypes.c_size_t()
    capi.call("wg_group_commuting", 0, w, T, G.ptr(dx), G.ptr(dz), 1 if mode == "full" else 0,
              order.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t)),
              sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t)), ctypes.byref(ng), None)
    out, q = [], 0
    for s in sizes[: ng.value]:
        out.append([int(v) for v in order[q:q + int(s)]])
        q += int(s)
    return out


@pytest.mark.parametrize("mode,count", [("qwc", 3), ("full", 4)])
def test_grouping_chunk_candidates_identical(tuner, oracle, mode, count):
    rng = seeded("tune-group", mode)
    n, T = 128, 5000 if mode == "qwc" else 2500
    _, x, z, _ = random_operator(rng, n, T, 0.05)
    want = oracle.group_commuting(n, x, z, mode)
    tuner.autotune_mode(capi.WG_TUNE_CACHED)
    for c in range(count):
        tuner.autotune_clear()
        tuner.autotune_import(f"group_{mode} 2 {lg(T)} 0 {c}\n")
        assert _groups(n, x, z, mode) == want
    tuner.autotune_clear()
    tuner.autotune_mode(capi.WG_TUNE_SEARCH)
    assert _groups(n, x, z, mode) == want
    assert tuner.autotune_export().startswith(f"group_{mode} 2 {lg(T)} 0 ")
