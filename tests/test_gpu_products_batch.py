"""Prepared product batches (wg_products_batch_*) against the oracle, bit for bit.

Each pair's result must equal the oracle's matmul + simplify (or the fused
path's cull) of that pair: masks, canonical order and coefficient bits.  The
batch is also captured in a CUDA graph and replayed after its coefficient
buffers are overwritten, and a run must not allocate.
"""

from __future__ import annotations

import zlib

import numpy as np
import pytest

from tests.conftest import random_operator
from wolfgang_b200 import capi

pytestmark = pytest.mark.gpu


def seeded(*key):
    return np.random.default_rng(zlib.crc32(repr(key).encode()))


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def oracle_pair(oracle, n, A, B, mode, atol=1e-12, rtol=0.0):
    raw = oracle.matmul(n, A[1:], B[1:], simplify=False)
    if mode == "fused":
        atol, rtol = 1e-12, 0.0  # the fused path's fixed cull; finite inputs
    return oracle.simplify(n, *raw, atol, rtol)


def uneven_pairs(rng, n, count, pool=None):
    pairs = []
    for k in range(count):
        nl = int(np.exp(rng.uniform(0, np.log(600))))
        nr = int(np.exp(rng.uniform(0, np.log(400))))
        p = rng.uniform(0.05, 0.4) if n <= 20 else rng.uniform(0.01, 0.08)
        A = random_operator(rng, n, nl, p, pool)
        B = random_operator(rng, n, nr, p, pool)
        pairs.append((A, B))
    return pairs


@pytest.mark.parametrize("n,count,pool,mode,rtol", [
    (12, 40, None, "simplify", 0.0),
    (12, 25, 30, "simplify", 0.0),     # duplicate-heavy operands: long equal-key runs
    (20, 30, None, "fused", 0.0),
    (70, 20, 60, "simplify", 0.05),    # two words, rtol cull
    (150, 12, None, "simplify", 0.0),  # three words
    (0, 5, None, "simplify", 0.0),     # no qubits: one key per pair
])
def test_products_batch_matches_oracle(cuda, oracle, n, count, pool, mode, rtol):
    from wolfgang_b200.products import ProductsBatch

    rng = seeded("pbatch", n, count, pool, mode)
    pairs = uneven_pairs(rng, n, count, pool)
    # an empty operand in the middle of the batch
    pairs.insert(count // 2, (random_operator(rng, n, 0, 0.1), random_operator(rng, n, 7, 0.1)))
    batch = ProductsBatch(pairs, mode=mode, atol=1e-12, rtol=rtol)
    batch.run()
    got = batch.results()
    assert batch.n_products == sum(len(A[3]) * len(B[3]) for A, B in pairs)
    for (A, B), g in zip(pairs, got):
        want = oracle_pair(oracle, n, A, B, mode, 1e-12, rtol)
        for a, b in zip(g, want):
            assert same_bits(a, b)
    batch.close()


def test_products_batch_graph_replay_with_new_coefficients(cuda, oracle):
    torch = cuda
    from wolfgang_b200.products import ProductsBatch

    rng = seeded("pbatch-graph")
    n = 30
    pairs = uneven_pairs(rng, n, 24, pool=80)
    batch = ProductsBatch(pairs)
    batch.capture()
    for trial in range(3):
        new = []
        for p, (A, B) in enumerate(pairs):
            lc = rng.normal(size=len(A[3])) + 1j * rng.normal(size=len(A[3]))
            rc = rng.normal(size=len(B[3])) + 1j * rng.normal(size=len(B[3]))
            if trial == 2 and p % 3 == 0:
                lc[: len(lc) // 2] = 0.0  # exact cancellations and culls
            batch.set_coefficients(p, lc, rc)
            new.append(((n, A[1], A[2], lc), (n, B[1], B[2], rc)))
        capi.call("wg_inject_alloc_failure", 1)  # a replay allocates nothing
        try:
            batch.replay()
            torch.cuda.synchronize()
        finally:
            capi.call("wg_inject_alloc_failure", 0)
        for (A, B), g in zip(new, batch.results()):
            for a, b in zip(g, oracle_pair(oracle, n, A, B, "simplify")):
                assert same_bits(a, b)
    batch.close()


def test_products_batch_equals_per_call_path(cuda):
    """The batch and wg_pauli_products (the per-call drop-in) agree bit for bit."""
    from tests import gpu_util as G
    from wolfgang_b200.products import ProductsBatch

    rng = seeded("pbatch-percall")
    n = 64
    pairs = uneven_pairs(rng, n, 16)
    batch = ProductsBatch(pairs)
    batch.run()
    for (A, B), g in zip(pairs, batch.results()):
        want = G.products(n, A[1:], B[1:], capi.WG_PRODUCTS_SIMPLIFY)
        for a, b in zip(g, want):
            assert same_bits(a, b)


def test_products_batch_rejects_bad_arguments(cuda):
    from wolfgang_b200.products import ProductsBatch

    rng = seeded("pbatch-bad")
    A = random_operator(rng, 10, 4, 0.3)
    with pytest.raises(ValueError, match="same num_qubits"):
        ProductsBatch([(A, random_operator(rng, 11, 4, 0.3))])
    with pytest.raises(ValueError, match="mode"):
        ProductsBatch([(A, A)], mode="raw")
    with pytest.raises(ValueError, match="tolerances"):
        ProductsBatch([(A, A)], atol=-1.0)


def test_products_batch_rejects_misaligned_coefficients(cuda):
    import ctypes

    torch = cuda
    rng = seeded("pbatch-align")
    A = random_operator(rng, 10, 4, 0.3)
    x, z = (torch.from_numpy(A[k].view(np.int64)).cuda() for k in (1, 2))
    c = torch.zeros(2 * len(A[3]) + 1, dtype=torch.float64, device="cuda")  # doubles from an 8-byte offset
    P = ctypes.c_void_p * 1
    S = ctypes.c_size_t * 1
    h = ctypes.c_void_p()
    with pytest.raises(ValueError, match="16-byte aligned"):
        capi.call("wg_products_batch_create", 0, 1, 1, P(x.data_ptr()), P(z.data_ptr()), P(c.data_ptr() + 8), S(4),
                  P(x.data_ptr()), P(z.data_ptr()), P(c.data_ptr() + 8), S(4), capi.WG_PRODUCTS_SIMPLIFY, 1e-12, 0.0,
                  ctypes.byref(h), None)


@pytest.mark.parametrize("rtol", [0.0, 0.2])
def test_products_batch_nonfinite_and_huge_coefficients(cuda, oracle, rtol):
    """An infinite |product| makes atol + rtol * max NaN (nothing of that pair
    survives); NaN products never raise the maximum; huge finite products
    overflow only where the reference's would."""
    from wolfgang_b200.products import ProductsBatch

    rng = seeded("pbatch-nonfinite", rtol)
    n = 16
    pairs = uneven_pairs(rng, n, 6, pool=40)
    special = [complex(np.inf, 0.5), complex(np.nan, 1.0), complex(1e200, -1e200), complex(1e300, 0.0)]
    for k, v in enumerate(special):
        A, B = pairs[k]
        c = A[3].copy()
        c[len(c) // 2] = v
        pairs[k] = ((A[0], A[1], A[2], c), B)
    batch = ProductsBatch(pairs, atol=1e-12, rtol=rtol)
    batch.run()
    for (A, B), g in zip(pairs, batch.results()):
        for a, b in zip(g, oracle_pair(oracle, n, A, B, "simplify", 1e-12, rtol)):
            assert same_bits(a, b)
    batch.close()
