"""Seeded synthetic workloads of the five benchmark configurations.

Operators are returned as ``(n, x, z, c)`` numpy arrays: ``x``/``z`` uint64 of
shape ``(T, words)`` (bit q%64 of word q//64 = X / Z part of qubit q), ``c``
complex128 of shape ``(T,)``.  Paulis are encoded X=(1,0), Y=(1,1), Z=(0,1).
Each configuration uses ``numpy.random.default_rng(20261203 + k)`` so every
machine regenerates the same inputs; no dataset is read.

  1  plain: 20 qubits, 4,096 terms, each qubit non-identity with p=0.25,
     complex N(0,1) coefficients; psi 2^20 complex Gaussian, normalised.
  2  products: 100 qubits, A 32,768 and B 16,384 terms of weight U{2,3,4}.
  3  commutation: 128 qubits, 262,144 terms, p=0.05.
  4  differentiable expectation: 26 qubits, 20,000 Hermitian terms with real
     N(0, 1/sqrt(T)) coefficients whose x-masks come from 2,000 distinct
     patterns (weight a in 0..4), term weight U{1..8}.
  5  batched: 512 (H, psi) pairs, n in U{8..24}, T log-uniform in
     [100, 50,000], weight U{1..6}, real N(0,1) coefficients.
  6  batched products: 256 products A_p * B_p on 64 qubits, term counts
     log-uniform in [16, 4,096] on each side, weight U{1..6}, complex N(0,1)
     coefficients (the product counterpart of 5).
"""

from __future__ import annotations

import numpy as np

SEED_BASE = 20261203


def rng_for(k: int) -> np.random.Generator:
    """Generator of workload k: PCG64 seeded with SEED_BASE + k."""
    return np.random.default_rng(SEED_BASE + k)


def words_for(n: int) -> int:
    return 0 if n == 0 else (n + 63) // 64


def pack_bits(bits: np.ndarray, n: int) -> np.ndarray:
    """(T, n) bool -> (T, words) uint64, qubit q -> bit q%64 of word q//64."""
    T = bits.shape[0]
    w = words_for(n)
    if w == 0:
        return np.zeros((T, 0), np.uint64)
    padded = np.zeros((T, 64 * w), np.uint8)
    padded[:, :n] = bits
    return np.packbits(padded, axis=1, bitorder="little").view("<u8").reshape(T, w).astype(np.uint64)


def paulis_to_xz(kind: np.ndarray, active: np.ndarray, n: int) -> tuple[np.ndarray, np.ndarray]:
    """kind in {0:X, 1:Y, 2:Z} where active."""
    xb = active & (kind < 2)
    zb = active & (kind > 0)
    return pack_bits(xb, n), pack_bits(zb, n)


def bernoulli_operator(rng: np.random.Generator, n: int, T: int, p: float, real: bool = False):
    active = rng.random((T, n)) < p
    kind = rng.integers(0, 3, size=(T, n))
    x, z = paulis_to_xz(kind, active, n)
    c = rng.normal(size=T) + (0.0 if real else 1j * rng.normal(size=T))
    return n, x, z, np.asarray(c, np.complex128)


def klocal_operator(rng: np.random.Generator, n: int, T: int, weights: np.ndarray, real: bool = False):
    """Each term: weight drawn from `weights`, distinct uniform qubits, X/Y/Z uniform."""
    w = rng.choice(weights, size=T)
    order = np.argsort(rng.random((T, n)), axis=1)
    active = np.zeros((T, n), bool)
    rows = np.arange(T)[:, None]
    cols = np.arange(n)[None, :]
    # the first w[t] qubits of the random permutation are non-identity
    rank = np.empty_like(order)
    rank[rows, order] = cols
    active = rank < w[:, None]
    kind = rng.integers(0, 3, size=(T, n))
    x, z = paulis_to_xz(kind, active, n)
    c = rng.normal(size=T) + (0.0 if real else 1j * rng.normal(size=T))
    return n, x, z, np.asarray(c, np.complex128)


def random_state(rng: np.random.Generator, n: int, dtype=np.complex128) -> np.ndarray:
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    return psi.astype(dtype)


def hamiltonian_20q_and_state():
    rng = rng_for(1)
    H = bernoulli_operator(rng, 20, 4096, 0.25)
    psi = random_state(rng, 20)
    return H, psi


def klocal_pair_100q(scale_a: int = 32768, scale_b: int = 16384):
    rng = rng_for(2)
    A = klocal_operator(rng, 100, scale_a, np.array([2, 3, 4]))
    B = klocal_operator(rng, 100, scale_b, np.array([2, 3, 4]))
    return A, B


def sparse_operator_128q(T: int = 262144):
    rng = rng_for(3)
    return bernoulli_operator(rng, 128, T, 0.05)


def xpattern_operator(n: int = 26, T: int = 20000, patterns: int = 2000, seed_offset: int = 0):
    """Hermitian H with x-masks from `patterns` distinct x-patterns."""
    rng = np.random.default_rng(SEED_BASE + 4 + seed_offset)
    pats: list[np.ndarray] = []
    seen: set[bytes] = set()
    while len(pats) < patterns:
        a = int(rng.integers(0, 5))
        sup = np.sort(rng.choice(n, size=a, replace=False)) if a else np.zeros(0, np.int64)
        key = sup.tobytes()
        if key in seen:
            continue
        seen.add(key)
        pats.append(sup)
    pat_w = np.array([len(p) for p in pats])
    active = np.zeros((T, n), bool)
    kind = np.zeros((T, n), np.int64)
    for t in range(T):
        w = int(rng.integers(1, 9))
        eligible = np.nonzero(pat_w <= w)[0]
        sup = pats[int(rng.choice(eligible))]
        active[t, sup] = True
        kind[t, sup] = rng.integers(0, 2, size=len(sup))  # X or Y on the pattern
        free = np.setdiff1d(np.arange(n), sup)
        extra = rng.choice(free, size=w - len(sup), replace=False) if w > len(sup) else np.zeros(0, np.int64)
        active[t, extra] = True
        kind[t, extra] = 2  # Z off the pattern
    x, z = paulis_to_xz(kind, active, n)
    c = rng.normal(scale=1.0 / np.sqrt(T), size=T).astype(np.complex128)
    return n, x, z, c


def state_26q(n: int = 26) -> np.ndarray:
    return random_state(np.random.default_rng(SEED_BASE + 40), n)


def uneven_pairs(count: int = 512, n_min: int = 8, n_max: int = 24, t_min: int = 100, t_max: int = 50000):
    """List of (n, T, seed) descriptors; operators/states are built per pair."""
    rng = rng_for(5)
    ns = rng.integers(n_min, n_max + 1, size=count)
    Ts = np.round(np.exp(rng.uniform(np.log(t_min), np.log(t_max), size=count))).astype(np.int64)
    return [(int(ns[i]), int(Ts[i]), SEED_BASE + 5000 + i) for i in range(count)]


def uneven_pair_operator(n: int, T: int, seed: int):
    rng = np.random.default_rng(seed)
    return klocal_operator(rng, n, T, np.arange(1, min(6, n) + 1), real=True)


def uneven_pair_state(n: int, seed: int, dtype=np.complex128) -> np.ndarray:
    return random_state(np.random.default_rng(seed + 1_000_000), n, dtype)


def uneven_product_pairs(count: int = 256, n: int = 64, t_min: int = 16, t_max: int = 4096):
    """List of (n, T_lhs, T_rhs, seed) descriptors of uneven products."""
    rng = rng_for(6)
    Ts = np.round(np.exp(rng.uniform(np.log(t_min), np.log(t_max), size=(count, 2)))).astype(np.int64)
    return [(n, int(a), int(b), SEED_BASE + 6000 + i) for i, (a, b) in enumerate(Ts)]


def uneven_product_operands(n: int, t_lhs: int, t_rhs: int, seed: int):
    rng = np.random.default_rng(seed)
    weights = np.arange(1, min(6, n) + 1)
    return klocal_operator(rng, n, t_lhs, weights), klocal_operator(rng, n, t_rhs, weights)
