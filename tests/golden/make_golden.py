"""Generates tests/golden/*.npz by running the reference's own C++ core.

Run in a checkout where oracle/_ref/libwgref.so was built from the reference
sources (``make -C oracle``):

    python tests/golden/make_golden.py

Each fixture stores seeded inputs and the reference's outputs for one case:
simplify, matmul (raw, simplified, fused path), commutation flags,
group_commuting (qwc and full), expectation values (complex128 and
complex64, general and all-diagonal) and Z-count expectations.  Names given
on the command line limit the run to those fixtures.  tests/test_golden.py checks the
oracle against them and tests/test_gpu_golden.py the device kernels.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle import Reference  # noqa: E402
from wolfgang_b200.workloads import bernoulli_operator, klocal_operator  # noqa: E402


def op(seed, n, T, p, pool=None):
    rng = np.random.default_rng(seed)
    if pool is None:
        return bernoulli_operator(rng, n, T, p)
    _, px, pz, _ = bernoulli_operator(rng, n, pool, p)
    pick = rng.integers(0, pool, size=T)
    c = rng.normal(size=T) + 1j * rng.normal(size=T)
    return n, px[pick].copy(), pz[pick].copy(), c.astype(np.complex128)


def main() -> None:
    ref = Reference()
    out: dict[str, dict[str, np.ndarray]] = {}

    for name, (seed, n, T, p, pool, atol, rtol) in {
        "simplify_w1_dups": (1, 20, 6000, 0.25, 500, 1e-12, 0.0),
        "simplify_w2_rtol": (2, 70, 3000, 0.05, 400, 1e-12, 0.02),
        "simplify_w3": (3, 150, 800, 0.03, 100, 0.0, 0.0),
        "simplify_cull": (4, 10, 2000, 0.3, 200, 0.7, 0.0),
    }.items():
        _, x, z, c = op(seed, n, T, p, pool)
        ox, oz, oc = ref.simplify(n, x, z, c, atol, rtol)
        out[name] = dict(n=np.int64(n), x=x, z=z, c=c, atol=np.float64(atol), rtol=np.float64(rtol),
                         out_x=ox, out_z=oz, out_c=oc)

    for name, (seed, n, nl, nr, p, pool, simp) in {
        "matmul_w1_raw": (10, 12, 40, 30, 0.3, None, 0),
        "matmul_w1": (11, 16, 300, 200, 0.25, None, 1),
        "matmul_w1_fused": (12, 12, 300, 200, 0.3, 40, 1),
        "matmul_w2_fused": (13, 70, 256, 200, 0.05, 30, 1),
    }.items():
        A = op(seed, n, nl, p, pool)
        B = op(seed + 100, n, nr, p)
        ox, oz, oc = ref.matmul(n, A[1:], B[1:], simplify=bool(simp))
        out[name] = dict(n=np.int64(n), lx=A[1], lz=A[2], lc=A[3], rx=B[1], rz=B[2], rc=B[3],
                         simplify=np.int64(simp), out_x=ox, out_z=oz, out_c=oc)
    rng = np.random.default_rng(14)
    A = klocal_operator(rng, 100, 256, np.array([2, 3, 4]))
    B = klocal_operator(rng, 100, 128, np.array([2, 3, 4]))
    ox, oz, oc = ref.matmul(100, A[1:], B[1:], simplify=True)
    out["matmul_config2_slice"] = dict(n=np.int64(100), lx=A[1], lz=A[2], lc=A[3], rx=B[1], rz=B[2], rc=B[3],
                                       simplify=np.int64(1), out_x=ox, out_z=oz, out_c=oc)

    for name, (seed, n, nl, nr, p) in {"commute_w1": (20, 30, 200, 333, 0.2),
                                       "commute_w2": (21, 128, 300, 257, 0.05)}.items():
        A = op(seed, n, nl, p)
        B = op(seed + 1, n, nr, p)
        out[name] = dict(n=np.int64(n), lx=A[1], lz=A[2], rx=B[1], rz=B[2], flags=ref.commutes(n, A[1:3], B[1:3]))

    for name, (seed, n, T, p, pool) in {"group_w1": (30, 10, 400, 0.2, None),
                                        "group_w2": (31, 128, 1500, 0.05, None)}.items():
        _, x, z, c = op(seed, n, T, p, pool)
        rec = dict(n=np.int64(n), x=x, z=z, c=c)
        for mode in ("qwc", "full"):
            groups = ref.group_commuting(n, x, z, c, mode)
            rec[f"{mode}_sizes"] = np.array([len(g[2]) for g in groups], np.int64)
            rec[f"{mode}_x"] = np.concatenate([g[0] for g in groups])
            rec[f"{mode}_z"] = np.concatenate([g[1] for g in groups])
            rec[f"{mode}_c"] = np.concatenate([g[2] for g in groups])
        out[name] = rec

    for name, (seed, n, T, p, diag, dtype) in {
        "expect_c128": (40, 12, 300, 0.25, False, np.complex128),
        "expect_c64": (41, 10, 120, 0.3, False, np.complex64),
        "expect_diag": (42, 10, 100, 0.3, True, np.complex128),
    }.items():
        _, x, z, c = op(seed, n, T, p)
        if diag:
            x[:] = 0
        rng = np.random.default_rng(seed + 7)
        psi = (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n))
        psi = (psi / np.linalg.norm(psi)).astype(dtype)
        e = ref.expectation(n, x, z, c, psi)
        out[name] = dict(n=np.int64(n), x=x, z=z, c=c, psi=psi, value=np.complex128(e))

    for name, (seed, n, T, p, rows) in {"zcounts_w1": (50, 10, 60, 0.3, 300),
                                        "zcounts_w2": (51, 100, 40, 0.05, 500)}.items():
        _, x, z, c = op(seed, n, T, p)
        x[:] = 0  # Z-count expectations take diagonal terms only
        rng = np.random.default_rng(seed + 9)
        w = (n + 63) // 64
        bits = rng.random((rows, n)) < 0.5
        padded = np.zeros((rows, 64 * w), np.uint8)
        padded[:, :n] = bits
        packed = np.packbits(padded, axis=1, bitorder="little").view("<u8").reshape(rows, w).astype(np.uint64)
        counts = rng.integers(0, 50, size=rows).astype(np.float64)
        e = ref.expectation_z_counts(n, x, z, c, packed, counts)
        out[name] = dict(n=np.int64(n), x=x, z=z, c=c, packed=packed, counts=counts, value=np.complex128(e))

    only = set(sys.argv[1:])
    written = [name for name in out if not only or name in only]
    for name in written:
        np.savez_compressed(HERE / f"{name}.npz", **out[name])
    print("wrote", len(written), "fixtures to", HERE)


if __name__ == "__main__":
    main()
