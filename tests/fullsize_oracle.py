"""Oracle work of the full-size parity tests, run in spawned worker processes.

TEST INFRASTRUCTURE (the checker).  Each worker regenerates the seeded
workload itself (the generators are loaded by file path, so no worker loads
the package's native libraries or touches the GPU) and returns digests or
small arrays: no large buffer crosses a process boundary.  The pool is
created with the "spawn" start method, so a worker never inherits a CUDA
context from the test process.
"""

from __future__ import annotations

import hashlib
import importlib.util
import multiprocessing as mp
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
_STATE: dict = {}


def workloads():
    """wolfgang_b200/workloads.py (numpy only), loaded without the package."""
    mod = sys.modules.get("wg_test_workloads")
    if mod is None:
        spec = importlib.util.spec_from_file_location("wg_test_workloads", ROOT / "wolfgang_b200" / "workloads.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules["wg_test_workloads"] = mod
    return mod


def digest(*arrays) -> str:
    """blake2b over the arrays' bytes (C order), in turn."""
    h = hashlib.blake2b(digest_size=20)
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(memoryview(a).cast("B") if a.size else b"")
    return h.hexdigest()


def pool(n: int | None = None):
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 2
    n = n or max(1, min(32, cores))
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    return mp.get_context("spawn").Pool(n, initializer=_init, initargs=(str(ROOT),))


def _init(root: str) -> None:
    if root not in sys.path:
        sys.path.insert(0, root)


# ------------------------------------------------------------ config 2

def products_range(args):
    """Oracle matmul + simplify of the 32,768 x 16,384 products workload over
    the key range [lo, hi): (survivor count, digest of x, z, coefficients)."""
    lo, hi, cap = args
    from oracle import Oracle

    if "products" not in _STATE:
        _STATE["products"] = workloads().klocal_pair_100q()
    A, B = _STATE["products"]
    ox, oz, oc = Oracle().matmul_keyrange(100, A[1:], B[1:], lo, hi, cap=cap)
    return len(oc), digest(ox, oz, oc)


# ------------------------------------------------------------ config 5

def pair_term_values(args):
    """Oracle <psi|P_k|psi> of pair (n, T, seed) for the listed terms, with the
    pair's seeded state stored as `dtype`; plus (H psi) at `idx` (complex128
    state only) and, when `full`, the pair's E in the reference's order."""
    n, T, seed, sample, idx, dtype, full = args
    from oracle import Oracle

    w = workloads()
    _, x, z, c = w.uneven_pair_operator(n, T, seed)
    psi = w.uneven_pair_state(n, seed, np.complex128 if dtype == "c128" else np.complex64)
    orc = Oracle()
    vals = orc.term_expectations(n, x[sample], z[sample], psi)
    hp = orc.hpsi_at(n, x, z, c, psi, idx) if dtype == "c128" and len(idx) else np.zeros(0, np.complex128)
    E = orc.expectation(n, x, z, c, psi) if full else None
    return vals, hp, E
