"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")
    config.addinivalue_line("markers", "slow: long-running full-size case")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference core library (oracle/_ref) was not built")
    return Reference()


@pytest.fixture(scope="session")
def cuda():
    """Skips CPU-only runs; on a GPU box, returns torch with the device ready."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


def random_operator(rng: np.random.Generator, n: int, T: int, p: float = 0.3, pool: int | None = None):
    """Random operator; with `pool`, terms are drawn from `pool` distinct keys (duplicates)."""
    from wolfgang_b200.workloads import bernoulli_operator

    if pool is None:
        return bernoulli_operator(rng, n, T, p)
    _, px, pz, _ = bernoulli_operator(rng, n, pool, p)
    pick = rng.integers(0, pool, size=T)
    c = rng.normal(size=T) + 1j * rng.normal(size=T)
    return n, px[pick].copy(), pz[pick].copy(), c.astype(np.complex128)
