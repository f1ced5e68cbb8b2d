"""Arithmetic that two kernels rely on, checked on the CPU.

* The expectation adjoint forms a quad's sign mask at a thread's first output
  j0 = hi + tid (hi a multiple of the tile size, >= 256 or 0; tid < 256) as
  parity(z & (hi ^ x)), staged once per tile by the CTA, XOR parity(z & tid),
  read from the plan's per-lane table: the two must equal parity(z & (j0 ^ x)).
* The bucketed sort's one-pass fine layout gives each coarse bucket
  slots * 2048 records; a coarse bucket whose fine buckets overflow falls back
  to packing them 32-aligned inside that room, which must hold its n items
  whenever the host admitted the call (n <= capacity <= 640 * target).
"""

from __future__ import annotations

import numpy as np

K_CAP = 2048        # records a fine bucket owns in the one-pass layout
K_FINE_MAX = 640    # fine buckets targeted per coarse bucket at most


def parity(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint64)
    bits = np.unpackbits(v.view(np.uint8)).reshape(*v.shape, 64)
    return bits.sum(axis=-1) & 1


def test_adjoint_sign_mask_splits_into_tile_and_lane_parts():
    rng = np.random.default_rng(7)
    for n in (8, 12, 20, 26, 40):
        tlog = min(n, 12)
        z = rng.integers(0, 1 << n, size=64, dtype=np.uint64)
        x = rng.integers(0, 1 << n, size=64, dtype=np.uint64)
        tiles = 1 << (n - tlog)
        hi = (rng.integers(0, tiles, size=64, dtype=np.uint64) << np.uint64(tlog))
        tid = rng.integers(0, min(256, 1 << tlog), size=64, dtype=np.uint64)
        j0 = hi + tid
        whole = parity(z & (j0 ^ x))
        split = parity(z & (hi ^ x)) ^ parity(z & tid)
        assert np.array_equal(whole, split)


def fine_slots(n: int, favg: int) -> int:
    t = max(1, min(K_FINE_MAX, -(-n // favg)))
    return t + t // 4 + 8


def test_packed_fallback_fits_the_one_pass_room():
    for favg in (32, 500, 896, 1024, 2048):
        for n in (1, 31, 1000, 262_144, 532_480, K_FINE_MAX * favg):
            if n > K_FINE_MAX * favg:  # the host sends such calls elsewhere
                continue
            slots = fine_slots(n, favg)
            packed = n + 31 * slots  # every fine bucket rounded up to 32 records
            assert packed <= slots * K_CAP, (favg, n, slots)
