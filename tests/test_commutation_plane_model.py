"""The bit-plane formulation of the commutation matrix, checked in numpy.

Terms l and r commute iff popc((lx & rz) ^ (lz & rx)) is even.  For a fixed
row l that parity, over all columns r at once, is the XOR over the qubits q in
l's support of (lx_q ? Zplane_q : 0) ^ (lz_q ? Xplane_q : 0), where Xplane_q /
Zplane_q are the bit-vectors over r of r's x / z bit on qubit q.  The device
kernel builds those planes for a block of columns in shared memory and, per
row, XORs the planes that the row's set bits select; the output bit is the
complement (1 = commute).
"""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("n,nl,nr,p", [(20, 40, 100, 0.3), (64, 30, 257, 0.1), (128, 25, 300, 0.05)])
def test_plane_xor_equals_parity(n, nl, nr, p):
    rng = np.random.default_rng(20261204 + n)
    lx, lz = rng.random((nl, n)) < p, rng.random((nl, n)) < p
    rx, rz = rng.random((nr, n)) < p, rng.random((nr, n)) < p
    # direct definition
    parity = ((lx[:, None, :] & rz[None, :, :]) ^ (lz[:, None, :] & rx[None, :, :])).sum(axis=2) % 2
    want = parity == 0
    # planes: X plane of qubit q is rx[:, q] over the columns, Z plane rz[:, q]
    xplane, zplane = rx.T, rz.T
    got = np.empty((nl, nr), bool)
    for i in range(nl):
        acc = np.zeros(nr, bool)
        for q in np.nonzero(lx[i])[0]:
            acc ^= zplane[q]  # a set x bit selects the rhs Z plane
        for q in np.nonzero(lz[i])[0]:
            acc ^= xplane[q]  # a set z bit selects the rhs X plane
        got[i] = ~acc
    assert np.array_equal(got, want)
