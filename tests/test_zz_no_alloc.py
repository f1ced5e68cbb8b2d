"""The no-allocation commutation entry point (wg_commutation_u8_noalloc).

It serves callers that cannot allocate device memory while they use the
library -- for example a framework that owns the whole device budget, or a
latency-critical loop that must not call cudaMalloc/cudaFree, which
synchronise the device.  Its scratch (the bit-packed matrix) is a static
device array, so this test checks, through the C-ABI, that two calls in a row
give exactly the flags of the ordinary path (wg_commutation_bits followed by
wg_bits_to_u8 with caller buffers), that it makes no allocation from the
library's memory pool, and that oversized requests are rejected.  This file is
collected last so that a stopping failure here comes after every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from tests.conftest import random_operator
from wolfgang_b200 import capi

pytestmark = pytest.mark.gpu


def _ordinary_flags(torch, w, A, B):
    nl, nr = len(A[0]), len(B[0])
    pitch = (nr + 31) // 32
    bits = torch.zeros(nl * pitch, dtype=torch.int32, device="cuda")
    out = torch.zeros(nl * nr, dtype=torch.uint8, device="cuda")
    capi.call("wg_commutation_bits", 0, w, A[0].data_ptr(), A[1].data_ptr(), nl, B[0].data_ptr(), B[1].data_ptr(),
              nr, bits.data_ptr(), pitch, 0, None)
    capi.call("wg_bits_to_u8", 0, bits.data_ptr(), nl, nr, pitch, out.data_ptr(), None)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def test_noalloc_matches_ordinary_path_twice(cuda):
    torch = cuda
    rng = np.random.default_rng(2718)
    cases = [(70, 700, 1100, 0.05), (20, 333, 97, 0.3)]  # two calls in a row, different shapes
    for n, nl, nr, p in cases:
        w = (n + 63) // 64
        A = random_operator(rng, n, nl, p)
        B = random_operator(rng, n, nr, p)
        dA = (_dev(torch, A[1]), _dev(torch, A[2]))
        dB = (_dev(torch, B[1]), _dev(torch, B[2]))
        want = _ordinary_flags(torch, w, dA, dB)
        out = torch.full((nl * nr,), 7, dtype=torch.uint8, device="cuda")
        # any allocation from the library's pool during the call would fail
        capi.call("wg_inject_alloc_failure", 1)
        try:
            capi.call("wg_commutation_u8_noalloc", 0, w, dA[0].data_ptr(), dA[1].data_ptr(), nl, dB[0].data_ptr(),
                      dB[1].data_ptr(), nr, out.data_ptr(), None)
        finally:
            capi.call("wg_inject_alloc_failure", 0)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), want)


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    torch = cuda
    dummy = torch.zeros(8, dtype=torch.int64, device="cuda")
    with pytest.raises(ValueError, match="32 MiB"):
        # 2^15 rows x 2^13 words x 4 bytes = 1 GiB > 32 MiB: rejected before any launch
        capi.call("wg_commutation_u8_noalloc", 0, 1, dummy.data_ptr(), dummy.data_ptr(), 1 << 15,
                  dummy.data_ptr(), dummy.data_ptr(), 1 << 18, dummy.data_ptr(), None)
