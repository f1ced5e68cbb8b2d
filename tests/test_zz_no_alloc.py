"""The no-allocation commutation entry point (wg_commutation_u8_noalloc).

It serves callers that cannot allocate device memory while they use the
library -- for example a framework that owns the whole device budget, or a
latency-critical loop that must not call cudaMalloc/cudaFree, which
synchronise the device.  Its scratch (the bit-packed matrix) is a static
device array, so this test checks, through the C-ABI, that calls in a row
give exactly the flags of the ordinary path (wg_commutation_bits followed by
wg_bits_to_u8 with caller buffers) and of the oracle, that they make no
allocation from the library's memory pool, that a request of exactly the
scratch size is accepted and a larger one rejected, that a call on a
non-default stream is ordered on that stream, and that a call after the first
can be captured in a CUDA graph and replayed on new inputs.  This file is
collected last so that a stopping failure here comes after every other test.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests.conftest import random_operator
from wolfgang_b200 import capi

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 32 << 20


def _ordinary_flags(torch, w, A, B, nl, nr):
    pitch = (nr + 31) // 32
    bits = torch.zeros(max(nl * pitch, 1), dtype=torch.int32, device="cuda")
    out = torch.zeros(nl * nr, dtype=torch.uint8, device="cuda")
    capi.call("wg_commutation_bits", 0, w, _p(A[0]), _p(A[1]), nl, _p(B[0]), _p(B[1]), nr, bits.data_ptr(), pitch, 0,
              None)
    capi.call("wg_bits_to_u8", 0, bits.data_ptr(), nl, nr, pitch, out.data_ptr(), None)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _p(t):
    return t.data_ptr() if t is not None and t.numel() > 0 else None


def _dev(torch, a):
    a = np.ascontiguousarray(a)
    if a.size == 0:
        return torch.zeros(1, dtype=torch.int64, device="cuda")
    return torch.from_numpy(a.view(np.int64)).cuda()


def _noalloc(torch, w, dA, dB, nl, nr, out, stream=None):
    # any allocation from the library's pool during the call would fail
    capi.call("wg_inject_alloc_failure", 1)
    try:
        capi.call("wg_commutation_u8_noalloc", 0, w, _p(dA[0]), _p(dA[1]), nl, _p(dB[0]), _p(dB[1]), nr,
                  out.data_ptr(), stream)
    finally:
        capi.call("wg_inject_alloc_failure", 0)


@pytest.mark.parametrize("n, nl, nr, p", [
    (70, 700, 1100, 0.05),   # two words, bit-plane kernel by the size rule
    (20, 333, 97, 0.3),      # one word, ballot kernel (few columns)
    (0, 45, 77, 0.0),        # no qubits: every pair commutes (fill path)
    (300, 130, 600, 0.02),   # five words: generic kernel
])
def test_noalloc_matches_ordinary_path_and_oracle_twice(cuda, oracle, n, nl, nr, p):
    torch = cuda
    rng = np.random.default_rng(2718 + n)
    w = 0 if n == 0 else (n + 63) // 64
    for _ in range(2):  # two calls in a row on the shared scratch
        A = random_operator(rng, n, nl, p)
        B = random_operator(rng, n, nr, p)
        dA = (_dev(torch, A[1]), _dev(torch, A[2]))
        dB = (_dev(torch, B[1]), _dev(torch, B[2]))
        want = _ordinary_flags(torch, w, dA, dB, nl, nr)
        out = torch.full((nl * nr,), 7, dtype=torch.uint8, device="cuda")
        _noalloc(torch, w, dA, dB, nl, nr, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got, want)
        assert np.array_equal(got.reshape(nl, nr), oracle.commutes(n, (A[1], A[2]), (B[1], B[2])))


def test_noalloc_accepts_exactly_its_scratch_size(cuda, oracle):
    torch = cuda
    nl, nr = 8192, 32768  # 8192 rows x 1024 words x 4 bytes = 32 MiB exactly
    assert nl * ((nr + 31) // 32) * 4 == SCRATCH_BYTES
    rng = np.random.default_rng(31)
    n = 40
    A = random_operator(rng, n, nl, 0.1)
    B = random_operator(rng, n, nr, 0.1)
    dA = (_dev(torch, A[1]), _dev(torch, A[2]))
    dB = (_dev(torch, B[1]), _dev(torch, B[2]))
    want = _ordinary_flags(torch, 1, dA, dB, nl, nr)
    out = torch.full((nl * nr,), 7, dtype=torch.uint8, device="cuda")
    _noalloc(torch, 1, dA, dB, nl, nr, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.array_equal(got, want)
    rows = slice(nl - 64, nl)  # the rows at the very end of the scratch, against the oracle
    assert np.array_equal(got.reshape(nl, nr)[rows], oracle.commutes(n, (A[1][rows], A[2][rows]), (B[1], B[2])))


def test_noalloc_on_a_side_stream(cuda, oracle):
    torch = cuda
    rng = np.random.default_rng(77)
    n, nl, nr = 90, 640, 900
    A = random_operator(rng, n, nl, 0.05)
    B = random_operator(rng, n, nr, 0.05)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        dA = (_dev(torch, A[1]), _dev(torch, A[2]))
        dB = (_dev(torch, B[1]), _dev(torch, B[2]))
        out = torch.full((nl * nr,), 7, dtype=torch.uint8, device="cuda")
        _noalloc(torch, 2, dA, dB, nl, nr, out, side.cuda_stream)
        got_dev = out.clone()  # ordered after the call on the same stream
    side.synchronize()
    assert np.array_equal(got_dev.cpu().numpy().reshape(nl, nr), oracle.commutes(n, (A[1], A[2]), (B[1], B[2])))


def test_noalloc_call_captured_in_a_cuda_graph(cuda, oracle):
    torch = cuda
    rng = np.random.default_rng(4242)
    n, nl, nr = 70, 700, 1100  # >= 512 x 512 terms: the bit-plane kernel
    A = random_operator(rng, n, nl, 0.05)
    B = random_operator(rng, n, nr, 0.05)
    dA = (_dev(torch, A[1]), _dev(torch, A[2]))
    dB = (_dev(torch, B[1]), _dev(torch, B[2]))
    out = torch.full((nl * nr,), 7, dtype=torch.uint8, device="cuda")
    _noalloc(torch, 2, dA, dB, nl, nr, out)  # first call on the device: resolves the scratch address
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        capi.call("wg_commutation_u8_noalloc", 0, 2, _p(dA[0]), _p(dA[1]), nl, _p(dB[0]), _p(dB[1]), nr,
                  out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    for trial in range(2):  # replay on new inputs written into the captured buffers
        A = random_operator(rng, n, nl, 0.05)
        B = random_operator(rng, n, nr, 0.05)
        dA[0].copy_(_dev(torch, A[1]))
        dA[1].copy_(_dev(torch, A[2]))
        dB[0].copy_(_dev(torch, B[1]))
        dB[1].copy_(_dev(torch, B[2]))
        out.fill_(7)
        graph.replay()
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().reshape(nl, nr), oracle.commutes(n, (A[1], A[2]), (B[1], B[2])))
    del graph


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    torch = cuda
    dummy = torch.zeros(8, dtype=torch.int64, device="cuda")
    with pytest.raises(ValueError, match="32 MiB"):
        # 2^15 rows x 2^13 words x 4 bytes = 1 GiB > 32 MiB: rejected before any launch
        capi.call("wg_commutation_u8_noalloc", 0, 1, dummy.data_ptr(), dummy.data_ptr(), 1 << 15,
                  dummy.data_ptr(), dummy.data_ptr(), 1 << 18, dummy.data_ptr(), None)
    with pytest.raises(ValueError, match="32 MiB"):
        # one word more than the scratch holds: 8192 rows x 1025 words x 4 bytes
        capi.call("wg_commutation_u8_noalloc", 0, 1, dummy.data_ptr(), dummy.data_ptr(), 8192,
                  dummy.data_ptr(), dummy.data_ptr(), 32768 + 1, dummy.data_ptr(), None)
