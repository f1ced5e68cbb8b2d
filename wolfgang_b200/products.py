"""Batched Pauli products on the B200: many lhs_p * rhs_p prepared once, run many times.

:class:`ProductsBatch` wraps the wg_products_batch_* C-ABI.  Creating it reads
every pair's masks once on the device (all products sorted by key, equal keys
grouped in nested-loop order, outputs sized); :meth:`ProductsBatch.run` then
forms, sums and culls the coefficients of every pair in a few launches with no
allocation and no host synchronisation, so it can be captured in a CUDA graph
(:meth:`capture` / :meth:`replay`) and replayed after the coefficients change
(:meth:`set_coefficients`).  Each pair's result equals
``lhs.matmul(rhs, simplify=True)`` (or the fused path's cull at 1e-12) bit for
bit.  torch supplies device memory and the current stream only.
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np
import torch

from . import capi

__all__ = ["ProductsBatch"]


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _operand(op, dev) -> tuple[int, torch.Tensor, torch.Tensor, torch.Tensor]:
    """(n, x int64 (T, W), z int64 (T, W), c complex128 (T,)) device tensors."""
    from . import PauliSum

    if isinstance(op, PauliSum):
        n = op.num_qubits
        x, z, c = op._packed()
    else:
        n, x, z, c = op

    def u64(a):
        if isinstance(a, torch.Tensor):
            return a.to(device=dev, dtype=torch.int64).contiguous()
        a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64))
        return torch.from_numpy(a.view(np.int64)).to(dev)

    ct = c if isinstance(c, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(np.asarray(c, np.complex128)))
    return int(n), u64(x), u64(z), ct.to(device=dev, dtype=torch.complex128).contiguous()


class ProductsBatch:
    """Simplified products of many operator pairs of uneven sizes.

    ``pairs`` is a sequence of ``(lhs, rhs)``; an operand is a ``PauliSum`` or
    a tuple ``(num_qubits, x, z, coeffs)`` of packed arrays or tensors.  All
    operands share one qubit count.  ``mode`` is ``"simplify"``
    (simplify(atol, rtol) per pair, the reference's non-fused path) or
    ``"fused"`` (cull at 1e-12, the reference's fused hash path).
    """

    def __init__(self, pairs: Sequence, mode: str = "simplify", atol: float = 1e-12, rtol: float = 0.0,
                 device: int | None = None) -> None:
        if mode not in ("simplify", "fused"):
            raise ValueError("mode must be 'simplify' or 'fused'")
        self.device = torch.cuda.current_device() if device is None else device
        dev = torch.device("cuda", self.device)
        ops = [(_operand(a, dev), _operand(b, dev)) for a, b in pairs]
        ns = {o[0] for ab in ops for o in ab}
        if len(ns) > 1:
            raise ValueError("every operand of a product batch needs the same num_qubits")
        self.num_qubits = ns.pop() if ns else 0
        self.words = 0 if self.num_qubits == 0 else (self.num_qubits + 63) // 64
        self._ops = ops  # the masks and coefficient buffers the batch reads
        n = len(ops)
        self.n_pairs = n
        P = ctypes.c_void_p * max(n, 1)
        S = ctypes.c_size_t * max(n, 1)

        def ptrs(k):
            return P(*[(ab[k // 3][1 + k % 3].data_ptr() if ab[k // 3][1 + k % 3].numel() else None) for ab in ops])

        lx, lz, lc, rx, rz, rc = (ptrs(k) for k in range(6))
        self.sizes = [(ab[0][3].numel(), ab[1][3].numel()) for ab in ops]
        nl = S(*[a for a, _ in self.sizes])
        nr = S(*[b for _, b in self.sizes])
        self.handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            capi.call("wg_products_batch_create", self.device, self.words, n, lx, lz, lc, nl, rx, rz, rc, nr,
                      capi.WG_PRODUCTS_SIMPLIFY if mode == "simplify" else capi.WG_PRODUCTS_FUSED, float(atol),
                      float(rtol), ctypes.byref(self.handle), _stream())
        cnt = ctypes.c_void_p()
        capi.call("wg_products_batch_counts", self.handle, ctypes.byref(cnt))
        self._counts_ptr = cnt.value
        np_, nk = ctypes.c_size_t(), ctypes.c_size_t()
        capi.call("wg_products_batch_info", self.handle, ctypes.byref(np_), ctypes.byref(nk))
        self.n_products, self.n_keys = np_.value, nk.value
        self.graph = None

    # ------------------------------------------------------------------ runs
    def run(self) -> None:
        """Enqueue one evaluation of every pair on the current stream."""
        capi.call("wg_products_batch_run", self.handle, _stream())

    def capture(self) -> None:
        """Record one run in a CUDA graph (after a warm-up run)."""
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.run()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.run()

    def replay(self) -> None:
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def set_coefficients(self, pair: int, lhs=None, rhs=None) -> None:
        """Overwrite pair ``pair``'s coefficient buffers in place (same term counts),
        ordered on the current stream; the next run or replay uses them."""
        for side, new in ((0, lhs), (1, rhs)):
            if new is None:
                continue
            buf = self._ops[pair][side][3]
            t = new if isinstance(new, torch.Tensor) else torch.from_numpy(np.asarray(new, np.complex128))
            if t.numel() != buf.numel():
                raise ValueError("coefficient count must match the operand's term count")
            buf.copy_(t.to(device=buf.device, dtype=torch.complex128).reshape(buf.shape))

    # --------------------------------------------------------------- results
    def counts(self) -> np.ndarray:
        """Term count of every pair's last result (synchronises the current stream)."""
        out = np.zeros(max(self.n_pairs, 1), np.uint64)
        torch.cuda.current_stream().synchronize()
        capi.call("wg_memcpy_dtoh", self.device, out.ctypes.data, self._counts_ptr, 8 * self.n_pairs, None)
        return out[: self.n_pairs]

    def result(self, pair: int, count: int | None = None):
        """Pair ``pair``'s last result as host arrays (x, z uint64 (U, W), c complex128 (U,))."""
        U = int(self.counts()[pair]) if count is None else int(count)
        x, z, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        cap = ctypes.c_size_t()
        capi.call("wg_products_batch_result", self.handle, pair, ctypes.byref(x), ctypes.byref(z), ctypes.byref(c),
                  ctypes.byref(cap))
        W = self.words
        hx = np.zeros((U, W), np.uint64)
        hz = np.zeros((U, W), np.uint64)
        hc = np.zeros(U, np.complex128)
        if U:
            if W:
                capi.call("wg_memcpy_dtoh", self.device, hx.ctypes.data, x.value, hx.nbytes, None)
                capi.call("wg_memcpy_dtoh", self.device, hz.ctypes.data, z.value, hz.nbytes, None)
            capi.call("wg_memcpy_dtoh", self.device, hc.ctypes.data, c.value, hc.nbytes, None)
        return hx, hz, hc

    def results(self) -> list:
        cnt = self.counts()
        return [self.result(p, int(cnt[p])) for p in range(self.n_pairs)]

    def close(self) -> None:
        self.graph = None
        if getattr(self, "handle", None) is not None and self.handle.value:
            capi.lib().wg_products_batch_destroy(self.handle)
        self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass
