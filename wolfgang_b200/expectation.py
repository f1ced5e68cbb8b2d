"""Statevector expectation on the B200: plans, autograd, batches and CUDA graphs.

Everything here calls the wg_* C-ABI (``capi``); torch provides device memory,
the current stream and autograd.  No torch type crosses the C-ABI.

* :class:`ExpectationPlan` -- one operator's x-grouping, built once on the
  device and reused for any number of statevectors (complex128, or complex64
  storage with FP64 accumulation).
* :func:`expectation` -- differentiable E = <psi|H|psi> for Hermitian H (real
  coefficients): backward gives dE/dc_k = <psi|P_k|psi> and dE/dpsi* = H psi,
  both produced by the same device pass as E.
* :class:`ExpectationBatch` -- many (H, psi) pairs of uneven sizes in one
  persistent launch (a device work queue over (pair, x-group, chunk) items),
  optionally captured in a CUDA graph and replayed.
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np
import torch

from . import capi

__all__ = ["ExpectationPlan", "ExpectationBatch", "expectation"]


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _device_u64(a, device) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.int64).contiguous()
    a = np.ascontiguousarray(np.asarray(a, dtype=np.uint64))
    return torch.from_numpy(a.view(np.int64)).to(device)


def _dtype_code(psi: torch.Tensor) -> int:
    if psi.dtype == torch.complex128:
        return capi.WG_DTYPE_C128
    if psi.dtype == torch.complex64:
        return capi.WG_DTYPE_C64
    raise TypeError("psi dtype must be complex64 or complex128")


class ExpectationPlan:
    """Device x-grouping of one operator (wg_expect_plan_t).

    ``op`` is a ``DevicePauliSum``, a ``PauliSum``, or a tuple
    ``(num_qubits, x, z, coeffs)`` of packed arrays / tensors (x, z uint64 with
    shape (T, words), coeffs complex128 (T,)).  num_qubits <= 63.
    """

    def __init__(self, op, device: int | None = None) -> None:
        from . import DevicePauliSum, PauliSum

        self.device = torch.cuda.current_device() if device is None else device
        dev = torch.device("cuda", self.device)
        self._keep = []
        if isinstance(op, DevicePauliSum):
            self.n, self.T = op.num_qubits, op.num_terms
            xp, zp, cp = op._pointers
            self._keep.append(op)
            if op.device != self.device:
                raise ValueError("DevicePauliSum lives on another device")
        else:
            if isinstance(op, PauliSum):
                n = op.num_qubits
                x, z, c = op._packed()
            else:
                n, x, z, c = op
            self.n = int(n)
            xt, zt = _device_u64(x, dev), _device_u64(z, dev)
            ct = torch.as_tensor(np.asarray(c, np.complex128) if not isinstance(c, torch.Tensor) else c,
                                 dtype=torch.complex128).to(dev).contiguous()
            self.T = int(ct.numel())
            self._keep += [xt, zt, ct]
            xp, zp, cp = xt.data_ptr(), zt.data_ptr(), ct.data_ptr()
        self.handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            capi.call("wg_expect_plan_create", self.device, self.n, self.T, xp or None, zp or None, cp or None,
                      ctypes.byref(self.handle), _stream())
        ng, nt = ctypes.c_size_t(), ctypes.c_size_t()
        capi.call("wg_expect_plan_info", self.handle, ctypes.byref(ng), ctypes.byref(nt))
        self.n_groups = ng.value

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            capi.lib().wg_expect_plan_destroy(self.handle)
        self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def set_coefficients(self, coeffs: torch.Tensor) -> None:
        """Replace the coefficients (same terms, original order) in place."""
        c = coeffs.to(device=f"cuda:{self.device}", dtype=torch.complex128).contiguous()
        if c.numel() != self.T:
            raise ValueError("coefficient count must match the plan's term count")
        capi.call("wg_expect_plan_set_coeffs", self.handle, c.data_ptr(), _stream())
        self._coeff_tensor = c  # keep alive until the copy has run

    def run(self, psi: torch.Tensor, terms: bool = False, hpsi: bool = False):
        """Returns (E complex128 tensor [2], e_k float64 [T] or None, H psi complex128 or None)."""
        psi = psi.contiguous()
        if psi.dim() != 1 or psi.numel() != (1 << self.n):
            raise ValueError("expectation_statevector requires len(psi) == 2 ** num_qubits")
        dev = psi.device
        res = torch.empty(2, dtype=torch.float64, device=dev)
        ev = torch.empty(max(self.T, 1), dtype=torch.float64, device=dev) if terms else None
        hp = torch.empty(1 << self.n, dtype=torch.complex128, device=dev) if hpsi else None
        capi.call("wg_expect_plan_run", self.handle, psi.data_ptr(), _dtype_code(psi), res.data_ptr(),
                  ev.data_ptr() if ev is not None else None, hp.data_ptr() if hp is not None else None, _stream())
        return res, (ev[: self.T] if ev is not None else None), hp


class _ExpectationFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coeffs, psi, plan):
        plan.set_coefficients(coeffs.detach())
        need_c = ctx.needs_input_grad[0]
        need_psi = ctx.needs_input_grad[1]
        res, ev, hp = plan.run(psi.detach(), terms=need_c, hpsi=need_psi)
        ctx.save_for_backward(ev if ev is not None else torch.empty(0), hp if hp is not None else torch.empty(0))
        ctx.psi_dtype = psi.dtype
        return res[0].clone()

    @staticmethod
    def backward(ctx, grad):
        ev, hp = ctx.saved_tensors
        gc = grad * ev if ctx.needs_input_grad[0] else None
        # E = <psi|H|psi> is real for Hermitian H; torch's convention for a real
        # loss L of complex z is grad = 2 dL/dz*, here 2 H psi.
        gpsi = (2.0 * grad * hp).to(ctx.psi_dtype) if ctx.needs_input_grad[1] else None
        return gc, gpsi, None


def expectation(plan: ExpectationPlan, coeffs: torch.Tensor, psi: torch.Tensor) -> torch.Tensor:
    """Differentiable <psi|H|psi> for H = sum_k coeffs[k] P_k (real coefficients).

    ``coeffs`` is a real float64 tensor of the plan's term count; ``psi`` a
    complex128 or complex64 tensor of length 2^n on the plan's device.
    """
    if coeffs.is_complex():
        raise TypeError("differentiable expectation needs real (Hermitian) coefficients")
    return _ExpectationFn.apply(coeffs, psi, plan)


class ExpectationBatch:
    """Many (plan, psi) pairs evaluated by one persistent launch.

    Outputs are preallocated device tensors: ``values`` (n_pairs, 2) float64,
    ``term_values[i]`` (T_i,) float64 and, with ``gradients=True``,
    ``hpsi[i]`` (2^n_i,) complex128.  :meth:`run` enqueues the kernels on the
    current stream; :meth:`capture` records them in a CUDA graph that
    :meth:`replay` re-launches with no host work.
    """

    def __init__(self, plans: Sequence[ExpectationPlan], psis: Sequence[torch.Tensor], gradients: bool = True):
        if len(plans) != len(psis) or not plans:
            raise ValueError("plans and psis must be non-empty and of equal length")
        self.plans = list(plans)
        self.psis = [p.contiguous() for p in psis]
        dtypes = {p.dtype for p in self.psis}
        if len(dtypes) != 1:
            raise TypeError("all statevectors of a batch share one dtype")
        self.dtype = _dtype_code(self.psis[0])
        dev = self.psis[0].device
        self.device = dev.index
        n = len(plans)
        self.values = torch.zeros(n, 2, dtype=torch.float64, device=dev)
        self.term_values = [torch.zeros(max(p.T, 1), dtype=torch.float64, device=dev) for p in plans]
        self.hpsi = [torch.zeros(1 << p.n, dtype=torch.complex128, device=dev) for p in plans] if gradients else None
        P = ctypes.c_void_p * n
        self._plans = P(*[p.handle.value for p in plans])
        self._psis = P(*[t.data_ptr() for t in self.psis])
        self._res = P(*[self.values[i].data_ptr() for i in range(n)])
        self._ev = P(*[t.data_ptr() for t in self.term_values])
        self._hp = P(*[t.data_ptr() for t in self.hpsi]) if gradients else None
        self.handle = ctypes.c_void_p()
        capi.call("wg_expect_batch_create", self.device, n, self._plans, self._psis, self.dtype, self._res, self._ev,
                  self._hp, ctypes.byref(self.handle), _stream())
        self.graph = None

    def run(self) -> None:
        capi.call("wg_expect_batch_run", self.handle, _stream())

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

    def close(self) -> None:
        self.graph = None
        if getattr(self, "handle", None) is not None and self.handle.value:
            capi.lib().wg_expect_batch_destroy(self.handle)
        self.handle = None

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass
