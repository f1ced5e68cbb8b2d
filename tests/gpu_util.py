"""Helpers for GPU tests: device buffers (torch-owned) and C-ABI calls."""

from __future__ import annotations

import ctypes

import numpy as np

from wolfgang_b200 import capi


def torch():
    import torch as _t

    return _t


def dev(a: np.ndarray):
    """numpy -> CUDA tensor with the same bytes (uint64/complex kept bitwise)."""
    t = torch()
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint64:
        return t.from_numpy(a.view(np.int64)).cuda()
    if a.dtype == np.uint32:
        return t.from_numpy(a.view(np.int32)).cuda()
    return t.from_numpy(a).cuda()


def host_u64(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


def ptr(t) -> int | None:
    return t.data_ptr() if t is not None and t.numel() > 0 else None


def operator_on_device(x, z, c):
    return dev(x), dev(z), dev(c)


def commutation_bits(n, A, B, algo=0, pitch=None):
    t = torch()
    w = 0 if n == 0 else (n + 63) // 64
    ax, az = dev(A[0]), dev(A[1])
    bx, bz = dev(B[0]), dev(B[1])
    nl, nr = len(A[0]), len(B[0])
    pitch = pitch or (nr + 31) // 32
    bits = t.full((max(nl * pitch, 1),), -1, dtype=t.int32, device="cuda")
    capi.call("wg_commutation_bits", 0, w, ptr(ax), ptr(az), nl, ptr(bx), ptr(bz), nr, ptr(bits), pitch, algo, None)
    t.cuda.synchronize()
    return bits.cpu().numpy().view(np.uint32)[: nl * pitch].reshape(nl, pitch)


def unpack_bits(bits: np.ndarray, cols: int) -> np.ndarray:
    rows = bits.shape[0]
    as_bytes = bits.view(np.uint8).reshape(rows, -1)
    flags = np.unpackbits(as_bytes, axis=1, bitorder="little")
    return flags[:, :cols]


def _take_outputs(n_words, ox, oz, oc, U):
    """Copy library-allocated outputs to host and free them."""
    x = np.zeros((U, n_words), np.uint64)
    z = np.zeros((U, n_words), np.uint64)
    c = np.zeros(U, np.complex128)
    L = capi.lib()
    if U:
        if n_words:
            capi.check(L.wg_memcpy_dtoh(0, x.ctypes.data, ox, x.nbytes, None))
            capi.check(L.wg_memcpy_dtoh(0, z.ctypes.data, oz, z.nbytes, None))
        capi.check(L.wg_memcpy_dtoh(0, c.ctypes.data, oc, c.nbytes, None))
    for p in (ox, oz, oc):
        if p:
            capi.check(L.wg_free(0, p, None))
    return x, z, c


def simplify(n, x, z, c, atol=1e-12, rtol=0.0):
    w = 0 if n == 0 else (n + 63) // 64
    dx, dz, dc = operator_on_device(x, z, c)
    ox, oz, oc = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    U = ctypes.c_size_t()
    capi.call("wg_simplify", 0, w, len(c), ptr(dx), ptr(dz), ptr(dc), atol, rtol, ctypes.byref(ox),
              ctypes.byref(oz), ctypes.byref(oc), ctypes.byref(U), None)
    return _take_outputs(w, ox.value, oz.value, oc.value, U.value)


def products(n, A, B, mode=capi.WG_PRODUCTS_SIMPLIFY, atol=1e-12, rtol=0.0):
    w = 0 if n == 0 else (n + 63) // 64
    ax, az, ac = operator_on_device(*A)
    bx, bz, bc = operator_on_device(*B)
    ox, oz, oc = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    U = ctypes.c_size_t()
    capi.call("wg_pauli_products", 0, w, ptr(ax), ptr(az), ptr(ac), len(A[2]), ptr(bx), ptr(bz), ptr(bc), len(B[2]),
              mode, atol, rtol, ctypes.byref(ox), ctypes.byref(oz), ctypes.byref(oc), ctypes.byref(U), None)
    return _take_outputs(w, ox.value, oz.value, oc.value, U.value)


class Plan:
    """wg_expect_plan_t owner."""

    def __init__(self, n, x, z, c):
        self.n = n
        self.T = len(c)
        self.dx, self.dz, self.dc = operator_on_device(x, z, c)
        self.h = ctypes.c_void_p()
        capi.call("wg_expect_plan_create", 0, n, self.T, ptr(self.dx), ptr(self.dz), ptr(self.dc),
                  ctypes.byref(self.h), None)

    def run(self, psi_dev, want_terms=False, want_hpsi=False):
        t = torch()
        dtype = capi.WG_DTYPE_C128 if psi_dev.dtype == t.complex128 else capi.WG_DTYPE_C64
        res = t.zeros(2, dtype=t.float64, device="cuda")
        ev = t.zeros(max(self.T, 1), dtype=t.float64, device="cuda") if want_terms else None
        hp = t.zeros(1 << self.n, dtype=t.complex128, device="cuda") if want_hpsi else None
        capi.call("wg_expect_plan_run", self.h, psi_dev.data_ptr(), dtype, res.data_ptr(),
                  ev.data_ptr() if ev is not None else None, hp.data_ptr() if hp is not None else None, None)
        t.cuda.synchronize()
        out = complex(res[0].item(), res[1].item())
        return out, (ev.cpu().numpy()[: self.T] if ev is not None else None), (hp.cpu().numpy() if hp is not None else None)

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            capi.lib().wg_expect_plan_destroy(self.h)
            self.h = None
