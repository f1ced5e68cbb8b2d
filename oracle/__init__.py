"""TEST INFRASTRUCTURE ONLY: ctypes loaders for the checkers.

* ``Oracle`` wraps ``_build/liboracle.so``, the scalar C++ restatement of the
  reference semantics (``oracle.cpp``).
* ``Reference`` wraps ``_ref/libwgref.so``, the reference's own CPU core compiled
  from its sources by ``Makefile`` (when the reference checkout was available
  at build time; the prebuilt library travels with the repository snapshot).
* ``ReferenceGPU`` wraps ``_ref/libwgref_cuda.so``, the reference's own CUDA
  path (src/cuda/*.cu built for sm_100a) with its CPU core, for timing it on
  the same GPU; it defines the reference's DevicePauliSum, so it is never
  loaded into a process that loads this repository's C++ layer.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline /
reference arm may import this package.  The product (``wolfgang_b200``) never
does.

Operators are passed as ``(n, x, z, c)``: ``x`` and ``z`` are uint64 arrays of
shape ``(T, words)``, ``c`` is complex128 of shape ``(T,)``.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libwgref.so"
REF_GPU_SO = HERE / "_ref" / "libwgref_cuda.so"

_sz = ctypes.c_size_t
_p = ctypes.c_void_p


def build() -> None:
    """Compile the oracle (and the reference core when its sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)


def _ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    return a.ctypes.data


def words_for(n: int) -> int:
    return 0 if n == 0 else (n + 63) // 64


def _u64(a, T: int, w: int) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64).reshape(T, w))


def _c128(c, T: int) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(c, dtype=np.complex128).reshape(T))


class OracleError(ValueError):
    pass


class Oracle:
    """Scalar restatement of the reference semantics (see oracle.h)."""

    def __init__(self, path: Path = ORACLE_SO) -> None:
        if not path.exists():
            build()
        self.lib = ctypes.CDLL(str(path))
        self.lib.or_last_error.restype = ctypes.c_char_p
        self.lib.or_abs.restype = ctypes.c_double
        self.lib.or_abs.argtypes = [ctypes.c_double, ctypes.c_double]

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise OracleError(self.lib.or_last_error().decode())

    def abs(self, re: float, im: float) -> float:
        return self.lib.or_abs(re, im)

    def simplify(self, n, x, z, c, atol=1e-12, rtol=0.0):
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        ox = np.zeros((T, w), np.uint64)
        oz = np.zeros((T, w), np.uint64)
        oc = np.zeros(T, np.complex128)
        out = _sz(0)
        self._check(self.lib.or_simplify(_sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                         ctypes.c_double(atol), ctypes.c_double(rtol),
                                         _p(_ptr(ox)), _p(_ptr(oz)), _p(_ptr(oc)), ctypes.byref(out)))
        u = out.value
        return ox[:u].copy(), oz[:u].copy(), oc[:u].copy()

    def matmul(self, n, lhs, rhs, simplify=True):
        lx, lz, lc = lhs
        rx, rz, rc = rhs
        w = words_for(n)
        nl, nr = len(lc), len(rc)
        lx, lz, lc = _u64(lx, nl, w), _u64(lz, nl, w), _c128(lc, nl)
        rx, rz, rc = _u64(rx, nr, w), _u64(rz, nr, w), _c128(rc, nr)
        P = nl * nr
        ox = np.zeros((P, w), np.uint64)
        oz = np.zeros((P, w), np.uint64)
        oc = np.zeros(P, np.complex128)
        out = _sz(0)
        self._check(self.lib.or_matmul(_sz(nl), _sz(nr), _sz(w), _p(_ptr(lx)), _p(_ptr(lz)), _p(_ptr(lc)),
                                       _p(_ptr(rx)), _p(_ptr(rz)), _p(_ptr(rc)), ctypes.c_int(int(simplify)),
                                       _p(_ptr(ox)), _p(_ptr(oz)), _p(_ptr(oc)), ctypes.byref(out)))
        u = out.value
        return ox[:u].copy(), oz[:u].copy(), oc[:u].copy()

    def matmul_keyrange(self, n, lhs, rhs, key_lo, key_hi, fused_threshold=False, cap=None):
        lx, lz, lc = lhs
        rx, rz, rc = rhs
        w = words_for(n)
        nl, nr = len(lc), len(rc)
        lx, lz, lc = _u64(lx, nl, w), _u64(lz, nl, w), _c128(lc, nl)
        rx, rz, rc = _u64(rx, nr, w), _u64(rz, nr, w), _c128(rc, nr)
        klo = np.ascontiguousarray(np.asarray(key_lo, np.uint64).reshape(2 * w))
        khi = np.ascontiguousarray(np.asarray(key_hi, np.uint64).reshape(2 * w))
        cap = cap if cap is not None else 1 << 22
        ox = np.zeros((cap, w), np.uint64)
        oz = np.zeros((cap, w), np.uint64)
        oc = np.zeros(cap, np.complex128)
        out = _sz(0)
        self._check(self.lib.or_matmul_keyrange(
            _sz(nl), _sz(nr), _sz(w), _p(_ptr(lx)), _p(_ptr(lz)), _p(_ptr(lc)),
            _p(_ptr(rx)), _p(_ptr(rz)), _p(_ptr(rc)), _p(_ptr(klo)), _p(_ptr(khi)),
            ctypes.c_int(int(fused_threshold)), _sz(cap), _p(_ptr(ox)), _p(_ptr(oz)), _p(_ptr(oc)),
            ctypes.byref(out)))
        u = out.value
        return ox[:u].copy(), oz[:u].copy(), oc[:u].copy()

    def matmul_uses_fused_path(self, n, lhs, rhs, simplify=True) -> bool:
        w = words_for(n)
        lx, lz, lc = lhs
        rx, rz, rc = rhs
        nl, nr = len(lc), len(rc)
        lx, lz = _u64(lx, nl, w), _u64(lz, nl, w)
        rx, rz = _u64(rx, nr, w), _u64(rz, nr, w)
        return bool(self.lib.or_matmul_uses_fused_path(_sz(nl), _sz(nr), _sz(w), _p(_ptr(lx)), _p(_ptr(lz)),
                                                       _p(_ptr(rx)), _p(_ptr(rz)), ctypes.c_int(int(simplify))))

    def commutes(self, n, lhs, rhs) -> np.ndarray:
        w = words_for(n)
        lx, lz = lhs[0], lhs[1]
        rx, rz = rhs[0], rhs[1]
        nl, nr = len(lx), len(rx)
        lx, lz = _u64(lx, nl, w), _u64(lz, nl, w)
        rx, rz = _u64(rx, nr, w), _u64(rz, nr, w)
        out = np.zeros(nl * nr, np.uint8)
        self._check(self.lib.or_commutes(_sz(nl), _sz(nr), _sz(w), _p(_ptr(lx)), _p(_ptr(lz)),
                                         _p(_ptr(rx)), _p(_ptr(rz)), _p(_ptr(out))))
        return out.reshape(nl, nr)

    def group_commuting(self, n, x, z, mode="qwc") -> list[list[int]]:
        T = len(x)
        w = words_for(n)
        x, z = _u64(x, T, w), _u64(z, T, w)
        order = np.zeros(max(T, 1), np.uintp)
        sizes = np.zeros(max(T, 1), np.uintp)
        ng = _sz(0)
        self._check(self.lib.or_group_commuting(_sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)),
                                                ctypes.c_int(1 if mode == "full" else 0),
                                                _p(_ptr(order)), _p(_ptr(sizes)), ctypes.byref(ng)))
        groups, p = [], 0
        for g in range(ng.value):
            s = int(sizes[g])
            groups.append([int(v) for v in order[p:p + s]])
            p += s
        return groups

    def expectation(self, n, x, z, c, psi) -> complex:
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        psi = np.ascontiguousarray(psi)
        dtype = 0 if psi.dtype == np.complex128 else 1
        out = np.zeros(2, np.float64)
        self._check(self.lib.or_expectation(_sz(T), _sz(n), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                            _p(_ptr(psi)), ctypes.c_int(dtype), _p(_ptr(out))))
        return complex(out[0], out[1])

    def term_expectations(self, n, x, z, psi) -> np.ndarray:
        T = len(x)
        w = words_for(n)
        x, z = _u64(x, T, w), _u64(z, T, w)
        psi = np.ascontiguousarray(psi)
        dtype = 0 if psi.dtype == np.complex128 else 1
        out = np.zeros(T, np.float64)
        self._check(self.lib.or_term_expectations(_sz(T), _sz(n), _p(_ptr(x)), _p(_ptr(z)),
                                                  _p(_ptr(psi)), ctypes.c_int(dtype), _p(_ptr(out))))
        return out

    def hpsi(self, n, x, z, c, psi) -> np.ndarray:
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        out = np.zeros(1 << n, np.complex128)
        self._check(self.lib.or_hpsi(_sz(T), _sz(n), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                     _p(_ptr(psi)), _p(_ptr(out))))
        return out

    def hpsi_at(self, n, x, z, c, psi, idx) -> np.ndarray:
        """(H psi)[idx] (complex128), the or_hpsi sum at the listed amplitudes only."""
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        idx = np.ascontiguousarray(np.asarray(idx, np.uint64))
        out = np.zeros(len(idx), np.complex128)
        self._check(self.lib.or_hpsi_at(_sz(T), _sz(n), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)), _p(_ptr(psi)),
                                        _sz(len(idx)), _p(_ptr(idx)), _p(_ptr(out))))
        return out

    def expectation_z_counts(self, n, x, z, c, packed, counts) -> complex:
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        rows = len(counts)
        packed = np.ascontiguousarray(np.asarray(packed, np.uint64).reshape(rows, w))
        counts = np.ascontiguousarray(np.asarray(counts, np.float64))
        out = np.zeros(2, np.float64)
        self._check(self.lib.or_expectation_z_counts(_sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                                     _sz(rows), _p(_ptr(packed)), _p(_ptr(counts)),
                                                     _p(_ptr(out))))
        return complex(out[0], out[1])


class Reference:
    """The reference's own CPU core (compiled from its sources), via ref_shim.cpp."""

    def __init__(self, path: Path = REF_SO) -> None:
        if not path.exists():
            raise FileNotFoundError(f"{path} was not built (reference sources unavailable)")
        self.lib = ctypes.CDLL(str(path), mode=os.RTLD_LOCAL)
        self.lib.wgref_last_error.restype = ctypes.c_char_p

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise OracleError(self.lib.wgref_last_error().decode())

    def simplify(self, n, x, z, c, atol=1e-12, rtol=0.0):
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        ox = np.zeros((max(T, 1), w), np.uint64)
        oz = np.zeros((max(T, 1), w), np.uint64)
        oc = np.zeros(max(T, 1), np.complex128)
        out = _sz(0)
        self._check(self.lib.wgref_simplify(_sz(n), _sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                            ctypes.c_double(atol), ctypes.c_double(rtol),
                                            _p(_ptr(ox)), _p(_ptr(oz)), _p(_ptr(oc)), ctypes.byref(out)))
        u = out.value
        return ox[:u].copy(), oz[:u].copy(), oc[:u].copy()

    def matmul(self, n, lhs, rhs, simplify=True, max_intermediate_terms=50_000_000):
        lx, lz, lc = lhs
        rx, rz, rc = rhs
        w = words_for(n)
        nl, nr = len(lc), len(rc)
        lx, lz, lc = _u64(lx, nl, w), _u64(lz, nl, w), _c128(lc, nl)
        rx, rz, rc = _u64(rx, nr, w), _u64(rz, nr, w), _c128(rc, nr)
        P = max(nl * nr, 1)
        ox = np.zeros((P, w), np.uint64)
        oz = np.zeros((P, w), np.uint64)
        oc = np.zeros(P, np.complex128)
        out = _sz(0)
        self._check(self.lib.wgref_matmul(_sz(n), _sz(nl), _sz(nr), _sz(w), _p(_ptr(lx)), _p(_ptr(lz)),
                                          _p(_ptr(lc)), _p(_ptr(rx)), _p(_ptr(rz)), _p(_ptr(rc)),
                                          ctypes.c_int(int(simplify)), _sz(max_intermediate_terms),
                                          _p(_ptr(ox)), _p(_ptr(oz)), _p(_ptr(oc)), ctypes.byref(out)))
        u = out.value
        return ox[:u].copy(), oz[:u].copy(), oc[:u].copy()

    def commutes(self, n, lhs, rhs, max_entries=None) -> np.ndarray:
        w = words_for(n)
        lx, lz = lhs[0], lhs[1]
        rx, rz = rhs[0], rhs[1]
        nl, nr = len(lx), len(rx)
        lx, lz = _u64(lx, nl, w), _u64(lz, nl, w)
        rx, rz = _u64(rx, nr, w), _u64(rz, nr, w)
        out = np.zeros(max(nl * nr, 1), np.uint8)
        me = max_entries if max_entries is not None else nl * nr
        self._check(self.lib.wgref_commutes(_sz(n), _sz(nl), _sz(nr), _sz(w), _p(_ptr(lx)), _p(_ptr(lz)),
                                            _p(_ptr(rx)), _p(_ptr(rz)), _sz(me), _p(_ptr(out))))
        return out[: nl * nr].reshape(nl, nr)

    def group_commuting(self, n, x, z, c, mode="qwc", max_terms_for_graph=50000):
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        ox = np.zeros((max(T, 1), w), np.uint64)
        oz = np.zeros((max(T, 1), w), np.uint64)
        oc = np.zeros(max(T, 1), np.complex128)
        sizes = np.zeros(max(T, 1), np.uintp)
        ng = _sz(0)
        self._check(self.lib.wgref_group_commuting(_sz(n), _sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                                   ctypes.c_int(1 if mode == "full" else 0),
                                                   _sz(max_terms_for_graph), _p(_ptr(ox)), _p(_ptr(oz)),
                                                   _p(_ptr(oc)), _p(_ptr(sizes)), ctypes.byref(ng)))
        groups, p = [], 0
        for g in range(ng.value):
            s = int(sizes[g])
            groups.append((ox[p:p + s].copy(), oz[p:p + s].copy(), oc[p:p + s].copy()))
            p += s
        return groups

    def expectation(self, n, x, z, c, psi) -> complex:
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        psi = np.ascontiguousarray(psi)
        dtype = 0 if psi.dtype == np.complex128 else 1
        out = np.zeros(2, np.float64)
        self._check(self.lib.wgref_expectation(_sz(n), _sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                               _p(_ptr(psi)), ctypes.c_int(dtype), _p(_ptr(out))))
        return complex(out[0], out[1])

    def expectation_z_counts(self, n, x, z, c, packed, counts) -> complex:
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        rows = len(counts)
        packed = np.ascontiguousarray(np.asarray(packed, np.uint64).reshape(rows, w))
        counts = np.ascontiguousarray(np.asarray(counts, np.float64))
        out = np.zeros(2, np.float64)
        self._check(self.lib.wgref_expectation_z_counts(_sz(n), _sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)),
                                                        _p(_ptr(c)), _sz(rows), _p(_ptr(packed)),
                                                        _p(_ptr(counts)), _p(_ptr(out))))
        return complex(out[0], out[1])

    def cpu_backend(self) -> str:
        buf = ctypes.create_string_buffer(512)
        self._check(self.lib.wgref_cpu_backend(buf, _sz(512)))
        return buf.value.decode()


class ReferenceGPU:
    """The reference's DevicePauliSum path on the GPU (ref_gpu_shim.cpp).

    Every method uploads the operands once, makes `warmup` untimed and `reps`
    timed calls of the reference's stock device-resident operation (each call
    synchronises before it returns) and returns (mean ms per call, result)."""

    def __init__(self, path: Path = REF_GPU_SO) -> None:
        if not path.exists():
            raise FileNotFoundError(f"{path} was not built (reference sources unavailable)")
        self.lib = ctypes.CDLL(str(path), mode=os.RTLD_LOCAL)
        self.lib.wgrefgpu_last_error.restype = ctypes.c_char_p

    @staticmethod
    def available() -> bool:
        return REF_GPU_SO.exists()

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise OracleError(self.lib.wgrefgpu_last_error().decode())

    def matmul(self, n, lhs, rhs, simplify=True, max_intermediate_terms=50_000_000, warmup=1, reps=3):
        lx, lz, lc = lhs
        rx, rz, rc = rhs
        w = words_for(n)
        nl, nr = len(lc), len(rc)
        lx, lz, lc = _u64(lx, nl, w), _u64(lz, nl, w), _c128(lc, nl)
        rx, rz, rc = _u64(rx, nr, w), _u64(rz, nr, w), _c128(rc, nr)
        ms, terms = ctypes.c_double(), _sz()
        self._check(self.lib.wgrefgpu_matmul(_sz(n), _sz(nl), _sz(nr), _sz(w), _p(_ptr(lx)), _p(_ptr(lz)),
                                             _p(_ptr(lc)), _p(_ptr(rx)), _p(_ptr(rz)), _p(_ptr(rc)),
                                             ctypes.c_int(int(simplify)), _sz(max_intermediate_terms),
                                             ctypes.c_int(warmup), ctypes.c_int(reps), ctypes.byref(ms),
                                             ctypes.byref(terms)))
        return ms.value, terms.value

    def simplify(self, n, x, z, c, atol=1e-12, rtol=0.0, warmup=1, reps=3):
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        ms, terms = ctypes.c_double(), _sz()
        self._check(self.lib.wgrefgpu_simplify(_sz(n), _sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                               ctypes.c_double(atol), ctypes.c_double(rtol), ctypes.c_int(warmup),
                                               ctypes.c_int(reps), ctypes.byref(ms), ctypes.byref(terms)))
        return ms.value, terms.value

    def commutes_device(self, n, lhs, rhs, warmup=1, reps=3):
        w = words_for(n)
        lx, lz = lhs[0], lhs[1]
        rx, rz = rhs[0], rhs[1]
        nl, nr = len(lx), len(rx)
        lx, lz = _u64(lx, nl, w), _u64(lz, nl, w)
        rx, rz = _u64(rx, nr, w), _u64(rz, nr, w)
        ms, count = ctypes.c_double(), ctypes.c_uint64()
        self._check(self.lib.wgrefgpu_commutes_device(_sz(n), _sz(nl), _sz(nr), _sz(w), _p(_ptr(lx)), _p(_ptr(lz)),
                                                      _p(_ptr(rx)), _p(_ptr(rz)), _sz(nl * nr), ctypes.c_int(warmup),
                                                      ctypes.c_int(reps), ctypes.byref(ms), ctypes.byref(count)))
        return ms.value, count.value

    def expectation(self, n, x, z, c, psi, warmup=1, reps=3):
        T = len(c)
        w = words_for(n)
        x, z, c = _u64(x, T, w), _u64(z, T, w), _c128(c, T)
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        ms = ctypes.c_double()
        out = np.zeros(2, np.float64)
        self._check(self.lib.wgrefgpu_expectation(_sz(n), _sz(T), _sz(w), _p(_ptr(x)), _p(_ptr(z)), _p(_ptr(c)),
                                                  _p(_ptr(psi)), ctypes.c_int(warmup), ctypes.c_int(reps),
                                                  ctypes.byref(ms), _p(_ptr(out))))
        return ms.value, complex(out[0], out[1])
