"""ctypes binding of the wg_* C-ABI (include/wg_pauli.h) in lib/libwgpauli.so.

This is the boundary the parity tests, the autograd wrapper and the batched
API call: plain pointers, sizes and status codes.  Device buffers come from
any CUDA allocator (torch tensors are used for that plumbing: ``tensor.data_ptr()``),
streams are ``cudaStream_t`` handles as integers (``torch.cuda.current_stream().cuda_stream``).
Status codes other than WG_OK raise: WG_ERR_INVALID -> ValueError, the others
-> RuntimeError, with the library's message.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libwgpauli.so"
HEADER = Path(__file__).resolve().parent.parent / "include" / "wg_pauli.h"

WG_OK = 0
WG_ERR_INVALID = 1
WG_ERR_OOM = 2
WG_ERR_CUDA = 3
WG_ERR_TIMEOUT = 4
WG_ERR_NO_DEVICE = 5
WG_DTYPE_C128 = 0
WG_DTYPE_C64 = 1
WG_PRODUCTS_RAW = 0
WG_PRODUCTS_SIMPLIFY = 1
WG_PRODUCTS_FUSED = 2
WG_SORT_AUTO = 0
WG_TUNE_OFF = 0
WG_TUNE_CACHED = 1
WG_TUNE_SEARCH = 2
WG_SORT_LSD = 1
WG_SORT_BUCKET = 2

_sz = ctypes.c_size_t
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_pvp = ctypes.POINTER(ctypes.c_void_p)
_psz = ctypes.POINTER(ctypes.c_size_t)

# name -> argtypes (all return int status unless listed in _RESTYPES)
_SIGNATURES: dict[str, list] = {
    "wg_last_error": [],
    "wg_abi_version": [],
    "wg_device_count": [ctypes.POINTER(_i)],
    "wg_runtime_versions": [ctypes.POINTER(_i), ctypes.POINTER(_i)],
    "wg_device_info": [_i, ctypes.c_char_p, _sz, ctypes.POINTER(_i), ctypes.POINTER(_i), _psz, ctypes.POINTER(_i)],
    "wg_malloc": [_i, _sz, _vp, _pvp],
    "wg_free": [_i, _vp, _vp],
    "wg_memcpy_htod": [_i, _vp, _vp, _sz, _vp],
    "wg_memcpy_dtoh": [_i, _vp, _vp, _sz, _vp],
    "wg_memcpy_dtod": [_i, _vp, _vp, _sz, _vp],
    "wg_memcpy_dtoh_chunked": [_i, _vp, _sz, _vp, _vp, _vp],
    "wg_memset": [_i, _vp, _i, _sz, _vp],
    "wg_stream_synchronize": [_i, _vp],
    "wg_device_synchronize": [_i],
    "wg_pointer_check": [_vp, _sz, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i)],
    "wg_inject_alloc_failure": [ctypes.c_long],
    "wg_kernel_launches": [ctypes.POINTER(ctypes.c_ulonglong)],
    "wg_profile_enable": [_i],
    "wg_profile_report": [ctypes.c_char_p, _sz],
    "wg_commutation_bits": [_i, _sz, _vp, _vp, _sz, _vp, _vp, _sz, _vp, _sz, _i, _vp],
    "wg_bits_to_u8": [_i, _vp, _sz, _sz, _sz, _vp, _vp],
    "wg_commutation_u8_noalloc": [_i, _sz, _vp, _vp, _sz, _vp, _vp, _sz, _vp, _vp],
    "wg_bits_count": [_i, _vp, _sz, _sz, _sz, _vp, _vp, ctypes.POINTER(ctypes.c_uint64), _vp],
    "wg_u8_count": [_i, _vp, _sz, _sz, _vp, _vp, ctypes.POINTER(ctypes.c_uint64), _vp],
    "wg_simplify": [_i, _sz, _sz, _vp, _vp, _vp, _d, _d, _pvp, _pvp, _pvp, _psz, _vp],
    "wg_pauli_products": [_i, _sz, _vp, _vp, _vp, _sz, _vp, _vp, _vp, _sz, _i, _d, _d, _pvp, _pvp, _pvp, _psz, _vp],
    "wg_products_batch_create": [_i, _sz, _sz, _pvp, _pvp, _pvp, _psz, _pvp, _pvp, _pvp, _psz, _i, _d, _d, _pvp,
                                 _vp],
    "wg_products_batch_run": [_vp, _vp],
    "wg_products_batch_result": [_vp, _sz, _pvp, _pvp, _pvp, _psz],
    "wg_products_batch_counts": [_vp, _pvp],
    "wg_products_batch_info": [_vp, _psz, _psz],
    "wg_products_batch_destroy": [_vp],
    "wg_autotune_set_mode": [_i],
    "wg_autotune_get_mode": [ctypes.POINTER(_i)],
    "wg_autotune_export": [ctypes.c_char_p, _sz, _psz],
    "wg_autotune_import": [ctypes.c_char_p],
    "wg_autotune_clear": [],
    "wg_set_sort_algorithm": [_i],
    "wg_last_sort_algorithm": [],
    "wg_set_bucket_fine_target": [ctypes.c_uint],
    "wg_set_bucket_one_pass": [ctypes.c_int],
    "wg_expect_plan_create": [_i, _sz, _sz, _vp, _vp, _vp, _pvp, _vp],
    "wg_expect_plan_destroy": [_vp],
    "wg_expect_plan_set_coeffs": [_vp, _vp, _vp],
    "wg_expect_plan_info": [_vp, _psz, _psz],
    "wg_expect_plan_run": [_vp, _vp, _i, _vp, _vp, _vp, _vp],
    "wg_expectation": [_i, _sz, _sz, _vp, _vp, _vp, _vp, _i, ctypes.POINTER(_d), _vp],
    "wg_expect_batched": [_i, _sz, _pvp, _pvp, _i, _pvp, _pvp, _pvp, _vp],
    "wg_expect_batch_create": [_i, _sz, _pvp, _pvp, _i, _pvp, _pvp, _pvp, _pvp, _vp],
    "wg_expect_batch_run": [_vp, _vp],
    "wg_expect_batch_destroy": [_vp],
    "wg_expectation_z_counts": [_i, _sz, _sz, _vp, _vp, _vp, _sz, _vp, _vp, ctypes.POINTER(_d), _vp],
    "wg_group_commuting": [_i, _sz, _sz, _vp, _vp, _i, _psz, _psz, _psz, _vp],
}
_RESTYPES = {"wg_last_error": ctypes.c_char_p}


class WGError(RuntimeError):
    def __init__(self, code: int, message: str) -> None:
        super().__init__(message)
        self.code = code


class WGInvalid(ValueError):
    code = WG_ERR_INVALID


_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """Load libwgpauli.so (raises if the native build is missing)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run `python wolfgang_b200/build.py`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, args in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = L
    return _lib


def check(status: int) -> None:
    if status == WG_OK:
        return
    msg = lib().wg_last_error().decode()
    if status == WG_ERR_INVALID:
        raise WGInvalid(msg)
    raise WGError(status, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def declared_functions() -> list[str]:
    """Entry points declared in include/wg_pauli.h."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(wg_\w+)\(", text, flags=re.M)))


def profile_enable(on: bool) -> None:
    check(lib().wg_profile_enable(1 if on else 0))


def profile_report() -> dict[str, tuple[int, float]]:
    """{kernel name: (launches, total ms)} since the last report."""
    buf = ctypes.create_string_buffer(1 << 16)
    check(lib().wg_profile_report(buf, len(buf)))
    out: dict[str, tuple[int, float]] = {}
    for item in buf.value.decode().split(";"):
        if item:
            name, count, ms = item.rsplit(":", 2)
            out[name] = (int(count), float(ms))
    return out


def set_sort_algorithm(algo: int) -> int:
    """Selects the sort-reduce algorithm (WG_SORT_*) process-wide; returns the previous one."""
    prev = _sort_setting[0]
    check(lib().wg_set_sort_algorithm(int(algo)))
    _sort_setting[0] = int(algo)
    return prev


def last_sort_algorithm() -> int:
    """WG_SORT_LSD or WG_SORT_BUCKET: the algorithm of this thread's last simplify / products result."""
    return int(lib().wg_last_sort_algorithm())


_sort_setting = [WG_SORT_AUTO]


def set_bucket_fine_target(items: int) -> None:
    """Target items per fine bucket of the bucketed sort (0: the default, 896); results do not change."""
    check(lib().wg_set_bucket_fine_target(int(items)))


def set_bucket_one_pass(on: bool) -> None:
    """Bucketed sort: fine partition written in one pass where memory allows (True, the default), or two."""
    check(lib().wg_set_bucket_one_pass(1 if on else 0))


def autotune_mode(mode: int | None = None) -> int:
    """Returns the autotuner mode (WG_TUNE_*); sets it first when ``mode`` is given."""
    if mode is not None:
        check(lib().wg_autotune_set_mode(int(mode)))
    m = _i(0)
    check(lib().wg_autotune_get_mode(ctypes.byref(m)))
    return m.value


def autotune_export() -> str:
    """The autotuner's cache as text, one '<op> <words> <a> <b> <choice>' line per class."""
    need = ctypes.c_size_t(0)
    check(lib().wg_autotune_export(None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(need.value + 64)
    check(lib().wg_autotune_export(buf, len(buf), ctypes.byref(need)))
    return buf.value.decode()


def autotune_import(text: str) -> None:
    check(lib().wg_autotune_import(text.encode()))


def autotune_clear() -> None:
    check(lib().wg_autotune_clear())


def kernel_launches() -> int:
    c = ctypes.c_ulonglong(0)
    check(lib().wg_kernel_launches(ctypes.byref(c)))
    return c.value


def device_count() -> int:
    c = _i(0)
    check(lib().wg_device_count(ctypes.byref(c)))
    return c.value
