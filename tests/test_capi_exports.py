"""The C-ABI library loads without a GPU and exports every declared entry point."""

from __future__ import annotations

import ctypes
import subprocess

from wolfgang_b200 import capi


def test_library_exports_every_declared_symbol():
    declared = capi.declared_functions()
    assert len(declared) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    # the ctypes table covers the whole header
    assert sorted(capi._SIGNATURES) == declared


def test_abi_calls_without_a_device():
    L = capi.lib()
    assert L.wg_abi_version() == 1
    n = ctypes.c_int(-1)
    assert L.wg_device_count(ctypes.byref(n)) == capi.WG_OK
    if n.value == 0:
        out = ctypes.c_void_p()
        rc = L.wg_malloc(0, 16, None, ctypes.byref(out))
        assert rc == capi.WG_ERR_NO_DEVICE
        assert b"no CUDA device" in L.wg_last_error()


def test_invalid_arguments_are_rejected_before_device_work():
    L = capi.lib()
    ox, oz, oc = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    u = ctypes.c_size_t()
    rc = L.wg_simplify(0, 1, 4, None, None, None, -1.0, 0.0, ctypes.byref(ox), ctypes.byref(oz),
                       ctypes.byref(oc), ctypes.byref(u), None)
    assert rc == capi.WG_ERR_INVALID and b"tolerances" in L.wg_last_error()
    rc = L.wg_pauli_products(0, 1, None, None, None, 1 << 33, None, None, None, 1 << 33, 1, 1e-12, 0.0,
                             ctypes.byref(ox), ctypes.byref(oz), ctypes.byref(oc), ctypes.byref(u), None)
    assert rc == capi.WG_ERR_INVALID
    rc = L.wg_commutation_bits(0, 1, None, None, 4, None, None, 100, None, 1, 0, None)
    assert rc == capi.WG_ERR_INVALID and b"pitch" in L.wg_last_error()
    plan = ctypes.c_void_p()
    rc = L.wg_expect_plan_create(0, 64, 1, None, None, None, ctypes.byref(plan), None)
    assert rc == capi.WG_ERR_INVALID and b"num_qubits <= 63" in L.wg_last_error()
    # empty inputs need no device
    rc = L.wg_simplify(0, 1, 0, None, None, None, 0.0, 0.0, ctypes.byref(ox), ctypes.byref(oz),
                       ctypes.byref(oc), ctypes.byref(u), None)
    assert rc == capi.WG_OK and u.value == 0 and ox.value is None


def _built_libraries():
    from wolfgang_b200 import build

    return [capi.LIB_PATH, capi.LIB_PATH.parent / "libwolfgang.so", build.module_path()]


def test_libraries_share_the_system_libstdcxx():
    """Every shared library links libstdc++ dynamically and exports no unique
    (u) symbols: a static copy would export the old std::string's empty
    representation, and libraries loaded after it would bind to it."""
    for path in _built_libraries():
        needed = subprocess.run(["readelf", "-d", str(path)], capture_output=True, text=True, check=True).stdout
        assert "libstdc++.so.6" in needed, path
        syms = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True,
                              check=True).stdout
        unique = [line.split()[-1] for line in syms.splitlines() if line.split()[1:2] == ["u"]]
        assert not unique, (path, unique[:5])


def test_torch_imports_after_the_package():
    """Importing the package (and its native libraries) before torch leaves
    torch's own library loading intact."""
    import sys

    code = "import wolfgang_quantum, wolfgang_b200.capi as c; c.lib(); import torch; print('ok')"
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                         cwd=str(capi.LIB_PATH.parents[2]))
    assert out.returncode == 0 and out.stdout.strip().endswith("ok"), (out.returncode, out.stderr[-2000:])


def test_bucket_fine_target_is_range_checked_before_device_work():
    for bad in (1, 31, 2049):
        try:
            capi.set_bucket_fine_target(bad)
        except capi.WGInvalid as e:
            assert "fine bucket target" in str(e)
        else:
            raise AssertionError(f"fine target {bad} accepted")
    capi.set_bucket_fine_target(1800)
    capi.set_bucket_fine_target(0)


def test_bucket_one_pass_setting_is_checked():
    for bad in (-1, 2):
        rc = capi.lib().wg_set_bucket_one_pass(bad)
        assert rc == capi.WG_ERR_INVALID and b"one-pass" in capi.lib().wg_last_error()
    capi.set_bucket_one_pass(False)
    capi.set_bucket_one_pass(True)


def test_chunked_download_needs_a_callback():
    L = capi.lib()
    rc = L.wg_memcpy_dtoh_chunked(0, None, 64, None, None, None)
    assert rc == capi.WG_ERR_INVALID and b"callback" in L.wg_last_error()
    assert L.wg_memcpy_dtoh_chunked(0, None, 0, None, None, None) == capi.WG_OK
