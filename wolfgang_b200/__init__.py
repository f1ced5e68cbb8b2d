"""B200-native (sm_100a) packed-Pauli hot path of sghowell/wolfgang.

The public operator types mirror the reference's ``wolfgang_quantum`` module:
``PauliSum``, ``DevicePauliSum``, ``DeviceCommutationMatrix`` and the device
helpers.  Compute methods run on the GPU through the wg_* C-ABI of
``lib/libwgpauli.so``; there is no CPU fallback, and importing this package
fails loudly when the native module has not been built
(``python wolfgang_b200/build.py``).
"""

from __future__ import annotations

from pathlib import Path

_PKG = Path(__file__).resolve().parent

try:
    from . import _wolfgang_core  # noqa: F401
except ImportError as exc:  # pragma: no cover - exercised only on a broken install
    raise ImportError(
        "wolfgang_b200 native module is not built; run `python wolfgang_b200/build.py` "
        f"(sm_100a CUDA toolchain required): {exc}"
    ) from exc

from ._wolfgang_core import (  # noqa: E402
    DeviceCommutationBits,
    DeviceCommutationMatrix,
    DevicePauliSum,
    PauliSum,
    cuda_available,
    cuda_devices,
    hip_available,
    hip_devices,
    metal_available,
    metal_devices,
)

__version__ = "0.2.3+b200"

__all__ = [
    "DeviceCommutationBits",
    "DeviceCommutationMatrix",
    "DevicePauliSum",
    "PauliSum",
    "__version__",
    "cuda_available",
    "cuda_devices",
    "hip_available",
    "hip_devices",
    "metal_available",
    "metal_devices",
]


def native_libraries() -> list[Path]:
    """Paths of the native libraries this package loads."""
    return [_PKG / "lib" / "libwgpauli.so", _PKG / "lib" / "libwolfgang.so", Path(_wolfgang_core.__file__)]
