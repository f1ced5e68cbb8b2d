"""``wolfgang_quantum`` names of sghowell/wolfgang, served by the B200 build.

``python/wolfgang_quantum/__init__.py:32-42`` of the reference exports these
names; code that imports them from ``wolfgang_quantum`` runs unchanged on the
sm_100a kernels of :mod:`wolfgang_b200`.
"""

from wolfgang_b200 import (  # noqa: F401
    DeviceCommutationBits,
    DeviceCommutationMatrix,
    DevicePauliSum,
    PauliSum,
    __version__,
    _wolfgang_core,
    cuda_available,
    cuda_devices,
    hip_available,
    hip_devices,
    metal_available,
    metal_devices,
)
from .openfermion import _install_pauli_sum_openfermion_methods
from .qiskit import _install_pauli_sum_qiskit_methods

# PauliSum.from_qiskit / to_qiskit / from_openfermion / to_openfermion, as the
# reference installs them (python/wolfgang_quantum/__init__.py:43-47)
_install_pauli_sum_qiskit_methods()
_install_pauli_sum_openfermion_methods()

__all__ = [
    "DeviceCommutationMatrix",
    "DevicePauliSum",
    "PauliSum",
    "__version__",
    "_wolfgang_core",
    "cuda_available",
    "cuda_devices",
    "hip_available",
    "hip_devices",
    "metal_available",
    "metal_devices",
]
