"""Qiskit ``SparsePauliOp`` <-> :class:`PauliSum` conversion.

Mirrors ``python/wolfgang_quantum/qiskit.py`` of the reference (names,
arguments, error types and messages).  Qiskit is imported only when an adapter
is called, so it stays an optional dependency.  Conversion goes through Pauli
labels and coefficients; no dense matrix is formed.  Qiskit labels put qubit 0
rightmost, the same order ``PauliSum.from_labels`` reads.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from wolfgang_b200 import PauliSum

QISKIT_INSTALL_HINT = "Install Wolfgang with the qiskit extra to use this adapter."

# explicit phase prefixes a Qiskit Pauli label may carry, longest first
_PREFIX_PHASE = (("-i", -1j), ("+i", 1j), ("i", 1j), ("-", -1.0 + 0j), ("+", 1.0 + 0j))


def _import_qiskit_quantum_info() -> Any:
    try:
        from qiskit import quantum_info
    except ImportError as exc:
        raise ImportError(QISKIT_INSTALL_HINT) from exc
    return quantum_info


def _split_phase(label: str) -> tuple[str, complex]:
    for prefix, phase in _PREFIX_PHASE:
        if label.startswith(prefix):
            return label[len(prefix):], phase
    return label, 1.0 + 0j


def from_qiskit(op: Any) -> PauliSum:
    """PauliSum of a ``SparsePauliOp``; label phase prefixes fold into the coefficients."""
    qi = _import_qiskit_quantum_info()
    if not isinstance(op, qi.SparsePauliOp):
        raise TypeError("PauliSum.from_qiskit expects qiskit.quantum_info.SparsePauliOp")
    labels = [str(s) for s in op.paulis.to_labels()]
    coeffs = np.asarray(op.coeffs, dtype=np.complex128)
    if len(labels) != len(coeffs):
        raise ValueError("SparsePauliOp label and coefficient counts differ")
    if not labels:
        return PauliSum.empty(int(op.num_qubits))
    plain, folded = [], []
    for label, coeff in zip(labels, coeffs):
        body, phase = _split_phase(label)
        plain.append(body)
        folded.append(complex(coeff) * phase)
    return PauliSum.from_labels(plain, folded)


def to_qiskit(self: PauliSum) -> Any:
    """``SparsePauliOp`` of a PauliSum: phase-free labels, every phase in the coefficients."""
    if not isinstance(self, PauliSum):
        raise TypeError("PauliSum.to_qiskit expects a PauliSum receiver")
    qi = _import_qiskit_quantum_info()
    labels, coeffs = self.to_labels()
    coeffs = np.asarray(coeffs, dtype=np.complex128)
    if self.num_terms == 0:
        empty = np.zeros((0, self.num_qubits), dtype=bool)
        return qi.SparsePauliOp(qi.PauliList.from_symplectic(empty, empty), coeffs=coeffs)
    return qi.SparsePauliOp(list(labels), coeffs=coeffs)


def _install_pauli_sum_qiskit_methods() -> None:
    PauliSum.from_qiskit = staticmethod(from_qiskit)
    PauliSum.to_qiskit = to_qiskit


__all__ = ["QISKIT_INSTALL_HINT", "from_qiskit", "to_qiskit"]
