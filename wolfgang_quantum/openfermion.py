"""OpenFermion ``QubitOperator`` <-> :class:`PauliSum` conversion.

Mirrors ``python/wolfgang_quantum/openfermion.py`` of the reference (names,
arguments, error types and messages).  OpenFermion is imported only when an
adapter is called.  Conversion reads the operator's sparse ``terms``
dictionary ({((qubit, 'X'|'Y'|'Z'), ...): coefficient}); no dense matrix is
formed.
"""

from __future__ import annotations

from typing import Any

from wolfgang_b200 import PauliSum

OPENFERMION_INSTALL_HINT = "Install Wolfgang with the openfermion extra to use this adapter."


def _import_qubit_operator_type() -> Any:
    try:
        from openfermion.ops.operators.qubit_operator import QubitOperator
    except ImportError as exc:
        raise ImportError(OPENFERMION_INSTALL_HINT) from exc
    return QubitOperator


def _width(num_qubits: int | None, terms: dict) -> int:
    if num_qubits is not None:
        if not isinstance(num_qubits, int):
            raise TypeError("num_qubits must be an integer or None")
        if num_qubits < 0:
            raise ValueError("num_qubits must be non-negative")
        return num_qubits
    # the largest non-identity qubit index + 1 (0 for identity-only or zero)
    return max((int(q) + 1 for term in terms for q, _ in term), default=0)


def from_openfermion(op: Any, num_qubits: int | None = None) -> PauliSum:
    """PauliSum of a ``QubitOperator``; the width is inferred when not given."""
    qubit_operator = _import_qubit_operator_type()
    if not isinstance(op, qubit_operator):
        raise TypeError("PauliSum.from_openfermion expects openfermion.ops.QubitOperator")
    width = _width(num_qubits, op.terms)
    if not op.terms:
        return PauliSum.empty(width)
    sparse = []
    for term, coeff in op.terms.items():
        qubits = [int(q) for q, _ in term]
        if any(q < 0 or q >= width for q in qubits):
            raise ValueError("OpenFermion term qubit index is out of range for num_qubits")
        sparse.append(("".join(str(p) for _, p in term), qubits, complex(coeff)))
    return PauliSum.from_sparse_list(sparse, width)


def to_openfermion(self: PauliSum) -> Any:
    """``QubitOperator`` of a PauliSum: identity terms become the empty term, no terms the zero operator."""
    if not isinstance(self, PauliSum):
        raise TypeError("PauliSum.to_openfermion expects a PauliSum receiver")
    qubit_operator = _import_qubit_operator_type()
    out = qubit_operator()
    for paulis, qubits, coeff in self.to_sparse_list():
        term = tuple((int(q), str(p)) for p, q in zip(paulis, qubits)) if paulis else ()
        out += qubit_operator(term, complex(coeff))
    return out


def _install_pauli_sum_openfermion_methods() -> None:
    PauliSum.from_openfermion = staticmethod(from_openfermion)
    PauliSum.to_openfermion = to_openfermion


__all__ = ["OPENFERMION_INSTALL_HINT", "from_openfermion", "to_openfermion"]
