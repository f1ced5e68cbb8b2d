"""Qiskit / OpenFermion adapters (wolfgang_quantum.qiskit, .openfermion).

Neither package is installed here, so minimal stand-ins for the parts the
adapters touch (``qiskit.quantum_info.SparsePauliOp`` / ``PauliList`` and
``openfermion.ops.operators.qubit_operator.QubitOperator``) are put into
``sys.modules`` for the tests that convert.  Cases follow the reference's
tests/test_qiskit_adapter.py and tests/test_openfermion_adapter.py: round
trips, endianness, identity and empty operators, phase prefixes, duplicate
terms, width inference and validation, wrong input types, and the install
hint when the package is missing.  Host-only: no GPU call.
"""

from __future__ import annotations

import builtins
import sys
import types

import numpy as np
import pytest

import wolfgang_quantum as wq
from wolfgang_quantum import PauliSum
from wolfgang_quantum.openfermion import OPENFERMION_INSTALL_HINT
from wolfgang_quantum.qiskit import QISKIT_INSTALL_HINT


# ---------------------------------------------------------------- stand-ins

class _PauliList:
    def __init__(self, labels):
        self._labels = list(labels)

    def to_labels(self):
        return list(self._labels)

    @classmethod
    def from_symplectic(cls, z, x):
        assert z.shape == x.shape
        return cls([])


class _SparsePauliOp:
    def __init__(self, data, coeffs=None):
        if isinstance(data, _PauliList):
            self.paulis = data
            self.num_qubits = 0
        else:
            labels = list(data)
            self.paulis = _PauliList(labels)
            self.num_qubits = len(labels[0].lstrip("+-i")) if labels else 0
        n = len(self.paulis.to_labels())
        self.coeffs = np.ones(n, np.complex128) if coeffs is None else np.asarray(coeffs, np.complex128)


class _QubitOperator:
    def __init__(self, term=None, coefficient=1.0):
        self.terms = {}
        if term is None:
            return
        if isinstance(term, str):
            term = tuple((int(t[1:]), t[0]) for t in term.split())
        self.terms[tuple(term)] = complex(coefficient)

    def __iadd__(self, other):
        for t, c in other.terms.items():
            self.terms[t] = self.terms.get(t, 0) + c
        return self

    def __add__(self, other):
        out = _QubitOperator()
        out += self
        out += other
        return out


@pytest.fixture
def fake_qiskit(monkeypatch):
    qiskit = types.ModuleType("qiskit")
    qi = types.ModuleType("qiskit.quantum_info")
    qi.SparsePauliOp = _SparsePauliOp
    qi.PauliList = _PauliList
    qiskit.quantum_info = qi
    monkeypatch.setitem(sys.modules, "qiskit", qiskit)
    monkeypatch.setitem(sys.modules, "qiskit.quantum_info", qi)
    return qi


@pytest.fixture
def fake_openfermion(monkeypatch):
    names = ["openfermion", "openfermion.ops", "openfermion.ops.operators", "openfermion.ops.operators.qubit_operator"]
    mods = {n: types.ModuleType(n) for n in names}
    mods["openfermion.ops.operators.qubit_operator"].QubitOperator = _QubitOperator
    for parent, child in zip(names, names[1:]):
        setattr(mods[parent], child.rsplit(".", 1)[1], mods[child])
    for n, m in mods.items():
        monkeypatch.setitem(sys.modules, n, m)
    return _QubitOperator


# ---------------------------------------------------------------- qiskit

@pytest.mark.parametrize("label", ["I", "X", "Y", "Z"])
def test_qiskit_single_qubit_round_trip(fake_qiskit, label):
    op = PauliSum.from_qiskit(_SparsePauliOp([label], coeffs=[0.5 - 2j]))
    assert op.num_qubits == 1 and op.num_terms == 1
    back = op.to_qiskit()
    assert back.paulis.to_labels() == [label]
    np.testing.assert_array_equal(back.coeffs, [0.5 - 2j])


def test_qiskit_endianness(fake_qiskit):
    # Qiskit puts qubit 0 rightmost: "XIZ" is Z on qubit 0 and X on qubit 2
    op = PauliSum.from_qiskit(_SparsePauliOp(["XIZ"], coeffs=[1.0]))
    (paulis, qubits, coeff), = op.to_sparse_list()
    assert sorted(zip(qubits, paulis)) == [(0, "Z"), (2, "X")]
    assert op.to_qiskit().paulis.to_labels() == ["XIZ"]


def test_qiskit_identity_and_empty(fake_qiskit):
    ident = PauliSum.from_qiskit(_SparsePauliOp(["III"], coeffs=[3.0]))
    assert ident.to_labels()[0] == ["III"]
    empty = PauliSum.from_qiskit(_SparsePauliOp(_PauliList([]), coeffs=[]))
    assert empty.num_terms == 0
    assert PauliSum.empty(2).to_qiskit().paulis.to_labels() == []


def test_qiskit_phase_prefixes_fold_into_coefficients(fake_qiskit):
    op = PauliSum.from_qiskit(_SparsePauliOp(["-iXYZ", "-III", "iIIZ", "+XXX"], coeffs=[2.0, 3.0, -4j, 1.0]))
    labels, coeffs = op.to_labels()
    assert list(labels) == ["XYZ", "III", "IIZ", "XXX"]
    np.testing.assert_array_equal(coeffs, [-2j, -3.0, 4.0, 1.0])


def test_qiskit_duplicates_kept_in_order(fake_qiskit):
    op = PauliSum.from_qiskit(_SparsePauliOp(["ZZ", "XI", "ZZ"], coeffs=[1.0, 2.0, 3.0]))
    labels, coeffs = op.to_labels()
    assert list(labels) == ["ZZ", "XI", "ZZ"]
    np.testing.assert_array_equal(coeffs, [1.0, 2.0, 3.0])


def test_qiskit_rejects_wrong_types(fake_qiskit):
    with pytest.raises(TypeError, match="expects qiskit.quantum_info.SparsePauliOp"):
        PauliSum.from_qiskit(object())
    from wolfgang_quantum.qiskit import to_qiskit

    with pytest.raises(TypeError, match="expects a PauliSum receiver"):
        to_qiskit(object())


def test_qiskit_missing_dependency_hint(monkeypatch):
    original = builtins.__import__

    def no_qiskit(name, *args, **kwargs):
        if name == "qiskit" or name.startswith("qiskit."):
            raise ModuleNotFoundError("No module named 'qiskit'")
        return original(name, *args, **kwargs)

    monkeypatch.setattr(builtins, "__import__", no_qiskit)
    with pytest.raises(ImportError, match=QISKIT_INSTALL_HINT):
        PauliSum.empty(1).to_qiskit()
    with pytest.raises(ImportError, match=QISKIT_INSTALL_HINT):
        PauliSum.from_qiskit(object())


def test_qiskit_loader_is_patchable(monkeypatch):
    """The reference's tests replace the module's loader; the same name works here."""
    import wolfgang_quantum.qiskit as adapter

    class FakeQI:
        SparsePauliOp = _SparsePauliOp
        PauliList = _PauliList

    monkeypatch.setattr(adapter, "_import_qiskit_quantum_info", lambda: FakeQI())
    assert PauliSum.from_qiskit(_SparsePauliOp(["ZX"], coeffs=[1j])).num_terms == 1


# ---------------------------------------------------------------- openfermion

def test_openfermion_round_trip(fake_openfermion):
    Q = fake_openfermion
    src = Q("X0 Z3", 0.5) + Q("Y1", -2j)
    op = PauliSum.from_openfermion(src)
    assert op.num_qubits == 4 and op.num_terms == 2
    back = op.to_openfermion()
    assert {tuple(sorted(t)): c for t, c in back.terms.items()} == \
        {tuple(sorted(t)): c for t, c in src.terms.items()}


def test_openfermion_identity_and_empty(fake_openfermion):
    Q = fake_openfermion
    ident = PauliSum.from_openfermion(Q((), 1.5))
    assert ident.num_qubits == 0 and ident.num_terms == 1
    assert ident.to_openfermion().terms == {(): 1.5}
    explicit = PauliSum.from_openfermion(Q((), 1.5), num_qubits=3)
    assert explicit.num_qubits == 3 and explicit.to_openfermion().terms == {(): 1.5}
    empty = PauliSum.from_openfermion(Q(), num_qubits=5)
    assert empty.num_qubits == 5 and empty.num_terms == 0 and empty.to_openfermion().terms == {}
    assert PauliSum.from_openfermion(Q()).num_qubits == 0


def test_openfermion_num_qubits_validation(fake_openfermion):
    Q = fake_openfermion
    with pytest.raises(ValueError, match="out of range"):
        PauliSum.from_openfermion(Q("X3", 1.0), num_qubits=3)
    with pytest.raises(TypeError, match="num_qubits must be an integer or None"):
        PauliSum.from_openfermion(Q("X0", 1.0), num_qubits=2.5)
    with pytest.raises(ValueError, match="num_qubits must be non-negative"):
        PauliSum.from_openfermion(Q("X0", 1.0), num_qubits=-1)


def test_openfermion_rejects_wrong_types(fake_openfermion):
    with pytest.raises(TypeError, match="expects openfermion.ops.QubitOperator"):
        PauliSum.from_openfermion(object())
    from wolfgang_quantum.openfermion import to_openfermion

    with pytest.raises(TypeError, match="expects a PauliSum receiver"):
        to_openfermion(object())


def test_openfermion_missing_dependency_hint(monkeypatch):
    original = builtins.__import__

    def no_openfermion(name, *args, **kwargs):
        if name == "openfermion" or name.startswith("openfermion."):
            raise ModuleNotFoundError("No module named 'openfermion'")
        return original(name, *args, **kwargs)

    monkeypatch.setattr(builtins, "__import__", no_openfermion)
    with pytest.raises(ImportError, match=OPENFERMION_INSTALL_HINT):
        PauliSum.empty(1).to_openfermion()
    with pytest.raises(ImportError, match=OPENFERMION_INSTALL_HINT):
        PauliSum.from_openfermion(object())


def test_importing_package_does_not_import_adapters_deps():
    assert "qiskit" not in sys.modules or isinstance(sys.modules["qiskit"], types.ModuleType)
    assert hasattr(wq.PauliSum, "from_qiskit") and hasattr(wq.PauliSum, "to_openfermion")
