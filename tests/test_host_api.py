"""Host-side API behaviour (no GPU): I/O, arithmetic, guardrails, errors.

Known answers restate the reference's public-API fixtures
(tests/test_phase2_io.py, test_phase5_arithmetic.py:396-412,
test_phase6_commutation_grouping.py:91-113 of sghowell/wolfgang 0.2.3).
"""

from __future__ import annotations

import numpy as np
import pytest

from wolfgang_quantum import PauliSum


def label_for(n: int, entries: dict[int, str]) -> str:
    chars = ["I"] * n
    for q, p in entries.items():
        chars[n - 1 - q] = p
    return "".join(chars)


def test_from_labels_round_trip():
    op = PauliSum.from_labels(["I", "X", "Y", "Z"], [1, 2.5, np.complex64(3 + 4j), -1j])
    labels, coeffs = op.to_labels()
    assert labels == ["I", "X", "Y", "Z"]
    assert op.num_qubits == 1 and op.num_terms == 4
    assert coeffs.dtype == np.complex128
    np.testing.assert_array_equal(coeffs, np.asarray([1, 2.5, 3 + 4j, -1j], np.complex128))


def test_default_coefficients_and_endianness():
    op = PauliSum.from_labels(["XXI", "IZZ", "YYI"])
    assert op.to_labels()[0] == ["XXI", "IZZ", "YYI"]
    np.testing.assert_array_equal(op.to_labels()[1], np.ones(3, np.complex128))
    assert PauliSum.from_labels(["XYZ"]).to_sparse_list() == [("ZYX", [0, 1, 2], 1.0 + 0.0j)]
    assert PauliSum.from_sparse_list([("ZX", [1, 4], 1.0)], num_qubits=5).to_labels()[0] == ["XIIZI"]


def test_sparse_list_preserves_order_and_sorts_qubits():
    op = PauliSum.from_sparse_list([("XZ", [4, 1], 2.0), ("Y", [0], -0.5j), ("", [], 3.0)], num_qubits=5)
    assert op.to_sparse_list() == [("ZX", [1, 4], 2.0 + 0.0j), ("Y", [0], -0.5j), ("", [], 3.0 + 0.0j)]
    assert op.to_labels()[0] == ["XIIZI", "IIIIY", "IIIII"]


def test_empty_operators():
    op = PauliSum.empty(5)
    assert (op.num_qubits, op.num_terms) == (5, 0)
    assert op.to_labels()[0] == [] and op.to_sparse_list() == []
    assert PauliSum.from_sparse_list([], num_qubits=3).num_terms == 0
    assert PauliSum(3, 2).to_labels()[0] == ["III", "III"]


@pytest.mark.parametrize(
    "call,match",
    [
        (lambda: PauliSum.from_labels("XYZ"), "not a single string"),
        (lambda: PauliSum.from_labels([]), "cannot infer num_qubits"),
        (lambda: PauliSum.from_labels(["XX", "X"]), "same length"),
        (lambda: PauliSum.from_labels(["XA"]), "only I, X, Y, or Z"),
        (lambda: PauliSum.from_labels(["X", "Y"], 1.0), "scalar coeffs"),
        (lambda: PauliSum.from_labels(["X", "Y"], [1.0]), "coefficient count"),
        (lambda: PauliSum.from_sparse_list([("X", [3], 1.0)], num_qubits=2), "out of range"),
        (lambda: PauliSum.from_sparse_list([("XX", [1, 1], 1.0)], num_qubits=2), "duplicate qubit"),
        (lambda: PauliSum.from_sparse_list([("XX", [1], 1.0)], num_qubits=2), "length must match"),
        (lambda: PauliSum.from_sparse_list([("Q", [1], 1.0)], num_qubits=2), "only I, X, Y, or Z"),
    ],
)
def test_parse_errors(call, match):
    with pytest.raises(ValueError, match=match):
        call()


def test_add_and_scalar_multiply_keep_order():
    a = PauliSum.from_labels(["XI", "IZ"], [1.0, 2.0])
    b = PauliSum.from_labels(["YY"], [3j])
    s = a + b
    assert s.to_labels()[0] == ["XI", "IZ", "YY"]
    np.testing.assert_array_equal(s.to_labels()[1], [1, 2, 3j])
    np.testing.assert_array_equal((2j * a).to_labels()[1], [2j, 4j])
    np.testing.assert_array_equal((a * 0).to_labels()[1], [0, 0])
    with pytest.raises(ValueError, match="same num_qubits"):
        a + PauliSum.from_labels(["X"])


def test_validation_precedes_device_access():
    """Argument errors are reported before any GPU work, so they hold on CPU."""
    a = PauliSum.from_labels(["XI", "IZ"], [1.0, 2.0])
    with pytest.raises(ValueError, match="same num_qubits"):
        a.matmul(PauliSum.from_labels(["X"]))
    with pytest.raises(ValueError, match="max_intermediate_terms"):
        a.matmul(a, max_intermediate_terms=3)
    with pytest.raises(ValueError, match="same num_qubits"):
        a.commutes_with(PauliSum.from_labels(["XXX"]))
    with pytest.raises(ValueError, match="max_commutation_matrix_entries"):
        PauliSum(1, 3).commutes_with(PauliSum(1, 4), max_commutation_matrix_entries=11)
    with pytest.raises(ValueError, match="tolerances must be non-negative"):
        a.simplify(atol=-1e-12)
    with pytest.raises(ValueError, match="tolerances must be non-negative"):
        a.simplify(rtol=float("nan"))
    with pytest.raises(ValueError, match="mode"):
        a.group_commuting(mode="diagonal")
    with pytest.raises(ValueError, match="strategy"):
        a.group_commuting(strategy="smallest_first")
    with pytest.raises(ValueError, match="2 \\*\\* num_qubits"):
        a.expectation_statevector(np.zeros(3, np.complex128))
    with pytest.raises(TypeError, match="complex64 or complex128"):
        a.expectation_statevector(np.zeros(4, np.float64))
    with pytest.raises(ValueError, match="diagonal"):
        a.expectation_z_counts({"00": 1})
    with pytest.raises(ValueError, match="non-negative"):
        PauliSum.from_labels(["ZI"]).expectation_z_counts({"00": -1})


def test_guardrail_overflow_messages():
    with pytest.raises(ValueError, match="commutation matrix entry count overflows"):
        PauliSum._checked_commutation_size_for_testing(lhs_terms=1 << 63, rhs_terms=2,
                                                       max_commutation_matrix_entries=1 << 63)
    with pytest.raises(ValueError, match="matmul intermediate term count overflows"):
        PauliSum._checked_matmul_size_for_testing(lhs_terms=1 << 63, rhs_terms=2, max_intermediate_terms=1 << 63)
    assert PauliSum._checked_matmul_size_for_testing(lhs_terms=3, rhs_terms=4, max_intermediate_terms=12) == 12


def test_empty_results_need_no_device():
    a = PauliSum.empty(3)
    assert a.simplify().num_terms == 0
    assert a.matmul(PauliSum.from_labels(["XXX"])).num_terms == 0
    assert a.group_commuting() == []
    assert a.expectation_statevector(np.zeros(8, np.complex128)) == 0j


def test_packed_round_trip():
    op = PauliSum.from_labels([label_for(70, {0: "X", 64: "Y", 69: "Z"}), label_for(70, {5: "Z"})], [1, 2])
    x, z, c = op._packed()
    assert x.shape == (2, 2) and x.dtype == np.uint64
    back = PauliSum._from_packed(70, x, z, c)
    assert back.to_labels()[0] == op.to_labels()[0]
    with pytest.raises(ValueError, match="above num_qubits"):
        PauliSum._from_packed(3, np.array([[8]], np.uint64), np.array([[0]], np.uint64), np.ones(1))


def test_public_packed_constructor_and_export():
    """from_packed / to_packed: the public forms of the packed constructor and
    export; they equal the label path and round-trip the storage exactly."""
    labels = [label_for(130, {0: "X", 64: "Y", 129: "Z"}), label_for(130, {5: "Z", 77: "X"}), "I" * 130]
    coeffs = [1 + 2j, -0.5, 3j]
    op = PauliSum.from_labels(labels, coeffs)
    x, z, c = op.to_packed()
    assert x.shape == (3, 3) and z.shape == (3, 3) and c.dtype == np.complex128
    back = PauliSum.from_packed(130, x, z, c)
    assert back.to_labels()[0] == op.to_labels()[0] == labels
    for a, b in zip(back.to_packed(), op.to_packed()):
        assert a.tobytes() == b.tobytes()
    with pytest.raises(ValueError, match="above num_qubits"):
        PauliSum.from_packed(3, np.array([[8]], np.uint64), np.array([[0]], np.uint64), np.ones(1))


def test_no_device_is_reported_as_runtime_error():
    import wolfgang_quantum as wq

    if wq.cuda_available():
        pytest.skip("a CUDA device is visible")
    with pytest.raises(RuntimeError, match="no CUDA device"):
        PauliSum.from_labels(["XX", "XX"]).simplify()
    with pytest.raises(RuntimeError, match="no CUDA device"):
        PauliSum.from_labels(["X"]).to_device()
    assert wq._wolfgang_core._cuda_status()["runtime_available"] is False
