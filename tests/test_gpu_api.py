"""The reference's public-API known answers, run through wolfgang_quantum on the GPU.

Fixtures restate tests/test_phase4_simplify.py:42-112, test_phase5_arithmetic.py
:328-436, test_phase6_commutation_grouping.py:55-184, test_phase8_expectation.py
:284-358 and test_phase11_cuda_kernels.py (DevicePauliSum parity) of
sghowell/wolfgang 0.2.3, written as new tests against the same public names.
"""

from __future__ import annotations

import numpy as np
import pytest

import wolfgang_quantum as wq
from wolfgang_quantum import DeviceCommutationMatrix, PauliSum

pytestmark = pytest.mark.gpu

PAULI = {
    "I": np.eye(2, dtype=np.complex128),
    "X": np.array([[0, 1], [1, 0]], np.complex128),
    "Y": np.array([[0, -1j], [1j, 0]], np.complex128),
    "Z": np.array([[1, 0], [0, -1]], np.complex128),
}


def dense(labels, coeffs):
    n = len(labels[0])
    m = np.zeros((1 << n, 1 << n), np.complex128)
    for lab, c in zip(labels, coeffs):
        t = PAULI[lab[0]]
        for p in lab[1:]:
            t = np.kron(t, PAULI[p])
        m += c * t
    return m


def label_for(n, entries):
    chars = ["I"] * n
    for q, p in entries.items():
        chars[n - 1 - q] = p
    return "".join(chars)


def labels_coeffs(op):
    labels, coeffs = op.to_labels()
    return list(labels), coeffs


@pytest.fixture(autouse=True)
def _gpu(cuda):
    return cuda


# ---------------------------------------------------------------- simplify

def test_simplify_one_word_canonical_order():
    op = PauliSum.from_labels(["Z", "X", "X", "I", "Z"], [1.0, 2.0, 3.0, 4.0, -0.25])
    labels, coeffs = labels_coeffs(op.simplify(atol=0.0, rtol=0.0))
    assert labels == ["I", "Z", "X"]
    np.testing.assert_array_equal(coeffs, [4.0, 0.75, 5.0])


def test_simplify_inclusive_threshold_with_rtol():
    op = PauliSum.from_labels(["X", "X", "Z", "Y"], [0.4, 0.6, 10.0, 1.0 + 1.0e-9])
    labels, coeffs = labels_coeffs(op.simplify(atol=0.0, rtol=0.1))
    assert labels == ["Z", "Y"]
    np.testing.assert_array_equal(coeffs, [10.0, 1.0 + 1.0e-9])


def test_simplify_all_zero_keeps_qubit_count():
    s = PauliSum.from_labels(["XX", "ZZ"], [1.0e-13, 0.0]).simplify()
    assert s.num_qubits == 2 and s.num_terms == 0


def test_simplify_multiword_order():
    n = 130
    q64z, q64x = label_for(n, {64: "Z"}), label_for(n, {64: "X"})
    q0z, q0x = label_for(n, {0: "Z"}), label_for(n, {0: "X"})
    op = PauliSum.from_labels([q0x, q64x, q0z, q64z], [4.0, 2.0, 3.0, 1.0])
    labels, coeffs = labels_coeffs(op.simplify(atol=0.0, rtol=0.0))
    assert labels == [q64z, q64x, q0z, q0x]
    np.testing.assert_array_equal(coeffs, [1.0, 2.0, 3.0, 4.0])


@pytest.mark.parametrize("n", [1, 65])
def test_duplicate_heavy_simplify(n):
    pool = ["I", "Z", "X", "Y"] if n == 1 else [label_for(n, {0: "X"}), label_for(n, {64: "Z"}),
                                                label_for(n, {0: "Y", 64: "X"}), label_for(n, {1: "Z", 64: "Y"})]
    labels = [pool[i % 4] for i in range(4096)]
    coeffs = [complex((i % 13) - 6, (i % 7) - 3) for i in range(4096)]
    sums = [sum(c for lab, c in zip(labels, coeffs) if lab == p) for p in pool]
    got = PauliSum.from_labels(labels, coeffs).simplify(atol=0.0, rtol=0.0)
    want = PauliSum.from_labels(pool, sums).simplify(atol=0.0, rtol=0.0)
    assert labels_coeffs(got)[0] == labels_coeffs(want)[0]
    np.testing.assert_array_equal(labels_coeffs(got)[1], labels_coeffs(want)[1])


# ---------------------------------------------------------------- products

PHASES = [("X", "Y", "Z", 1j), ("Y", "X", "Z", -1j), ("Y", "Z", "X", 1j), ("Z", "Y", "X", -1j),
          ("Z", "X", "Y", 1j), ("X", "Z", "Y", -1j)]


@pytest.mark.parametrize("a,b,label,coeff", PHASES)
def test_single_qubit_phase_fixtures(a, b, label, coeff):
    labels, coeffs = labels_coeffs(PauliSum.from_labels([a]) @ PauliSum.from_labels([b]))
    assert labels == [label]
    np.testing.assert_array_equal(coeffs, [coeff])


def test_nested_loop_order_without_simplify():
    lhs = PauliSum.from_labels(["XI", "IZ"], [1.0, 2.0])
    rhs = PauliSum.from_labels(["IY", "ZI"], [3.0, 4.0])
    labels, coeffs = labels_coeffs(lhs.matmul(rhs, simplify=False))
    assert labels == ["XY", "YI", "IX", "ZZ"]
    np.testing.assert_array_equal(coeffs, [3.0, -4j, -6j, 8.0])


def test_products_combine_duplicates():
    op = PauliSum.from_labels(["X", "Y"], [1.0, 1.0])
    labels, coeffs = labels_coeffs(op @ op)
    assert labels == ["I"]
    np.testing.assert_array_equal(coeffs, [2.0])


@pytest.mark.parametrize("n", [1, 2, 3])
def test_matmul_matches_dense_matrices(n):
    rng = np.random.default_rng(500 + n)
    letters = np.array(list("IXYZ"))
    la = ["".join(rng.choice(letters, n)) for _ in range(4)]
    lb = ["".join(rng.choice(letters, n)) for _ in range(3)]
    ca = rng.normal(size=4) + 1j * rng.normal(size=4)
    cb = rng.normal(size=3) + 1j * rng.normal(size=3)
    prod = PauliSum.from_labels(la, ca) @ PauliSum.from_labels(lb, cb)
    got_labels, got_coeffs = labels_coeffs(prod)
    np.testing.assert_allclose(dense(got_labels, got_coeffs) if got_labels else 0, dense(la, ca) @ dense(lb, cb),
                               atol=1e-12)


def test_matmul_guardrail():
    with pytest.raises(ValueError, match="max_intermediate_terms"):
        PauliSum(1, 3).matmul(PauliSum(1, 4), max_intermediate_terms=11)


# ---------------------------------------------------------------- commutation

def test_commutes_with_shapes():
    x = PauliSum.from_labels(["X"])
    zz = PauliSum.from_labels(["Z"])
    rhs = PauliSum.from_labels(["X", "Y", "I"], [1.0, 2.0, 3.0])
    lhs = PauliSum.from_labels(["X", "Z"], [1.0, 2.0])
    assert x.commutes_with(x) is True
    assert x.commutes_with(zz) is False
    v = x.commutes_with(rhs)
    assert v.dtype == np.bool_ and v.shape == (3,) and v.flags.writeable
    np.testing.assert_array_equal(v, [True, False, True])
    np.testing.assert_array_equal(lhs.commutes_with(x), [True, False])
    m = lhs.commutes_with(rhs)
    assert m.shape == (2, 3)
    np.testing.assert_array_equal(m, [[True, False, True], [False, False, True]])


def test_commutation_symmetry():
    rng = np.random.default_rng(1979)
    letters = np.array(list("IXYZ"))
    for _ in range(10):
        a = PauliSum.from_labels(["".join(rng.choice(letters, 4)) for _ in range(int(rng.integers(2, 8)))])
        b = PauliSum.from_labels(["".join(rng.choice(letters, 4)) for _ in range(int(rng.integers(2, 8)))])
        np.testing.assert_array_equal(a.commutes_with(b), b.commutes_with(a).T)


# ---------------------------------------------------------------- grouping

GROUP_OP = (["XI", "IX", "XX", "YY", "ZI", "IZ", "II"], [1.0, -2.0, 3.0, 4.0, 5.0, -6.0, 7.0])


def _qwc(a, b):
    return all(p == "I" or q == "I" or p == q for p, q in zip(a, b))


def _full(a, b):
    par = 0
    for p, q in zip(a, b):
        par ^= int((p in "XY" and q in "ZY") != (p in "ZY" and q in "XY"))
    return par == 0


@pytest.mark.parametrize("mode", ["qwc", "full"])
def test_groups_valid_and_deterministic(mode):
    op = PauliSum.from_labels(*GROUP_OP)
    groups = [labels_coeffs(g)[0] for g in op.group_commuting(mode=mode)]
    again = [labels_coeffs(g)[0] for g in op.group_commuting(mode=mode)]
    assert groups == again
    pred = _qwc if mode == "qwc" else _full
    for g in groups:
        for i, a in enumerate(g):
            for b in g[i + 1:]:
                assert pred(a, b)
    assert sorted(sum(groups, [])) == sorted(GROUP_OP[0])


def test_group_greedy_order_fixture():
    groups = PauliSum.from_labels(["II", "XI", "XX", "IZ"], [1.0, 2.0, 3.0, 4.0]).group_commuting(mode="qwc")
    assert [labels_coeffs(g)[0] for g in groups] == [["XX", "XI", "II"], ["IZ"]]
    np.testing.assert_array_equal(labels_coeffs(groups[0])[1], [3.0, 2.0, 1.0])


def test_streaming_equals_graph():
    op = PauliSum.from_labels(*GROUP_OP)
    a = [labels_coeffs(g)[0] for g in op.group_commuting(mode="full")]
    b = [labels_coeffs(g)[0] for g in op.group_commuting(mode="full", max_terms_for_graph=0)]
    assert a == b


# ---------------------------------------------------------------- expectation

def _state(width, dtype):
    rng = np.random.default_rng(9100 + width)
    raw = (rng.normal(size=1 << width) + 1j * rng.normal(size=1 << width)).astype(dtype)
    return raw / np.linalg.norm(raw)


@pytest.mark.parametrize("width", range(1, 9))
def test_expectation_matches_dense(width):
    rng = np.random.default_rng(8100 + width)
    letters = np.array(list("IXYZ"))
    k = min(10, 2 + width)
    labels = ["".join(rng.choice(letters, width)) for _ in range(k)]
    coeffs = rng.normal(size=k) + 1j * rng.normal(size=k)
    psi = _state(width, np.complex128)
    op = PauliSum.from_labels(labels, coeffs)
    expected = np.vdot(psi, dense(labels, coeffs) @ psi)
    assert op.expectation_statevector(psi) == pytest.approx(expected, abs=1e-11)
    assert op.to_device().expectation_statevector(psi) == pytest.approx(expected, abs=1e-11)


def test_expectation_complex64():
    labels, coeffs = ["XI", "YZ", "II"], [0.5 - 0.25j, -1.25 + 0.75j, 0.125]
    op = PauliSum.from_labels(labels, coeffs)
    p128 = _state(2, np.complex128)
    p64 = p128.astype(np.complex64)
    assert op.expectation_statevector(p128) == pytest.approx(np.vdot(p128, dense(labels, coeffs) @ p128), abs=1e-12)
    e64 = np.vdot(p64.astype(np.complex128), dense(labels, coeffs) @ p64.astype(np.complex128))
    assert op.expectation_statevector(p64) == pytest.approx(e64, abs=1e-6)


def test_expectation_diagonal_duplicates():
    base = ["ZZII", "IZZI", "ZIIZ", "IIZZ", "ZIZI"]
    labels = [base[i % 5] for i in range(80)]
    coeffs = [complex(np.sin(i + 1) * 0.125, np.cos(i + 3) * 0.0625) for i in range(80)]
    psi = _state(4, np.complex128)
    op = PauliSum.from_labels(labels, coeffs)
    assert op.expectation_statevector(psi) == pytest.approx(np.vdot(psi, dense(labels, coeffs) @ psi), abs=1e-11)


def test_expectation_empty_and_zero_qubits():
    assert PauliSum.empty(2).expectation_statevector(np.array([1, 0, 0, 0], np.complex128)) == 0j
    ident = PauliSum.from_sparse_list([("", [], 2.5 - 0.75j)], num_qubits=0)
    assert ident.expectation_statevector(np.array([1.0 + 0j])) == pytest.approx(2.5 - 0.75j)


def test_expectation_cuda_array_interface_and_validation(cuda):
    t = cuda
    rng = np.random.default_rng(3)
    labels = ["XZY", "ZZI", "IYX"]
    coeffs = [0.3, -1.1j, 0.7]
    op = PauliSum.from_labels(labels, coeffs).to_device()
    psi = _state(3, np.complex128)
    expected = np.vdot(psi, dense(labels, coeffs) @ psi)
    dpsi = t.from_numpy(psi).cuda()
    assert op.expectation_statevector(dpsi) == pytest.approx(expected, abs=1e-12)
    assert op.expectation_statevector(dpsi.to(t.complex64)) == pytest.approx(expected, abs=1e-6)

    class Fake:
        def __init__(self, **iface):
            self.__cuda_array_interface__ = iface

    with pytest.raises(TypeError, match="typestr"):
        op.expectation_statevector(Fake(shape=(8,), typestr="<f8", data=(dpsi.data_ptr(), False), version=3))
    with pytest.raises(ValueError, match="1-dimensional"):
        op.expectation_statevector(Fake(shape=(2, 4), typestr="<c16", data=(dpsi.data_ptr(), False), version=3))
    with pytest.raises(ValueError, match="2 \\*\\* num_qubits"):
        op.expectation_statevector(Fake(shape=(4,), typestr="<c16", data=(dpsi.data_ptr(), False), version=3))
    with pytest.raises(TypeError, match="non-null"):
        op.expectation_statevector(Fake(shape=(8,), typestr="<c16", data=(0, False), version=3))
    host = np.zeros(8, np.complex128)
    with pytest.raises(ValueError, match="device memory"):
        op.expectation_statevector(Fake(shape=(8,), typestr="<c16", data=(host.ctypes.data, False), version=3))
    # 2^36 amplitudes (1 TiB) cannot lie inside the allocation behind a small
    # tensor: the extent check rejects it on the host, before any kernel runs.
    wide = PauliSum.from_sparse_list([("Z", [35], 1.0)], num_qubits=36).to_device()
    small = t.zeros(4, dtype=t.complex128, device="cuda")
    with pytest.raises(ValueError, match="backing allocation"):
        wide.expectation_statevector(Fake(shape=(1 << 36,), typestr="<c16", data=(small.data_ptr(), False), version=3))


# ---------------------------------------------------------------- DevicePauliSum

def test_device_round_trip_and_metadata():
    op = PauliSum.from_labels(["XYZ", "IZI"], [1, 2j])
    d = op.to_device()
    assert (d.num_qubits, d.num_terms, d.device, d.backend) == (3, 2, 0, "cuda")
    assert d.to_host().to_labels()[0] == op.to_labels()[0]
    assert wq.cuda_available()
    assert wq.cuda_devices()[0]["compute_capability"][0] >= 10


def test_device_simplify_and_matmul_match_host():
    rng = np.random.default_rng(77)
    letters = np.array(list("IXYZ"))
    labels = ["".join(rng.choice(letters, 70)) for _ in range(300)]
    op = PauliSum.from_labels(labels, rng.normal(size=300) + 1j * rng.normal(size=300))
    d = op.to_device()
    assert labels_coeffs(d.simplify().to_host())[0] == labels_coeffs(op.simplify())[0]
    a = labels_coeffs(d.matmul(d).to_host())
    b = labels_coeffs(op.matmul(op))
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])
    raw = d.matmul(d, simplify=False)
    assert raw.num_terms == 300 * 300


def test_device_commutation_outputs():
    rng = np.random.default_rng(11)
    letters = np.array(list("IXYZ"))
    a = PauliSum.from_labels(["".join(rng.choice(letters, 6)) for _ in range(17)])
    b = PauliSum.from_labels(["".join(rng.choice(letters, 6)) for _ in range(23)])
    want = a.commutes_with(b)
    da, db = a.to_device(), b.to_device()
    np.testing.assert_array_equal(da.commutes_with(db), want)
    out = np.zeros(17 * 23, np.bool_)
    da.commutes_with_into(db, out)
    np.testing.assert_array_equal(out.reshape(17, 23), want)
    m = da.commutes_with_device(db)
    assert m.shape == (17, 23) and m.dtype == "uint8" and m.num_entries == 17 * 23
    np.testing.assert_array_equal(m.to_host(), want)
    assert m.count_commuting() == int(want.sum())
    np.testing.assert_array_equal(m.count_commuting(axis=1), want.sum(axis=1))
    np.testing.assert_array_equal(m.count_commuting(axis=0), want.sum(axis=0))
    assert m.conflict_degrees() == int((~want).sum())
    reuse = DeviceCommutationMatrix.empty((17, 23))
    assert da.commutes_with_device(db, output=reuse) is reuse
    np.testing.assert_array_equal(reuse.to_host(), want)
    bits = da.commutes_with_bits(db)
    assert bits.count_commuting() == int(want.sum())
    with pytest.raises(ValueError, match="output shape"):
        da.commutes_with_device(db, output=DeviceCommutationMatrix.empty((2, 2)))


def test_device_commutation_matrix_dlpack():
    """DeviceCommutationMatrix.__dlpack__ (reference .pyi:29-30,
    bindings/python/pauli_sum_py.cpp:663-821): a read-only view of the dense
    uint8 buffer that torch imports without a copy, lifetime-tied to the
    matrix, with the reference's refusals."""
    import gc

    import torch

    rng = np.random.default_rng(12)
    letters = np.array(list("IXYZ"))
    a = PauliSum.from_labels(["".join(rng.choice(letters, 7)) for _ in range(31)])
    b = PauliSum.from_labels(["".join(rng.choice(letters, 7)) for _ in range(45)])
    want = a.commutes_with(b)
    m = a.to_device().commutes_with_device(b.to_device())
    assert m.__dlpack_device__() == (2, 0)
    t = torch.from_dlpack(m)
    assert t.dtype == torch.uint8 and tuple(t.shape) == (31, 45) and t.device == torch.device("cuda", 0)
    assert t.data_ptr() == m.__cuda_array_interface__["data"][0]  # a view of the matrix, not a copy
    np.testing.assert_array_equal(t.cpu().numpy().astype(bool), want)
    np.testing.assert_array_equal(t.cpu().numpy().astype(bool), m.to_host())
    # the view keeps the buffer alive after the matrix object is dropped
    del m
    gc.collect()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(t.cpu().numpy().astype(bool), want)

    m = a.to_device().commutes_with_device(b.to_device())
    cap = m.__dlpack__(max_version=(1, 0))  # an unconsumed capsule is freed with it
    del cap
    gc.collect()
    with pytest.raises(BufferError, match="copy=True"):
        m.__dlpack__(max_version=(1, 0), copy=True)
    with pytest.raises(BufferError, match=r"max_version >= \(1, 0\)"):
        m.__dlpack__()
    with pytest.raises(BufferError, match=r"max_version >= \(1, 0\)"):
        m.__dlpack__(max_version=(0, 8))
    with pytest.raises(ValueError, match="stream=0 is ambiguous"):
        m.__dlpack__(stream=0, max_version=(1, 0))
    with pytest.raises(ValueError, match="non-negative"):
        m.__dlpack__(stream=-1, max_version=(1, 0))
    with pytest.raises(TypeError, match="stream must be None or an integer"):
        m.__dlpack__(stream="s", max_version=(1, 0))
    with pytest.raises(ValueError, match=r"\(major, minor\) tuple"):
        m.__dlpack__(max_version=(1,))
    with pytest.raises(ValueError, match="uint32"):
        m.__dlpack__(max_version=(-1, 0))
    # an explicit copy through torch is allowed (torch copies after importing the view)
    c = torch.from_dlpack(m, copy=False)
    assert c.data_ptr() == m.__cuda_array_interface__["data"][0]


def test_device_errors():
    d = PauliSum.from_labels(["XX"]).to_device()
    with pytest.raises(ValueError, match="same num_qubits"):
        d.matmul(PauliSum.from_labels(["X"]).to_device())
    with pytest.raises(ValueError, match="ordinal"):
        PauliSum.from_labels(["X"]).to_device(device=999)
    with pytest.raises(RuntimeError, match="HIP"):
        PauliSum.from_labels(["X"]).to_device(backend="hip")


@pytest.mark.parametrize("op", ["simplify", "matmul"])
def test_large_host_operands_through_staging(oracle, op):
    """Host operands of 32 MiB or more go to the device through pinned staging
    (two 64 MiB buffers filled by several host threads while the DMA engine
    drains the other): simplify of 2.4 million terms on 100 qubits (x, z and
    the coefficients 38 MB each, a third of the keys repeated) and matmul with
    that operand on the left, built with the public from_packed, equal the
    oracle bit for bit."""
    from wolfgang_b200.workloads import klocal_operator

    rng = np.random.default_rng(641)
    T = 2_400_000
    _, x, z, c = klocal_operator(rng, 100, T, np.array([2, 3, 4]))
    x[2 * T // 3:], z[2 * T // 3:] = x[:T // 3], z[:T // 3]
    assert x.nbytes >= 32 << 20 and c.nbytes >= 32 << 20
    A = PauliSum.from_packed(100, x, z, c)
    if op == "simplify":
        got = A.simplify().to_packed()
        want = oracle.simplify(100, x, z, c)
    else:
        _, bx, bz, bc = klocal_operator(rng, 100, 3, np.array([1, 2]))
        got = A.matmul(PauliSum.from_packed(100, bx, bz, bc), max_intermediate_terms=3 * T).to_packed()
        want = oracle.matmul(100, (x, z, c), (bx, bz, bc), simplify=True)
    for g, w in zip(got, want):
        assert np.ascontiguousarray(g).tobytes() == np.ascontiguousarray(w).tobytes()


@pytest.mark.parametrize("n", [0, 20])
def test_large_host_result_narrow_words(oracle, n):
    """The large-result path with no mask words (0 qubits: only the
    coefficient vector is filled) and with one word: raw products of 4,096 x
    1,100 terms (4.5e6 terms, 72 MB of coefficients) equal the oracle."""
    from tests.conftest import random_operator

    rng = np.random.default_rng(642 + n)
    A = random_operator(rng, n, 4096, 0.3)
    B = random_operator(rng, n, 1100, 0.3)
    hA = PauliSum.from_packed(n, A[1], A[2], A[3])
    hB = PauliSum.from_packed(n, B[1], B[2], B[3])
    got = hA.matmul(hB, simplify=False, max_intermediate_terms=4096 * 1100).to_packed()
    want = oracle.matmul(n, A[1:], B[1:], simplify=False)
    assert len(got[2]) * 16 > 64 << 20
    for g, w in zip(got, want):
        assert np.ascontiguousarray(g).tobytes() == np.ascontiguousarray(w).tobytes()


@pytest.mark.parametrize("simplify", [True, False])
def test_large_host_result_through_public_matmul(oracle, simplify):
    """A host result above 64 MB takes the large-result path (storage reserved,
    each vector grown by appending the downloaded chunks piece by piece behind
    fault-ahead helpers): the public PauliSum.matmul result equals the oracle
    bit for bit."""
    from wolfgang_b200.workloads import klocal_operator

    rng = np.random.default_rng(640)
    A = klocal_operator(rng, 100, 4096, np.array([2, 3, 4]))
    B = klocal_operator(rng, 100, 2300, np.array([2, 3, 4]))  # 9.4e6 products: each vector spans many 2 MiB pieces and 8 MiB chunks
    hA = PauliSum._from_packed(100, A[1], A[2], A[3])
    hB = PauliSum._from_packed(100, B[1], B[2], B[3])
    x, z, c = hA.matmul(hB, simplify=simplify, max_intermediate_terms=len(A[3]) * len(B[3]))._packed()
    want = oracle.matmul(100, A[1:], B[1:], simplify=simplify)
    assert len(c) * 48 > 64 << 20
    for got, w in zip((x, z, c), want):
        assert np.ascontiguousarray(got).tobytes() == np.ascontiguousarray(w).tobytes()
