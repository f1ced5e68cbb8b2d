"""The oracle reproduces the committed golden vectors (made by the reference core).

The fixtures under tests/golden/ were produced by tests/golden/make_golden.py,
which runs the reference's own C++ core compiled from its sources; they pin the
oracle wherever that library is absent.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("name", ["simplify_w1_dups", "simplify_w2_rtol", "simplify_w3", "simplify_cull"])
def test_simplify_golden(oracle, name):
    g = load(name)
    got = oracle.simplify(int(g["n"]), g["x"], g["z"], g["c"], float(g["atol"]), float(g["rtol"]))
    for a, b in zip(got, (g["out_x"], g["out_z"], g["out_c"])):
        assert same_bits(a, b)


@pytest.mark.parametrize("name", ["matmul_w1_raw", "matmul_w1", "matmul_w1_fused", "matmul_w2_fused",
                                  "matmul_config2_slice"])
def test_matmul_golden(oracle, name):
    g = load(name)
    got = oracle.matmul(int(g["n"]), (g["lx"], g["lz"], g["lc"]), (g["rx"], g["rz"], g["rc"]),
                        simplify=bool(g["simplify"]))
    for a, b in zip(got, (g["out_x"], g["out_z"], g["out_c"])):
        assert same_bits(a, b)


@pytest.mark.parametrize("name", ["commute_w1", "commute_w2"])
def test_commute_golden(oracle, name):
    g = load(name)
    assert np.array_equal(oracle.commutes(int(g["n"]), (g["lx"], g["lz"]), (g["rx"], g["rz"])), g["flags"])


@pytest.mark.parametrize("name", ["group_w1", "group_w2"])
@pytest.mark.parametrize("mode", ["qwc", "full"])
def test_group_golden(oracle, name, mode):
    g = load(name)
    groups = oracle.group_commuting(int(g["n"]), g["x"], g["z"], mode)
    assert [len(k) for k in groups] == list(g[f"{mode}_sizes"])
    order = np.concatenate(groups)
    assert same_bits(g["x"][order], g[f"{mode}_x"])
    assert same_bits(g["c"][order], g[f"{mode}_c"])


@pytest.mark.parametrize("name", ["expect_c128", "expect_c64", "expect_diag"])
def test_expectation_golden(oracle, name):
    g = load(name)
    assert oracle.expectation(int(g["n"]), g["x"], g["z"], g["c"], g["psi"]) == complex(g["value"])


@pytest.mark.parametrize("name", ["zcounts_w1", "zcounts_w2"])
def test_z_counts_golden(oracle, name):
    g = load(name)
    got = oracle.expectation_z_counts(int(g["n"]), g["x"], g["z"], g["c"], g["packed"], g["counts"])
    assert got == complex(g["value"])
