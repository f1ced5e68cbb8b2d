"""The autotuner's host side (no GPU): mode, and the cache's text form.

The cache maps a shape class (operation, mask words, log2 sizes) to the index
of the candidate tile / schedule that measured fastest; it moves between
processes as text lines "<op> <words> <a> <b> <choice>".
"""

from __future__ import annotations

import pytest

from wolfgang_b200 import capi


@pytest.fixture()
def tuner():
    mode = capi.autotune_mode()
    capi.autotune_clear()
    yield capi
    capi.autotune_clear()
    capi.autotune_mode(mode)


def test_mode_round_trip(tuner):
    assert tuner.autotune_mode(capi.WG_TUNE_OFF) == capi.WG_TUNE_OFF
    assert tuner.autotune_mode(capi.WG_TUNE_SEARCH) == capi.WG_TUNE_SEARCH
    assert tuner.autotune_mode(capi.WG_TUNE_CACHED) == capi.WG_TUNE_CACHED
    with pytest.raises(ValueError, match="autotune mode"):
        tuner.autotune_mode(7)


def test_import_export_round_trip(tuner):
    text = "commute 2 18 18 2\nbucket 2 30 0 4\n# a comment\n\ngroup_qwc 2 18 0 1\ngroup_full 1 15 0 3\n"
    tuner.autotune_import(text)
    lines = sorted(tuner.autotune_export().splitlines())
    assert lines == sorted(["commute 2 18 18 2", "bucket 2 30 0 4", "group_qwc 2 18 0 1", "group_full 1 15 0 3"])
    tuner.autotune_import("commute 2 18 18 0\n")  # a class is replaced, not duplicated
    assert "commute 2 18 18 0" in tuner.autotune_export().splitlines()
    assert len(tuner.autotune_export().splitlines()) == 4
    tuner.autotune_clear()
    assert tuner.autotune_export() == ""


@pytest.mark.parametrize("line,msg", [
    ("commute 2 18 18", "expected"),
    ("commute 2 18 18 1 9", "expected"),
    ("transpose 1 1 1 0", "unknown operation"),
    ("commute 2 18 18 5", "out of range"),   # five commutation candidates: 0-4
    ("group_qwc 1 10 0 3", "out of range"),  # three qwc chunk lengths
    ("bucket 1 70 0 1", "out of range"),
])
def test_import_rejects_bad_lines(tuner, line, msg):
    with pytest.raises(ValueError, match=msg):
        tuner.autotune_import(line + "\n")
    assert tuner.autotune_export() == ""  # a rejected text adds nothing
