"""bench.py's isolation of the reference's CPU timings (no GPU needed): a
function run in a child process returns its result through JSON, and a
child that dies or fails yields None (the bench then reports the reference
as unavailable instead of ending)."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_child_returns_the_result():
    peak, kind = bench._in_child("_peaks", attempts=1, timeout_s=120.0)
    assert kind in ("measured", "fallback") and peak > 0


def test_child_failure_is_none(capsys):
    assert bench._in_child("no_such_function", attempts=2, timeout_s=120.0) is None
    err = capsys.readouterr().err
    assert err.count("no_such_function: attempt") == 2


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref")), reason="reference build absent")
def test_reference_griffin_lim_in_child():
    r = bench._in_child("_ref_griffin_lim", attempts=2, timeout_s=300.0, N=256, H=64, F=64)
    assert r is not None
    assert r.get("kind") == "reference" or "unavailable" in r
