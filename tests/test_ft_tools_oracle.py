"""The grid-pipeline checker (the reference's own ft_tools_cffi.cpp built
into oracle/_ref/) reproduces the committed fixtures, and its shape rule (CPU
only; skipped where the reference tree was not available to build it)."""
import os

import numpy as np
import pytest

from oracle import ft_tools as ft
from tests.golden.make_ft_golden import CASES, structs

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.skipif(not ft.available(), reason="oracle/_ref not built (needs the reference tree)")


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(REPO, "tests", "golden", "ft_tools_cases.npz"))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_reference_reproduces_fixture(gold, case):
    name, polar, T, F, spec, plan, quant, contrast = case
    ok, ra, rb = ft.apply(gold[name + "/a"], gold[name + "/b"], T, F, *structs(spec, plan, quant, contrast),
                          polar=bool(polar))
    assert ok == int(gold[name + "/ok"])
    assert np.array_equal(ra, gold[name + "/ra"]) and np.array_equal(rb, gold[name + "/rb"])


def test_shape_mismatch_leaves_arrays():
    a = np.arange(64, dtype=np.float32)
    b = -a
    ok, ra, rb = ft.apply(a, b, 8, 8, plan=ft.ResamplePlan(2, 1, 3, 1, 1))
    assert ok == 0 and np.array_equal(ra, a) and np.array_equal(rb, b)
