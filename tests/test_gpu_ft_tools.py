"""The GPU grid pipeline (ft_apply_complex_pipeline / ft_apply_polar_pipeline)
against the reference's own ft_tools.hpp: the committed fixtures, and (where
oracle/_ref is present) random grids of larger sizes."""
import os

import numpy as np
import pytest
import torch

from tests.golden.make_ft_golden import CASES
from tests.helpers import assert_close

pytestmark = pytest.mark.gpu

api = pytest.importorskip("fftfree_b200.api")
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# Products and sums follow the reference's order; sin / cos / atan2 / hypot /
# exp / pow are CUDA's, a few ulp from the host's, which can move a
# quantizer cell across a rounding boundary (one magnitude step); sums over a
# whole axis are FP64 here against the reference's running float sums.
# Measured worst case on 257 x 513 grids: 5.7e-6.
TOL = 1e-5


def _structs(spec, plan, quant, contrast):
    return (api.FtGridSpec(*spec) if spec else None, api.FtResamplePlan(*plan) if plan else None,
            api.FtQuantizerConfig(*quant) if quant else None, api.FtContrastConfig(*contrast) if contrast else None)


def _compare(polar, ga, gb, ra, rb, what):
    if polar:
        assert_close(ga, ra, TOL, what + " magnitude")
        assert_close(ga * np.exp(1j * gb.astype(np.float64)), ra * np.exp(1j * rb.astype(np.float64)), TOL,
                     what + " value")
    else:
        assert_close(ga + 1j * gb, ra + 1j * rb, TOL, what)


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(REPO, "tests", "golden", "ft_tools_cases.npz"))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("device", [False, True])
def test_pipeline_matches_reference_fixture(gold, case, device):
    name, polar, T, F, spec, plan, quant, contrast = case
    a = gold[name + "/a"].copy()
    b = gold[name + "/b"].copy()
    if device:
        da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        ok = api.ft_apply_pipeline(da, db, T, F, *_structs(spec, plan, quant, contrast), polar=bool(polar))
        torch.cuda.synchronize()
        ga, gb = da.cpu().numpy(), db.cpu().numpy()
    else:
        ok = api.ft_apply_pipeline(a, b, T, F, *_structs(spec, plan, quant, contrast), polar=bool(polar))
        ga, gb = a, b
    assert ok == int(gold[name + "/ok"])
    if not ok:
        assert np.array_equal(ga, gold[name + "/a"]) and np.array_equal(gb, gold[name + "/b"])
        return
    _compare(polar, ga, gb, gold[name + "/ra"], gold[name + "/rb"], name)


def test_pipeline_argument_checks():
    a = np.zeros(16, np.float32)
    assert api.ft_apply_pipeline(a, None, 4, 4) == 0
    assert api.ft_apply_pipeline(a, a.copy(), 0, 4) == 0
    assert api.ft_apply_pipeline(a, a.copy(), 4, -1, polar=True) == 0


@pytest.mark.parametrize("polar", [False, True])
@pytest.mark.parametrize("kt,kf", [(3, 3), (0, 7), (9, 0), (0, 0)])
def test_pipeline_random_grids_against_reference(polar, kt, kf):
    from oracle import ft_tools as ft
    if not ft.available():
        pytest.skip("oracle/_ref not built")
    T, F = 257, 513
    rng = np.random.default_rng(kt * 31 + kf + polar)
    if polar:
        a = rng.uniform(0, 3, (T, F)).astype(np.float32)
        b = rng.uniform(-np.pi, np.pi, (T, F)).astype(np.float32)
    else:
        a = rng.standard_normal((T, F)).astype(np.float32)
        b = rng.standard_normal((T, F)).astype(np.float32)
    spec, plan, quant, contrast = (0.0, 0.0, 1.0, 21.533203125), (2, 2, 2, 2, 1), (1, 110.0, 0.02, 0.6, 5.0), \
        (1, kt, kf, 0.01, 0.6, 0.9, 1)
    ok, ra, rb = ft.apply(a, b, T, F, ft.GridSpec(*spec), ft.ResamplePlan(*plan), ft.QuantizerConfig(*quant),
                          ft.ContrastConfig(*contrast), polar=polar)
    ga, gb = a.copy(), b.copy()
    assert api.ft_apply_pipeline(ga, gb, T, F, *_structs(spec, plan, quant, contrast), polar=polar) == ok == 1
    _compare(polar, ga, gb, ra, rb, f"random {T}x{F}")
