"""2-D transforms (fftfree_execute_2d) against the oracle's fft_inplace_2d
restatement, and bit-identical to the same two axes run as contiguous
batched transforms with an explicit transpose."""
import numpy as np
import pytest
import torch

from oracle.oracle import fft_2d
from tests.helpers import assert_close, ctx_kwargs, oracle_for, tol_for

pytestmark = pytest.mark.gpu

api = pytest.importorskip("fftfree_b200.api")


def _mats(batch, rows, cols, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((batch, cols, rows)) + 1j * rng.standard_normal((batch, cols, rows))).astype(
        np.complex64)


def _pair(rows, cols, kw0=None, kw1=None):
    k0 = ctx_kwargs(rows, **(kw0 or {}))
    k1 = ctx_kwargs(cols, **(kw1 or {}))
    return api.FftContext.full_v2(**k0), api.FftContext.full_v2(**k1), oracle_for(k0), oracle_for(k1)


@pytest.mark.parametrize("rows,cols,batch", [(2, 2, 1), (16, 64, 3), (64, 16, 2), (256, 256, 2), (1024, 512, 1),
                                             (4096, 64, 1), (8, 8192, 2), (32, 2048, 1), (2, 4096, 5),
                                             (64, 16384, 1), (4, 65536, 1), (16384, 8, 1)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_2d_matches_oracle(rows, cols, batch, inverse):
    c0, c1, o0, o1 = _pair(rows, cols, dict(inverse=inverse), dict(inverse=inverse))
    X = _mats(batch, rows, cols, rows + 3 * cols + inverse)
    out = np.zeros_like(X)
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), rows, cols, batch) == 1
    ok, ref = fft_2d(o0, o1, X)
    assert ok
    assert_close(out, ref, tol_for(rows * cols), "2-D")


@pytest.mark.parametrize("rows,cols", [(64, 128), (512, 1024), (16, 8192), (2048, 4)])
def test_2d_bit_identical_to_two_batched_passes(rows, cols):
    c0, c1, _, _ = _pair(rows, cols, dict(kernel=2), dict(kernel=2))
    batch = 2
    X = _mats(batch, rows, cols, 5)
    out = np.zeros_like(X)
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), rows, cols, batch) == 1
    y = np.zeros_like(X)
    assert c0.execute_c2c(X.view(np.float32), y.view(np.float32), batch * cols) == 1
    yt = np.ascontiguousarray(y.transpose(0, 2, 1))  # (batch, rows, cols): rows contiguous
    z = np.zeros_like(yt)
    assert c1.execute_c2c(yt.view(np.float32), z.view(np.float32), batch * rows) == 1
    want = np.ascontiguousarray(z.transpose(0, 2, 1))
    assert np.array_equal(out.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("kw0,kw1", [
    (dict(kernel=0, transform=1), dict(kernel=0, store_polar=1)),
    (dict(kernel=2, inverse=1, reduce_magnitude=1), dict(kernel=0, transform=2, half_spectrum=1, inverse=1)),
    (dict(kernel=0, transform=2, half_spectrum=1, inverse=1), dict(kernel=2)),
    (dict(kernel=2, store_polar=1), dict(kernel=0, transform=1)),
])
def test_2d_plan_hooks_match_oracle(kw0, kw1):
    rows, cols, batch = 128, 256, 2
    c0, c1, o0, o1 = _pair(rows, cols, kw0, kw1)
    # (A polar output of the first axis feeds its phases to the second one,
    # so only cases whose first-axis phases are well conditioned are used:
    # the phase of a real C2R output flips between -pi and pi with the sign of
    # a rounding-level imaginary part.)
    X = _mats(batch, rows, cols, 9)
    out = np.zeros_like(X)
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), rows, cols, batch) == 1
    ok, ref = fft_2d(o0, o1, X)
    assert ok
    if kw1.get("store_polar"):
        assert_close(out.real, ref.real, tol_for(rows * cols), "2-D polar magnitude")
        got = out.real * np.exp(1j * out.imag.astype(np.float64))
        want = ref.real * np.exp(1j * ref.imag.astype(np.float64))
        assert_close(got, want, tol_for(rows * cols), "2-D polar value")
    else:
        assert_close(out, ref, tol_for(rows * cols), "2-D")


@pytest.mark.parametrize("rows,cols", [(256, 512), (32, 16384)])
def test_2d_in_place_on_device(rows, cols):
    c0, c1, o0, o1 = _pair(rows, cols)
    X = _mats(3, rows, cols, 11)
    d = torch.from_numpy(X.view(np.float32).copy()).cuda()
    assert api.execute_2d(c0, c1, d, d, rows, cols, 3) == 1
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(np.complex64).reshape(X.shape)
    ok, ref = fft_2d(o0, o1, X)
    assert_close(got, ref, tol_for(rows * cols), "2-D in place")


def test_2d_argument_checks():
    c0, c1, _, _ = _pair(16, 32)
    X = _mats(1, 16, 32, 0)
    out = np.zeros_like(X)
    L = api.lib()
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), 32, 16, 1) == 0
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), 16, 32, 0) == 0
    assert L.fftfree_execute_2d(None, c1.handle, api._fp(X.view(np.float32)), api._fp(out.view(np.float32)), 16,
                                32, 1) == 0
