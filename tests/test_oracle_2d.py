"""The oracle's 2-D transform (axis-0 columns, transpose, axis-1 rows) against
numpy's float64 fft2 (CPU only)."""
import numpy as np
import pytest

from oracle.oracle import OracleContext, fft_2d
from tests.helpers import assert_close, tol_for


@pytest.mark.parametrize("rows,cols,batch", [(8, 16, 1), (64, 4, 3), (2, 256, 2), (128, 128, 1)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_oracle_2d_matches_fft2(rows, cols, batch, inverse):
    rng = np.random.default_rng(rows * 7 + cols + inverse)
    X = (rng.standard_normal((batch, cols, rows)) + 1j * rng.standard_normal((batch, cols, rows))).astype(
        np.complex64)
    ok, Y = fft_2d(OracleContext(N=rows, inverse=inverse), OracleContext(N=cols, inverse=inverse), X)
    assert ok
    A = X.astype(np.complex128).transpose(0, 2, 1)  # A[b, r, c]
    ref = np.fft.ifft2(A) if inverse else np.fft.fft2(A)
    assert_close(Y.transpose(0, 2, 1), ref, tol_for(rows * cols), "2-D")


def test_oracle_2d_rejects_mismatched_plan():
    X = np.zeros((1, 8, 16), np.complex64)
    ok, _ = fft_2d(OracleContext(N=8), OracleContext(N=16), X)
    assert not ok
