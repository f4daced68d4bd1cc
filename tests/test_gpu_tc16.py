"""The split-FP16 tensor-core variant of the multi-pass C2C transforms
(FFTFREE_TC16=1): same results as an FP64 DFT within the parity bar,
forward and inverse, for the sizes whose 256-point groups it computes."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

api = pytest.importorskip("fftfree_b200.api")


@pytest.mark.parametrize("N", [1 << 15, 1 << 16, 1 << 17])
@pytest.mark.parametrize("inverse", [0, 1])
def test_tc16_c2c(monkeypatch, N, inverse):
    B = 12
    rng = np.random.default_rng(3)
    z = (rng.standard_normal((B, N)) + 1j * rng.standard_normal((B, N))).astype(np.complex64)
    ref = np.fft.ifft(z.astype(np.complex128), axis=1) if inverse else np.fft.fft(z.astype(np.complex128), axis=1)
    dx = torch.from_numpy(z.view(np.float32)).cuda()
    errs = {}
    for tc in ("0", "1"):
        monkeypatch.setenv("FFTFREE_TC16", tc)
        c = api.FftContext.full_v2(N, kernel=2, inverse=inverse)
        dy = torch.empty_like(dx)
        assert c.execute_c2c(dx, dy, B) == 1
        got = dy.cpu().numpy().view(np.complex64).astype(np.complex128)
        errs[tc] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        c.close()
    print(f"N={N} inverse={inverse}: rel-L2 vs FP64 fp32 {errs['0']:.3e}, split-fp16 tensor core {errs['1']:.3e}")
    assert errs["1"] <= 1e-5 * math.log2(N)
    assert errs["0"] <= 1e-5 * math.log2(N)


@pytest.mark.parametrize("B", [1, 8, 13, 4096])
@pytest.mark.parametrize("inverse", [0, 1])
def test_tc05_c2c256(monkeypatch, B, inverse):
    # FFTFREE_TC16=2: the 256-point transforms on the tcgen05 tensor cores
    # (k_tc05.cu), against an FP64 DFT at the parity bar and beside the FP32
    # engine; transforms of very different scale keep their own precision
    # (per-transform power-of-two scaling before each FP16 split)
    N = 256
    rng = np.random.default_rng(B + 10 * inverse)
    z = (rng.standard_normal((B, N)) + 1j * rng.standard_normal((B, N))).astype(np.complex64)
    if B >= 8:
        z[1] *= np.float32(1e20)
        z[2] *= np.float32(1e-20)
        z[3] = 0
    ref = np.fft.ifft(z.astype(np.complex128), axis=1) if inverse else np.fft.fft(z.astype(np.complex128), axis=1)
    dx = torch.from_numpy(z.view(np.float32)).cuda()
    got = {}
    for tc in ("0", "2"):
        monkeypatch.setenv("FFTFREE_TC16", tc)
        c = api.FftContext.full_v2(N, kernel=2, inverse=inverse)
        dy = torch.full_like(dx, float("nan"))
        assert c.execute_c2c(dx, dy, B) == 1
        got[tc] = dy.cpu().numpy().view(np.complex64).astype(np.complex128)
        c.close()
    for tc, g in got.items():
        for b in range(B):
            den = np.linalg.norm(ref[b])
            err = np.linalg.norm(g[b] - ref[b]) / den if den > 0 else np.linalg.norm(g[b])
            assert err <= 1e-5 * math.log2(N), (tc, b, err)
