"""Pins the CPU oracle against the reference's own known-answer cases.

Each case reproduces a reference test (seeded input, shape, tolerance) from
tests/golden/kat_cases.npz (see make_golden.py) and checks the oracle the way
that test checks the library: max complex |difference| against the DFT within
the test's tolerance, for both executors.  CPU only.
"""
import numpy as np
import pytest

from oracle.oracle import OracleContext, plan_twiddles
from oracle import fp64

C2C_CASES = (["single_thread_n8_b3", "prepared_n64_b4", "stockham_n256_b128_s1337",
              "stockham_n256_b128_s2337", "twiddle_meta_n16_b5", "consensus_n8_b3"]
             + [f"extended_n{N}_b{B}" for N in (2, 4, 8, 16, 32) for B in (1, 3, 16)])


def _maxabs(a, b):
    return float(np.max(np.abs(np.asarray(a, np.complex128) - np.asarray(b, np.complex128))))


@pytest.mark.parametrize("case", C2C_CASES)
@pytest.mark.parametrize("kernel", [1, 2])
def test_oracle_matches_reference_test_dft(kat, case, kernel):
    x = kat[case + "__input"]
    exp = kat[case + "__expected"]
    tol = float(kat[case + "__tol"][0])
    N = x.shape[1]
    ok, y, _ = OracleContext(N=N, kernel=kernel).fft_columns(x)
    assert ok
    assert _maxabs(y, exp) <= tol


def test_oracle_roundtrip_n16(kat):
    # tests/fftfree_tests.cpp:176-220: forward then inverse, error < 1e-5
    x = kat["roundtrip_n16_b8__input"]
    _, y, _ = OracleContext(N=16, inverse=0).fft_columns(x)
    _, z, _ = OracleContext(N=16, inverse=1).fft_columns(y)
    assert _maxabs(z, x) < 1e-5


@pytest.mark.parametrize("N", [1, 2, 4, 8, 16])
def test_oracle_multin_metadata_finite(kat, N):
    # tests/fftfree_tests.cpp:1273-1351: CT with all seven kinds, finite output
    x = kat[f"multin_meta_n{N}__input"]
    S = int(np.log2(N))
    tw = max(sum(1 << s for s in range(S)), 1)
    meta = {"Twiddle": tw, "LayoutMap": N}
    if S > 0:
        meta.update({"StageSnapshot": N * S, "StageParams": S, "ButterflyPairs": N * S,
                     "StageInvariant": S, "TwiddleIndexMap": N * S})
    ok, y, bufs = OracleContext(N=N, kernel=1).fft_columns(x, meta)
    assert ok and np.all(np.isfinite(y.view(np.float32)))
    assert _maxabs(y, kat[f"multin_meta_n{N}__expected"]) < 1e-4


def test_oracle_plain_fft_cffi(kat):
    # tests/cffi_stft_compare_test.cpp:344-404 (R2C, full spectrum, CT)
    pcm = kat["cffi_plain_fft__input"]
    ctx = OracleContext(N=1024, transform=1, pad_mode=1)
    n, re, im, mag = ctx.execute_batched(pcm, pad_mode=1)
    assert n == 1
    got = re[0] + 1j * im[0]
    assert _maxabs(got, kat["cffi_plain_fft__expected"]) <= 1e-4
    assert np.allclose(mag[0], np.abs(got), rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("kernel", [0, 2])
def test_oracle_batched_stft_cffi(kat, kernel):
    # tests/cffi_stft_compare_test.cpp:406-475 (N=W=512, H=128, Hann, R2C)
    pcm = kat["cffi_batched_stft__input"]
    N, W, H, frames = (int(v) for v in kat["cffi_batched_stft__meta"])
    ctx = OracleContext(N=N, window=W, hop=H, transform=1, pad_mode=1, kernel=kernel,
                        apply_windows=1, analysis_kind=1, synthesis_kind=1)
    n, re, im, _ = ctx.execute_batched(pcm, pad_mode=1)
    assert n == frames
    assert _maxabs(re + 1j * im, kat["cffi_batched_stft__expected"]) <= 1e-4


def test_consensus_metadata_structure(kat):
    # tests/fftfree_tests.cpp:921-1086: both executors agree, layout maps are
    # permutations, twiddle metadata equals the plan table.
    x = kat["consensus_n8_b3__input"]
    N, S = 8, 3
    meta = {"Twiddle": 7, "LayoutMap": N, "StageSnapshot": N * S, "StageParams": S,
            "ButterflyPairs": N * S, "StageInvariant": S, "TwiddleIndexMap": N * S}
    ok1, y1, m1 = OracleContext(N=N, kernel=1).fft_columns(x, meta)
    ok2, y2, m2 = OracleContext(N=N, kernel=2).fft_columns(x, meta)
    assert ok1 and ok2
    tol = 20e-5
    assert _maxabs(y1, y2) <= tol
    for m in (m1, m2):
        lay = np.rint(m["LayoutMap"].real).astype(int)
        assert sorted(lay.tolist()) == list(range(N))
    W = plan_twiddles(N)
    for s in range(S):
        mm = 1 << s
        step = N // (2 * mm)
        for j in range(mm):
            assert abs(m1["Twiddle"][mm - 1 + j] - W[j * step]) <= tol
    assert _maxabs(m1["Twiddle"], m2["Twiddle"]) <= tol


def test_undersized_metadata_rejected():
    # writers throw std::invalid_argument on short buffers (eigen_fft.hpp:1551-1553)
    x = np.zeros((1, 8), np.complex64)
    ok, _, _ = OracleContext(N=8, kernel=1).fft_columns(x, {"ButterflyPairs": 8})
    assert not ok


def test_fp64_oracle_agrees(kat):
    x = kat["stockham_n256_b128_s1337__input"]
    ctx = OracleContext(N=256, kernel=2)
    _, y, _ = ctx.fft_columns(x)
    assert fp64.rel_l2(y, fp64.fft_columns(ctx, x)) < 1e-6
