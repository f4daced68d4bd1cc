"""Regenerate tests/golden/kat_cases.npz.

The reference's tests hold no stored vectors: each case draws its input from a
seeded std::mt19937 / std::mt19937_64 + std::normal_distribution and compares
the library against a DFT (Eigen::FFT) within a stated tolerance.  This script
reproduces those inputs bit for bit with kat_inputs.cpp (libstdc++ generators,
same seeds, same draw order), computes the float64 DFT that stands in for the
test's DFT, and stores input, expected output and the test's own tolerance per
case.  Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _load(d, name):
    return np.fromfile(os.path.join(d, name + ".f32"), dtype=np.float32)


def _cmatrix(flat, N, B):
    """Interleaved (r, c) row-major draw -> (B, N) complex64 transforms."""
    z = flat.view(np.complex64).reshape(N, B)
    return np.ascontiguousarray(z.T)


def main() -> int:
    sys.path.insert(0, REPO)
    from oracle import fp64  # noqa: F401  (shared helpers; FP64 math below)

    cases = {}
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "kat_inputs")
        subprocess.run(["g++", "-O1", "-std=c++17", os.path.join(HERE, "kat_inputs.cpp"),
                        "-o", exe], check=True)
        subprocess.run([exe, td], check=True)

        def c2c_case(name, fname, N, B, tol, inverse_roundtrip=False, kind="c2c"):
            x = _cmatrix(_load(td, fname), N, B)
            exp = np.fft.fft(x.astype(np.complex128), axis=1)
            cases[name + "__input"] = x
            cases[name + "__expected"] = (x if inverse_roundtrip else exp).astype(np.complex64)
            cases[name + "__meta"] = np.array([N, B, int(inverse_roundtrip)], np.int64)
            cases[name + "__tol"] = np.array([tol], np.float64)

        # tests/fftfree_tests.cpp:176-220 roundtrip, tol 1e-5 (f32) on |x - ifft(fft(x))|
        c2c_case("roundtrip_n16_b8", "roundtrip_n16_b8", 16, 8, 1e-5, inverse_roundtrip=True)
        # :331-365 single-thread CT vs DFT, tol 10 * 1e-5
        c2c_case("single_thread_n8_b3", "single_thread_n8_b3_s1381", 8, 3, 1e-4)
        # :418-501 prepared transform, tol 10 * 1e-5
        c2c_case("prepared_n64_b4", "prepared_n64_b4", 64, 4, 1e-4)
        # :718-844 Stockham vs CT vs DFT, real-only inputs, tol 256 * 1e-5
        c2c_case("stockham_n256_b128_s1337", "stockham_n256_b128_s1337", 256, 128, 256e-5)
        c2c_case("stockham_n256_b128_s2337", "stockham_n256_b128_s2337", 256, 128, 256e-5)
        # :846-919 twiddle metadata capture, tol 10 * 1e-5
        c2c_case("twiddle_meta_n16_b5", "twiddle_meta_n16_b5_s2025", 16, 5, 1e-4)
        # :921-1086 seven-kind consensus, tol 20 * 1e-5
        c2c_case("consensus_n8_b3", "consensus_n8_b3_s2026", 8, 3, 20e-5)
        # :1088-1271 extended consensus, tol 50 * 1e-5
        for N in (2, 4, 8, 16, 32):
            for B in (1, 3, 16):
                c2c_case(f"extended_n{N}_b{B}", f"extended_n{N}_b{B}", N, B, 50e-5)
        # :1273-1351 multi-N metadata dump (finite-output check only)
        for N in (1, 2, 4, 8, 16):
            c2c_case(f"multin_meta_n{N}", f"multin_meta_n{N}", N, 3, float("inf"))

        # tests/cffi_stft_compare_test.cpp:344-404: fft_execute on N=1024, R2C,
        # full spectrum, no window; max-abs tolerance 1e-4.
        pcm = _load(td, "cffi_plain_fft_pcm")
        cases["cffi_plain_fft__input"] = pcm
        cases["cffi_plain_fft__expected"] = np.fft.fft(pcm.astype(np.float64)).astype(np.complex64)
        cases["cffi_plain_fft__tol"] = np.array([1e-4])
        # :406-475: fft_execute_batched, N=W=512, H=128, Hann (symmetric, W-1
        # denominator), R2C, full spectrum; max-abs tolerance 1e-4.
        pcm = _load(td, "cffi_batched_stft_pcm")
        W, H, N = 512, 128, 512
        n = np.arange(W)
        hann = (0.5 * (1.0 - np.cos(2.0 * np.pi * n / (W - 1)))).astype(np.float32)
        frames = 1 + (len(pcm) - W) // H
        fr = np.stack([pcm[f * H: f * H + W].astype(np.float64) * hann.astype(np.float64)
                       for f in range(frames)])
        cases["cffi_batched_stft__input"] = pcm
        cases["cffi_batched_stft__expected"] = np.fft.fft(fr, n=N, axis=1).astype(np.complex64)
        cases["cffi_batched_stft__tol"] = np.array([1e-4])
        cases["cffi_batched_stft__meta"] = np.array([N, W, H, frames], np.int64)

    out = os.path.join(HERE, "kat_cases.npz")
    np.savez_compressed(out, **cases)
    print("wrote", out, "cases:", len([k for k in cases if k.endswith("__input")]))
    return 0


if __name__ == "__main__":
    sys.exit(main())
