"""The CPU restatement of the streaming buffers, Griffin-Lim and phase
inference (CPU only): the initial-phase generator against libstdc++'s own
std::mt19937 + uniform_real_distribution<float>, and properties of the
restated drivers."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import stream_gl as sg
from oracle.oracle import OracleContext

_MT_SRC = r"""
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
int main(int argc, char** argv) {
  const unsigned seed = (unsigned)std::strtoul(argv[1], nullptr, 0);
  const int n = std::atoi(argv[2]);
  const float kPi = 3.14159265358979323846f;
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> d(-kPi, kPi);
  for (int i = 0; i < n; ++i) {
    const float v = d(rng);
    unsigned u;
    std::memcpy(&u, &v, 4);
    std::printf("%08x\n", u);
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def mt_prog(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("mt")
    src = os.path.join(d, "mt.cpp")
    exe = os.path.join(d, "mt")
    with open(src, "w") as f:
        f.write(_MT_SRC)
    subprocess.run([gxx, "-O2", "-o", exe, src], check=True)
    return exe


@pytest.mark.parametrize("seed", [sg.GL_DEFAULT_SEED, 1, 12345, 0xFFFFFFFF])
def test_initial_phases_match_libstdcxx(mt_prog, seed):
    n = 4000
    out = subprocess.run([mt_prog, str(seed), str(n)], capture_output=True, text=True, check=True).stdout.split()
    ref = np.array([int(x, 16) for x in out], np.uint32)
    got = sg.mt19937_uniform_float(n, seed, -np.float32(np.pi), np.float32(np.pi))
    assert np.array_equal(got.view(np.uint32), ref)


def _gl_ctx(N, H):
    fwd = OracleContext(N=N, transform=1, half_spectrum=1, window=N, hop=H, apply_windows=1, analysis_kind=1,
                        pad_mode=1)
    inv = OracleContext(N=N, inverse=1, transform=2, half_spectrum=1, window=N, hop=H, pad_mode=1)
    return fwd, inv


def test_griffin_lim_reduces_inconsistency():
    """More iterations give a smaller spectral inconsistency (the quantity
    Griffin-Lim descends) on the magnitude of a real signal."""
    N, H, frames = 64, 16, 24
    fwd, inv = _gl_ctx(N, H)
    t = np.arange((frames - 1) * H + N)
    x = (np.sin(0.21 * t) + 0.5 * np.sin(0.05 * t + 1.0)).astype(np.float32)
    n, _, _, mag = fwd.execute_batched(x, pad_mode=1, max_frames=frames)
    assert n == frames
    errs = []
    for iters in (1, 4, 16):
        ok, re, im = sg.griffin_lim(fwd, inv, mag, frames, H, True, iters)
        assert ok == 1
        np.testing.assert_allclose(np.hypot(re, im), mag, rtol=1e-5, atol=1e-6)
        errs.append(sg.spectral_convergence(mag, fwd, inv, re, im, frames, H))
    assert errs[0] > errs[1] > errs[2], errs


def test_griffin_lim_rejects_mismatched_half_spectrum():
    fwd, _ = _gl_ctx(64, 16)
    inv = OracleContext(N=64, inverse=1, half_spectrum=0, hop=16)
    ok, _, _ = sg.griffin_lim(fwd, inv, np.ones(5 * 33, np.float32), 5, 16, True, 2)
    assert ok == 0


def test_stream_chunks_equal_one_batch():
    """Frames produced by pushing a signal in ragged chunks equal the frames of
    one batched call over the whole signal."""
    N, H = 64, 24
    ctx = OracleContext(N=N, transform=1, half_spectrum=1, window=48, hop=H, apply_windows=1, analysis_kind=2)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, 1000).astype(np.float32)
    st = sg.StreamOracle(ctx)
    got = []
    pos = 0
    for c in [5, 100, 1, 48, 300, 7, 539]:
        n, re, im, _ = st.push_pcm(x[pos: pos + c])
        pos += c
        if n:
            got.append(re + 1j * im)
    got = np.concatenate(got)
    n, re, im, _ = ctx.execute_batched(x, pad_mode=2)
    assert got.shape[0] == n
    np.testing.assert_array_equal(got, re + 1j * im)


def test_stream_spectrum_final_flush_reconstructs():
    """push_spectrum with COLA normalisation and a FINAL flush returns the
    overlap-added inverse of a forward STFT: the signal itself."""
    N, H = 64, 16
    fwd = OracleContext(N=N, transform=1, half_spectrum=1, window=N, hop=H)
    inv = OracleContext(N=N, inverse=1, transform=2, half_spectrum=1, window=N, hop=H, cola_mode=1)
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, 15 * H + N).astype(np.float32)
    n, re, im, _ = fwd.execute_batched(x, pad_mode=2)
    st = sg.StreamOracle(inv)
    y = st.push_spectrum(re, im, n, flush_mode=sg.FLUSH_FINAL)
    assert len(y) == (n - 1) * H + N
    np.testing.assert_allclose(y, x[: len(y)], rtol=0, atol=2e-5)


def test_phase_min_keeps_magnitude():
    N, frames = 64, 5
    rng = np.random.default_rng(5)
    mag = rng.uniform(0.1, 2.0, (frames, N // 2 + 1)).astype(np.float32)
    re, im = sg.phase_min(mag, frames, N, True)
    np.testing.assert_allclose(np.hypot(re, im), mag, rtol=1e-4)


def test_phase_linear_advance():
    N, H, frames = 32, 8, 4
    mag = np.ones((frames, N // 2 + 1), np.float32)
    re, im = sg.phase_linear(mag, frames, N, H, True)
    ph = np.angle(re + 1j * im)
    k = np.arange(N // 2 + 1)
    want = np.angle(np.exp(1j * 2 * np.pi * k * H / N * 3))
    np.testing.assert_allclose(np.angle(np.exp(1j * (ph[3] - want))), 0, atol=1e-5)


def test_stream_spectrum_hop_beyond_frame():
    """A hop longer than the frame: each frame emits all of its N samples
    (the emit count is min(hop, N)), so the stream is the frames back to back."""
    N, H = 32, 48
    fwd = OracleContext(N=N, transform=1, half_spectrum=1, window=N, hop=N)
    inv = OracleContext(N=N, inverse=1, transform=2, half_spectrum=1, window=N, hop=H)
    rng = np.random.default_rng(6)
    x = rng.uniform(-1, 1, 5 * N).astype(np.float32)
    n, re, im, _ = fwd.execute_batched(x, pad_mode=2)
    assert n == 5
    st = sg.StreamOracle(inv)
    y = st.push_spectrum(re, im, n)
    assert len(y) == n * N
    np.testing.assert_allclose(y, x, rtol=0, atol=2e-5)


def test_griffin_lim_full_spectrum():
    """Full (non-half) spectra: the iterations keep the target magnitudes and
    leave the DC / Nyquist imaginary parts alone."""
    N, H, frames = 32, 8, 12
    fwd = OracleContext(N=N, transform=0, half_spectrum=0, window=N, hop=H, apply_windows=1, analysis_kind=1)
    inv = OracleContext(N=N, inverse=1, transform=0, half_spectrum=0, window=N, hop=H)
    t = np.arange((frames - 1) * H + N)
    x = np.sin(0.3 * t).astype(np.float32)
    n, _, _, mag = fwd.execute_batched(x, pad_mode=1, max_frames=frames)
    ok, re, im = sg.griffin_lim(fwd, inv, mag, frames, H, False, 3)
    assert ok == 1 and re.shape == (frames, N)
    np.testing.assert_allclose(np.hypot(re, im), mag, rtol=1e-5, atol=1e-6)
