"""FP64 restatement of the magnitude STFT and of its gradient.

TEST INFRASTRUCTURE ONLY: the checker of the GPU adjoint kernel, never a
product path.

Forward: the framing of fft_execute_batched (fft_cffi.cpp:765-791: frame f
is pcm[f*H .. f*H + W) times the analysis window, zero beyond the signal end
and from W up to N; frame count fft_cffi.cpp:710-750), a full-length DFT,
bins 0..N/2 (R2C half spectrum, DC and Nyquist imag cleared as in
eigen_fft.hpp:2544-2554) and |X| (reduce_magnitude, fft_cffi.cpp:813-824).

Gradient of sum(g * |X|) with respect to the signal -- no counterpart in the
reference, derived here: with V[k] = g[k] X[k] / |X[k]| (0 where |X| = 0),
  dL/ds[n] = Re sum_{k=0}^{N/2} V[k] e^{+2 pi i k n / N}
and dL/dx[t] = sum over frames f covering t of w[t - fH] dL/ds_f[t - fH].
The spectrum sum is evaluated with numpy's float64 inverse real FFT.
"""
from __future__ import annotations

import numpy as np


def frame_count(length: int, N: int, W: int, H: int, pad_mode: int = 1) -> int:
    """fft_cffi.cpp:710-750 (W <= N)."""
    if length < W:
        return 1 if pad_mode == 1 else 0
    return 1 + (length - W) // H


def _frames(x: np.ndarray, N: int, W: int, H: int, win, frames: int):
    L = x.shape[-1]
    out = np.zeros(x.shape[:-1] + (frames, N), np.float64)
    cnts = []
    for f in range(frames):
        s = f * H
        cnt = max(0, min(W, L - s))
        seg = x[..., s: s + cnt].astype(np.float64)
        if win is not None:
            seg = seg * np.asarray(win, np.float64)[:cnt]
        out[..., f, :cnt] = seg
        cnts.append(cnt)
    return out, cnts


def stft_mag64(x: np.ndarray, N: int, W: int, H: int, win=None, pad_mode: int = 1) -> np.ndarray:
    """(signals, L) float -> (signals, frames, N/2+1) float64 |X|."""
    x = np.atleast_2d(np.asarray(x))
    F = frame_count(x.shape[-1], N, W, H, pad_mode)
    fr, _ = _frames(x, N, W, H, win, F)
    return np.abs(np.fft.rfft(fr, axis=-1))


def stft_mag_grad64(x: np.ndarray, g: np.ndarray, N: int, W: int, H: int, win=None,
                    pad_mode: int = 1) -> np.ndarray:
    """d(sum(g * |STFT x|))/dx in float64, shaped (signals, L)."""
    x = np.atleast_2d(np.asarray(x))
    S, L = x.shape
    F = frame_count(L, N, W, H, pad_mode)
    fr, cnts = _frames(x, N, W, H, win, F)
    X = np.fft.rfft(fr, axis=-1)
    mag = np.abs(X)
    g = np.asarray(g, np.float64).reshape(S, F, N // 2 + 1)
    V = np.where(mag > 0, g * X / np.where(mag > 0, mag, 1.0), 0.0)
    # Re sum_{k=0}^{N/2} V[k] e^{+i theta k n} = (N/2) irfft(V') with the two
    # edge bins doubled (irfft counts bins 1..N/2-1 twice, the edges once).
    Vp = V.copy()
    Vp[..., 0] *= 2.0
    Vp[..., -1] *= 2.0
    ds = np.fft.irfft(Vp, n=N, axis=-1) * (N / 2.0)
    if win is not None:
        ds = ds * np.asarray(win, np.float64)[:N] if len(win) >= N else ds * np.pad(np.asarray(win, np.float64), (0, N - len(win)))
    grad = np.zeros((S, L), np.float64)
    for f in range(F):
        cnt = cnts[f]
        grad[:, f * H: f * H + cnt] += ds[:, f, :cnt]
    return grad
