"""FP64 restatement of the fftfree batched STFT/FFT semantics.

TEST INFRASTRUCTURE ONLY.  Same data flow as the float32 oracle
(fftfree_oracle.c) -- framing fft_cffi.cpp:765-791, hooks
eigen_fft.hpp:2484-2596, output copy fft_cffi.cpp:813-824, complex batch + OLA
fft_cffi.cpp:1042-1340 -- but every arithmetic step is float64 and the DFT is
numpy's float64 FFT.  It answers "how far is a float32 result from the exact
transform of the same float32 inputs" (windows are the same float32 taps).
"""
from __future__ import annotations

import numpy as np


def _mode(t: int) -> int:
    return t if 0 <= t <= 3 else 0


def pre_transform(ctx, X: np.ndarray) -> np.ndarray:
    """eigen_fft.hpp:2484-2533 (Cooley-Tukey executor only)."""
    N = ctx.N
    X = X.copy()
    m = _mode(ctx.transform)
    if m == 1:
        X.imag = 0.0
    elif m == 2 and ctx.half_spectrum:
        if ctx.store_polar:
            mag = X[:, : N // 2 + 1].real.copy()
            ph = X[:, : N // 2 + 1].imag.copy()
            X[:, : N // 2 + 1] = mag * np.cos(ph) + 1j * mag * np.sin(ph)
        X[:, 0] = X[:, 0].real
        X[:, N // 2] = X[:, N // 2].real
        if N // 2 > 1:
            X[:, N - np.arange(1, N // 2)] = np.conj(X[:, 1: N // 2])
    return X


def post_transform(ctx, X: np.ndarray) -> np.ndarray:
    """eigen_fft.hpp:2535-2596."""
    N = ctx.N
    X = X.copy()
    m = _mode(ctx.transform)
    r2c_half = (m == 1 and ctx.half_spectrum)
    if r2c_half:
        X[:, 0] = X[:, 0].real
        X[:, N // 2] = X[:, N // 2].real
        X[:, N // 2 + 1:] = 0
    upper = N // 2 + 1 if r2c_half else N
    if ctx.store_polar:
        v = X[:, :upper]
        X[:, :upper] = np.abs(v) + 1j * np.angle(v)
        return X
    if ctx.reduce_magnitude:
        X[:, :upper] = np.abs(X[:, :upper])
        return X
    if m == 2:
        X.imag = 0.0
    return X


def fft_columns(ctx, X: np.ndarray) -> np.ndarray:
    """(B, N) complex -> hooks + DFT (+1/N when inverse) in float64."""
    X = np.asarray(X, dtype=np.complex128).reshape(-1, ctx.N)
    if ctx.kernel != 2:
        X = pre_transform(ctx, X)
    Y = np.fft.ifft(X, axis=1) if ctx.inverse else np.fft.fft(X, axis=1)
    return post_transform(ctx, Y)


def frames_matrix(ctx, pcm: np.ndarray, frames: int) -> np.ndarray:
    N = ctx.N
    W = ctx.window or N
    H = ctx.hop or W
    pcm64 = np.asarray(pcm, dtype=np.float32).astype(np.float64)
    out = np.zeros((frames, N), np.complex128)
    win = np.asarray(ctx.analysis_win, np.float32).astype(np.float64)
    for f in range(frames):
        start = f * H
        cnt = min(W, len(pcm64) - start) if start < len(pcm64) else 0
        seg = pcm64[start: start + cnt]
        if ctx.apply_windows:
            seg = seg * win[:cnt]
        out[f, :cnt] = seg
    return out


def execute_batched(ctx, pcm: np.ndarray, pad_mode: int = 1, max_frames: int = 0):
    frames = ctx.frame_count(len(pcm), pad_mode, max_frames)
    if frames == 0:
        return 0, None, None, None
    Y = fft_columns(ctx, frames_matrix(ctx, pcm, frames))
    bins = ctx.bins
    v = Y[:, :bins]
    mag = v.real.copy() if ctx.store_polar else np.abs(v)
    return frames, v.real.copy(), v.imag.copy(), mag


def execute_complex_batched(ctx, in_real: np.ndarray, in_imag: np.ndarray, frames: int,
                            max_frames: int = 0):
    N = ctx.N
    bins = ctx.bins
    if max_frames and frames > max_frames:
        frames = max_frames
    X = np.zeros((frames, N), np.complex128)
    r = np.asarray(in_real, np.float32).astype(np.float64).reshape(-1, bins)[:frames]
    i = np.asarray(in_imag, np.float32).astype(np.float64).reshape(-1, bins)[:frames]
    X[:, :bins] = r + 1j * i
    if ctx.half_spectrum and _mode(ctx.transform) == 2:
        X[:, 0] = X[:, 0].real
        ny = N // 2
        if ny < bins:
            X[:, ny] = X[:, ny].real
        maxk = ny if bins > ny + 1 else bins - 1
        if maxk > 1:
            ks = np.arange(1, maxk)
            X[:, N - ks] = np.conj(X[:, ks])
    Y = fft_columns(ctx, X)
    s = Y.real.copy()
    if ctx.apply_windows:
        s = s * np.asarray(ctx.synthesis_win, np.float32).astype(np.float64)[None, :]
    if not ctx.apply_ola:
        return frames, s
    W = ctx.window if ctx.window > 0 else N
    H = ctx.hop if ctx.hop > 0 else W
    total = frames * N
    out = np.zeros(total)
    norm = np.zeros(total) if ctx.cola_mode == 1 else None
    if ctx.apply_windows:
        wgt = (np.asarray(ctx.analysis_win, np.float32).astype(np.float64)
               * np.asarray(ctx.synthesis_win, np.float32).astype(np.float64))
    else:
        wgt = np.ones(N)
    for f in range(frames):
        t0 = f * H
        t1 = min(t0 + N, total)
        if t1 > t0:
            out[t0:t1] += s[f, : t1 - t0]
            if norm is not None:
                norm[t0:t1] += wgt[: t1 - t0]
    if norm is not None:
        nz = norm > 1e-12
        out[nz] /= norm[nz]
    return frames, out.reshape(frames, N)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, np.float64 if not np.iscomplexobj(a) else np.complex128)
    b = np.asarray(b, np.float64 if not np.iscomplexobj(b) else np.complex128)
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)
