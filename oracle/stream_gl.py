"""CPU restatement of the reference's host drivers over the batched transforms:
the streaming STFT / ISTFT buffers (fft_cffi.cpp:1342-1742), Griffin-Lim
(phase_infer.hpp:68-210 behind fft_cffi.cpp:2176-2248) and the two phase
inference modes (phase_infer.hpp:35-65, fft_cffi.cpp:2083-2168).

TEST INFRASTRUCTURE ONLY: the checker of the GPU library's streaming, phase
and Griffin-Lim entry points.  Every transform goes through the C oracle
(``OracleContext``), every host step is restated here in float32 numpy in the
reference's order of operations.
"""
from __future__ import annotations

import numpy as np

from .oracle import OracleContext

GL_DEFAULT_SEED = 0x47D7BFAD
FLUSH_NONE, FLUSH_PARTIAL, FLUSH_FINAL = 0, 1, 2  # fft_cffi.hpp:316-320
COLA_NORMALIZE = 1


def mt19937_uniform_float(count: int, seed: int, a: float, b: float) -> np.ndarray:
    """``std::uniform_real_distribution<float>(a, b)`` over ``std::mt19937(seed)``
    as libstdc++ evaluates it: one 32-bit draw per value,
    u = float(x) / 2^32 (1 - 2^-24 when that rounds to 1), then u * (b - a) + a
    in float32.  numpy's legacy MT19937 seeding is the generator's init_genrand
    (Matsumoto and Nishimura, 1998), the seeding of ``std::mt19937(seed)``."""
    rs = np.random.RandomState(seed & 0xFFFFFFFF)
    x = rs.randint(0, 2 ** 32, size=count, dtype=np.uint64).astype(np.uint32)
    u = x.astype(np.float32) / np.float32(4294967296.0)
    one_minus = np.nextafter(np.float32(1), np.float32(0))
    u = np.where(u >= np.float32(1), one_minus, u).astype(np.float32)
    fa, fb = np.float32(a), np.float32(b)
    return (u * (fb - fa) + fa).astype(np.float32)


def griffin_lim(fwd: OracleContext, inv: OracleContext, mag: np.ndarray, frames: int, hop: int, half: bool,
                iterations: int = 0, pad_mode: int = 1, seed: int = GL_DEFAULT_SEED):
    """fft_griffin_lim (fft_cffi.cpp:2176-2248 -> phase_infer.hpp:69-210).
    Returns (ok, re, im) as (frames, bins) float32 arrays."""
    N = inv.N if inv.N > 0 else fwd.N
    if half != bool(inv.half_spectrum) or half != bool(fwd.half_spectrum):
        return 0, None, None
    if hop <= 0:
        hop = inv.hop if inv.hop > 0 else (fwd.hop if fwd.hop > 0 else N)
    plan_n = fwd.N if fwd.N else inv.N
    if fwd.N and inv.N and fwd.N != inv.N:
        plan_n = inv.N
    bins = plan_n // 2 + 1 if half else plan_n
    total = bins * frames
    ola_len = (frames - 1) * hop + plan_n
    iters = iterations if iterations > 0 else 32
    mag = np.asarray(mag, np.float32).reshape(-1)[:total]
    kpi = np.float32(np.pi)
    ang = mt19937_uniform_float(total, seed if seed else GL_DEFAULT_SEED, -kpi, kpi)
    re = (mag * np.cos(ang)).astype(np.float32)
    im = (mag * np.sin(ang)).astype(np.float32)
    for _ in range(iters):
        produced, fr = inv.execute_complex_batched(re, im, frames, max_frames=frames)
        if produced == 0:
            return 0, re.reshape(frames, bins), im.reshape(frames, bins)
        uf = min(produced, frames)
        ola = np.zeros(ola_len, np.float32)
        w = np.zeros(ola_len, np.float32)
        for f in range(uf):
            s = f * hop
            if s + plan_n > ola_len:
                break
            ola[s: s + plan_n] += fr[f, :plan_n]
            w[s: s + plan_n] += np.float32(1)
        nz = w > 0
        ola[nz] = ola[nz] / w[nz]
        ff, tr, ti, _ = fwd.execute_batched(ola, pad_mode=pad_mode, max_frames=frames)
        if ff == 0:
            return 0, re.reshape(frames, bins), im.reshape(frames, bins)
        n = min(ff, frames) * bins
        ph = np.arctan2(ti.reshape(-1)[:n], tr.reshape(-1)[:n]).astype(np.float32)
        re[:n] = mag[:n] * np.cos(ph)
        im[:n] = mag[:n] * np.sin(ph)
        if half:
            for f in range(min(ff, frames)):
                im[f * bins] = 0
                if plan_n % 2 == 0 and bins > 1:
                    im[f * bins + bins - 1] = 0
    return 1, re.reshape(frames, bins), im.reshape(frames, bins)


def spectral_convergence(mag: np.ndarray, fwd: OracleContext, inv: OracleContext, re, im, frames, hop):
    """|| |STFT(ISTFT(X))| - mag || / || mag || after one more inverse + OLA
    + forward pass of Griffin-Lim: the quantity its iterations reduce."""
    plan_n = inv.N
    bins = re.shape[-1]
    _, fr = inv.execute_complex_batched(re, im, frames, max_frames=frames)
    ola_len = (frames - 1) * hop + plan_n
    ola = np.zeros(ola_len, np.float64)
    w = np.zeros(ola_len, np.float64)
    for f in range(frames):
        ola[f * hop: f * hop + plan_n] += fr[f]
        w[f * hop: f * hop + plan_n] += 1
    ola = (ola / np.maximum(w, 1)).astype(np.float32)
    ff, _, _, m = fwd.execute_batched(ola, pad_mode=1, max_frames=frames)
    m = m.reshape(-1)[: ff * bins].astype(np.float64)
    ref = np.asarray(mag, np.float64).reshape(-1)[: ff * bins]
    return float(np.linalg.norm(m - ref) / max(np.linalg.norm(ref), 1e-30))


class StreamOracle:
    """Streaming buffers of one context (fft_cffi.cpp:1342-1742)."""

    def __init__(self, ctx: OracleContext):
        self.ctx = ctx
        self.buffer = np.zeros(0, np.float32)
        self.queue = np.zeros(0, np.float32)
        self.accum = None
        self.norm = None

    @property
    def W(self):
        return self.ctx.window if self.ctx.window > 0 else self.ctx.N

    @property
    def H(self):
        return self.ctx.hop if self.ctx.hop > 0 else self.W

    def available_frames(self):
        """fft_cffi.cpp:1368-1375."""
        if len(self.buffer) < self.W:
            return 0
        return 1 + (len(self.buffer) - self.W) // self.H

    def push_pcm(self, pcm, max_frames=0):
        """fft_stream_push_pcm (fft_cffi.cpp:1508-1595): frames of the backlog
        through execute_batched with pad_mode 2; returns (frames, re, im, mag)."""
        if pcm is not None and len(pcm):
            self.buffer = np.concatenate([self.buffer, np.asarray(pcm, np.float32)])
        frames = self.available_frames()
        if frames == 0:
            return 0, None, None, None
        if max_frames and frames > max_frames:
            frames = max_frames
        pcm_len = min(self.W + (frames - 1) * self.H, len(self.buffer))
        chunk = np.zeros(pcm_len, np.float32)
        for f in range(frames):
            s = f * self.H
            e = min(s + self.W, pcm_len)
            src = self.buffer[s: e]
            chunk[s: s + len(src)] = src
        n, re, im, mag = self.ctx.execute_batched(chunk, pad_mode=2, max_frames=frames)
        if n == 0:
            return 0, None, None, None
        self.buffer = self.buffer[n * self.H:]
        return n, re, im, mag

    def _cola_weight(self):
        if not self.ctx.apply_windows:
            return np.ones(self.ctx.N, np.float32)
        return (self.ctx.analysis_win * self.ctx.synthesis_win).astype(np.float32)

    def _emit(self, max_samples):
        take = len(self.queue)
        if max_samples and take > max_samples:
            take = max_samples
        out = self.queue[:take].copy()
        self.queue = self.queue[take:]
        return out

    def push_spectrum(self, re, im, frames, max_samples=0, flush_mode=FLUSH_NONE):
        """fft_stream_push_spectrum (fft_cffi.cpp:1597-1742): inverse frames
        overlap-added into the accumulator; hop samples (the whole frame on the
        last frame of a FINAL flush) leave per frame, divided by the summed
        window product under COLA normalisation.  Returns the emitted samples."""
        N = max(self.ctx.N, 1)
        if self.accum is None or len(self.accum) != N:
            self.accum = np.zeros(N, np.float32)
        use_norm = self.ctx.cola_mode == COLA_NORMALIZE
        if use_norm:
            if self.norm is None or len(self.norm) != N:
                self.norm = np.zeros(N, np.float32)
        else:
            self.norm = None
        queued = []
        if frames > 0:
            produced, fr = self.ctx.execute_complex_batched(re, im, frames, max_frames=frames)
            produced = min(produced, frames)
            wgt = self._cola_weight()
            for f in range(produced):
                self.accum += fr[f]
                if use_norm:
                    self.norm += wgt
                emit = N if (flush_mode == FLUSH_FINAL and f + 1 == produced) else self.H
                emit = min(emit, N)
                s = self.accum[:emit].copy()
                if use_norm:
                    d = self.norm[:emit]
                    big = np.abs(d) > np.float32(1e-12)
                    s[big] = s[big] / d[big]
                queued.append(s)
                self.accum = np.concatenate([self.accum[emit:], np.zeros(emit, np.float32)])
                if use_norm:
                    self.norm = np.concatenate([self.norm[emit:], np.zeros(emit, np.float32)])
        if flush_mode == FLUSH_FINAL and frames == 0:
            s = self.accum.copy()
            if self.norm is not None:
                big = np.abs(self.norm) > np.float32(1e-12)
                s[big] = s[big] / self.norm[big]
            queued.append(s)
            self.accum[:] = 0
            if self.norm is not None:
                self.norm[:] = 0
        if queued:
            self.queue = np.concatenate([self.queue] + queued)
        return self._emit(max_samples)


def phase_linear(mag, frames, N, hop, half):
    """phase_infer.hpp:35-65: phi[f, k] = f * 2 pi k hop / N in float64."""
    bins = N // 2 + 1 if half else N
    hop = hop if hop > 0 else N
    mag = np.asarray(mag, np.float64).reshape(frames, bins)
    k = np.arange(bins)
    dphi = 2.0 * np.pi * (k % N) * hop / N
    re = np.empty((frames, bins), np.float32)
    im = np.empty((frames, bins), np.float32)
    phi = np.zeros(bins)
    for f in range(frames):
        re[f] = mag[f] * np.cos(phi)
        im[f] = mag[f] * np.sin(phi)
        phi = phi + dphi
    return re, im


def phase_min(mag, frames, N, half):
    """fft_cffi.cpp:2100-2160: minimum phase from the real cepstrum; the two
    N-point transforms are the oracle's column transforms (inverse, then
    forward), every step in float32."""
    bins = N // 2 + 1 if half else N
    mag = np.asarray(mag, np.float32).reshape(frames, bins)
    eps = np.float32(1e-20)
    lg = np.log(np.maximum(eps, mag)).astype(np.float32)
    spec = np.zeros((frames, N), np.complex64)
    spec[:, 0] = lg[:, 0]
    if half:
        for k in range(1, N // 2):
            spec[:, k] = lg[:, k]
            spec[:, N - k] = lg[:, k]
        if N % 2 == 0:
            spec[:, N // 2] = lg[:, N // 2]
    else:
        spec[:, 1:] = lg[:, 1:N]
    ok, t, _ = OracleContext(N=N, inverse=1).fft_columns(spec)
    assert ok
    t[:, 1:(N + 1) // 2] *= np.float32(2)
    t[:, N // 2 + 1:] = 0
    ok, s, _ = OracleContext(N=N, inverse=0).fft_columns(t)
    assert ok
    a = np.exp(s.real[:, :bins].astype(np.float32))
    ph = s.imag[:, :bins].astype(np.float32)
    return (a * np.cos(ph)).astype(np.float32), (a * np.sin(ph)).astype(np.float32)
