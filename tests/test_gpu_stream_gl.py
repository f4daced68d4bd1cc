"""Streaming buffers, Griffin-Lim and phase inference of the CUDA library
against their CPU restatement over the oracle (same contexts, same inputs)."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import stream_gl as sg
from tests.helpers import assert_close, ctx_kwargs, oracle_for, tol_for

pytestmark = pytest.mark.gpu

api = pytest.importorskip("fftfree_b200.api")
_fp = api._fp


def _gl_pair(N, H, window_kind=1):
    fk = ctx_kwargs(N, transform=1, half_spectrum=1, window=N, hop=H, apply_windows=1, analysis_kind=window_kind)
    ik = ctx_kwargs(N, inverse=1, transform=2, half_spectrum=1, window=N, hop=H)
    return (api.FftContext.full_v2(**fk), api.FftContext.full_v2(**ik), oracle_for(fk), oracle_for(ik))


def _signal(frames, H, N, seed):
    t = np.arange((frames - 1) * H + N)
    rng = np.random.default_rng(seed)
    return (np.sin(0.031 * t) + 0.4 * np.sin(0.17 * t + 0.5) + 0.05 * rng.standard_normal(t.size)).astype(
        np.float32)


def _gpu_gl(fc, ic, mag, frames, H, iters, seed, device_mag=False):
    bins = mag.shape[-1]
    re = np.zeros(frames * bins, np.float32)
    im = np.zeros(frames * bins, np.float32)
    m = torch.from_numpy(np.ascontiguousarray(mag)).cuda() if device_mag else np.ascontiguousarray(mag)
    ok = api.lib().fft_griffin_lim(fc.handle, ic.handle, _fp(m), frames, H, 1, iters, 1, seed, _fp(re), _fp(im))
    return ok, re.reshape(frames, bins), im.reshape(frames, bins)


@pytest.mark.parametrize("N,H,frames,iters", [(256, 64, 16, 1), (256, 64, 16, 4), (1024, 256, 12, 3),
                                              (64, 16, 40, 2)])
def test_griffin_lim_matches_oracle(N, H, frames, iters):
    fc, ic, fo, io = _gl_pair(N, H)
    x = _signal(frames, H, N, N + iters)
    n, _, _, mag = fo.execute_batched(x, pad_mode=1, max_frames=frames)
    assert n == frames
    ok, re, im = _gpu_gl(fc, ic, mag, frames, H, iters, 7)
    rok, rre, rim = sg.griffin_lim(fo, io, mag, frames, H, True, iters, 1, 7)
    assert ok == 1 and rok == 1
    # The initial phases are bit-identical; each iteration adds transform
    # rounding (rel-L2 <= 1e-5 log2 N per transform) and a few-ulp difference
    # of atan2/cos/sin, which the next projections carry forward.
    assert_close(re + 1j * im, rre + 1j * rim, 4 * iters * tol_for(N), "griffin-lim spectrum")
    np.testing.assert_allclose(np.hypot(re, im), mag, rtol=1e-5, atol=1e-5)
    assert np.all(im[:, 0] == 0) and np.all(im[:, -1] == 0)


def _gl_case(N, H, frames, iters, half=True, fwd_extra=None, seed=5):
    """GPU and oracle Griffin-Lim on the STFT magnitudes of a test signal."""
    fk = ctx_kwargs(N, transform=1, half_spectrum=1 if half else 0, window=N, hop=H, apply_windows=1,
                    analysis_kind=1, **(fwd_extra or {}))
    ik = ctx_kwargs(N, inverse=1, transform=2, half_spectrum=1 if half else 0, window=N, hop=H)
    fc, ic = api.FftContext.full_v2(**fk), api.FftContext.full_v2(**ik)
    fo, io = oracle_for(fk), oracle_for(ik)
    plain = oracle_for(ctx_kwargs(N, transform=1, half_spectrum=1 if half else 0, window=N, hop=H,
                                  apply_windows=1, analysis_kind=1))
    x = _signal(frames, H, N, N + iters + H)
    n, _, _, mag = plain.execute_batched(x, pad_mode=1, max_frames=frames)
    assert n == frames
    bins = mag.shape[-1]
    re = np.zeros(frames * bins, np.float32)
    im = np.zeros(frames * bins, np.float32)
    return fc, ic, fo, io, np.ascontiguousarray(mag), re, im


def _run_gl(fc, ic, mag, frames, H, half, iters, seed, re, im):
    return api.lib().fft_griffin_lim(fc.handle, ic.handle, _fp(mag), frames, H, 1 if half else 0, iters, 1, seed,
                                     _fp(re), _fp(im))


@pytest.mark.parametrize("N,H,frames,iters", [(64, 80, 10, 3), (128, 128, 9, 2), (256, 300, 6, 2)])
def test_griffin_lim_hop_at_or_beyond_frame(N, H, frames, iters):
    # H > N leaves samples no frame covers: the overlap-add runs over the
    # (frames-1)*H + N samples of the reference, zero in the gaps.
    fc, ic, fo, io, mag, re, im = _gl_case(N, H, frames, iters)
    assert _run_gl(fc, ic, mag, frames, H, True, iters, 11, re, im) == 1
    rok, rre, rim = sg.griffin_lim(fo, io, mag, frames, H, True, iters, 1, 11)
    assert rok == 1
    assert_close(re + 1j * im, (rre + 1j * rim).reshape(-1), 4 * iters * tol_for(N), "griffin-lim spectrum")


@pytest.mark.parametrize("N,H,frames,iters", [(256, 64, 12, 3), (64, 16, 20, 2)])
def test_griffin_lim_full_spectrum(N, H, frames, iters):
    # full-spectrum contexts: the projection runs in the STFT's general
    # (two-sided) epilogue
    fc, ic, fo, io, mag, re, im = _gl_case(N, H, frames, iters, half=False)
    assert mag.shape[-1] == N
    assert _run_gl(fc, ic, mag, frames, H, False, iters, 3, re, im) == 1
    rok, rre, rim = sg.griffin_lim(fo, io, mag, frames, H, False, iters, 1, 3)
    assert rok == 1
    assert_close(re + 1j * im, (rre + 1j * rim).reshape(-1), 4 * iters * tol_for(N), "griffin-lim spectrum")


@pytest.mark.parametrize("extra", [dict(store_polar=1), dict(reduce_magnitude=1)])
def test_griffin_lim_polar_forward_context(extra):
    # A forward context that stores polar values or magnitudes: the
    # projection reads its (re, im) outputs as the reference does, through
    # the separate projection kernel.
    N, H, frames, iters = 128, 32, 14, 2
    fc, ic, fo, io, mag, re, im = _gl_case(N, H, frames, iters, fwd_extra=extra)
    assert _run_gl(fc, ic, mag, frames, H, True, iters, 9, re, im) == 1
    rok, rre, rim = sg.griffin_lim(fo, io, mag, frames, H, True, iters, 1, 9)
    assert rok == 1
    # atan2 of (|X|, arg X) amplifies rounding near the branch cut less than
    # a spectrum would; compare as the other cases do
    assert_close(re + 1j * im, (rre + 1j * rim).reshape(-1), 4 * iters * tol_for(N), "griffin-lim spectrum")


def test_griffin_lim_contexts_on_one_stream():
    # both contexts on one caller stream: no cross-stream events, same result
    N, H, frames, iters = 256, 64, 16, 4
    fc, ic, fo, io, mag, re, im = _gl_case(N, H, frames, iters)
    assert _run_gl(fc, ic, mag, frames, H, True, iters, 7, re, im) == 1
    s = torch.cuda.Stream()
    fc.set_stream(s.cuda_stream)
    ic.set_stream(s.cuda_stream)
    re2, im2 = np.zeros_like(re), np.zeros_like(im)
    assert _run_gl(fc, ic, mag, frames, H, True, iters, 7, re2, im2) == 1
    assert np.array_equal(re, re2) and np.array_equal(im, im2)
    fc.set_stream(0)
    ic.set_stream(0)
    re3, im3 = np.zeros_like(re), np.zeros_like(im)
    assert _run_gl(fc, ic, mag, frames, H, True, iters, 7, re3, im3) == 1
    assert np.array_equal(re, re3) and np.array_equal(im, im3)


def test_griffin_lim_converges_and_device_magnitude():
    N, H, frames = 512, 128, 32
    fc, ic, fo, io = _gl_pair(N, H)
    x = _signal(frames, H, N, 3)
    _, _, _, mag = fo.execute_batched(x, pad_mode=1, max_frames=frames)
    errs = []
    for iters in (1, 8, 32):
        ok, re, im = _gpu_gl(fc, ic, mag, frames, H, iters, 0)
        assert ok == 1
        errs.append(sg.spectral_convergence(mag, fo, io, re, im, frames, H))
    assert errs[0] > errs[1] > errs[2], errs
    ok, dre, dim = _gpu_gl(fc, ic, mag, frames, H, 8, 0, device_mag=True)
    ok2, hre, him = _gpu_gl(fc, ic, mag, frames, H, 8, 0)
    assert ok == ok2 == 1
    assert np.array_equal(dre, hre) and np.array_equal(dim, him)


def test_griffin_lim_argument_checks():
    fc, ic, _, _ = _gl_pair(64, 16)
    mag = np.ones((4, 33), np.float32)
    re = np.zeros(4 * 33, np.float32)
    L = api.lib()
    assert L.fft_griffin_lim(fc.handle, ic.handle, _fp(mag), 4, 16, 1, 2, 1, 0, _fp(re), _fp(re)) == 0
    assert L.fft_griffin_lim(fc.handle, ic.handle, _fp(mag), 4, 16, 0, 2, 1, 0, _fp(re),
                             _fp(np.zeros_like(re))) == 0
    assert L.fft_griffin_lim(fc.handle, ic.handle, _fp(mag), 0, 16, 1, 2, 1, 0, _fp(re),
                             _fp(np.zeros_like(re))) == 0


@pytest.mark.parametrize("W,H,kind", [(64, 16, 1), (48, 24, 2), (64, 64, 0)])
def test_stream_push_pcm_matches_oracle(W, H, kind):
    N = 64
    kw = ctx_kwargs(N, transform=1, half_spectrum=1, window=W, hop=H, apply_windows=1, analysis_kind=kind,
                    reduce_magnitude=1)
    ctx = api.FftContext.full_v2(**kw)
    st = sg.StreamOracle(oracle_for(kw))
    bins = N // 2 + 1
    rng = np.random.default_rng(W + H)
    x = rng.uniform(-1, 1, 1500).astype(np.float32)
    L = api.lib()
    pos = 0
    total = 0
    for c, mf in [(5, 0), (100, 0), (1, 0), (48, 2), (300, 0), (7, 0), (539, 3), (500, 0), (0, 0)]:
        chunk = np.ascontiguousarray(x[pos: pos + c])
        pos += c
        cap = 128 * bins
        re = np.zeros(cap, np.float32)
        im = np.zeros(cap, np.float32)
        mg = np.zeros(cap, np.float32)
        n = L.fft_stream_push_pcm(ctx.handle, _fp(chunk), c, _fp(re), _fp(im), _fp(mg), mf, 0)
        rn, rre, rim, rmg = st.push_pcm(chunk, mf)
        assert n == rn
        assert L.fft_stream_backlog_samples(ctx.handle) == len(st.buffer)
        assert L.fft_stream_pending_frames(ctx.handle) == st.available_frames()
        if n:
            k = n * bins
            assert_close(re[:k] + 1j * im[:k], (rre + 1j * rim).ravel(), tol_for(N), "stream spectrum")
            assert_close(mg[:k], rmg.ravel(), tol_for(N), "stream magnitude")
        total += n
    assert total > 0
    L.fft_stream_reset(ctx.handle)
    assert L.fft_stream_backlog_samples(ctx.handle) == 0


@pytest.mark.parametrize("cola,win", [(1, 1), (0, 0), (1, 0)])
def test_stream_push_spectrum_matches_oracle(cola, win):
    N, H = 128, 32
    kw = ctx_kwargs(N, inverse=1, transform=2, half_spectrum=1, window=N, hop=H, apply_windows=win,
                    analysis_kind=1, synthesis_kind=1, cola_mode=cola)
    ctx = api.FftContext.full_v2(**kw)
    st = sg.StreamOracle(oracle_for(kw))
    bins = N // 2 + 1
    rng = np.random.default_rng(cola + 2 * win)
    L = api.lib()
    got, ref = [], []
    for frames, ms, fl in [(3, 50, 0), (1, 40, 1), (5, 0, 0), (0, 0, 0), (2, 0, sg.FLUSH_FINAL),
                          (0, 0, sg.FLUSH_FINAL), (4, 0, 0), (0, 0, sg.FLUSH_FINAL)]:
        re = rng.standard_normal(max(frames, 1) * bins).astype(np.float32)
        im = rng.standard_normal(max(frames, 1) * bins).astype(np.float32)
        out = np.zeros(4096, np.float32)
        n = L.fft_stream_push_spectrum(ctx.handle, _fp(re), _fp(im), frames, _fp(out), ms, fl)
        r = st.push_spectrum(re, im, frames, ms, fl)
        assert n == len(r)
        assert L.fft_stream_pending_pcm(ctx.handle) == len(st.queue)
        got.append(out[:n])
        ref.append(r)
    got = np.concatenate(got)
    ref = np.concatenate(ref)
    assert got.size > 0
    assert_close(got, ref, tol_for(N), "stream pcm")


@pytest.mark.parametrize("N,half", [(64, 1), (256, 1), (128, 0), (4096, 1)])
def test_phase_infer_matches_oracle(N, half):
    frames, H = 6, N // 4
    bins = N // 2 + 1 if half else N
    rng = np.random.default_rng(N)
    mag = rng.uniform(0.05, 2.0, frames * bins).astype(np.float32)
    L = api.lib()
    for mode in (0, 1):
        h = L.phase_init(N, H, half, mode, 0)
        assert h
        re = np.zeros(frames * bins, np.float32)
        im = np.zeros_like(re)
        try:
            assert L.phase_infer_execute(h, _fp(mag), frames, _fp(re), _fp(im)) == frames
        finally:
            L.phase_free(h)
        if mode == 0:
            rre, rim = sg.phase_linear(mag, frames, N, H, bool(half))
            np.testing.assert_allclose(re, rre.ravel(), rtol=1e-6, atol=1e-6)
            np.testing.assert_allclose(im, rim.ravel(), rtol=1e-6, atol=1e-6)
        else:
            rre, rim = sg.phase_min(mag, frames, N, bool(half))
            assert_close(re + 1j * im, (rre + 1j * rim).ravel(), 10 * tol_for(N), "minimum phase")


def test_stream_push_pcm_large_pushes_device_input_and_null_outputs():
    """Pushes larger than the device backlog's first allocation (it grows and
    compacts), a device-resident chunk, and a push with NULL outputs (the
    frames are consumed, as in the reference)."""
    N, W, H = 256, 256, 64
    kw = ctx_kwargs(N, transform=1, half_spectrum=1, window=W, hop=H, apply_windows=1, analysis_kind=1)
    ctx = api.FftContext.full_v2(**kw)
    st = sg.StreamOracle(oracle_for(kw))
    bins = N // 2 + 1
    rng = np.random.default_rng(77)
    L = api.lib()
    for n_in, dev, mf, null_out in [(100_000, False, 0, False), (70_001, True, 500, False), (3, False, 0, True),
                                    (150_000, False, 0, False), (0, False, 0, False)]:
        x = rng.uniform(-1, 1, n_in).astype(np.float32)
        src = torch.from_numpy(x).cuda() if dev else x
        cap = (n_in + 1024) // H + 2
        re = np.zeros(cap * bins, np.float32)
        im = np.zeros_like(re)
        mg = np.zeros_like(re)
        if null_out:
            n = L.fft_stream_push_pcm(ctx.handle, _fp(src) if n_in else None, n_in, None, None, None, mf, 0)
        else:
            n = L.fft_stream_push_pcm(ctx.handle, _fp(src) if n_in else None, n_in, _fp(re), _fp(im), _fp(mg), mf, 0)
        rn, rre, rim, rmg = st.push_pcm(x, mf)
        assert n == rn
        assert L.fft_stream_backlog_samples(ctx.handle) == len(st.buffer)
        if n and not null_out:
            k = n * bins
            assert_close(re[:k] + 1j * im[:k], (rre + 1j * rim).ravel(), tol_for(N), "stream spectrum")


def test_stream_push_spectrum_long_queue():
    """Many frames per push with the queue drained in small pieces: the
    device queue grows while samples are pending."""
    N, H = 128, 32
    kw = ctx_kwargs(N, inverse=1, transform=2, half_spectrum=1, window=N, hop=H, apply_windows=1,
                    analysis_kind=1, synthesis_kind=1, cola_mode=1)
    ctx = api.FftContext.full_v2(**kw)
    st = sg.StreamOracle(oracle_for(kw))
    bins = N // 2 + 1
    rng = np.random.default_rng(5)
    L = api.lib()
    got, ref = [], []
    for frames, ms, fl in [(300, 1000, 0), (400, 3000, 0), (0, 0, 0), (250, 0, sg.FLUSH_FINAL), (0, 0, 0)]:
        re = rng.standard_normal(max(frames, 1) * bins).astype(np.float32)
        im = rng.standard_normal(max(frames, 1) * bins).astype(np.float32)
        out = np.zeros(64000, np.float32)
        n = L.fft_stream_push_spectrum(ctx.handle, _fp(re), _fp(im), frames, _fp(out), ms, fl)
        r = st.push_spectrum(re, im, frames, ms, fl)
        assert n == len(r)
        assert L.fft_stream_pending_pcm(ctx.handle) == len(st.queue)
        got.append(out[:n])
        ref.append(r)
    assert_close(np.concatenate(got), np.concatenate(ref), tol_for(N), "stream pcm")
