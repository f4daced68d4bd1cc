"""The host-driver restatement (oracle/stream_gl.py) pinned to the reference
itself (CPU only): streaming STFT / ISTFT buffers, Griffin-Lim and both phase
inference modes of the reference's own C ABI (oracle/_ref/libfftfree_ref.so)
against the restatement on the same inputs.  Data moves and float32 sums are
bit-identical; steps through libm (atan2, sin, cos, log, exp: the reference
calls glibc, the restatement numpy) agree within a few ulp per value."""
import numpy as np
import pytest

from oracle import reflib
from oracle import stream_gl as sg
from tests.helpers import assert_close, ctx_kwargs, oracle_for, tol_for

pytestmark = pytest.mark.skipif(not reflib.available(), reason="oracle/_ref not built (needs the reference tree)")
fp = reflib.fp


@pytest.mark.parametrize("W,H,kind", [(64, 16, 1), (48, 24, 2), (64, 64, 0)])
def test_stream_push_pcm(W, H, kind):
    N = 64
    kw = ctx_kwargs(N, transform=1, half_spectrum=1, window=W, hop=H, apply_windows=1, analysis_kind=kind,
                    reduce_magnitude=1)
    ctx = reflib.RefContext.full_v2(**kw)
    L = ctx.L
    st = sg.StreamOracle(oracle_for(kw))
    bins = N // 2 + 1
    x = np.random.default_rng(W + H).uniform(-1, 1, 1500).astype(np.float32)
    pos = total = 0
    for c, mf in [(5, 0), (100, 0), (1, 0), (48, 2), (300, 0), (7, 0), (539, 3), (500, 0), (0, 0)]:
        chunk = np.ascontiguousarray(x[pos: pos + c])
        pos += c
        re, im, mg = (np.zeros(128 * bins, np.float32) for _ in range(3))
        n = L.fft_stream_push_pcm(ctx.h, fp(chunk), c, fp(re), fp(im), fp(mg), mf, 0)
        rn, rre, rim, rmg = st.push_pcm(chunk, mf)
        assert n == rn
        assert L.fft_stream_backlog_samples(ctx.h) == len(st.buffer)
        assert L.fft_stream_pending_frames(ctx.h) == st.available_frames()
        if n:
            k = n * bins
            assert np.array_equal(re[:k], rre.ravel()) and np.array_equal(im[:k], rim.ravel())
            assert np.array_equal(mg[:k], rmg.ravel())
        total += n
    assert total > 0
    ctx.close()


@pytest.mark.parametrize("cola,win", [(1, 1), (0, 0), (1, 0)])
def test_stream_push_spectrum(cola, win):
    N, H = 128, 32
    kw = ctx_kwargs(N, inverse=1, transform=2, half_spectrum=1, window=N, hop=H, apply_windows=win,
                    analysis_kind=1, synthesis_kind=1, cola_mode=cola)
    ctx = reflib.RefContext.full_v2(**kw)
    L = ctx.L
    st = sg.StreamOracle(oracle_for(kw))
    bins = N // 2 + 1
    rng = np.random.default_rng(cola + 2 * win)
    for frames, ms, fl in [(3, 50, 0), (1, 40, 1), (5, 0, 0), (0, 0, 0), (2, 0, sg.FLUSH_FINAL),
                          (0, 0, sg.FLUSH_FINAL), (4, 0, 0), (0, 0, sg.FLUSH_FINAL)]:
        re = rng.standard_normal(max(frames, 1) * bins).astype(np.float32)
        im = rng.standard_normal(max(frames, 1) * bins).astype(np.float32)
        out = np.zeros(4096, np.float32)
        n = L.fft_stream_push_spectrum(ctx.h, fp(re), fp(im), frames, fp(out), ms, fl)
        r = st.push_spectrum(re, im, frames, ms, fl)
        assert n == len(r)
        assert L.fft_stream_pending_pcm(ctx.h) == len(st.queue)
        assert np.array_equal(out[:n], r)
    ctx.close()


@pytest.mark.parametrize("N,H,frames,iters", [(64, 16, 12, 4), (256, 64, 9, 8)])
def test_griffin_lim(N, H, frames, iters):
    fkw = ctx_kwargs(N, transform=1, half_spectrum=1, window=N, hop=H, apply_windows=1, analysis_kind=1)
    ikw = ctx_kwargs(N, inverse=1, transform=2, half_spectrum=1, window=N, hop=H)
    fc, ic = reflib.RefContext.full_v2(**fkw), reflib.RefContext.full_v2(**ikw)
    fo, io = oracle_for(fkw), oracle_for(ikw)
    t = np.arange((frames - 1) * H + N)
    x = (np.sin(0.21 * t) + 0.5 * np.sin(0.05 * t + 1.0)).astype(np.float32)
    n, _, _, mag = fo.execute_batched(x, pad_mode=1, max_frames=frames)
    assert n == frames
    bins = N // 2 + 1
    m = np.ascontiguousarray(mag.ravel())
    re, im = np.zeros(frames * bins, np.float32), np.zeros(frames * bins, np.float32)
    ok = fc.L.fft_griffin_lim(fc.h, ic.h, fp(m), frames, H, 1, iters, 1, 7, fp(re), fp(im))
    rok, rre, rim = sg.griffin_lim(fo, io, mag, frames, H, True, iters, 1, 7)
    assert ok == rok == 1
    assert_close(re + 1j * im, (rre + 1j * rim).ravel(), 4 * iters * tol_for(N), "griffin-lim spectrum")
    fc.close()
    ic.close()


@pytest.mark.parametrize("N,half", [(64, 1), (256, 1), (128, 0)])
def test_phase_infer(N, half):
    frames, H = 6, N // 4
    bins = N // 2 + 1 if half else N
    mag = np.random.default_rng(N).uniform(0.05, 2.0, frames * bins).astype(np.float32)
    L = reflib.lib()
    for mode in (0, 1):
        h = L.phase_init(N, H, half, mode, 0)
        assert h
        re, im = np.zeros(frames * bins, np.float32), np.zeros(frames * bins, np.float32)
        try:
            assert L.phase_infer_execute(h, fp(mag), frames, fp(re), fp(im)) == frames
        finally:
            L.phase_free(h)
        if mode == 0:
            rre, rim = sg.phase_linear(mag, frames, N, H, bool(half))
            np.testing.assert_allclose(re, rre.ravel(), rtol=1e-6, atol=1e-6)
            np.testing.assert_allclose(im, rim.ravel(), rtol=1e-6, atol=1e-6)
        else:
            rre, rim = sg.phase_min(mag, frames, N, bool(half))
            assert_close(re + 1j * im, (rre + 1j * rim).ravel(), tol_for(N), "minimum phase")
