"""GPU parity of the C ABI's remaining entry points against the reference
itself (its own fft_cffi.cpp, built into oracle/_ref/libfftfree_ref.so and
pinned bit-exact to the oracle by tests/test_ref_pin.py) and the oracle:

  * the recovery path, fft_execute_batched / fft_execute_complex_batched with
    enable_backup=1 under host-injected dropouts (fft_cffi.cpp:826-1027,
    1168-1340): the same restore-observer calls, recovered frames within the
    bar, abandoned frames equal to the reference's restored input;
  * fft_pcm_to_channels (fft_cffi.cpp:431-513), fft_init / fft_init_ex pad
    rules and the FFTFREE_DEFAULT_KERNEL override (:540-658),
    fft_stft_execute (:1458-1466), fft_config_window / _custom (:1983-2032);
  * every window kind and normalisation (fft_cffi.cpp:163-208);
  * the batched-C2C configuration at its full size (N=4096 x 16,384, re / im
    N(0,1) from numpy default_rng(1)), checked on a row sample.

Floating-point outputs: rel-L2 <= 1e-5 * log2(N) against the reference.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import fftfree_b200 as ff
from oracle import reflib
from oracle.oracle import OracleContext
from tests.helpers import assert_close, compare_spectrum, ctx_kwargs, oracle_for, tol_for

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not reflib.available(), reason="oracle/_ref not built (needs the reference tree)")
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _reset(L):
    L.fft_set_workerpool_dropout_pattern(0, 0, 0)
    L.fft_set_workerpool_dropout_single(-1)
    L.fft_set_workerpool_dropout_persistent(0)
    L.fft_set_workerpool_debug_dropout(0)
    L.fft_clear_workerpool_dropout_history()


@pytest.fixture
def observer():
    calls = []
    cb = ff.RESTORE_OBSERVER(lambda s, e: calls.append((s, e)))
    ff.lib().fft_register_restore_observer(cb)
    yield calls
    ff.lib().fft_register_restore_observer(ff.RESTORE_OBSERVER())
    _reset(ff.lib())
    if reflib.available():
        _reset(reflib.lib())


# name, setup(lib), frames: the dropout controls of fft_cffi.hpp:232-268
_SCENARIOS = [
    ("none", lambda L: None, 10),
    ("stripe_one_shot", lambda L: L.fft_set_workerpool_dropout_pattern(4, 1, 0), 10),
    ("single_one_shot", lambda L: L.fft_set_workerpool_dropout_single(2), 5),
    ("single_persistent", lambda L: (L.fft_set_workerpool_dropout_single(3),
                                     L.fft_set_workerpool_dropout_persistent(1)), 6),
    ("stripe_persistent", lambda L: (L.fft_set_workerpool_dropout_pattern(4, 1, 0),
                                     L.fft_set_workerpool_dropout_persistent(1)), 10),
    ("stripe2_persistent", lambda L: (L.fft_set_workerpool_dropout_pattern(5, 2, 1),
                                      L.fft_set_workerpool_dropout_persistent(1)), 12),
]


def _given_up(setup, frames):
    """Frames the GPU library's host coordinator leaves restored for this
    dropout setting (its CPU debug entry, deterministic)."""
    L = ff.lib()
    _reset(L)
    setup(L)
    raw = ctypes.create_string_buffer(frames)
    L.fftfree_debug_recovery_plan(frames, raw)
    _reset(L)
    return [bool(b) for b in raw.raw[:frames]]


def _ref_backup_run(kw, setup, run, expect_calls, expect_given_up, transformed, attempts=6):
    """The reference's recovery path on 2 worker threads, or None.  Its pool
    is not deterministic under every dropout mode (runs were seen where a
    one-shot dropout left a frame restored, or a persistent one gave up on
    another frame), so it is run up to `attempts` times and the first run
    with the expected observer calls and frames left restored is returned.
    The coordinator itself is pinned to the reference on the CPU
    (tests/test_ref_pin.py); here the reference run, when one agrees, also
    checks the values of the frames it left restored."""
    L = reflib.lib()
    try:
        for _ in range(attempts):
            _reset(L)
            setup(L)
            reflib.observer_attach(L)
            c = reflib.RefContext.full_v2(**kw)
            out = run(c)
            c.close()
            calls = sorted(reflib.observer_calls(L))
            given = [not transformed(out, f) for f in range(len(expect_given_up))]
            if calls == expect_calls and given == expect_given_up:
                return out
        return None
    finally:
        _reset(L)


@needs_ref
@pytest.mark.parametrize("name,setup,frames", _SCENARIOS, ids=[s[0] for s in _SCENARIOS])
@pytest.mark.parametrize("N,W,H", [(64, 64, 64), (256, 200, 64)])
def test_backup_batched_against_reference(observer, name, setup, frames, N, W, H):
    """Recovered frames: the transform (against the oracle, pinned bit-exact
    to the reference).  Given-up frames: the restored, windowed frame samples
    as (re, 0, |re|), as the reference leaves them (fft_cffi.cpp:954-1026)."""
    kw = ctx_kwargs(N, threads=2, window=W, hop=H, transform=1, allow_outer_parallel=1, apply_windows=1,
                    analysis_kind=1)
    pcm = np.random.default_rng(frames + N).uniform(-1, 1, (frames - 1) * H + W).astype(np.float32)
    o = oracle_for(kw)
    assert o.frame_count(len(pcm), 1) == frames
    given_up = _given_up(setup, frames)
    observer.clear()  # the debug plan reported to the same observer
    L = ff.lib()
    _reset(L)
    setup(L)
    ctx = ff.FftContext.full_v2(**kw)
    re, im, mg = (np.zeros(frames * N, np.float32) for _ in range(3))
    assert ctx.execute_batched(pcm, re, im, mg, enable_backup=1) == frames
    ctx.close()
    ours = sorted(observer)
    _, ore, oim, omg = o.execute_batched(pcm)
    ore, oim, omg = ore.ravel(), oim.ravel(), omg.ravel()
    ref = _ref_backup_run(kw, setup, lambda c: c.execute_batched(pcm, frames, N, enable_backup=1), ours, given_up,
                          lambda out, f: np.array_equal(out[1][f * N:(f + 1) * N], ore[f * N:(f + 1) * N]))
    for f in range(frames):
        s = slice(f * N, (f + 1) * N)
        if not given_up[f]:
            assert_close(re[s] + 1j * im[s], ore[s] + 1j * oim[s], tol_for(N), f"frame {f}")
            assert_close(mg[s], omg[s], tol_for(N), f"frame {f} magnitude")
        else:
            seg = np.zeros(N, np.float32)
            seg[:W] = pcm[f * H: f * H + W] * o.analysis_win[:W]
            assert np.array_equal(re[s], seg) and not np.any(im[s]) and np.array_equal(mg[s], np.abs(seg))
            if ref is not None:
                _, rre, rim, rmg = ref
                assert np.array_equal(re[s], rre[s]) and np.array_equal(im[s], rim[s])
                assert np.array_equal(mg[s], rmg[s])


@needs_ref
@pytest.mark.parametrize("name,setup,frames", _SCENARIOS, ids=[s[0] for s in _SCENARIOS])
def test_backup_complex_batched_against_reference(observer, name, setup, frames):
    """Recovered frames: the inverse transform times the synthesis window.
    Given-up frames: the restored input -- the Hermitian-mirrored spectrum's
    real part times the synthesis window -- as the reference leaves them
    (fft_cffi.cpp:1168-1340)."""
    N = 128
    kw = ctx_kwargs(N, threads=2, inverse=1, transform=2, half_spectrum=1, window=N, hop=32, apply_windows=1,
                    synthesis_kind=1, allow_outer_parallel=1)
    bins = N // 2 + 1
    rng = np.random.default_rng(frames)
    ri = rng.standard_normal(frames * bins).astype(np.float32)
    ii = rng.standard_normal(frames * bins).astype(np.float32)
    given_up = _given_up(setup, frames)
    observer.clear()  # the debug plan reported to the same observer
    L = ff.lib()
    _reset(L)
    setup(L)
    ctx = ff.FftContext.full_v2(**kw)
    out = np.zeros(frames * N, np.float32)
    assert ctx.execute_complex_batched(ri, ii, frames, out, enable_backup=1) == frames
    ctx.close()
    ours = sorted(observer)
    o = oracle_for(kw)
    _, oo = o.execute_complex_batched(ri, ii, frames)
    oo = oo.ravel()
    ref = _ref_backup_run(kw, setup, lambda c: c.execute_complex_batched(ri, ii, frames, N, enable_backup=1),
                          ours, given_up, lambda r, f: np.array_equal(r[1][f * N:(f + 1) * N], oo[f * N:(f + 1) * N]))
    for f in range(frames):
        s = slice(f * N, (f + 1) * N)
        if not given_up[f]:
            assert_close(out[s], oo[s], tol_for(N), f"frame {f}")
        else:
            spec = ri[f * bins:(f + 1) * bins]
            full = np.concatenate([spec, spec[1:N // 2][::-1]])  # real part of the mirrored spectrum
            assert_close(out[s], full * o.synthesis_win[:N], 1e-6, f"restored frame {f}")
            if ref is not None:
                assert_close(out[s], ref[1][s], 1e-6, f"restored frame {f} (reference)")


@needs_ref
@pytest.mark.parametrize("n", [1, 3, 5, 100, 1000, 1024, 3000])
def test_pcm_to_channels(n):
    x = np.random.default_rng(n).uniform(-1, 1, n).astype(np.float32)
    got = [np.zeros(n, np.float32) for _ in range(3)]
    ff.lib().fft_pcm_to_channels(*(reflib.fp(a) for a in [x] + got), n, 1)
    ref = [np.zeros(n, np.float32) for _ in range(3)]
    reflib.lib().fft_pcm_to_channels(*(reflib.fp(a) for a in [x] + ref), n, 1)
    P = 1 << max(0, (n - 1).bit_length())
    tol = tol_for(P)
    assert_close(got[0] + 1j * got[1], ref[0] + 1j * ref[1], tol, "pcm_to_channels")
    assert_close(got[2], ref[2], tol, "pcm_to_channels magnitude")


@needs_ref
@pytest.mark.parametrize("n", [1, 2, 3, 100, 256, 1000, 4096, 5000])
@pytest.mark.parametrize("pad_mode", [0, 1, 2])
@pytest.mark.parametrize("kernel,radix", [(0, 0), (1, 0), (2, 0), (2, 4), (0, 8)])
def test_init_ex_pad_rules(n, pad_mode, kernel, radix):
    """fft_init_ex / fft_init pad a non-power-of-two N up only when
    pad_mode == 1 and refuse it otherwise; the context size is the
    reference's."""
    L, R = ff.lib(), reflib.lib()
    for fn in ("fft_init_ex", "fft_init"):
        extra = (0, 0) if fn == "fft_init_ex" else ()
        h = getattr(L, fn)(n, 1, 1, 0, kernel, radix, None, 0, pad_mode, *extra)
        r = getattr(R, fn)(n, 1, 1, 0, kernel, radix, None, 0, pad_mode, *extra)
        try:
            assert bool(h) == bool(r), fn
            if h:
                assert L.fft_ctx_size(h) == R.fft_ctx_size(r)
                assert L.fftfree_ctx_kernel(h) == kernel
        finally:
            L.fft_free(h)
            R.fft_free(r)


@needs_ref
def test_init_ex_executes_like_reference():
    """A padded fft_init_ex context (N=1000 -> 1024) through fft_execute and
    fft_execute_batched, against the reference's own context."""
    L, R = ff.lib(), reflib.lib()
    h = L.fft_init_ex(1000, 1, 1, 0, 2, 0, None, 0, 1, 512, 128)
    r = R.fft_init_ex(1000, 1, 1, 0, 2, 0, None, 0, 1, 512, 128)
    try:
        x = np.random.default_rng(9).uniform(-1, 1, 5000).astype(np.float32)
        for fn_args in (("fft_execute", 700), ("fft_execute_batched",)):
            got = [np.zeros(1024 * 40, np.float32) for _ in range(3)]
            ref = [np.zeros(1024 * 40, np.float32) for _ in range(3)]
            if fn_args[0] == "fft_execute":
                a = L.fft_execute(h, reflib.fp(x), *(reflib.fp(g) for g in got), fn_args[1])
                b = R.fft_execute(r, reflib.fp(x), *(reflib.fp(g) for g in ref), fn_args[1])
            else:
                a = L.fft_execute_batched(h, reflib.fp(x), x.size, *(reflib.fp(g) for g in got), 1, 0, 0)
                b = R.fft_execute_batched(r, reflib.fp(x), x.size, *(reflib.fp(g) for g in ref), 1, 0, 0)
            assert a == b and a > 0
            k = 1024 if fn_args[0] == "fft_execute" else a * 1024
            assert_close(got[0][:k] + 1j * got[1][:k], ref[0][:k] + 1j * ref[1][:k], tol_for(1024), fn_args[0])
            assert_close(got[2][:k], ref[2][:k], tol_for(1024), fn_args[0] + " magnitude")
    finally:
        L.fft_free(h)
        R.fft_free(r)


@pytest.mark.parametrize("token,expect", [("stockham", 1), ("CT", 0), ("external", 2), ("2", 2), ("auto", 0),
                                          ("bogus", 0)])
def test_default_kernel_env(token, expect):
    """FFTFREE_DEFAULT_KERNEL replaces kernel 0 in fft_init / fft_init_ex
    with the header's constant (fft_cffi.cpp:104-159, 553-558): 'stockham'
    yields FFT_KERNEL_STOCKHAM = 1, which the executor switch reads as
    Cooley-Tukey, and 'ct' yields FFT_KERNEL_COOLEYTUKEY = 0, which counts as
    no override (quirks kept as they are).  The override is read once per
    process, so each token runs in a fresh interpreter."""
    code = ("import sys; sys.path.insert(0, %r); import fftfree_b200 as ff; L = ff.lib(); "
            "h = L.fft_init_ex(64, 1, 1, 0, 0, 0, None, 0, 1, 0, 0); k0 = L.fftfree_ctx_kernel(h); L.fft_free(h); "
            "h = L.fft_init_ex(64, 1, 1, 0, 2, 0, None, 0, 1, 0, 0); k2 = L.fftfree_ctx_kernel(h); L.fft_free(h); "
            "print('KERNELS', k0, k2)" % REPO)
    env = dict(os.environ, FFTFREE_DEFAULT_KERNEL=token)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert f"KERNELS {expect} 2" in r.stdout, r.stdout + r.stderr


@needs_ref
@pytest.mark.parametrize("max_frames", [0, 3])
def test_stft_execute(max_frames):
    kw = ctx_kwargs(512, window=512, hop=128, transform=1, half_spectrum=1, reduce_magnitude=1, pad_mode=1)
    x = np.random.default_rng(4).uniform(-1, 1, 3000).astype(np.float32)
    bins, cap = 257, 64 * 257
    ctx = ff.FftContext.full_v2(**kw)
    got = [np.zeros(cap, np.float32) for _ in range(3)]
    n = ff.lib().fft_stft_execute(ctx.handle, reflib.fp(x), x.size, *(reflib.fp(g) for g in got), max_frames)
    rc = reflib.RefContext.full_v2(**kw)
    ref = [np.zeros(cap, np.float32) for _ in range(3)]
    rn = rc.L.fft_stft_execute(rc.h, reflib.fp(x), x.size, *(reflib.fp(g) for g in ref), max_frames)
    rc.close()
    # the same call as fft_execute_batched(pad_mode=1, backup=0)
    b = [np.zeros(cap, np.float32) for _ in range(3)]
    nb = ctx.execute_batched(x, *b, pad_mode=1, max_frames=max_frames)
    ctx.close()
    assert n == rn == nb > 0
    k = n * bins
    compare_spectrum(kw, [g[:k] for g in got], [r[:k] for r in ref], tol_for(512))
    assert all(np.array_equal(g[:k], c[:k]) for g, c in zip(got, b))


@needs_ref
@pytest.mark.parametrize("custom", [0, 1])
def test_config_window_rebuilds_and_disables(custom):
    """fft_config_window / _custom rebuild the windows and leave window
    application off (fft_cffi.cpp:2006, 2029): on a v2 context created with
    windows applied, later calls run unwindowed, like the reference's."""
    N, W, H = 256, 256, 64
    kw = ctx_kwargs(N, window=W, hop=H, transform=1, half_spectrum=1, apply_windows=1, analysis_kind=1,
                    synthesis_kind=1)
    x = np.random.default_rng(6).uniform(-1, 1, 4000).astype(np.float32)
    ctx = ff.FftContext.full_v2(**kw)
    rc = reflib.RefContext.full_v2(**kw)
    if custom:
        w = np.hanning(W).astype(np.float32)
        assert ff.lib().fft_config_window_custom(ctx.handle, reflib.fp(w), W, reflib.fp(w), W, 1, 1) == 1
        assert rc.L.fft_config_window_custom(rc.h, reflib.fp(w), W, reflib.fp(w), W, 1, 1) == 1
    else:
        assert ff.lib().fft_config_window(ctx.handle, 3, 2, 0.0, 0.0, 2, 1) == 1
        assert rc.L.fft_config_window(rc.h, 3, 2, 0.0, 0.0, 2, 1) == 1
    o = oracle_for(kw)
    nf = o.frame_count(x.size, 1)
    bins = o.bins
    got = [np.zeros(nf * bins, np.float32) for _ in range(3)]
    assert ctx.execute_batched(x, *got) == nf
    rn, *ref = rc.execute_batched(x, nf, bins)
    assert rn == nf
    compare_spectrum(kw, got, ref, tol_for(N))
    # unwindowed: the same as a context that never had windows
    plain = oracle_for(dict(kw, apply_windows=0))
    _, pre, pim, _ = plain.execute_batched(x)
    assert_close(got[0] + 1j * got[1], (pre + 1j * pim).ravel(), tol_for(N), "windows disabled")
    # and the complex batch of an inverse context after reconfiguration
    ikw = dict(kw, inverse=1, transform=2, apply_ola=1, cola_mode=1)
    ictx = ff.FftContext.full_v2(**ikw)
    irc = reflib.RefContext.full_v2(**ikw)
    assert ff.lib().fft_config_window(ictx.handle, 1, 1, 0.0, 0.0, 0, 1) == 1
    assert irc.L.fft_config_window(irc.h, 1, 1, 0.0, 0.0, 0, 1) == 1
    out = np.zeros(nf * N, np.float32)
    assert ictx.execute_complex_batched(got[0], got[1], nf, out) == nf
    irn, rout = irc.execute_complex_batched(got[0], got[1], nf, N)
    assert irn == nf
    assert_close(out, rout, tol_for(N), "complex batch after fft_config_window")
    for c in (ctx, ictx):
        c.close()
    for c in (rc, irc):
        c.close()


_WINDOWS = [(4, 0.0), (4, 0.3), (4, 1.0), (5, 0.0), (5, 8.6), (3, 0.0), (9, 0.0)]


@needs_ref
@pytest.mark.parametrize("kind,p1", _WINDOWS)
@pytest.mark.parametrize("norm", [0, 1, 2])
def test_windows_against_reference(kind, p1, norm):
    """Tukey (alpha p1, default 0.5), the Kaiser placeholder, an unknown kind
    and L2 / area normalisation, on the analysis side (STFT) and the
    synthesis side (complex batch with overlap-add and COLA)."""
    N, W, H = 256, 200, 50
    kw = ctx_kwargs(N, window=W, hop=H, transform=1, half_spectrum=1, apply_windows=1, analysis_kind=kind,
                    analysis_p1=p1, synthesis_kind=kind, synthesis_p1=p1, norm_policy=norm)
    x = np.random.default_rng(kind * 7 + norm).uniform(-1, 1, 3000).astype(np.float32)
    ctx = ff.FftContext.full_v2(**kw)
    rc = reflib.RefContext.full_v2(**kw)
    o = oracle_for(kw)
    nf = o.frame_count(x.size, 1)
    got = [np.zeros(nf * o.bins, np.float32) for _ in range(3)]
    assert ctx.execute_batched(x, *got) == nf
    rn, *ref = rc.execute_batched(x, nf, o.bins)
    assert rn == nf
    compare_spectrum(kw, got, ref, tol_for(N))
    ctx.close()
    rc.close()
    ikw = dict(kw, inverse=1, transform=2, apply_ola=1, cola_mode=1)
    ictx = ff.FftContext.full_v2(**ikw)
    irc = reflib.RefContext.full_v2(**ikw)
    out = np.zeros(nf * N, np.float32)
    assert ictx.execute_complex_batched(got[0], got[1], nf, out) == nf
    irn, rout = irc.execute_complex_batched(got[0], got[1], nf, N)
    assert irn == nf
    assert_close(out, rout, tol_for(N), "synthesis window + COLA")
    ictx.close()
    irc.close()


@pytest.mark.parametrize("kernel,inverse", [(2, 0), (2, 1), (1, 0)])
def test_config2_full_batch_seed1(kernel, inverse):
    """The batched-C2C configuration at full size: 16,384 transforms of 4096
    points, re / im i.i.d. N(0,1) from numpy default_rng(1) (PCG64), on the
    device; 256 rows spread over the batch against the oracle (the
    reference's float path)."""
    import torch
    N, B = 4096, 16384
    z = np.random.default_rng(1).standard_normal((B, N, 2), dtype=np.float32)
    x = torch.from_numpy(z).cuda()
    y = torch.empty_like(x)
    ctx = ff.FftContext.full_v2(N, kernel=kernel, inverse=inverse)
    assert ctx.execute_c2c(x, y, B) == 1
    torch.cuda.synchronize()
    rows = np.linspace(0, B - 1, 256).astype(np.int64)
    got = y[torch.from_numpy(rows).cuda()].cpu().numpy()
    ctx.close()
    xs = z[rows, :, 0] + 1j * z[rows, :, 1]
    _, ref, _ = OracleContext(N=N, kernel=kernel, inverse=inverse).fft_columns(xs.astype(np.complex64))
    assert_close(got[..., 0] + 1j * got[..., 1], ref, tol_for(N), "config-2 row sample")
    # every row: the batch has no stale or skipped transform (energy per row,
    # Parseval: sum |Y|^2 = N^(1 - 2 inverse) sum |X|^2)
    e_in = (x.double() ** 2).sum(dim=(1, 2))
    e_out = (y.double() ** 2).sum(dim=(1, 2))
    scale = float(N) if not inverse else 1.0 / N
    assert float(((e_out / (scale * e_in)) - 1).abs().max()) < 1e-4


@pytest.mark.parametrize("N,H", [(64, 16), (64, 24), (256, 64), (32, 32), (64, 10), (128, 12)])
@pytest.mark.parametrize("cola", [0, 1])
def test_overlap_add_is_the_frame_order_sum(N, H, cola):
    # fft_cffi.cpp:1295-1320: the internal overlap-add is the float sum of the
    # frames in frame order over frames*N samples, divided by the frame count
    # covering each sample under COLA normalisation.  The GPU's own frames
    # (apply_ola off) summed that way in numpy must equal its OLA output bit
    # for bit, on the 16-byte path (N, H multiples of 4) and the scalar one.
    nf = 37
    bins = N // 2 + 1
    rng = np.random.default_rng(N * 100 + H + cola)
    re = rng.standard_normal(nf * bins).astype(np.float32)
    im = rng.standard_normal(nf * bins).astype(np.float32)
    base = dict(inverse=1, transform=2, half_spectrum=1, window=N, hop=H, cola_mode=cola)
    fctx = ff.FftContext.full_v2(**ctx_kwargs(N, **base))
    octx = ff.FftContext.full_v2(**ctx_kwargs(N, apply_ola=1, **base))
    frames = np.zeros(nf * N, np.float32)
    out = np.zeros(nf * N, np.float32)
    assert fctx.execute_complex_batched(re, im, nf, frames) == nf
    assert octx.execute_complex_batched(re, im, nf, out) == nf
    exp = np.zeros(nf * N, np.float32)
    cnt = np.zeros(nf * N, np.float32)
    fr = frames.reshape(nf, N)
    for f in range(nf):
        s = f * H
        e = min(s + N, nf * N)
        if e > s:
            exp[s:e] += fr[f, :e - s]
            cnt[s:e] += np.float32(1)
    if cola:
        nz = cnt > np.float32(1e-12)
        exp[nz] = exp[nz] / cnt[nz]
    assert np.array_equal(out, exp)
    fctx.close()
    octx.close()
