"""The oracle pinned to the reference itself (CPU only).

The reference's own C ABI (fft_cffi.cpp + ft_tools_cffi.cpp, unchanged,
compiled into oracle/_ref/libfftfree_ref.so with IEEE arithmetic) runs the
same inputs as the oracle; every floating-point output must be bit-identical,
and so must every integer metadata kind, frame count and return code.  This
covers the hook quirks (pre-hook only on Cooley-Tukey, store_polar on
time-domain output, DC / Nyquist zeroing, inverse scale before the post-hook),
every window kind and normalisation, the OLA / COLA complex batch and all
eleven metadata kinds.  Skipped where the reference tree was not available to
build the library.
"""
import itertools

import numpy as np
import pytest

from oracle import reflib
from oracle.oracle import OracleContext, build_window
from tests.helpers import ctx_kwargs, oracle_for

pytestmark = pytest.mark.skipif(not reflib.available(), reason="oracle/_ref not built (needs the reference tree)")

META = {"Twiddle": 0, "LayoutMap": 1, "StageSnapshot": 2, "StageParams": 3, "ButterflyPairs": 4,
        "StageInvariant": 5, "TwiddleIndexMap": 6, "Omega": 7, "StageSnapshotAll": 8, "ButterflyPairsAll": 9,
        "TwiddleIndexMapAll": 10}


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def ref_batched(kw, pcm, pad_mode=1, max_frames=0, enable_backup=0):
    o = oracle_for(kw)
    nf = o.frame_count(len(pcm), pad_mode, max_frames)
    c = reflib.RefContext.full_v2(**kw)
    try:
        return c.execute_batched(pcm, nf, o.bins, pad_mode=pad_mode, enable_backup=enable_backup,
                                 max_frames=max_frames)
    finally:
        c.close()


def check_batched(kw, pcm, pad_mode=1, max_frames=0):
    o = oracle_for(kw)
    n, re, im, mag = o.execute_batched(pcm, pad_mode=pad_mode, max_frames=max_frames)
    rn, rre, rim, rmag = ref_batched(kw, pcm, pad_mode, max_frames)
    assert n == rn
    assert bits_equal(re.ravel(), rre) and bits_equal(im.ravel(), rim) and bits_equal(mag.ravel(), rmag)
    return n


# -- fft_execute_batched -----------------------------------------------------
_COMBOS = list(itertools.product([0, 1, 2], [0, 1, 2, 3], [0, 1], [(0, 0), (1, 0), (0, 1), (1, 1)], [0, 1],
                                 [(64, 16, 0), (48, 16, 1)]))


@pytest.mark.parametrize("kernel,transform,half,rp,inverse,wh", _COMBOS)
def test_batched_every_option_n64(kernel, transform, half, rp, inverse, wh):
    W, H, win = wh
    kw = ctx_kwargs(64, kernel=kernel, transform=transform, half_spectrum=half, reduce_magnitude=rp[0],
                    store_polar=rp[1], inverse=inverse, window=W, hop=H, apply_windows=win, analysis_kind=1,
                    synthesis_kind=1)
    pcm = np.random.default_rng(7).uniform(-1, 1, 700).astype(np.float32)
    assert check_batched(kw, pcm) > 0


@pytest.mark.parametrize("N", [1, 2, 4, 8, 16, 32, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 65536])
@pytest.mark.parametrize("kernel", [0, 1, 2])
def test_batched_sizes(N, kernel):
    kw = ctx_kwargs(N, kernel=kernel, transform=1, half_spectrum=1, window=N, hop=max(1, N // 4))
    pcm = np.random.default_rng(N).uniform(-1, 1, 4 * N + 3).astype(np.float32)
    check_batched(kw, pcm)


def test_config1_exact_call():
    """The reference's own plain R2C STFT call: 65,536 samples, W=1024, H=256,
    Stockham, radix 4, half spectrum, magnitude -> 253 x 513."""
    kw = ctx_kwargs(1024, kernel=2, radix=4, window=1024, hop=256, transform=1, reduce_magnitude=1,
                    half_spectrum=1, allow_outer_parallel=1)
    pcm = np.random.default_rng(0).uniform(-1, 1, 65536).astype(np.float32)
    assert check_batched(kw, pcm) == 253


@pytest.mark.parametrize("radix,pattern", [(0, None), (1, None), (2, None), (4, None), (8, None), (16, None),
                                           (3, None), (0, [4, 4, 2]), (0, [16, 16])])
def test_radix_options(radix, pattern):
    kw = ctx_kwargs(1024, kernel=2, radix=radix, radix_pattern=pattern, transform=1, half_spectrum=1,
                    reduce_magnitude=1, window=1024, hop=256)
    pcm = np.random.default_rng(3).uniform(-1, 1, 8000).astype(np.float32)
    check_batched(kw, pcm)


@pytest.mark.parametrize("pad_mode,ctx_pad", list(itertools.product([0, 1, 2], [0, 1, 2])))
@pytest.mark.parametrize("length", [0, 1, 50, 63, 64, 65, 100, 257, 300])
def test_frame_count_and_padding(pad_mode, ctx_pad, length):
    kw = ctx_kwargs(64, window=64, hop=32, transform=1, pad_mode=ctx_pad)
    pcm = np.random.default_rng(length).standard_normal(length).astype(np.float32)
    check_batched(kw, pcm, pad_mode=pad_mode)


@pytest.mark.parametrize("max_frames", [1, 5, 1000])
def test_max_frames(max_frames):
    kw = ctx_kwargs(256, window=200, hop=64, transform=1, half_spectrum=1)
    pcm = np.random.default_rng(1).standard_normal(4000).astype(np.float32)
    check_batched(kw, pcm, max_frames=max_frames)


def test_window_longer_than_n_refused():
    kw = ctx_kwargs(64, window=128, hop=32)
    rn, *_ = ref_batched(kw, np.ones(4096, np.float32))
    o = oracle_for(kw)
    assert rn == 0 and o.execute_batched(np.ones(4096, np.float32))[0] == 0


# -- windows (fft_cffi.cpp:163-208) ------------------------------------------
_WINDOWS = [(0, 0.0), (1, 0.0), (2, 0.0), (3, 0.0), (4, 0.0), (4, 0.3), (4, 1.0), (5, 0.0), (5, 8.6), (9, 0.0)]


@pytest.mark.parametrize("kind,p1", _WINDOWS)
@pytest.mark.parametrize("norm", [0, 1, 2])
def test_analysis_windows(kind, p1, norm):
    """Every window kind (Tukey with its alpha p1 and the 0.5 default, the
    Kaiser placeholder, an unknown kind) and each normalisation, through the
    framed transform with windows applied: the taps the oracle builds are the
    reference's."""
    kw = ctx_kwargs(64, window=48, hop=16, transform=1, half_spectrum=1, apply_windows=1, analysis_kind=kind,
                    analysis_p1=p1, norm_policy=norm)
    pcm = np.random.default_rng(11).uniform(-1, 1, 500).astype(np.float32)
    check_batched(kw, pcm)
    # ones in, rect framing: bin 0 of frame 0 is the sum of the taps
    o = oracle_for(kw)
    _, re, _, _ = o.execute_batched(np.ones(48, np.float32), pad_mode=1)
    w = build_window(kind, 48, p1, 0.0, norm)
    assert abs(float(re[0, 0]) - float(np.sum(w, dtype=np.float64))) <= 1e-4 * max(1.0, float(np.abs(w).sum()))


# -- fft_execute_complex_batched (fft_cffi.cpp:1042-1340) --------------------
_CPLX = list(itertools.product([0, 1, 2], [0, 1, 2, 3], [0, 1], [(0, 0), (1, 0), (0, 1)], [0, 1],
                               [(0, 0, 0), (1, 0, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)]))


@pytest.mark.parametrize("kernel,transform,half,rp,inverse,wol", _CPLX)
def test_complex_batched_every_option_n64(kernel, transform, half, rp, inverse, wol):
    win, ola, cola = wol
    N, frames = 64, 7
    kw = ctx_kwargs(N, kernel=kernel, transform=transform, half_spectrum=half, reduce_magnitude=rp[0],
                    store_polar=rp[1], inverse=inverse, window=N, hop=16, apply_windows=win, apply_ola=ola,
                    cola_mode=cola, analysis_kind=1, synthesis_kind=2)
    bins = N // 2 + 1 if half else N
    rng = np.random.default_rng(5)
    re = rng.standard_normal(frames * bins).astype(np.float32)
    im = rng.standard_normal(frames * bins).astype(np.float32)
    o = oracle_for(kw)
    n, out = o.execute_complex_batched(re, im, frames)
    c = reflib.RefContext.full_v2(**kw)
    rn, rout = c.execute_complex_batched(re, im, frames, N)
    c.close()
    assert n == rn
    assert bits_equal(out.ravel(), rout[: out.size])


# -- the C++ batched transform and its metadata (eigen_fft.hpp:1477-1888) ----
@pytest.mark.parametrize("N", [2, 4, 8, 64, 256])
@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("opts", [(0, 0, 0, 0, 0), (0, 0, 0, 0, 1), (1, 1, 0, 1, 0), (1, 1, 1, 0, 0),
                                  (1, 0, 0, 0, 0), (2, 1, 0, 1, 1), (2, 1, 0, 0, 1), (3, 0, 0, 0, 0)])
def test_metadata_every_kind(N, kernel, opts):
    transform, half, red, polar, inverse = opts
    B = 5
    rng = np.random.default_rng(N + kernel)
    x = (rng.standard_normal((B, N)) + 1j * rng.standard_normal((B, N))).astype(np.complex64)
    S = int(np.log2(N))
    counts = {"Twiddle": N, "LayoutMap": N, "StageParams": S, "ButterflyPairs": N * S, "TwiddleIndexMap": N * S,
              "Omega": N, "StageSnapshot": N * S, "StageInvariant": S, "StageSnapshotAll": N * S * B,
              "ButterflyPairsAll": N * S * B, "TwiddleIndexMapAll": N * S * B}
    o = OracleContext(N=N, kernel=kernel, transform=transform, half_spectrum=half, reduce_magnitude=red,
                      store_polar=polar, inverse=inverse)
    ok, xo, mo = o.fft_columns(x, counts)
    p = reflib.RefPlan(N, inverse, kernel, transform, red, polar, half)
    xr = x.copy()
    rok, mr = p.execute(xr, {META[k]: c for k, c in counts.items()})
    p.close()
    assert ok and rok
    assert bits_equal(xo.view(np.float32), xr.view(np.float32))
    for k in counts:
        assert bits_equal(mo[k].view(np.float32), mr[META[k]].view(np.float32)), k


def test_metadata_short_buffer_refused():
    N = 64
    x = np.ones((2, N), np.complex64)
    o = OracleContext(N=N, kernel=1)
    ok, _, _ = o.fft_columns(x, {"ButterflyPairs": N})
    p = reflib.RefPlan(N, 0, 1)
    rok, _ = p.execute(x.copy(), {META["ButterflyPairs"]: N})
    p.close()
    assert ok == rok


# -- the reference tests' own known-answer cases ------------------------------
@pytest.mark.parametrize("kernel", [1, 2])
def test_kat_cases_oracle_equals_reference(kat, kernel):
    """The seeded inputs of the reference's tests (regenerated with
    libstdc++'s generators): the reference meets each test's own tolerance
    against the DFT, and the oracle's columns are the reference's, bit for
    bit, for both executors."""
    from tests.test_oracle_kat import C2C_CASES
    for name in C2C_CASES:
        x = np.ascontiguousarray(kat[name + "__input"], np.complex64)
        B, N = x.shape
        ok, xo, _ = OracleContext(N=N, kernel=kernel).fft_columns(x)
        p = reflib.RefPlan(N, 0, kernel)
        xr = x.copy()
        rok, _ = p.execute(xr)
        p.close()
        assert ok and rok, name
        err = np.max(np.abs(xr.astype(np.complex128) - kat[name + "__expected"].astype(np.complex128)))
        assert err <= float(kat[name + "__tol"][0]), name
        assert bits_equal(xo.view(np.float32), xr.view(np.float32)), name


# -- the recovery path (fft_cffi.cpp:826-1027) --------------------------------
def test_backup_without_dropout_equals_fast_path():
    kw = ctx_kwargs(256, threads=4, window=256, hop=64, transform=1, half_spectrum=1, allow_outer_parallel=1)
    pcm = np.random.default_rng(2).uniform(-1, 1, 9000).astype(np.float32)
    fast = ref_batched(kw, pcm, enable_backup=0)
    backup = ref_batched(kw, pcm, enable_backup=1)
    assert fast[0] == backup[0] and all(bits_equal(a, b) for a, b in zip(fast[1:], backup[1:]))


# -- the recovery coordinator: observer calls and given-up frames -------------
_SCENARIOS = [
    ("stripe_one_shot", lambda L: L.fft_set_workerpool_dropout_pattern(4, 1, 0), 10),
    ("single_one_shot", lambda L: L.fft_set_workerpool_dropout_single(2), 5),
    ("single_persistent", lambda L: (L.fft_set_workerpool_dropout_single(3),
                                     L.fft_set_workerpool_dropout_persistent(1)), 6),
    ("clamped_pattern", lambda L: L.fft_set_workerpool_dropout_pattern(3, 7, 1), 4),
    ("stripe_persistent", lambda L: (L.fft_set_workerpool_dropout_pattern(4, 1, 0),
                                     L.fft_set_workerpool_dropout_persistent(1)), 10),
    ("stripe2_persistent", lambda L: (L.fft_set_workerpool_dropout_pattern(5, 2, 1),
                                      L.fft_set_workerpool_dropout_persistent(1)), 12),
]


def _reset(L):
    L.fft_set_workerpool_dropout_pattern(0, 0, 0)
    L.fft_set_workerpool_dropout_single(-1)
    L.fft_set_workerpool_dropout_persistent(0)
    L.fft_set_workerpool_debug_dropout(0)
    L.fft_clear_workerpool_dropout_history()


@pytest.mark.parametrize("name,setup,frames", _SCENARIOS, ids=[s[0] for s in _SCENARIOS])
def test_recovery_coordinator_matches_reference(name, setup, frames):
    """The host coordinator of the GPU library (its CPU debug entry
    fftfree_debug_recovery_plan) against the reference's recovery path on a
    2-thread WorkerPool: the same restore-observer calls and the same frames
    given up (left as their restored input in the reference's output).  The
    reference's pool is not deterministic under every mode, so it gets up to
    eight runs to produce the coordinator's outcome."""
    import ctypes
    import fftfree_b200 as ff
    ours = []
    cb = ff.RESTORE_OBSERVER(lambda s, e: ours.append((s, e)))
    L = ff.lib()
    L.fft_register_restore_observer(cb)
    try:
        _reset(L)
        setup(L)
        raw = ctypes.create_string_buffer(frames)
        L.fftfree_debug_recovery_plan(frames, raw)
        given_up = [bool(b) for b in raw.raw[:frames]]
    finally:
        L.fft_register_restore_observer(ff.RESTORE_OBSERVER())
        _reset(L)
    N = 64
    kw = ctx_kwargs(N, threads=2, window=N, hop=N, transform=1, allow_outer_parallel=1)
    pcm = np.random.default_rng(frames).uniform(-1, 1, N * frames).astype(np.float32)
    R = reflib.lib()
    _, ore, _, _ = oracle_for(kw).execute_batched(pcm)
    for _ in range(8):
        _reset(R)
        setup(R)
        reflib.observer_attach(R)
        n, re, im, mag = ref_batched(kw, pcm, enable_backup=1)
        calls = sorted(reflib.observer_calls(R))
        ref_given = [not bits_equal(re[f * N:(f + 1) * N], ore[f]) for f in range(frames)]
        if calls == sorted(ours) and ref_given == given_up:
            break
    _reset(R)
    assert calls == sorted(ours)
    assert ref_given == given_up
    assert n == frames
    for f in range(frames):
        s = slice(f * N, (f + 1) * N)
        if given_up[f]:
            assert np.array_equal(re[s], pcm[s]) and not np.any(im[s]) and np.array_equal(mag[s], np.abs(pcm[s]))
