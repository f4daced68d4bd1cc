"""Parity of the CUDA path (through the C ABI) with the oracle.

Every test here runs kernels on cuda:0 via libfft_cffi.so and compares the
outputs with the CPU oracle on the same seeded inputs: rel-L2 <= 1e-5*log2(N)
for floating-point outputs, exact equality for frame counts and return codes.
"""
import itertools

import numpy as np
import pytest

import fftfree_b200 as ff
from oracle.oracle import OracleContext
from tests.helpers import assert_close, compare_spectrum, ctx_kwargs, oracle_for, tol_for

pytestmark = pytest.mark.gpu


def run_batched(kw, pcm, pad_mode=1, max_frames=0):
    ctx = ff.FftContext.full_v2(**kw)
    ref = oracle_for(kw)
    nf = ref.frame_count(len(pcm), pad_mode, max_frames)
    bins = ref.bins
    cap = max(nf, 1) * bins
    re = np.zeros(cap, np.float32); im = np.zeros(cap, np.float32); mag = np.zeros(cap, np.float32)
    n = ctx.execute_batched(pcm, re, im, mag, pad_mode=pad_mode, max_frames=max_frames)
    rn, rre, rim, rmag = ref.execute_batched(pcm, pad_mode=pad_mode, max_frames=max_frames)
    ctx.close()
    assert n == rn == nf
    k = n * bins
    return (re[:k], im[:k], mag[:k]), (rre.ravel(), rim.ravel(), rmag.ravel())


# -- fft_execute_batched: every option combination at N=64 -----------------
_COMBOS = list(itertools.product([0, 2], [0, 1, 2, 3], [0, 1], [(0, 0), (1, 0), (0, 1), (1, 1)], [0, 1],
                                 [(64, 16, 0), (48, 16, 1)]))


@pytest.mark.parametrize("kernel,transform,half,rp,inverse,wh", _COMBOS)
def test_batched_all_options_n64(kernel, transform, half, rp, inverse, wh):
    W, H, win = wh
    kw = ctx_kwargs(64, kernel=kernel, transform=transform, half_spectrum=half, reduce_magnitude=rp[0],
                    store_polar=rp[1], inverse=inverse, window=W, hop=H, apply_windows=win, analysis_kind=1,
                    synthesis_kind=1)
    pcm = np.random.default_rng(7).uniform(-1, 1, 700).astype(np.float32)
    got, ref = run_batched(kw, pcm)
    compare_spectrum(kw, got, ref, tol_for(64))


@pytest.mark.parametrize("N", [1, 2, 4, 8, 16, 32, 128, 256, 512, 2048, 4096, 8192, 16384])
@pytest.mark.parametrize("kernel", [0, 2])
def test_batched_sizes(N, kernel):
    kw = ctx_kwargs(N, kernel=kernel, transform=1, half_spectrum=1, window=N, hop=max(1, N // 4))
    pcm = np.random.default_rng(N).uniform(-1, 1, 4 * N + 3).astype(np.float32)
    got, ref = run_batched(kw, pcm)
    compare_spectrum(kw, got, ref, tol_for(N))


@pytest.mark.parametrize("radix,pattern", [(0, None), (2, None), (4, None), (8, None), (16, None),
                                           (0, [4, 4, 2]), (0, [16, 16])])
def test_radix_options(radix, pattern):
    kw = ctx_kwargs(1024, kernel=2, radix=radix, radix_pattern=pattern, transform=1, half_spectrum=1,
                    reduce_magnitude=1, window=1024, hop=256)
    pcm = np.random.default_rng(3).uniform(-1, 1, 8000).astype(np.float32)
    got, ref = run_batched(kw, pcm)
    compare_spectrum(kw, got, ref, tol_for(1024))


@pytest.mark.parametrize("pad_mode,ctx_pad", [(0, 0), (0, 1), (0, 2), (1, 0), (2, 0)])
@pytest.mark.parametrize("length", [50, 64, 100, 257, 300])
def test_frame_count_and_padding(pad_mode, ctx_pad, length):
    kw = ctx_kwargs(64, window=64, hop=32, transform=1, pad_mode=ctx_pad)
    pcm = np.random.default_rng(length).standard_normal(length).astype(np.float32)
    ctx = ff.FftContext.full_v2(**kw)
    ref = oracle_for(kw)
    nf = ref.frame_count(length, pad_mode)
    cap = max(nf, 1) * 64
    re = np.zeros(cap, np.float32); im = np.zeros_like(re); mag = np.zeros_like(re)
    n = ctx.execute_batched(pcm, re, im, mag, pad_mode=pad_mode)
    assert n == nf
    if n:
        _, rre, rim, rmag = ref.execute_batched(pcm, pad_mode=pad_mode)
        compare_spectrum(kw, (re[: n * 64], im[: n * 64], mag[: n * 64]),
                         (rre.ravel(), rim.ravel(), rmag.ravel()), tol_for(64))


def test_max_frames_and_w_gt_n():
    pcm = np.random.default_rng(1).standard_normal(4000).astype(np.float32)
    kw = ctx_kwargs(256, window=256, hop=64, transform=1, half_spectrum=1)
    got, ref = run_batched(kw, pcm, max_frames=5)
    compare_spectrum(kw, got, ref, tol_for(256))
    # W > N is refused (fft_cffi.cpp:718-721)
    ctx = ff.FftContext.full_v2(**ctx_kwargs(64, window=128, hop=32))
    out = np.zeros(4096, np.float32)
    assert ctx.execute_batched(pcm, out, out.copy(), out.copy()) == 0


# -- reference known-answer cases through the GPU ---------------------------
def test_kat_cffi_plain_fft(kat):
    pcm = kat["cffi_plain_fft__input"]
    ctx = ff.FftContext.full_v2(1024, transform=1, pad_mode=1)
    re = np.zeros(1024, np.float32); im = np.zeros_like(re); mag = np.zeros_like(re)
    assert ctx.execute(pcm, re, im, mag) == 1
    got = re + 1j * im
    assert np.max(np.abs(got - kat["cffi_plain_fft__expected"])) <= 1e-4
    ref = OracleContext(N=1024, transform=1, pad_mode=1)
    _, rre, rim, _ = ref.execute_batched(pcm, pad_mode=1)
    assert_close(got, rre[0] + 1j * rim[0], tol_for(1024))


@pytest.mark.parametrize("kernel", [0, 2])
def test_kat_cffi_batched_stft(kat, kernel):
    pcm = kat["cffi_batched_stft__input"]
    N, W, H, frames = (int(v) for v in kat["cffi_batched_stft__meta"])
    kw = ctx_kwargs(N, window=W, hop=H, transform=1, kernel=kernel, apply_windows=1, analysis_kind=1,
                    synthesis_kind=1)
    got, ref = run_batched(kw, pcm)
    g = (got[0] + 1j * got[1]).reshape(frames, N)
    assert np.max(np.abs(g - kat["cffi_batched_stft__expected"])) <= 1e-4
    compare_spectrum(kw, got, ref, tol_for(N))


C2C_KATS = (["single_thread_n8_b3", "prepared_n64_b4", "stockham_n256_b128_s1337",
             "stockham_n256_b128_s2337", "twiddle_meta_n16_b5", "consensus_n8_b3"]
            + [f"extended_n{N}_b{B}" for N in (2, 4, 8, 16, 32) for B in (1, 3, 16)])


@pytest.mark.parametrize("case", C2C_KATS)
@pytest.mark.parametrize("kernel", [1, 2])
def test_kat_c2c(kat, case, kernel):
    x = np.ascontiguousarray(kat[case + "__input"])
    B, N = x.shape
    ctx = ff.FftContext.full_v2(N, kernel=kernel)
    out = np.zeros_like(x)
    assert ctx.execute_c2c(x.view(np.float32), out.view(np.float32), B) == 1
    assert np.max(np.abs(out - kat[case + "__expected"])) <= float(kat[case + "__tol"][0])
    _, ref, _ = OracleContext(N=N, kernel=kernel).fft_columns(x)
    assert_close(out, ref, tol_for(N))


def test_kat_roundtrip(kat):
    x = np.ascontiguousarray(kat["roundtrip_n16_b8__input"])
    f = ff.FftContext.full_v2(16, inverse=0)
    i = ff.FftContext.full_v2(16, inverse=1)
    y = np.zeros_like(x); z = np.zeros_like(x)
    assert f.execute_c2c(x.view(np.float32), y.view(np.float32), 8) == 1
    assert i.execute_c2c(y.view(np.float32), z.view(np.float32), 8) == 1
    assert np.max(np.abs(z - x)) < 1e-5


# -- C2C extension with every hook combination ------------------------------
@pytest.mark.parametrize("N", [1, 2, 8, 64, 1024, 4096, 8192])
@pytest.mark.parametrize("kernel,transform,half,polar,reduce,inverse", [
    (0, 0, 0, 0, 0, 0), (2, 0, 0, 0, 0, 1), (0, 1, 1, 0, 0, 0), (0, 1, 1, 1, 0, 0), (2, 1, 1, 0, 1, 0),
    (0, 2, 1, 0, 0, 1), (0, 2, 1, 1, 0, 1), (2, 2, 1, 1, 0, 1), (0, 3, 0, 0, 1, 0), (0, 2, 0, 0, 0, 1)])
def test_c2c_hooks(N, kernel, transform, half, polar, reduce, inverse):
    rng = np.random.default_rng(N + 31 * transform)
    B = max(1, 4096 // N)
    x = (rng.standard_normal((B, N)) + 1j * rng.standard_normal((B, N))).astype(np.complex64)
    if polar and transform == 2:
        x = (np.abs(x) + 1j * rng.uniform(-np.pi, np.pi, x.shape)).astype(np.complex64)
    ctx = ff.FftContext.full_v2(N, kernel=kernel, transform=transform, half_spectrum=half, store_polar=polar,
                                reduce_magnitude=reduce, inverse=inverse)
    out = np.zeros_like(x)
    assert ctx.execute_c2c(x.view(np.float32), out.view(np.float32), B) == 1
    oc = OracleContext(N=N, kernel=kernel, transform=transform, half_spectrum=half, store_polar=polar,
                       reduce_magnitude=reduce, inverse=inverse)
    _, ref, _ = oc.fft_columns(x)
    if polar:
        assert_close(out.real, ref.real, tol_for(N), "polar magnitude")
        assert_close(out.real * np.exp(1j * out.imag.astype(np.float64)),
                     ref.real * np.exp(1j * ref.imag.astype(np.float64)), tol_for(N), "polar value")
    else:
        assert_close(out, ref, tol_for(N))


# -- fft_execute_complex_batched --------------------------------------------
_CB = list(itertools.product([0, 2], [0, 1, 2], [0, 1], [0, 1], [0, 1], [(0, 0), (1, 0), (1, 1)]))


@pytest.mark.parametrize("kernel,transform,half,polar,inverse,wo", _CB)
def test_complex_batched_options(kernel, transform, half, polar, inverse, wo):
    N, W, H = 64, 64, 16
    win, ola = wo
    kw = ctx_kwargs(N, kernel=kernel, transform=transform, half_spectrum=half, store_polar=polar,
                    inverse=inverse, window=W, hop=H, apply_windows=win, apply_ola=ola, analysis_kind=1,
                    synthesis_kind=1, cola_mode=1)
    ctx = ff.FftContext.full_v2(**kw)
    ref = oracle_for(kw)
    bins = ref.bins
    frames = 9
    rng = np.random.default_rng(kernel + 3 * transform + 7 * half)
    re = rng.standard_normal(frames * bins).astype(np.float32)
    im = rng.standard_normal(frames * bins).astype(np.float32)
    if polar:
        re = np.abs(re)
        im = rng.uniform(-np.pi, np.pi, frames * bins).astype(np.float32)
    out = np.zeros(frames * N, np.float32)
    n = ctx.execute_complex_batched(re, im, frames, out)
    rn, rout = ref.execute_complex_batched(re, im, frames)
    assert n == rn == frames
    assert_close(out, rout.ravel(), tol_for(N))


@pytest.mark.parametrize("N", [2, 16, 256, 1024, 4096, 8192])
def test_complex_batched_c2r_sizes(N):
    kw = ctx_kwargs(N, transform=2, half_spectrum=1, store_polar=1, inverse=1, kernel=0)
    ctx = ff.FftContext.full_v2(**kw)
    ref = oracle_for(kw)
    frames = 6
    rng = np.random.default_rng(N)
    bins = N // 2 + 1
    re = np.abs(rng.standard_normal(frames * bins)).astype(np.float32)
    im = rng.uniform(-np.pi, np.pi, frames * bins).astype(np.float32)
    out = np.zeros(frames * N, np.float32)
    assert ctx.execute_complex_batched(re, im, frames, out) == frames
    _, rout = ref.execute_complex_batched(re, im, frames)
    assert_close(out, rout.ravel(), tol_for(N))


# -- device pointers ----------------------------------------------------------
def test_device_pointer_path():
    torch = pytest.importorskip("torch")
    N, W, H = 1024, 1024, 256
    kw = ctx_kwargs(N, kernel=2, radix=4, window=W, hop=H, transform=1, reduce_magnitude=1, half_spectrum=1,
                    allow_outer_parallel=1)
    pcm = np.random.default_rng(0).uniform(-1, 1, 65536).astype(np.float32)
    ref = oracle_for(kw)
    nf = ref.frame_count(len(pcm), 1)
    bins = N // 2 + 1
    d_pcm = torch.from_numpy(pcm).cuda()
    d_re = torch.zeros(nf * bins, device="cuda"); d_im = torch.zeros_like(d_re); d_mag = torch.zeros_like(d_re)
    ctx = ff.FftContext.full_v2(**kw)
    assert ctx.execute_batched(d_pcm, d_re, d_im, d_mag, pcm_len=len(pcm), pad_mode=1) == nf == 253
    torch.cuda.synchronize()
    _, rre, rim, rmag = ref.execute_batched(pcm, pad_mode=1)
    compare_spectrum(kw, (d_re.cpu().numpy(), d_im.cpu().numpy(), d_mag.cpu().numpy()),
                     (rre.ravel(), rim.ravel(), rmag.ravel()), tol_for(N))


def test_deterministic_repeat():
    kw = ctx_kwargs(4096, kernel=2, window=4096, hop=1024, transform=1, half_spectrum=1)
    pcm = np.random.default_rng(5).standard_normal(40000).astype(np.float32)
    a, _ = run_batched(kw, pcm)
    b, _ = run_batched(kw, pcm)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


# -- multi-pass (four-step) sizes ---------------------------------------------
@pytest.mark.parametrize("N", [1 << 14, 1 << 15, 1 << 16, 1 << 17, 1 << 18, 1 << 20])
@pytest.mark.parametrize("kernel,inverse,transform,half,polar", [(2, 0, 0, 0, 0), (0, 1, 0, 0, 0),
                                                                  (0, 0, 1, 1, 1), (2, 1, 2, 1, 0)])
def test_c2c_multipass(N, kernel, inverse, transform, half, polar):
    B = max(1, (1 << 17) // N)
    rng = np.random.default_rng(N + 7 * transform)
    x = (rng.standard_normal((B, N)) + 1j * rng.standard_normal((B, N))).astype(np.complex64)
    ctx = ff.FftContext.full_v2(N, kernel=kernel, inverse=inverse, transform=transform, half_spectrum=half,
                                store_polar=polar)
    out = np.zeros_like(x)
    assert ctx.execute_c2c(x.view(np.float32), out.view(np.float32), B) == 1
    _, ref, _ = OracleContext(N=N, kernel=kernel, inverse=inverse, transform=transform, half_spectrum=half,
                              store_polar=polar).fft_columns(x)
    if polar:
        assert_close(out.real * np.exp(1j * out.imag.astype(np.float64)),
                     ref.real * np.exp(1j * ref.imag.astype(np.float64)), tol_for(N), "polar value")
    else:
        assert_close(out, ref, tol_for(N))


def test_c2c_multipass_chunks():
    # N = 65536: the L2-sized scratch holds 64 transforms, so 130 spans 3 chunks
    N, B = 1 << 16, 130
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((B, N)) + 1j * rng.standard_normal((B, N))).astype(np.complex64)
    ctx = ff.FftContext.full_v2(N, kernel=2)
    out = np.zeros_like(x)
    assert ctx.execute_c2c(x.view(np.float32), out.view(np.float32), B) == 1
    rows = [0, 63, 64, 100, 129]
    _, ref, _ = OracleContext(N=N, kernel=2).fft_columns(x[rows])
    assert_close(out[rows], ref, tol_for(N))


@pytest.mark.parametrize("N", [1 << 15, 1 << 16, 1 << 17])
@pytest.mark.parametrize("opts", [dict(transform=1, half_spectrum=1, reduce_magnitude=1),
                                  dict(transform=1, half_spectrum=1, store_polar=1, apply_windows=1,
                                       analysis_kind=1),
                                  dict(transform=0, half_spectrum=0, kernel=2, inverse=1)])
def test_stft_multipass(N, opts):
    kw = ctx_kwargs(N, window=N, hop=N // 4, **opts)
    pcm = np.random.default_rng(N).uniform(-1, 1, 2 * N + 100).astype(np.float32)
    got, ref = run_batched(kw, pcm)
    compare_spectrum(kw, got, ref, tol_for(N))


@pytest.mark.parametrize("N", [1 << 14, 1 << 15, 1 << 16])
@pytest.mark.parametrize("ola", [0, 1])
def test_complex_batched_multipass(N, ola):
    kw = ctx_kwargs(N, transform=2, half_spectrum=1, store_polar=1, inverse=1, window=N, hop=N // 2,
                    apply_windows=1, apply_ola=ola, analysis_kind=1, synthesis_kind=1, cola_mode=1)
    ctx = ff.FftContext.full_v2(**kw)
    ref = oracle_for(kw)
    frames = 3
    bins = N // 2 + 1
    rng = np.random.default_rng(N + ola)
    re = np.abs(rng.standard_normal(frames * bins)).astype(np.float32)
    im = rng.uniform(-np.pi, np.pi, frames * bins).astype(np.float32)
    out = np.zeros(frames * N, np.float32)
    assert ctx.execute_complex_batched(re, im, frames, out) == frames
    _, rout = ref.execute_complex_batched(re, im, frames)
    assert_close(out, rout.ravel(), tol_for(N))
