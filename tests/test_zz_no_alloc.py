"""fftfree_execute_complex_batched_noalloc -- the entry point for callers
that cannot allocate GPU memory while they run (real-time audio threads,
processes whose GPU memory is reserved up front by another allocator).

Checks, through the C ABI, that two calls in a row give the same result as
the existing fft_execute_complex_batched entry point (within the parity
tolerance), that the calls allocate no device memory, and that the limits
(device buffers only, frames * N within the fixed scratch) are enforced.
Kept in a file that pytest collects last."""
import numpy as np
import pytest

import fftfree_b200 as ff
from tests.helpers import assert_close, tol_for

pytestmark = pytest.mark.gpu

MAX_SAMPLES = 1 << 22


def _ctx(N, W, H):
    return ff.FftContext.full_v2(N, inverse=1, transform=ff.FFT_TRANSFORM_C2R, half_spectrum=1, window=W,
                                 hop=H, apply_windows=1, apply_ola=1, analysis_kind=ff.FFT_WINDOW_HANN,
                                 synthesis_kind=ff.FFT_WINDOW_HANN, cola_mode=ff.FFT_COLA_NORMALIZE)


def test_noalloc_matches_existing_entry_point_twice():
    torch = pytest.importorskip("torch")
    N, W, H, frames = 1024, 1024, 256, 96
    bins = N // 2 + 1
    g = torch.Generator(device="cuda").manual_seed(9)
    re = torch.randn(frames * bins, device="cuda", generator=g)
    im = torch.randn(frames * bins, device="cuda", generator=g)
    ref = torch.zeros(frames * N, device="cuda")
    out = [torch.full((frames * N,), float("nan"), device="cuda") for _ in range(2)]
    ctx = _ctx(N, W, H)
    L = ff.lib()
    fp = ff.api._fp
    assert ctx.execute_complex_batched(re, im, frames, ref) == frames
    # first call on the device does the one-time symbol lookup
    assert L.fftfree_execute_complex_batched_noalloc(ctx.handle, fp(re), fp(im), frames, fp(out[0]), 0) == frames
    torch.cuda.synchronize()
    # free device memory is device-wide (another process can move it), so a
    # few measured pairs are taken and one unchanged pair suffices
    unchanged = False
    for _ in range(4):
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for o in out:
            assert L.fftfree_execute_complex_batched_noalloc(ctx.handle, fp(re), fp(im), frames, fp(o), 0) == frames
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        if free1 == free0:
            unchanged = True
            break
    assert unchanged, "the no-alloc calls changed free device memory"
    r = ref.cpu().numpy()
    for o in out:
        assert_close(o.cpu().numpy(), r, tol_for(N), "noalloc vs fft_execute_complex_batched")
    ctx.close()


def test_noalloc_without_overlap_add():
    torch = pytest.importorskip("torch")
    N, frames = 256, 40
    ctx = ff.FftContext.full_v2(N, inverse=1, transform=ff.FFT_TRANSFORM_C2R, half_spectrum=1, store_polar=1)
    bins = N // 2 + 1
    g = torch.Generator(device="cuda").manual_seed(3)
    re = torch.rand(frames * bins, device="cuda", generator=g)
    im = (torch.rand(frames * bins, device="cuda", generator=g) - 0.5) * 6.0
    ref = torch.zeros(frames * N, device="cuda")
    out = torch.zeros(frames * N, device="cuda")
    assert ctx.execute_complex_batched(re, im, frames, ref) == frames
    fp = ff.api._fp
    for _ in range(2):
        assert ff.lib().fftfree_execute_complex_batched_noalloc(ctx.handle, fp(re), fp(im), frames, fp(out),
                                                               0) == frames
        assert_close(out.cpu().numpy(), ref.cpu().numpy(), tol_for(N))


def test_noalloc_limits():
    torch = pytest.importorskip("torch")
    N = 4096
    ctx = _ctx(N, N, N // 4)
    bins = N // 2 + 1
    frames = MAX_SAMPLES // N + 1  # one frame beyond the fixed scratch
    re = torch.zeros(frames * bins, device="cuda")
    im = torch.zeros_like(re)
    out = torch.zeros(frames * N, device="cuda")
    fp = ff.api._fp
    L = ff.lib()
    assert L.fftfree_execute_complex_batched_noalloc(ctx.handle, fp(re), fp(im), frames, fp(out), 0) == 0
    # within the limit it runs
    assert L.fftfree_execute_complex_batched_noalloc(ctx.handle, fp(re), fp(im), frames - 1, fp(out), 0) == \
        frames - 1
    # sizes beyond one pass are refused; a half-spectrum C2R context of
    # 16384 points runs (its transform is an 8192-point one)
    big = _ctx(16384, 16384, 4096)
    bb = 16384 // 2 + 1
    re2 = torch.randn(8 * bb, device="cuda")
    im2 = torch.randn(8 * bb, device="cuda")
    out2 = torch.zeros(8 * 16384, device="cuda")
    ref2 = torch.zeros(8 * 16384, device="cuda")
    assert big.execute_complex_batched(re2, im2, 8, ref2) == 8
    assert L.fftfree_execute_complex_batched_noalloc(big.handle, fp(re2), fp(im2), 8, fp(out2), 0) == 8
    assert_close(out2.cpu().numpy(), ref2.cpu().numpy(), tol_for(16384))
    c2c = ff.FftContext.full_v2(16384, inverse=1)
    assert L.fftfree_execute_complex_batched_noalloc(c2c.handle, fp(re2), fp(im2), 1, fp(out2), 0) == 0
    # host buffers are refused (they would need staging allocations)
    h = np.zeros(bins * 4, np.float32)
    ho = np.zeros(N * 4, np.float32)
    assert L.fftfree_execute_complex_batched_noalloc(ctx.handle, fp(h), fp(h), 4, fp(ho), 0) == 0
