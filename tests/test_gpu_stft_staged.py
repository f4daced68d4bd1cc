"""The staged STFT kernel (FFTFREE_STFT_STAGED=1: each block bulk-copies its
frames' sample span and the window into shared memory) against the default
kernel, through the C ABI: the same arithmetic on the same samples, so the
outputs must be bit-identical -- including blocks whose frames run past the
signal's end, which load from global memory instead."""
import numpy as np
import pytest

from tests.helpers import assert_close, tol_for

pytestmark = pytest.mark.gpu

api = pytest.importorskip("fftfree_b200.api")
torch = pytest.importorskip("torch")


def _run(monkeypatch, staged, N, H, length, reduce, apply_windows):
    monkeypatch.setenv("FFTFREE_STFT_STAGED", "1" if staged else "0")
    ctx = api.FftContext.full_v2(N, kernel=2, window=N, hop=H, transform=1, half_spectrum=1,
                                 reduce_magnitude=reduce, apply_windows=apply_windows, analysis_kind=1)
    g = torch.Generator(device="cuda").manual_seed(N + H + length)
    pcm = torch.rand(length, device="cuda", generator=g) * 2 - 1
    frames = ctx.frame_count(length, 1)
    bins = N // 2 + 1
    out = [torch.zeros(frames * bins, device="cuda") for _ in range(3)]
    assert ctx.execute_batched(pcm, *out, pcm_len=length) == frames
    torch.cuda.synchronize()
    res = [o.cpu().numpy() for o in out]
    ctx.close()
    return pcm.cpu().numpy(), res


@pytest.mark.parametrize("N,H,length,reduce,win", [
    (1024, 256, 65536, 1, 1),     # the config-1 shape
    (1024, 256, 65536 + 300, 0, 0),  # a partial last frame: its block loads from global memory
    (2048, 512, 100000, 1, 1),
    (256, 64, 20000, 0, 1),
    (64, 16, 5000, 1, 0),
    (4096, 1024, 70000, 0, 1),
])
def test_staged_equals_default(monkeypatch, N, H, length, reduce, win):
    _, a = _run(monkeypatch, False, N, H, length, reduce, win)
    pcm, b = _run(monkeypatch, True, N, H, length, reduce, win)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    # and the magnitudes are those of the FP64 transform of the frames
    from oracle import grad64
    from oracle import oracle as orc
    ref = grad64.stft_mag64(pcm[None, :], N, N, H, orc.build_window(1, N) if win else None)
    assert ref.size == b[2].size
    assert_close(b[2], ref.ravel(), tol_for(N))
