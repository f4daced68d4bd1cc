"""Host-buffer calls large enough to be split into overlapping upload /
compute / download chunks give the same results as the same call on device
buffers (one launch over the whole batch)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

api = pytest.importorskip("fftfree_b200.api")


@pytest.mark.parametrize("pinned", [False, True])
def test_c2c_host_pipeline_matches_device(pinned):
    N, B = 4096, 3000  # 94 MiB each way: several chunks, the last one short
    rng = np.random.default_rng(21)
    x = rng.standard_normal((B, N, 2)).astype(np.float32)
    c = api.FftContext.full_v2(N, kernel=2)
    if pinned:
        hx = torch.from_numpy(x).pin_memory()
        hy = torch.empty_like(hx).pin_memory()
    else:
        hx = torch.from_numpy(x)
        hy = torch.zeros_like(hx)
    assert c.execute_c2c(hx, hy, B) == 1
    dx = hx.cuda()
    dy = torch.empty_like(dx)
    assert c.execute_c2c(dx, dy, B) == 1
    torch.cuda.synchronize()
    assert torch.equal(hy, dy.cpu())
    # mixed: device input, host output
    hy2 = torch.zeros_like(hx)
    assert c.execute_c2c(dx, hy2, B) == 1
    assert torch.equal(hy2, hy)


def test_stft_host_pipeline_matches_device():
    N, H = 1024, 256
    L = 1 << 24  # 64 MiB of samples, 3 x 128 MiB of planar output
    rng = np.random.default_rng(22)
    pcm = rng.uniform(-1, 1, L).astype(np.float32)
    c = api.FftContext.full_v2(N, kernel=2, window=N, hop=H, transform=1, reduce_magnitude=1, half_spectrum=1,
                               apply_windows=1, analysis_kind=1)
    frames = 1 + (L - N) // H
    bins = N // 2 + 1
    re = np.zeros(frames * bins, np.float32)
    im = np.zeros_like(re)
    mg = np.zeros_like(re)
    assert c.execute_batched(pcm, re, im, mg) == frames
    dp = torch.from_numpy(pcm).cuda()
    dre = torch.empty(frames * bins, device="cuda")
    dim = torch.empty_like(dre)
    dmg = torch.empty_like(dre)
    assert c.execute_batched(dp, dre, dim, dmg, pcm_len=L) == frames
    torch.cuda.synchronize()
    np.testing.assert_array_equal(re, dre.cpu().numpy())
    np.testing.assert_array_equal(im, dim.cpu().numpy())
    np.testing.assert_array_equal(mg, dmg.cpu().numpy())
