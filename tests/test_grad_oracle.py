"""The FP64 gradient oracle of the magnitude STFT against FP64 finite
differences, torch float64 autograd and torch.stft (CPU only)."""
import numpy as np
import pytest
import torch

from oracle import grad64
from oracle import oracle as orc


def _torch_mag64(x, N, W, H, win):
    """|STFT| in float64 with torch ops (frames by unfold, zero-padded to N)."""
    fr = x.unfold(-1, W, H) if x.shape[-1] >= W else torch.nn.functional.pad(x, (0, W - x.shape[-1])).unsqueeze(-2)
    if win is not None:
        fr = fr * torch.as_tensor(win, dtype=torch.float64)[:W]
    fr = torch.nn.functional.pad(fr, (0, N - W))
    return torch.fft.rfft(fr, dim=-1).abs()


def _case(seed, S, L, N, W, H, kind):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (S, L)).astype(np.float32)
    win = orc.build_window(kind, W) if kind else None
    F = grad64.frame_count(L, N, W, H)
    g = rng.standard_normal((S, F, N // 2 + 1))
    return x, win, g


@pytest.mark.parametrize("S,L,N,W,H,kind", [
    (2, 300, 64, 48, 16, 1),
    (3, 257, 32, 32, 8, 2),
    (1, 1000, 128, 100, 37, 0),
    (2, 64, 64, 64, 16, 3),
])
def test_grad64_matches_torch_autograd(S, L, N, W, H, kind):
    x, win, g = _case(11, S, L, N, W, H, kind)
    xt = torch.tensor(x, dtype=torch.float64, requires_grad=True)
    mag = _torch_mag64(xt, N, W, H, win)
    np.testing.assert_allclose(mag.detach().numpy(), grad64.stft_mag64(x, N, W, H, win), rtol=1e-12, atol=1e-12)
    (mag * torch.tensor(g)).sum().backward()
    ours = grad64.stft_mag_grad64(x, g, N, W, H, win)
    np.testing.assert_allclose(ours, xt.grad.numpy(), rtol=1e-10, atol=1e-10)


def test_grad64_finite_differences():
    """FP64 central differences on 4 signals of 256 samples, W = N = 64, H = 16,
    Hann, loss sum((|X| - T)^2) with T the magnitude of another signal."""
    rng = np.random.default_rng(4)
    S, L, N, W, H = 4, 256, 64, 64, 16
    x = rng.uniform(-1, 1, (S, L))
    y = rng.uniform(-1, 1, (S, L))
    win = orc.build_window(1, W).astype(np.float64)
    T = grad64.stft_mag64(y, N, W, H, win)

    def loss(z):
        return float(((grad64.stft_mag64(z, N, W, H, win) - T) ** 2).sum())

    g = 2.0 * (grad64.stft_mag64(x, N, W, H, win) - T)
    ana = grad64.stft_mag_grad64(x, g, N, W, H, win)
    eps = 1e-6
    fd = np.zeros_like(x)
    for s in range(S):
        for t in range(L):
            xp = x.copy()
            xp[s, t] += eps
            xm = x.copy()
            xm[s, t] -= eps
            fd[s, t] = (loss(xp) - loss(xm)) / (2 * eps)
    err = np.linalg.norm(ana - fd) / np.linalg.norm(fd)
    assert err < 1e-7, err


def test_grad64_matches_torch_stft_full_window():
    """W = N: the framing equals torch.stft(center=False) with a symmetric Hann."""
    rng = np.random.default_rng(5)
    S, L, N, H = 2, 4096, 256, 64
    x = rng.uniform(-1, 1, (S, L))
    win = orc.build_window(1, N).astype(np.float64)
    ref = torch.stft(torch.tensor(x), n_fft=N, hop_length=H,
                     window=torch.hann_window(N, periodic=False, dtype=torch.float64), center=False,
                     onesided=True, return_complex=True).abs().transpose(-1, -2).numpy()
    # the library's window taps are float32 (built in float64, then rounded)
    np.testing.assert_allclose(grad64.stft_mag64(x, N, N, H, win), ref, rtol=1e-5, atol=1e-5)


def test_grad64_partial_frame():
    """A signal shorter than the window (pad_mode 1) gives one zero-padded frame."""
    x, win, g = _case(7, 2, 40, 64, 64, 16, 1)
    assert grad64.frame_count(40, 64, 64, 16) == 1
    xt = torch.tensor(x, dtype=torch.float64, requires_grad=True)
    mag = _torch_mag64(xt, 64, 64, 16, win)
    (mag * torch.tensor(g)).sum().backward()
    np.testing.assert_allclose(grad64.stft_mag_grad64(x, g, 64, 64, 16, win), xt.grad.numpy(), rtol=1e-10,
                               atol=1e-10)
