"""Differentiable STFT magnitude on the GPU: the forward and adjoint kernels
against the FP64 oracle (oracle/grad64.py), torch float64 and finite
differences, the torch.autograd.Function, and gradient phase recovery beside
fft_griffin_lim."""
import math

import numpy as np
import pytest
import torch

from oracle import grad64
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

ag = pytest.importorskip("fftfree_b200.autograd")
api = pytest.importorskip("fftfree_b200.api")


def tol(N):
    """rel-L2 bound: 1e-5 * log2(N)."""
    return 1e-5 * max(1.0, math.log2(N))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def sinusoids(S, L, seed, n_sin=8, noise_var=0.01):
    """Sum of n_sin sinusoids per signal, frequency U(0, fs/2), amplitude
    U[0.1, 1], phase U[0, 2 pi), plus N(0, noise_var) noise (sigma = sqrt)."""
    rng = np.random.default_rng(seed)
    t = np.arange(L, dtype=np.float64)
    x = np.zeros((S, L), np.float64)
    for s in range(S):
        f = rng.uniform(0.0, 0.5, n_sin)
        a = rng.uniform(0.1, 1.0, n_sin)
        p = rng.uniform(0.0, 2 * np.pi, n_sin)
        x[s] = (a[:, None] * np.sin(2 * np.pi * f[:, None] * t[None, :] + p[:, None])).sum(0)
    x += rng.normal(0.0, math.sqrt(noise_var), (S, L))
    return x.astype(np.float32)


WIN = {None: 0, "hann": 1, "hamming": 2, "blackman": 3}


def window_of(kind, W):
    return orc.build_window(WIN[kind], W) if WIN[kind] else None


CASES = [
    # signals, length, N, W, H, window
    (1, 4096, 4, 4, 1, "hann"),
    (2, 3000, 16, 16, 4, None),
    (3, 5000, 64, 48, 16, "hamming"),
    (2, 9000, 256, 256, 64, "hann"),
    (4, 20000, 1024, 1024, 256, "hann"),
    (2, 40000, 2048, 2048, 512, "hann"),
    (1, 50000, 4096, 3000, 700, "blackman"),
    (1, 70000, 16384, 16384, 4096, "hann"),
    (2, 777, 64, 64, 100, "hann"),    # hop > window: samples between frames get 0
    (3, 50, 64, 64, 16, "hann"),      # shorter than the window: one zero-padded frame
    # sliding-window adjoint (hop N / 2^q, q <= 3): several runs of frames per signal
    (3, 33333, 512, 400, 256, "hann"),
    (2, 20000, 128, 128, 16, "hann"),
    (2, 10000, 256, 256, 256, None),
    (2, 100, 512, 512, 128, "hann"),
    (1, 300000, 8192, 8192, 2048, "hann"),
    (2, 26624, 2048, 2048, 512, "hann"),  # 49 frames: three runs of 16 and a last run of one frame
]


@pytest.mark.parametrize("S,L,N,W,H,kind", CASES)
def test_forward_matches_fp64(S, L, N, W, H, kind):
    x = sinusoids(S, L, 100 + N)
    plan = ag.StftPlan(N, H, W, kind)
    mag = plan.magnitude(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = grad64.stft_mag64(x, N, W, H, window_of(kind, W))
    assert mag.shape == ref.shape
    assert rel_l2(mag, ref) <= tol(N)


def test_forward_equals_abi_stft():
    """One signal: the same magnitudes as fft_execute_batched with reduce_magnitude."""
    x = sinusoids(1, 65536, 0)[0]
    N, W, H = 1024, 1024, 256
    plan = ag.StftPlan(N, H, W, "hann")
    mag = plan.magnitude(torch.from_numpy(x).cuda()).cpu().numpy()
    ctx = api.FftContext.full_v2(N, kernel=2, pad_mode=1, window=W, hop=H, transform=1, reduce_magnitude=1,
                                 half_spectrum=1, apply_windows=1, analysis_kind=1, synthesis_kind=1)
    F = plan.frames(len(x))
    re = np.zeros(F * (N // 2 + 1), np.float32)
    im = np.zeros_like(re)
    mg = np.zeros_like(re)
    assert ctx.execute_batched(x, re, im, mg) == F
    np.testing.assert_array_equal(mag.reshape(-1), mg)


def _loss_grad(x, N, W, H, kind, seed):
    """Upstream gradient of sum((|X| - T)^2) with T the magnitude of another signal."""
    y = sinusoids(x.shape[0], x.shape[1], seed)
    win = window_of(kind, W)
    T = grad64.stft_mag64(y, N, W, H, win)
    M = grad64.stft_mag64(x, N, W, H, win)
    return (2.0 * (M - T)).astype(np.float32)


@pytest.mark.parametrize("S,L,N,W,H,kind", CASES)
def test_backward_matches_fp64(S, L, N, W, H, kind):
    x = sinusoids(S, L, 200 + N)
    g = _loss_grad(x, N, W, H, kind, 300 + N)
    plan = ag.StftPlan(N, H, W, kind)
    gx = plan.magnitude_backward(torch.from_numpy(x).cuda(), torch.from_numpy(g).cuda()).cpu().numpy()
    ref = grad64.stft_mag_grad64(x, g, N, W, H, window_of(kind, W))
    err = rel_l2(gx, ref)
    assert err <= tol(N), err
    # samples that no frame covers are exactly zero
    covered = np.zeros(L, bool)
    for f in range(plan.frames(L)):
        covered[f * H: f * H + W] = True
    assert np.all(gx[:, ~covered] == 0.0)


@pytest.mark.parametrize("N,H", [(64, 16), (1024, 256)])
def test_backward_random_upstream(N, H):
    """A generic upstream gradient (not a loss of |X|): every bin weighs in,
    the smallest |X| included."""
    S, L = 3, 20000
    x = sinusoids(S, L, 7)
    F = grad64.frame_count(L, N, N, H)
    g = np.random.default_rng(8).standard_normal((S, F, N // 2 + 1)).astype(np.float32)
    plan = ag.StftPlan(N, H, N, "hann")
    gx = plan.magnitude_backward(torch.from_numpy(x).cuda(), torch.from_numpy(g).cuda()).cpu().numpy()
    ref = grad64.stft_mag_grad64(x, g, N, N, H, window_of("hann", N))
    err = rel_l2(gx, ref)
    print(f"random upstream N={N}: rel-L2 {err:.3e}")
    assert err <= 10 * tol(N), err


def test_backward_deterministic():
    x = torch.from_numpy(sinusoids(4, 30000, 9)).cuda()
    plan = ag.StftPlan(2048, 512, 2048, "hann")
    g = torch.randn((4, plan.frames(30000), plan.bins), device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    a = plan.magnitude_backward(x, g)
    b = plan.magnitude_backward(x, g)
    assert torch.equal(a, b)


@pytest.mark.parametrize("S,L,N,W,H,kind", CASES)
def test_backward_from_saved_phasor(S, L, N, W, H, kind):
    """The forward pass that saves X / |X| and the backward that starts from it."""
    x = sinusoids(S, L, 400 + N)
    g = _loss_grad(x, N, W, H, kind, 500 + N)
    plan = ag.StftPlan(N, H, W, kind)
    xt = torch.from_numpy(x).cuda()
    mag, ph = plan.magnitude_phasor(xt)
    assert torch.equal(mag, plan.magnitude(xt))  # same kernel, same magnitudes
    gx = plan.magnitude_backward_phasor(ph, torch.from_numpy(g).cuda(), L).cpu().numpy()
    ref = grad64.stft_mag_grad64(x, g, N, W, H, window_of(kind, W))
    err = rel_l2(gx, ref)
    assert err <= tol(N), err
    # the saved phasor is X / |X| (checked where |X| is not tiny)
    F = plan.frames(L)
    fr = np.zeros((S, F, N))
    win = window_of(kind, W)
    for f in range(F):
        cnt = max(0, min(W, L - f * H))
        seg = x[:, f * H: f * H + cnt].astype(np.float64)
        fr[:, f, :cnt] = seg * (win[:cnt] if win is not None else 1.0)
    X = np.fft.rfft(fr, axis=-1)
    big = np.abs(X) > 1e-3 * np.abs(X).max()
    u = ph.cpu().numpy().astype(np.complex128)
    assert np.max(np.abs(u[big] - X[big] / np.abs(X[big]))) < 1e-3
    assert np.allclose(np.abs(u[big]), 1.0, atol=1e-6)


def test_autograd_function():
    """Both backward sources through torch.autograd: the saved phase (the
    default while it fits the plan's budget) and the recomputed spectrum."""
    S, L, N, H = 2, 12000, 512, 128
    x0 = torch.from_numpy(sinusoids(S, L, 10)).cuda()
    T = torch.from_numpy(sinusoids(S, L, 11)).cuda()
    for budget, phase_path in ((1 << 30, True), (0, False)):
        plan = ag.StftPlan(N, H, N, "hann", phase_budget=budget)
        x = x0.clone().requires_grad_(True)
        assert plan.stores_phase(x) == phase_path
        tgt = ag.stft_magnitude(T, plan).detach()
        mag = ag.stft_magnitude(x, plan)
        loss = (mag - tgt).square().sum()
        loss.backward()
        up = 2 * (mag.detach() - tgt)
        if phase_path:
            direct = plan.magnitude_backward_phasor(plan.magnitude_phasor(x.detach())[1], up, L)
        else:
            direct = plan.magnitude_backward(x.detach(), up)
        assert torch.equal(x.grad, direct)
        ref = grad64.stft_mag_grad64(x.detach().cpu().numpy(), up.cpu().numpy(), N, N, H, window_of("hann", N))
        assert rel_l2(x.grad.cpu().numpy(), ref) <= tol(N)


def test_finite_differences_fp64():
    """4 signals x 256 samples, W = N = 64, H = 16: the GPU gradient against
    FP64 central differences of the FP64 loss."""
    S, L, N, W, H = 4, 256, 64, 64, 16
    x = sinusoids(S, L, 4)
    y = sinusoids(S, L, 5)
    win = window_of("hann", W).astype(np.float64)
    T = grad64.stft_mag64(y, N, W, H, win)
    x64 = x.astype(np.float64)

    def loss(z):
        return float(((grad64.stft_mag64(z, N, W, H, win) - T) ** 2).sum())

    plan = ag.StftPlan(N, H, W, "hann")
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    ((ag.stft_magnitude(xt, plan) - torch.from_numpy(T.astype(np.float32)).cuda()) ** 2).sum().backward()
    ours = xt.grad.cpu().numpy()
    eps = 1e-6
    fd = np.zeros_like(x64)
    for s in range(S):
        for t in range(L):
            xp = x64.copy()
            xp[s, t] += eps
            xm = x64.copy()
            xm[s, t] -= eps
            fd[s, t] = (loss(xp) - loss(xm)) / (2 * eps)
    err = rel_l2(ours, fd)
    print(f"FD check: rel-L2 {err:.3e}")
    assert err <= tol(N)


def test_differentiation_workload_full_size():
    """64 signals x 262,144 samples (8 sinusoids + noise), W = N = 2048,
    H = 512: 509 frames x 1025 bins; forward against torch.stft in float64
    and backward against the FP64 oracle, both within 1e-5 * log2(N)."""
    S, L, N, H = 64, 262144, 2048, 512
    x = sinusoids(S, L, 4)
    y = sinusoids(S, L, 44)
    plan = ag.StftPlan(N, H, N, "hann")
    xt = torch.from_numpy(x).cuda()
    mag = plan.magnitude(xt)
    T = plan.magnitude(torch.from_numpy(y).cuda())
    g = 2 * (mag - T)
    gx = plan.magnitude_backward(xt, g).cpu().numpy()
    gxp = plan.magnitude_backward_phasor(plan.magnitude_phasor(xt)[1], g, L).cpu().numpy()
    mag = mag.cpu().numpy()
    g = g.cpu().numpy()
    assert mag.shape == (S, 509, 1025)
    win = torch.hann_window(N, periodic=False, dtype=torch.float64)
    num_f = den_f = num_b = den_b = num_p = 0.0
    for s0 in range(0, S, 8):
        xs = x[s0: s0 + 8]
        ref = torch.stft(torch.from_numpy(xs.astype(np.float64)), n_fft=N, hop_length=H, window=win, center=False,
                         onesided=True, return_complex=True).abs().transpose(-1, -2).numpy()
        num_f += float(np.sum((mag[s0: s0 + 8] - ref) ** 2))
        den_f += float(np.sum(ref ** 2))
        rb = grad64.stft_mag_grad64(xs, g[s0: s0 + 8], N, N, H, window_of("hann", N))
        num_b += float(np.sum((gx[s0: s0 + 8] - rb) ** 2))
        num_p += float(np.sum((gxp[s0: s0 + 8] - rb) ** 2))
        den_b += float(np.sum(rb ** 2))
    ef, eb, ep = math.sqrt(num_f / den_f), math.sqrt(num_b / den_b), math.sqrt(num_p / den_b)
    print(f"differentiation workload: forward rel-L2 {ef:.3e} (vs torch.stft fp64, fp32 taps), "
          f"backward rel-L2 {eb:.3e} (recomputed spectrum), {ep:.3e} (saved phasor)")
    # torch's window is the exact float64 Hann, ours the float32 taps: add their rounding
    assert ef <= tol(N) + 1e-6
    assert eb <= tol(N)
    assert ep <= tol(N)


def _griffin_lim_signal(target, N, W, H, L, iters, seed):
    """fft_griffin_lim (fft_cffi.cpp:2176-2248) on the target magnitudes, then
    the signal its last iterate stands for (inverse + count-normalised
    overlap-add, as in its loop)."""
    F = target.shape[0]
    fwd = api.FftContext.full_v2(N, kernel=2, pad_mode=1, window=W, hop=H, transform=1, half_spectrum=1,
                                 apply_windows=1, analysis_kind=1, synthesis_kind=1)
    inv = api.FftContext.full_v2(N, inverse=1, kernel=2, pad_mode=1, window=W, hop=H, transform=2, half_spectrum=1)
    re = np.zeros(F * (N // 2 + 1), np.float32)
    im = np.zeros_like(re)
    mag = np.ascontiguousarray(target.reshape(-1), np.float32)
    ok = api.lib().fft_griffin_lim(fwd.handle, inv.handle, api._fp(mag), F, H, 1, iters, 1, seed, api._fp(re),
                                   api._fp(im))
    assert ok == 1
    frames = np.zeros(F * N, np.float32)
    assert inv.execute_complex_batched(re, im, F, frames) == F
    ola = np.zeros((F - 1) * H + N, np.float64)
    cnt = np.zeros_like(ola)
    for f in range(F):
        ola[f * H: f * H + N] += frames[f * N: (f + 1) * N]
        cnt[f * H: f * H + N] += 1
    ola = np.where(cnt > 0, ola / np.maximum(cnt, 1), 0.0)
    out = np.zeros(L, np.float32)
    n = min(L, len(ola))
    out[:n] = ola[:n]
    return out


def test_phase_recovery_beside_griffin_lim():
    """100 gradient steps from random noise towards a magnitude target, next to
    100 Griffin-Lim iterations on the same target; both reported as spectral
    convergence || |X| - T || / || T ||."""
    N, W, H, L = 512, 512, 128, 32768
    x = sinusoids(1, L, 12)[0]
    plan = ag.StftPlan(N, H, W, "hann")
    target = plan.magnitude(torch.from_numpy(x).cuda())
    rec, hist = ag.phase_recovery(target[None], plan, L, steps=100, lr=0.05, seed=3)
    sc_grad = hist[-1]
    gl = _griffin_lim_signal(target.cpu().numpy(), N, W, H, L, 100, 7)
    sc_gl = ag.spectral_convergence(plan.magnitude(torch.from_numpy(gl).cuda())[None], target[None])
    print(f"phase recovery: spectral convergence start {hist[0]:.4f}, gradient x100 {sc_grad:.4f}, "
          f"Griffin-Lim x100 {sc_gl:.4f}")
    assert sc_grad < 0.5 * hist[0]
    assert np.isfinite(sc_gl)


@pytest.mark.parametrize("S,L,N,W,H,kind", [(2, 9000, 256, 256, 64, "hann"), (3, 5000, 64, 48, 16, "hamming"),
                                            (4, 20000, 1024, 1024, 256, "hann"), (2, 40000, 2048, 2048, 512, "hann"),
                                            (1, 70000, 16384, 16384, 4096, "hann"), (2, 3000, 16, 16, 4, None),
                                            (3, 50, 64, 64, 16, "hann")])
def test_fused_l2_loss_matches_fp64(S, L, N, W, H, kind):
    """stft_magnitude_l2_loss: the loss sum((|X| - T)^2) against FP64 and its
    gradient (one fused forward kernel, the scaled adjoint kernel) against
    the FP64 gradient 2 (|X| - T) d|X|/dx, with an upstream gradient that
    stays on the device; the target's gradient -2 (|X| - T)."""
    x = sinusoids(S, L, 300 + N)
    y = sinusoids(S, L, 400 + N)
    win = window_of(kind, W)
    M64 = grad64.stft_mag64(x, N, W, H, win)
    T = grad64.stft_mag64(y, N, W, H, win).astype(np.float32)
    plan = ag.StftPlan(N, H, W, kind)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    tt = torch.from_numpy(T).cuda().requires_grad_(True)
    loss = ag.stft_magnitude_l2_loss(xt, tt, plan)
    up = torch.tensor(0.75, device="cuda")
    loss.backward(up)
    ref_loss = float(((M64 - T.astype(np.float64)) ** 2).sum())
    assert abs(float(loss) - ref_loss) <= tol(N) * ref_loss
    g64 = 2.0 * 0.75 * (M64 - T.astype(np.float64))
    ref = grad64.stft_mag_grad64(x, g64, N, W, H, win)
    assert rel_l2(xt.grad.cpu().numpy(), ref) <= tol(N)
    assert rel_l2(tt.grad.cpu().numpy(), -g64) <= tol(N)
    # the same loss through the unfused path (magnitude + torch ops)
    xt2 = torch.from_numpy(x).cuda().requires_grad_(True)
    l2 = (ag.stft_magnitude(xt2, plan) - tt.detach()).square().sum()
    l2.backward(up)
    assert abs(float(l2) - float(loss)) <= tol(N) * float(loss)
    assert rel_l2(xt.grad.cpu().numpy(), xt2.grad.cpu().numpy()) <= tol(N)
    plan.close()


def test_fused_l2_loss_deterministic_and_budget_fallback():
    """Two runs give the same loss and gradient bits; a plan whose phase
    budget is exceeded takes the unfused path with the same result."""
    S, L, N, H = 2, 40000, 2048, 512
    x = torch.from_numpy(sinusoids(S, L, 7)).cuda()
    plan = ag.StftPlan(N, H, N, "hann")
    T = plan.magnitude(x.roll(1, 0)).detach()
    outs = []
    for _ in range(2):
        xr = x.clone().requires_grad_(True)
        loss = ag.stft_magnitude_l2_loss(xr, T, plan)
        loss.backward()
        outs.append((float(loss), xr.grad.clone()))
    assert outs[0][0] == outs[1][0] and torch.equal(outs[0][1], outs[1][1])
    small = ag.StftPlan(N, H, N, "hann", phase_budget=0)
    xr = x.clone().requires_grad_(True)
    loss = ag.stft_magnitude_l2_loss(xr, T, small)
    loss.backward()
    assert abs(float(loss) - outs[0][0]) <= tol(N) * outs[0][0]
    assert rel_l2(xr.grad.cpu().numpy(), outs[0][1].cpu().numpy()) <= tol(N)
    plan.close()
    small.close()
