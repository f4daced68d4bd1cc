"""Differentiable STFT magnitude on the GPU.

``StftPlan`` owns a forward R2C half-spectrum context of the library
(``fft_init_full_v2`` with the reference's framing, window and pad rule) and
``stft_magnitude`` is a ``torch.autograd.Function`` over its two kernels:

* forward: ``fftfree_stft_magnitude`` -- the batched STFT kernel of
  ``fft_execute_batched`` with a magnitude-only epilogue;
* backward: ``fftfree_stft_magnitude_backward`` -- the adjoint kernel
  (magnitude/phase chain rule, conjugate-transposed half-spectrum transform,
  gather form of the overlap-add adjoint of framing), which recomputes the
  spectrum from the saved signal instead of storing it.

While the saved phasor of a call fits the plan's ``phase_budget`` (bytes),
the forward pass instead writes the unit phasor X / |X| beside |X|
(``fftfree_stft_magnitude_phasor``) and the backward starts from it
(``fftfree_stft_magnitude_backward_phasor``): one transform per frame
instead of two.  Longer signals keep the recompute path, which stores
nothing beyond the signal.

Both run on torch's current CUDA stream and never synchronise the host.
The reference has no autograd path; its ``train_mipmap_weights.py``
(lines 395-415) approximates the adjoint with a forward STFT.

``phase_recovery`` drives the signal from random noise towards a target
magnitude by gradient steps through this Function; it is the gradient
counterpart of ``fft_griffin_lim`` (fft_cffi.cpp:2176-2248).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Tuple

import torch

from . import api

WINDOWS = {"rect": 0, "rectangular": 0, None: 0, "hann": 1, "hamming": 2, "blackman": 3, "tukey": 4}


class StftPlan:
    """Magnitude STFT of n_fft points, window length ``win_length`` (<= n_fft),
    hop ``hop``; ``window`` is one of the reference's analysis windows
    (fft_cffi.cpp:163-208, symmetric, denominator W-1) or None for none."""

    def __init__(self, n_fft: int, hop: int, win_length: Optional[int] = None, window: Optional[str] = "hann",
                 window_param: float = 0.0, pad_mode: int = 1, device: Optional[int] = None,
                 phase_budget: int = 1 << 30):
        if n_fft < 2 or n_fft & (n_fft - 1) or n_fft > 16384:
            raise ValueError("n_fft must be a power of two in [2, 16384]")
        self.n_fft = int(n_fft)
        self.hop = int(hop)
        self.win_length = int(win_length or n_fft)
        self.window = window
        self.pad_mode = int(pad_mode)
        self.bins = self.n_fft // 2 + 1
        self.phase_budget = int(phase_budget)
        if window not in WINDOWS:
            raise ValueError(f"unknown window {window!r}")
        self.device = torch.cuda.current_device() if device is None else int(device)
        with torch.cuda.device(self.device):
            self.ctx = api.FftContext.full_v2(
                self.n_fft, threads=1, lanes=1, inverse=0, kernel=2, radix=0, pad_mode=self.pad_mode,
                window=self.win_length, hop=self.hop, transform=1, reduce_magnitude=1, store_polar=0,
                half_spectrum=1, silent_crash_reports=1, apply_windows=1 if WINDOWS[window] else 0,
                analysis_kind=WINDOWS[window], analysis_p1=window_param, synthesis_kind=WINDOWS[window],
                synthesis_p1=window_param)
        if not self.ctx.handle:
            raise RuntimeError("fft_init_full_v2 failed for the magnitude STFT plan")
        self.ctx.set_async(1)

    def frames(self, length: int) -> int:
        """Frames per signal under fft_execute_batched's framing rule
        (fft_cffi.cpp:710-750)."""
        W, H = self.win_length, self.hop
        if length < W:
            return 1 if self.pad_mode == 1 else 0
        return 1 + (length - W) // H

    def _check(self, x: torch.Tensor) -> torch.Tensor:
        if not x.is_cuda or x.dtype != torch.float32:
            raise TypeError("signals must be a float32 CUDA tensor")
        if x.dim() not in (1, 2):
            raise ValueError("signals must be (length,) or (signals, length)")
        if x.device.index != self.device:
            raise ValueError(f"plan lives on cuda:{self.device}, signals on {x.device}")
        return x.contiguous()

    def _bind_stream(self):
        self.ctx.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def magnitude(self, x: torch.Tensor) -> torch.Tensor:
        """|STFT| as (signals, frames, n_fft/2+1) (no leading dim for 1-D x)."""
        x = self._check(x)
        x2 = x.view(1, -1) if x.dim() == 1 else x
        S, L = x2.shape
        F = self.frames(L)
        out = torch.empty((S, F, self.bins), dtype=torch.float32, device=x.device)
        if F == 0:
            raise ValueError("signal shorter than one frame")
        self._bind_stream()
        got = self.ctx.stft_magnitude(x2, S, L, out)
        if got != F:
            raise RuntimeError(f"fftfree_stft_magnitude returned {got} frames, expected {F}")
        return out[0] if x.dim() == 1 else out

    def stores_phase(self, x: torch.Tensor) -> bool:
        """True when the forward pass of ``x`` saves the unit phasor X / |X|
        for the backward (its size within ``phase_budget``) rather than
        leaving the spectrum to be recomputed."""
        S = 1 if x.dim() == 1 else x.shape[0]
        return S * self.frames(x.shape[-1]) * self.bins * 8 <= self.phase_budget

    def magnitude_phasor(self, x: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
        """(|STFT|, STFT / |STFT|) with the layout of ``magnitude``, the
        phasor complex64 and 0 where |X| = 0."""
        x = self._check(x)
        x2 = x.view(1, -1) if x.dim() == 1 else x
        S, L = x2.shape
        F = self.frames(L)
        if F == 0:
            raise ValueError("signal shorter than one frame")
        mag = torch.empty((S, F, self.bins), dtype=torch.float32, device=x.device)
        ph = torch.empty((S, F, self.bins), dtype=torch.complex64, device=x.device)
        self._bind_stream()
        got = self.ctx.stft_magnitude_phasor(x2, S, L, mag, ph)
        if got != F:
            raise RuntimeError(f"fftfree_stft_magnitude_phasor returned {got} frames, expected {F}")
        return (mag[0], ph[0]) if x.dim() == 1 else (mag, ph)

    def magnitude_backward_phasor(self, phasor: torch.Tensor, grad_mag: torch.Tensor, length: int) -> torch.Tensor:
        """d(sum(grad_mag * |STFT x|))/dx from the phasor ``magnitude_phasor``
        saved; (signals, length), or (length,) for a 2-D phasor."""
        ph = phasor.contiguous()
        if ph.dtype != torch.complex64:
            raise TypeError("phasor must be complex64")
        S = 1 if ph.dim() == 2 else ph.shape[0]
        F = self.frames(length)
        g = grad_mag.to(dtype=torch.float32).contiguous()
        if ph.numel() != S * F * self.bins or g.numel() != ph.numel() or not g.is_cuda or not ph.is_cuda:
            raise ValueError("phasor / grad_mag do not match the forward output")
        gx = torch.empty((S, length), dtype=torch.float32, device=ph.device)
        self._bind_stream()
        got = self.ctx.stft_magnitude_backward_phasor(ph, S, length, g, gx)
        if got != F:
            raise RuntimeError(f"fftfree_stft_magnitude_backward_phasor returned {got} frames, expected {F}")
        return gx[0] if ph.dim() == 2 else gx

    def magnitude_l2(self, x: torch.Tensor, target: torch.Tensor):
        """One pass for the spectral L2 loss: (partial sums of (|X| - T)^2,
        residual |X| - T, unit phasor), the residual and phasor in the layout
        of ``magnitude``; the loss is the sum of the partial sums."""
        x = self._check(x)
        x2 = x.view(1, -1) if x.dim() == 1 else x
        S, L = x2.shape
        F = self.frames(L)
        if F == 0:
            raise ValueError("signal shorter than one frame")
        tg = target.to(device=x.device, dtype=torch.float32).contiguous()
        if tg.numel() != S * F * self.bins:
            raise ValueError("target does not match the magnitude STFT's shape")
        res = torch.empty((S, F, self.bins), dtype=torch.float32, device=x.device)
        ph = torch.empty((S, F, self.bins), dtype=torch.complex64, device=x.device)
        parts = torch.empty(self.ctx.stft_l2_partials(S * F), dtype=torch.float32, device=x.device)
        self._bind_stream()
        got = self.ctx.stft_magnitude_l2(x2, S, L, tg, res, ph, parts)
        if got != F:
            raise RuntimeError(f"fftfree_stft_magnitude_l2 returned {got} frames, expected {F}")
        return parts, res, ph

    def magnitude_backward_phasor_scaled(self, phasor: torch.Tensor, grad_mag: torch.Tensor, length: int,
                                         scale: Optional[torch.Tensor], factor: float) -> torch.Tensor:
        """``magnitude_backward_phasor`` times factor (times the one-element
        CUDA tensor ``scale``, read by the kernel)."""
        ph = phasor.contiguous()
        S = 1 if ph.dim() == 2 else ph.shape[0]
        F = self.frames(length)
        g = grad_mag.to(dtype=torch.float32).contiguous()
        if ph.numel() != S * F * self.bins or g.numel() != ph.numel():
            raise ValueError("phasor / grad_mag do not match the forward output")
        sc = None
        if scale is not None:
            sc = scale.to(device=ph.device, dtype=torch.float32).reshape(1).contiguous()
        gx = torch.empty((S, length), dtype=torch.float32, device=ph.device)
        self._bind_stream()
        got = self.ctx.stft_magnitude_backward_phasor_scaled(ph, S, length, g, gx, sc, factor)
        if got != F:
            raise RuntimeError(f"fftfree_stft_magnitude_backward_phasor_scaled returned {got} frames, expected {F}")
        return gx[0] if ph.dim() == 2 else gx

    def magnitude_backward(self, x: torch.Tensor, grad_mag: torch.Tensor) -> torch.Tensor:
        """d(sum(grad_mag * |STFT x|))/dx, shaped like x."""
        x = self._check(x)
        x2 = x.view(1, -1) if x.dim() == 1 else x
        S, L = x2.shape
        F = self.frames(L)
        g = grad_mag.to(dtype=torch.float32).contiguous()
        if g.numel() != S * F * self.bins or not g.is_cuda:
            raise ValueError("grad_mag does not match the forward output")
        gx = torch.empty_like(x2)
        self._bind_stream()
        got = self.ctx.stft_magnitude_backward(x2, S, L, g, gx)
        if got != F:
            raise RuntimeError(f"fftfree_stft_magnitude_backward returned {got} frames, expected {F}")
        return gx.view_as(x)

    def close(self):
        if getattr(self, "ctx", None) is not None:
            self.ctx.close()
            self.ctx = None


class _StftMagnitude(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, plan: StftPlan) -> torch.Tensor:
        ctx.plan = plan
        ctx.length = x.shape[-1]
        ctx.with_phase = plan.stores_phase(x)
        if ctx.with_phase:
            mag, ph = plan.magnitude_phasor(x)
            ctx.save_for_backward(ph)
        else:
            mag = plan.magnitude(x)
            ctx.save_for_backward(x)  # long signals: the spectrum is recomputed, not stored
        return mag

    @staticmethod
    def backward(ctx, grad_mag: torch.Tensor):
        (saved,) = ctx.saved_tensors
        if ctx.with_phase:
            return ctx.plan.magnitude_backward_phasor(saved, grad_mag, ctx.length), None
        return ctx.plan.magnitude_backward(saved, grad_mag), None


def stft_magnitude(x: torch.Tensor, plan: StftPlan) -> torch.Tensor:
    """Differentiable |STFT x| through the library's kernels."""
    return _StftMagnitude.apply(x, plan)


class _StftMagnitudeL2(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: torch.Tensor, target: torch.Tensor, plan: StftPlan) -> torch.Tensor:
        parts, res, ph = plan.magnitude_l2(x, target)
        ctx.plan = plan
        ctx.length = x.shape[-1]
        ctx.x_dim = x.dim()
        ctx.save_for_backward(ph, res)
        return parts.sum()

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        ph, res = ctx.saved_tensors
        gx = None
        if ctx.needs_input_grad[0]:
            gx = ctx.plan.magnitude_backward_phasor_scaled(ph, res, ctx.length, grad_out, 2.0)
            if ctx.x_dim == 1:
                gx = gx.reshape(-1)
        gt = None
        if ctx.needs_input_grad[1]:
            gt = res * (-2.0 * grad_out)
            if ctx.x_dim == 1:
                gt = gt[0]
        return gx, gt, None


def stft_magnitude_l2_loss(x: torch.Tensor, target: torch.Tensor, plan: StftPlan) -> torch.Tensor:
    """sum((|STFT x| - target)^2), differentiable, fused: one forward kernel
    writes the residual, the unit phasor and the loss's partial sums; the
    backward is one adjoint kernel scaled by the upstream gradient on the
    device.  Signals whose phasor exceeds the plan's ``phase_budget`` take
    ``stft_magnitude`` and torch's elementwise ops instead."""
    if not plan.stores_phase(x):
        return (stft_magnitude(x, plan) - target).square().sum()
    return _StftMagnitudeL2.apply(x, target, plan)


def spectral_convergence(mag: torch.Tensor, target: torch.Tensor) -> float:
    """|| |X| - T ||_F / || T ||_F."""
    return float(torch.linalg.vector_norm(mag - target) / torch.linalg.vector_norm(target))


def phase_recovery(target: torch.Tensor, plan: StftPlan, length: int, steps: int = 100, lr: float = 0.05,
                   seed: int = 0, x0: Optional[torch.Tensor] = None) -> Tuple[torch.Tensor, List[float]]:
    """Find a signal whose STFT magnitude matches ``target`` by ``steps`` Adam
    steps on sum((|STFT x| - target)^2), starting from seeded uniform noise
    (or ``x0``).  Returns the signal and the spectral convergence before each
    step and after the last."""
    signals = target.shape[0] if target.dim() == 3 else 1
    if x0 is None:
        gen = torch.Generator(device=target.device).manual_seed(seed)
        x0 = (torch.rand((signals, length), generator=gen, device=target.device) * 2 - 1) * 0.1
    x = x0.detach().clone().reshape(signals, length).requires_grad_(True)
    tgt = target.reshape(signals, -1, plan.bins)
    # |X| of a unit-amplitude sinusoid under a W-tap window is about W/4:
    # the step is scaled to the signal amplitude the target implies
    scale = float(tgt.abs().max())
    opt = torch.optim.Adam([x], lr=lr * max(4.0 * scale / plan.win_length, 1e-12))
    history = []
    for _ in range(steps):
        opt.zero_grad(set_to_none=True)
        mag = stft_magnitude(x, plan)
        history.append(spectral_convergence(mag.detach(), tgt))
        loss = (mag - tgt).square().sum()
        loss.backward()
        opt.step()
    with torch.no_grad():
        history.append(spectral_convergence(stft_magnitude(x, plan), tgt))
    out = x.detach()
    return (out[0] if target.dim() == 2 else out), history


_PLANS: Dict[Tuple, StftPlan] = {}


def plan_for(n_fft: int, hop: int, win_length: Optional[int] = None, window: Optional[str] = "hann",
             device: Optional[int] = None) -> StftPlan:
    """A cached StftPlan per (n_fft, hop, win_length, window, device)."""
    dev = torch.cuda.current_device() if device is None else int(device)
    key = (n_fft, hop, win_length or n_fft, window, dev)
    p = _PLANS.get(key)
    if p is None:
        p = _PLANS[key] = StftPlan(n_fft, hop, win_length, window, device=dev)
    return p
