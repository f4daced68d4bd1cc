"""Sharding of the batched STFT / FFT over the ranks of a process group (one
process per GPU).

The units of the path are independent (frames of a signal, transforms of a
batch, items of a ragged batch), so a multi-GPU run partitions them with no
data-path collective: every rank transforms a contiguous range of frames
(or transforms) on its own GPU.  A single long signal splits by frame range;
the rank's samples are the frames' span, W - H samples of halo beyond its
last hop, read directly from the caller's buffer.  An all-gather is needed
only when one rank must hold the whole output (``gather_frames``).

The frame rule of fft_execute_batched (fft_cffi.cpp:710-750) makes every
frame but a lone partial one full, so a span of f1 - f0 frames starting at
f0 * H holds exactly those frames: running the context's own call on it
with max_frames = f1 - f0 gives the same frames, bit for bit, as the
single-GPU call.
"""
from __future__ import annotations

from typing import Tuple


def frame_range(total: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [f0, f1) of ``total`` units for ``rank`` of ``world``
    (the first total % world ranks take one more)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(max(int(total), 0), world)
    f0 = rank * base + min(rank, extra)
    return f0, f0 + base + (1 if rank < extra else 0)


def sample_span(f0: int, f1: int, W: int, H: int, pcm_len: int) -> Tuple[int, int]:
    """Samples [s0, s1) that frames f0 .. f1 - 1 read (frame f covers
    f * H .. f * H + W, clipped to the signal)."""
    if f1 <= f0:
        s = min(f0 * H, pcm_len)
        return s, s
    s0 = f0 * H
    return s0, min(pcm_len, (f1 - 1) * H + W)


def stft_shard(ctx, pcm, pcm_len: int, out_real, out_imag, out_mag, rank: int, world: int, pad_mode: int = 1,
               max_frames: int = 0):
    """This rank's frames of ``fft_execute_batched(ctx, pcm, pcm_len, ...)``.

    ``pcm`` is the whole signal (a CUDA tensor, host array or device
    address; only this rank's span is read); the outputs receive this rank's
    frames, frame-major from their start.  Returns (f0, frames) -- the rank's
    first global frame and how many it wrote."""
    from . import api

    total = ctx.frame_count(pcm_len, pad_mode, max_frames)
    f0, f1 = frame_range(total, rank, world)
    if f1 <= f0:
        return f0, 0
    W = ctx.window_length()
    H = ctx.hop_length()
    s0, s1 = sample_span(f0, f1, W, H, pcm_len)
    base = api.address(pcm)
    n = ctx.execute_batched(base + 4 * s0, out_real, out_imag, out_mag, pcm_len=s1 - s0, pad_mode=pad_mode,
                            max_frames=f1 - f0)
    return f0, n


def gather_frames(local, total: int, rank: int, world: int, group=None):
    """All-gather per-rank frame blocks (torch tensors of shape (frames_r,
    bins), ranks in order) into the (total, bins) tensor on every rank.
    Blocks are padded to the largest rank's frame count for the collective."""
    import torch
    import torch.distributed as dist

    bins = local.shape[1]
    most = frame_range(total, 0, world)[1]  # rank 0 holds the most frames
    buf = torch.zeros((most, bins), dtype=local.dtype, device=local.device)
    buf[: local.shape[0]] = local
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = []
    for r in range(world):
        f0, f1 = frame_range(total, r, world)
        out.append(parts[r][: f1 - f0])
    return torch.cat(out, 0)


def max_over_ranks(value: float, device="cpu", group=None) -> float:
    """The largest ``value`` over the ranks (timings: a multi-GPU step takes
    as long as its slowest rank)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
