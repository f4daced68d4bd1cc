"""The multi-GPU path's host logic on CPU ranks (gloo, world size 2).

A multi-GPU run splits the frames of a signal (or the transforms of a batch)
into contiguous per-rank ranges with no data-path collective; the timing of
a step is the maximum over ranks; an all-gather assembles the output where
one rank needs all of it.  Here two gloo ranks on 127.0.0.1 run that logic
(fftfree_b200.shard) with the oracle as each rank's transform: the gathered
frames are bit-identical to the single-process result for every frame rule,
and the timing reduction returns the slowest rank's value on every rank.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fftfree_b200.shard import frame_range, sample_span

WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, cases, q):
    import datetime

    import torch
    import torch.distributed as dist

    from fftfree_b200.shard import frame_range, gather_frames, max_over_ranks, sample_span
    from oracle.oracle import OracleContext

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        results = []
        for (N, W, H, L, pad, seed) in cases:
            ctx = OracleContext(N=N, window=W, hop=H, transform=1, half_spectrum=1, pad_mode=pad)
            pcm = np.random.default_rng(seed).uniform(-1, 1, L).astype(np.float32)
            total = ctx.frame_count(L, pad)
            f0, f1 = frame_range(total, rank, world)
            s0, s1 = sample_span(f0, f1, W, H, L)
            if f1 > f0:
                n, re, im, mag = ctx.execute_batched(pcm[s0:s1], pad_mode=pad, max_frames=f1 - f0)
                assert n == f1 - f0, (n, f0, f1)
                local = torch.from_numpy(np.stack([re, im, mag], -1).reshape(n, -1).copy())
            else:
                local = torch.zeros((0, 3 * ctx.bins), dtype=torch.float32)
            full = gather_frames(local, total, rank, world)
            results.append(full.numpy())
        slowest = max_over_ranks(1.5 + rank)
        q.put((rank, results, slowest))
    finally:
        dist.destroy_process_group()


# (N, W, H, signal length, pad mode, seed): even and uneven splits, a frame
# count below the world size, a partial lone frame, W < N
CASES = [(256, 256, 64, 5000, 1, 1), (256, 200, 50, 4096, 2, 2), (64, 64, 16, 64 + 16, 1, 3),
         (128, 128, 32, 90, 1, 4), (1024, 1024, 256, 65536, 1, 0)]


def test_frame_range_partitions():
    for total in (0, 1, 2, 3, 7, 253, 1000):
        for world in (1, 2, 3, 8):
            spans = [frame_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    assert sample_span(2, 5, 1024, 256, 65536) == (512, 4 * 256 + 1024)
    assert sample_span(0, 1, 1024, 256, 300) == (0, 300)
    with pytest.raises(ValueError):
        frame_range(10, 2, 2)


def test_two_gloo_ranks_match_single_process():
    from oracle.oracle import OracleContext

    ctxm = mp.get_context("spawn")
    q = ctxm.Queue()
    port = _free_port()
    procs = [ctxm.Process(target=_rank_main, args=(r, WORLD, port, CASES, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(WORLD):
        rank, results, slowest = q.get(timeout=240)
        got[rank] = (results, slowest)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in range(WORLD):
        assert got[rank][1] == 1.5 + (WORLD - 1)  # the slowest rank's value on every rank
    for i, (N, W, H, L, pad, seed) in enumerate(CASES):
        ctx = OracleContext(N=N, window=W, hop=H, transform=1, half_spectrum=1, pad_mode=pad)
        pcm = np.random.default_rng(seed).uniform(-1, 1, L).astype(np.float32)
        n, re, im, mag = ctx.execute_batched(pcm, pad_mode=pad)
        want = np.stack([re, im, mag], -1).reshape(n, -1)
        for rank in range(WORLD):
            full = got[rank][0][i]
            assert full.shape == want.shape
            assert np.array_equal(full.view(np.uint32), want.view(np.uint32)), (i, rank)
