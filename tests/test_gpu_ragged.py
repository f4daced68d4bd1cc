"""Ragged batches (one persistent launch over mixed sizes) against the
per-size contexts of fft_execute_batched and an FP64 DFT."""
import math
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

api = pytest.importorskip("fftfree_b200.api")


def tol(N):
    return 1e-5 * max(1.0, math.log2(N))


def workload(count, seed=2, lo=6, hi=17):
    """sizes 2^e, e uniform in [lo, hi), then the signals in order, from one generator."""
    rng = np.random.default_rng(seed)
    e = rng.integers(lo, hi, count)
    sizes = [1 << int(v) for v in e]
    pcm = np.concatenate([rng.uniform(-1, 1, n) for n in sizes]).astype(np.float32)
    return sizes, pcm


def run_plan(plan, pcm, device=True):
    if device:
        dp = torch.from_numpy(pcm).cuda()
        outs = [torch.empty(plan.bins, device="cuda") for _ in range(3)]
        assert plan.execute(dp, *outs) == 1
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in outs]
    outs = [np.zeros(plan.bins, np.float32) for _ in range(3)]
    assert plan.execute(pcm, *outs) == 1
    return outs


def ctx_radix(c):
    """The pass radix a context's single-pass plan runs (largest pass)."""
    import ctypes
    buf = (ctypes.c_int * 16)()
    n = api.lib().fftfree_ctx_schedule(c.handle, buf, 16)
    return max(buf[:n]) if n else 0


def per_item(sizes, pcm, radix=None, **flags):
    """fft_execute_batched per item on a context of its size (the reference's
    usage); `radix` collects each size's pass radix."""
    ctxs, res = {}, []
    off = 0
    for n in sizes:
        c = ctxs.get(n)
        if c is None:
            c = ctxs[n] = api.FftContext.full_v2(n, kernel=2, pad_mode=1, window=n, hop=n, transform=1,
                                                 half_spectrum=1, **flags)
            if radix is not None:
                radix[n] = ctx_radix(c)
        b = n // 2 + 1
        re, im, mg = (np.zeros(b, np.float32) for _ in range(3))
        assert c.execute_batched(pcm[off: off + n], re, im, mg) == 1
        res.append((re, im, mg))
        off += n
    return res


@pytest.mark.parametrize("flags", [{}, {"reduce_magnitude": 1}, {"store_polar": 1}])
def test_ragged_matches_per_size_contexts(monkeypatch, flags):
    """With the tuner off, a size that runs the single-pass engine with the
    same pass radix as its context is bit-identical to fft_execute_batched;
    every size agrees with an FP64 DFT and with the context within tolerance
    (32768 points, one block's single pass where the context takes two
    passes, and 65536, the two-half path)."""
    monkeypatch.setenv("FFTFREE_TUNE", "0")
    sizes, pcm = workload(300)
    plan = api.RaggedPlan(sizes, flags.get("reduce_magnitude", 0), flags.get("store_polar", 0))
    assert plan.samples == len(pcm) and plan.bins == sum(n // 2 + 1 for n in sizes)
    re, im, mg = run_plan(plan, pcm)
    radix = {}
    ref = per_item(sizes, pcm, radix=radix, **flags)
    off = po = 0
    same = 0
    for n, (rre, rim, rmg) in zip(sizes, ref):
        b = n // 2 + 1
        got = (re[off: off + b], im[off: off + b], mg[off: off + b])
        if n <= 16384 and plan.schedule(n) == radix[n]:
            same += 1
            for g, r in zip(got, (rre, rim, rmg)):
                np.testing.assert_array_equal(g, r)
        else:
            X = np.fft.rfft(pcm[po: po + n].astype(np.float64))
            X[0] = X[0].real
            X[-1] = X[-1].real
            if flags.get("store_polar"):
                assert np.linalg.norm(got[0] - np.abs(X)) <= tol(n) * np.linalg.norm(np.abs(X))
                np.testing.assert_array_equal(got[0], got[2])  # mag = re with store_polar
                big = np.abs(X) > 1e-3 * np.abs(X).max()
                dph = np.angle(np.exp(1j * (got[1][big] - np.angle(X[big]))))
                assert np.max(np.abs(dph)) < 1e-3
            elif flags.get("reduce_magnitude"):
                assert np.linalg.norm(got[0] - np.abs(X)) <= tol(n) * np.linalg.norm(np.abs(X))
                assert np.all(got[1] == 0)
            else:
                Z = got[0] + 1j * got[1]
                assert np.linalg.norm(Z - X) <= tol(n) * np.linalg.norm(X)
                np.testing.assert_allclose(got[2], np.abs(Z), rtol=1e-6, atol=1e-6)
            # and within tolerance of the per-size context
            assert np.linalg.norm(got[2] - rmg) <= tol(n) * np.linalg.norm(rmg)
        off += b
        po += n
    assert same > 100  # most sizes share the context's radix


def test_ragged_host_buffers_and_graph_reuse(monkeypatch, tmp_path):
    """Host and device buffers give the same bits; repeated executes reuse
    the captured graph, new buffers capture again; the tuner writes its cache."""
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("FFTFREE_TUNE_CACHE", str(cache))
    sizes, pcm = workload(200, seed=5)
    plan = api.RaggedPlan(sizes)
    first = run_plan(plan, pcm, device=True)
    again = run_plan(plan, pcm, device=True)
    host = run_plan(plan, pcm, device=False)
    for a, b, c in zip(first, again, host):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(a, c)
    assert plan.launch_count() >= 3
    text = cache.read_text()
    assert text.startswith("ragged r2c")
    for n in set(sizes):
        if n <= 8192 and n >= 64:
            assert plan.schedule(n) in (4, 8, 16)
    # a second plan over the same workload reads the cached choices
    plan2 = api.RaggedPlan(sizes)
    for n in set(sizes):
        assert plan2.schedule(n) == plan.schedule(n)
    np.testing.assert_array_equal(run_plan(plan2, pcm)[2], first[2])


def test_ragged_tuner_tile_sizes(monkeypatch, tmp_path):
    """The tuner's tile size (block-loads of frames per claimed tile): a
    workload with many frames of a few small sizes lets it try tiles of 1, 2
    and 4 block-loads; whatever it picks is a whole number of block-loads,
    it is cached beside the radix, and the outputs are the same bits as the
    tuner-off plan's wherever the radix is the same (the tile only changes
    which block takes which frames)."""
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("FFTFREE_TUNE_CACHE", str(cache))
    rng = np.random.default_rng(21)
    sizes = [int(v) for v in rng.choice([64, 256, 1024, 2048], 6000)]
    pcm = np.concatenate([rng.uniform(-1, 1, n).astype(np.float32) for n in sizes])
    plan = api.RaggedPlan(sizes)
    got = run_plan(plan, pcm)
    lines = [ln.split() for ln in cache.read_text().splitlines()]
    assert lines and all(len(ln) == 6 and ln[0] == "ragged" for ln in lines)
    monkeypatch.setenv("FFTFREE_TUNE", "0")
    base = api.RaggedPlan(sizes)
    ref = run_plan(base, pcm)
    for n in set(sizes):
        T = max(1, (n // 2) // plan.schedule(n))
        per = max(1, 1024 // T)
        assert plan.tile(n) in (per, 2 * per, 4 * per), (n, plan.tile(n), per)
        assert base.tile(n) == max(1, 1024 // max(1, (n // 2) // base.schedule(n)))
    off = 0
    for n in sizes:
        b = n // 2 + 1
        if plan.schedule(n) == base.schedule(n):
            for g, r in zip(got, ref):
                np.testing.assert_array_equal(g[off: off + b], r[off: off + b])
        off += b
    assert plan.tile(65536) == 1 and plan.tile(3) == 0


def test_ragged_small_sizes_and_rejects():
    sizes = [4, 8, 16, 32, 64, 4, 128, 65536, 8]
    rng = np.random.default_rng(9)
    pcm = rng.uniform(-1, 1, sum(sizes)).astype(np.float32)
    plan = api.RaggedPlan(sizes)
    re, im, mg = run_plan(plan, pcm)
    off = po = 0
    for n in sizes:
        b = n // 2 + 1
        X = np.fft.rfft(pcm[po: po + n].astype(np.float64))
        Z = re[off: off + b] + 1j * im[off: off + b]
        assert np.linalg.norm(Z - X) <= tol(n) * np.linalg.norm(X)
        off += b
        po += n
    for bad in ([3], [2], [131072], [64, 100]):
        with pytest.raises(RuntimeError):
            api.RaggedPlan(bad)


def test_ragged_config_workload():
    """The configuration's draw: 4096 signals, sizes 2^6 .. 2^16 from seed 2;
    every item within tolerance of an FP64 DFT."""
    sizes, pcm = workload(4096)
    plan = api.RaggedPlan(sizes)
    re, im, mg = run_plan(plan, pcm)
    off = po = 0
    worst = 0.0
    for n in sizes:
        b = n // 2 + 1
        X = np.fft.rfft(pcm[po: po + n].astype(np.float64))
        Z = re[off: off + b] + 1j * im[off: off + b]
        err = np.linalg.norm(Z - X) / np.linalg.norm(X)
        worst = max(worst, err / tol(n))
        off += b
        po += n
    print(f"ragged 4096: worst rel-L2 / tolerance = {worst:.3e}")
    assert worst <= 1.0


def test_ragged_mixed_framing_against_oracle():
    """Ragged mixes of size AND framing (fftfree_ragged_plan_stft): every
    item against the oracle's fft_execute_batched with pad_mode 1 on a
    context of its (N, W, H, analysis window) -- frames of W <= N samples
    every H, zero-padded, a lone partial frame for a short signal, Hann /
    Hamming / Tukey / rectangular taps -- within 1e-5 log2 N, sizes 4 ..
    65536 (the two-half path included)."""
    from oracle.oracle import OracleContext
    rng = np.random.default_rng(12)
    items = []  # (N, length, W, H, kind, p1)
    for N in (4, 16, 64, 256, 1024, 2048, 4096, 8192, 16384, 32768, 65536):
        for W, H, kind, p1 in ((N, N, 0, 0.0), (max(2, 3 * N // 4), max(1, N // 4), 1, 0.0),
                               (N, max(1, N // 2), 2, 0.0), (max(2, N // 2), max(1, N // 8), 4, 0.3)):
            length = int(rng.integers(1, 5)) * W + int(rng.integers(0, H)) if N <= 8192 else W + H + 5
            items.append((N, length, W, H, kind, p1))
    items.append((1024, 300, 1024, 256, 1, 0.0))   # shorter than one frame: a partial frame
    items.append((65536, 70000, 65536, 4096, 1, 0.0))
    order = rng.permutation(len(items))
    items = [items[i] for i in order]
    sig = [rng.uniform(-1, 1, it[1]).astype(np.float32) for it in items]
    pcm = np.concatenate(sig)
    plan = api.RaggedPlan([it[0] for it in items], lengths=[it[1] for it in items], window=[it[2] for it in items],
                          hop=[it[3] for it in items], window_kind=[it[4] for it in items],
                          window_param=[it[5] for it in items])
    re, im, mg = run_plan(plan, pcm)
    off = 0
    for i, ((N, L, W, H, kind, p1), x) in enumerate(zip(items, sig)):
        o = OracleContext(N=N, window=W, hop=H, transform=1, half_spectrum=1, apply_windows=1, analysis_kind=kind,
                          analysis_p1=p1, pad_mode=1)
        n, rre, rim, rmg = o.execute_batched(x, pad_mode=1)
        assert plan.frames(i) == n, (N, L, W, H)
        k = n * (N // 2 + 1)
        Z = re[off: off + k] + 1j * im[off: off + k]
        R = (rre + 1j * rim).ravel()
        assert np.linalg.norm(Z - R) <= tol(N) * np.linalg.norm(R), (N, L, W, H, kind)
        assert np.linalg.norm(mg[off: off + k] - rmg.ravel()) <= tol(N) * np.linalg.norm(rmg), (N, L, W, H, kind)
        off += k
    assert off == plan.bins
