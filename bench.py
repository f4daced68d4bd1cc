"""Benchmark of the batched FFT hot path on B200 (one JSON line on stdout).

Workload (N=1 line): batched C2C forward, N = 4096 points x 16,384 transforms,
complex64, inputs re/im i.i.d. N(0,1) from numpy default_rng(1), Stockham
order -- the batched-C2C configuration of the reference (fft_inplace_batched
over a 4096 x 16384 column-major matrix), the one configuration of the metric
that is both bandwidth-bound and one-GPU-sized (the plain STFT configuration
is a single 65,536-sample call, reported as a latency leg, with its shape on
a long signal as a throughput leg).  One step = one pass over the whole batch.

  value  -- device-resident throughput: algorithmic bytes (input read once +
            output written once, 1 GiB per pass) / device time, all ranks.
  e2e    -- the same transform through the public C ABI with pinned HOST
            buffers: H2D of the input, kernel, D2H of the output, per step.
  roofline -- the FFT kernel alone, timed with CUDA events on its stream,
            against the measured HBM copy bandwidth.
  cpu_baseline -- the reference's own C++ executor (built from its unchanged
            sources with its Release flags into oracle/_ref) on the host
            cores, over the whole batch, for about 15 s.

--impl reference times that same reference CPU path alone, K steps of the
whole batch.  Multi-GPU (torchrun): every rank runs its own batch (weak
scaling, no data-path collective); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import math
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "STFT GB/s (% HBM peak); autograd fwd+bwd vs plain fwd at rel-L2<=1e-5 vs FP64"
N_FFT = 4096
BATCH = 16384
BYTES_PER_PASS = 2 * N_FFT * BATCH * 8  # read + write, complex64


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic():
    """DRAM bytes per launch of the C2C kernel from the committed ncu summary."""
    try:
        with open(os.path.join(REPO, "profiles", "k_fft_c2c_n4096.md")) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    return int(line.split(":", 1)[1])
    except Exception:
        pass
    return None


class ClockSampler:
    """SM clocks, power and throttle reasons sampled during the timed region:
    through NVML (opened before the region, one sample as it starts, then
    every millisecond, one as it ends: the region may last only
    milliseconds), nvidia-smi every 200 ms where NVML is unavailable.
    Reads only."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.source = None
        self._stop = threading.Event()
        self._t = None
        self._nvml = None

    def _open_nvml(self):
        import pynvml
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        bits = [getattr(pynvml, "nvmlClocksEventReasonHwSlowdown", 0x8),
                getattr(pynvml, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
                getattr(pynvml, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
                getattr(pynvml, "nvmlClocksEventReasonSwPowerCap", 0x4)]
        reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        self._nvml = (pynvml, h, bits, reasons, mx)
        self.source = "nvml, 1 ms"

    def _sample_nvml(self):
        pynvml, h, bits, reasons, mx = self._nvml
        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
        pw = pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0
        r = reasons(h)
        self.samples.append([str(sm), str(mx), f"{pw:.1f}"] + ["Active" if r & b else "Not Active" for b in bits])

    def _run(self):
        if self._nvml:
            try:
                while not self._stop.wait(0.001):
                    self._sample_nvml()
                return
            except Exception:
                pass
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self.source = "nvidia-smi, 200 ms"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        try:
            self._open_nvml()
            self._sample_nvml()
        except Exception:
            self._nvml = None
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if self._nvml:
            try:
                self._sample_nvml()
                self._nvml[0].nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and
                          s[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples), "source": self.source}


def _seed1_batch(seed: int = 1):
    """The configuration's input: 16,384 transforms of 4096 points, re / im
    i.i.d. N(0,1) from numpy default_rng(seed) (PCG64), drawn in float64 and
    stored as complex64 rows (B, N, 2)."""
    import numpy as np
    return np.random.default_rng(seed).standard_normal((BATCH, N_FFT, 2)).astype(np.float32)


def _cpu_reference_run(steps: int, warmup: int, budget_s: float = None):
    """The reference's own batched C2C (eigfft::fft_inplace_batched, Stockham,
    eigen_fft.hpp:3152-3175) compiled with its Release flags (oracle/_ref),
    on a WorkerPool of all host cores (at most 16, its thread limit), over
    the WHOLE configuration batch per step.  Falls back to the oracle's C
    port of the same executor where the reference build is absent.
    Returns (seconds per step, threads, kind, sample text)."""
    import numpy as np
    threads = max(1, min(16, os.cpu_count() or 1))
    X = _seed1_batch().view(np.complex64).reshape(BATCH, N_FFT)
    Y = np.empty_like(X)
    from oracle import reflib
    if os.path.exists(reflib.release_path()):
        L = reflib.release_lib()
        plan = reflib.RefPlan(N_FFT, 0, 2, threads=threads, L=L)
        run = lambda: plan.execute(Y)  # noqa: E731
        kind = "reference"
        what = (f"the reference's own C++ ({os.path.basename(reflib.release_path())}: fft_cffi sources "
                f"unchanged, -O3 -ffast-math)")
    else:
        from oracle.oracle import OracleContext
        ctx = OracleContext(N=N_FFT, kernel=2)
        holder = {}
        run = lambda: holder.__setitem__("y", ctx.fft_columns(Y, threads=threads))  # noqa: E731
        kind = "port"
        what = "the oracle's C port of the reference executor"
    for _ in range(warmup):
        Y[:] = X
        run()
    times = []
    t_end = time.perf_counter() + (budget_s or 1e30)
    while len(times) < steps and (budget_s is None or time.perf_counter() < t_end or len(times) < 3):
        Y[:] = X
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    dt = sum(times) / len(times)
    sample = (f"all {BATCH} transforms (N={N_FFT} C2C forward, Stockham order, seed-1 draw) per step, "
              f"mean of {len(times)} steps after {warmup} warm-up, {what}, {threads} WorkerPool threads")
    return dt, threads, kind, sample


def _in_child(func: str, attempts: int = 3, timeout_s: float = 180.0, **kw):
    """Runs bench.<func>(**kw) in a fresh Python process (no CUDA context) and
    returns its JSON-able result, or None when every attempt died or ran past
    timeout_s.  The reference's WorkerPool has crashed intermittently on the
    GPU box's 16 host threads (a segfault or abort in its own code, during or
    after a call); in a child process such a crash costs one attempt, not the
    bench.  The end of a failed attempt's stderr goes to this stderr."""
    code = ("import json, sys; sys.path.insert(0, %r); import bench; "
            "print('@@RESULT ' + json.dumps(bench.%s(**json.loads(sys.argv[1]))), flush=True)" % (REPO, func))
    for attempt in range(attempts):
        try:
            r = subprocess.run([sys.executable, "-c", code, json.dumps(kw)], capture_output=True, text=True,
                               timeout=timeout_s)
        except subprocess.TimeoutExpired:
            sys.stderr.write(f"[bench] {func}: attempt {attempt + 1} ran past {timeout_s:.0f} s\n")
            continue
        for line in r.stdout.splitlines():
            if line.startswith("@@RESULT "):
                return json.loads(line[len("@@RESULT "):])
        sys.stderr.write(f"[bench] {func}: attempt {attempt + 1} exited {r.returncode}: "
                         f"{r.stderr.strip()[-300:]}\n")
    return None


def _cpu_reference_child(steps: int, warmup: int, budget_s: float = None):
    dt, threads, kind, sample = _cpu_reference_run(steps=steps, warmup=warmup, budget_s=budget_s)
    return {"dt": dt, "threads": threads, "kind": kind, "sample": sample}


def cpu_baseline(budget_s: float = 15.0):
    """The reference's CPU path on the host cores (bounded: about budget_s),
    in a child process."""
    r = _in_child("_cpu_reference_child", timeout_s=budget_s + 120.0, steps=1000, warmup=1, budget_s=budget_s)
    if r is None:
        return {"unavailable": "the reference's CPU run crashed in every attempt (its WorkerPool)"}
    return {"value": round(BYTES_PER_PASS / r["dt"] / 1e9, 3), "unit": "GB/s", "cores": r["threads"],
            "kind": r["kind"], "sample": r["sample"]}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    # a step is about 0.1 s of the reference on 16 threads: generous room
    r = _in_child("_cpu_reference_child", timeout_s=120.0 + 5.0 * (args.steps + args.warmup), steps=args.steps,
                  warmup=args.warmup)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's CPU run crashed in every attempt "
                                                              "(a segfault in its own WorkerPool)"}), flush=True)
        return 0
    dt, threads, kind, sample = r["dt"], r["threads"], r["kind"], r["sample"]
    value = BYTES_PER_PASS / dt / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
            "data": "synthetic",
            "config": {"workload": f"batched C2C forward N={N_FFT} x {BATCH} transforms complex64 (Stockham order), "
                                   f"N(0,1) re/im from numpy default_rng(1); host CPU",
                       "parallelism": f"{threads} host threads"},
            "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# Single-kernel workloads for profiling (ncu -k <kernel> -s <warm-up> -c 1):
# device-resident inputs larger than L2, one library call per launch.
CASES = {
    "c2c_n4096_b8192": "C2C N=4096 x 8192 complex64, Stockham, fftfree_execute_c2c",
    "stft_n1024_h256": "STFT N=W=1024 H=256 on 128 x 65536 samples, radix option 4, reduce_magnitude, half",
    "mag_n2048": "magnitude STFT N=W=2048 H=512, 64 x 262144 samples (autograd plain forward)",
    "mag_phasor_n2048": "magnitude + unit phasor STFT N=W=2048 H=512, 64 x 262144 samples (autograd forward)",
    "grad_phasor_n2048": "magnitude STFT gradient from the saved phasor, N=W=2048 H=512, 64 x 262144",
    "mag_l2_n2048": "fused spectral L2 loss forward (residual, phasor, partial sums), N=W=2048 H=512, 64 x 262144",
    "grad_recompute_n2048": "magnitude STFT gradient with the spectrum recomputed, N=W=2048 H=512, 64 x 262144",
    "c2c_n65536_b512": "C2C N=65536 x 512 complex64, four-step (two passes)",
    "ragged_4096": "ragged batch: 4096 R2C signals, N = 2^e, e uniform in 6..16 (seed 2), one persistent launch",
    "fft2d_4096x4096_b4": "2-D C2C of 4 column-major 4096 x 4096 complex64 matrices (column pass + strided row pass)",
    "r2c_n4096_polar_b8192": "R2C N=W=H=4096, half spectrum, store_polar, 8192 frames (fft_execute_batched)",
    "c2r_n4096_polar_b8192": "C2R N=4096 half spectrum polar input (Cooley-Tukey pre-hook), 8192 frames "
                             "(fft_execute_complex_batched)",
    "c2c_n256_b262144": "C2C N=256 x 262144 complex64, one pass (FFTFREE_TC16=2: the tcgen05 split-FP16 kernel)",
    "griffin_lim_n1024_h256": "fft_griffin_lim, N=W=1024 H=256 Hann, 4096 frames x 513 bins, 32 iterations "
                              "(device magnitudes and outputs)",
}


def run_case(args):
    import torch
    import fftfree_b200 as ff
    from fftfree_b200 import autograd as ag

    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    g = torch.Generator(device="cuda").manual_seed(1)
    name = args.case
    if name == "c2c_n4096_b8192":
        x = torch.randn(8192, 4096, 2, device="cuda", generator=g)
        y = torch.empty_like(x)
        c = ff.FftContext.full_v2(4096, kernel=2)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        fn, nbytes = (lambda: c.execute_c2c(x, y, 8192)), 2 * x.numel() * 4
    elif name == "c2c_n256_b262144":
        x = torch.randn(262144, 256, 2, device="cuda", generator=g)
        y = torch.empty_like(x)
        c = ff.FftContext.full_v2(256, kernel=2)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        fn, nbytes = (lambda: c.execute_c2c(x, y, 262144)), 2 * x.numel() * 4
    elif name == "c2c_n65536_b512":
        x = torch.randn(512, 65536, 2, device="cuda", generator=g)
        y = torch.empty_like(x)
        c = ff.FftContext.full_v2(65536, kernel=2)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        fn, nbytes = (lambda: c.execute_c2c(x, y, 512)), 2 * x.numel() * 4
    elif name == "fft2d_4096x4096_b4":
        x = torch.randn(4 * 4096 * 4096 * 2, device="cuda", generator=g)
        y = torch.empty_like(x)
        c = ff.FftContext.full_v2(4096, kernel=2)
        c1 = ff.FftContext.full_v2(4096, kernel=2)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        fn, nbytes = (lambda: ff.execute_2d(c, c1, x, y, 4096, 4096, 4)), 2 * x.numel() * 4
    elif name == "ragged_4096":
        import numpy as np
        rng = np.random.default_rng(2)
        sizes = [1 << int(v) for v in rng.integers(6, 17, 4096)]
        pcm = torch.from_numpy(np.concatenate([rng.uniform(-1, 1, n) for n in sizes]).astype(np.float32)).cuda()
        plan = ff.RaggedPlan(sizes)
        plan.set_stream(stream.cuda_stream)
        re, im, mg = (torch.empty(plan.bins, device="cuda") for _ in range(3))
        fn, nbytes = (lambda: plan.execute(pcm, re, im, mg)), plan.samples * 4 + 3 * plan.bins * 4
    elif name in ("r2c_n4096_polar_b8192", "c2r_n4096_polar_b8192"):
        B, N = 8192, 4096
        bins = N // 2 + 1
        pcm = torch.rand(B * N, device="cuda", generator=g) * 2 - 1
        re, im, mg = (torch.empty(B * bins, device="cuda") for _ in range(3))
        c = ff.FftContext.full_v2(N, kernel=2, window=N, hop=N, transform=1, half_spectrum=1, store_polar=1)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        c.execute_batched(pcm, re, im, mg, pcm_len=B * N)
        if name.startswith("r2c"):
            fn, nbytes = (lambda: c.execute_batched(pcm, re, im, mg, pcm_len=B * N)), B * N * 4 + 3 * B * bins * 4
        else:
            ci = ff.FftContext.full_v2(N, kernel=0, inverse=1, transform=2, half_spectrum=1, store_polar=1)
            ci.set_stream(stream.cuda_stream)
            ci.set_async(True)
            out = torch.empty(B * N, device="cuda")
            fn, nbytes = (lambda: ci.execute_complex_batched(re, im, B, out)), 2 * B * bins * 4 + B * N * 4
    elif name == "griffin_lim_n1024_h256":
        N, H, F, iters = 1024, 256, 4096, 32
        bins = N // 2 + 1
        mag = torch.rand(F * bins, device="cuda", generator=g)
        re, im = torch.empty_like(mag), torch.empty_like(mag)
        fc = ff.FftContext.full_v2(N, kernel=2, window=N, hop=H, transform=1, half_spectrum=1, apply_windows=1,
                                   analysis_kind=1)
        ic = ff.FftContext.full_v2(N, kernel=2, inverse=1, transform=2, half_spectrum=1, window=N, hop=H)
        for c in (fc, ic):
            c.set_stream(stream.cuda_stream)
        L = ff.api.lib()

        def fn():
            if L.fft_griffin_lim(fc.handle, ic.handle, ff.api._fp(mag), F, H, 1, iters, 1, 7, ff.api._fp(re),
                                 ff.api._fp(im)) != 1:
                raise RuntimeError("fft_griffin_lim failed")
        ola = (F - 1) * H + N
        # per iteration: inverse (spectra in, frames out), overlap-add (frames
        # in, signal out), projected STFT (signal and magnitudes in, spectra out)
        nbytes = iters * (2 * F * bins * 4 + F * N * 4 + F * N * 4 + ola * 4 + ola * 4 + F * bins * 4
                          + 2 * F * bins * 4)
    elif name == "stft_n1024_h256":
        L = 128 * 65536
        pcm = torch.rand(L, device="cuda", generator=g) * 2 - 1
        frames, bins = 1 + (L - 1024) // 256, 513
        re = torch.empty(frames * bins, device="cuda")
        im, mg = torch.empty_like(re), torch.empty_like(re)
        c = ff.FftContext.full_v2(1024, kernel=2, radix=4, window=1024, hop=256, transform=1, reduce_magnitude=1,
                                  half_spectrum=1)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        fn, nbytes = (lambda: c.execute_batched(pcm, re, im, mg, pcm_len=L)), L * 4 + 3 * frames * bins * 4
    else:
        S, L = 64, 262144
        x = torch.rand(S, L, device="cuda", generator=g) * 2 - 1
        plan = ag.StftPlan(2048, 512, 2048, "hann")
        F, bins = plan.frames(L), plan.bins
        up = torch.randn(S, F, bins, device="cuda", generator=g)
        ph = plan.magnitude_phasor(x)[1]
        spec = S * F * bins * 4
        tgt = torch.rand(S, F, bins, device="cuda", generator=g)
        fn, nbytes = {
            "mag_l2_n2048": (lambda: plan.magnitude_l2(x, tgt), S * L * 4 + 4 * spec),
            "mag_n2048": (lambda: plan.magnitude(x), S * L * 4 + spec),
            "mag_phasor_n2048": (lambda: plan.magnitude_phasor(x), S * L * 4 + 3 * spec),
            "grad_phasor_n2048": (lambda: plan.magnitude_backward_phasor(ph, up, L), 3 * spec + S * L * 4),
            "grad_recompute_n2048": (lambda: plan.magnitude_backward(x, up), 2 * S * L * 4 + spec),
        }[name]
    for _ in range(args.warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(args.steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / args.steps
    print(json.dumps({"case": name, "what": CASES[name], "ms": round(ms, 4),
                      "GB/s": round(nbytes / (ms * 1e-3) / 1e9, 1)}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-legs", action="store_true")
    ap.add_argument("--case", choices=sorted(CASES),
                    help="run one kernel workload (W warm-up + K timed launches) and print its timing; "
                         "the profiling entry point")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import fftfree_b200 as ff

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    peak, peak_kind = _peaks()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    x_host = _seed1_batch(1 + rank)
    x = torch.from_numpy(x_host).cuda()
    y = torch.empty_like(x)
    ctx = ff.FftContext.full_v2(N_FFT, kernel=2)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_async(True)

    def step():
        if ctx.execute_c2c(x, y, BATCH) != 1:
            raise RuntimeError("fftfree_execute_c2c failed")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = ctx.launch_count()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        t_start = torch.cuda.Event(enable_timing=True)
        t_stop = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for i in range(args.steps):
            evs[i][0].record(stream)
            step()
            evs[i][1].record(stream)
        t_stop.record(stream)
        torch.cuda.synchronize()
    launches = ctx.launch_count() - launches0
    total_ms = t_start.elapsed_time(t_stop)
    kern_ms = [a.elapsed_time(b) for a, b in evs]
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = BYTES_PER_PASS * world * args.steps / (total_ms * 1e-3) / 1e9
    kern_avg = sum(kern_ms) / len(kern_ms)
    achieved = BYTES_PER_PASS / (kern_avg * 1e-3) / 1e9

    # secondary legs on the same device (information; not the headline).  One
    # GPU only: under torchrun the other ranks would wait for rank 0's legs
    # in the next collective.
    legs = {}
    if rank == 0 and world == 1 and not args.no_legs:
        legs = measure_legs(ff, torch, stream)

    # e2e through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        hx = torch.empty(BATCH, N_FFT, 2, pin_memory=True)
        hx.copy_(torch.from_numpy(x_host))
        hy = torch.empty_like(hx).pin_memory()
        ctx_h = ff.FftContext.full_v2(N_FFT, kernel=2)
        for _ in range(2):
            ctx_h.execute_c2c(hx, hy, BATCH)
        n_e2e = max(3, min(args.steps, 10))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n_e2e):
            if ctx_h.execute_c2c(hx, hy, BATCH) != 1:
                raise RuntimeError("e2e call failed")
        dt = (time.perf_counter() - t0) / n_e2e
        e2e_val = BYTES_PER_PASS / dt / 1e9
        if dist:
            t = torch.tensor([dt], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_val = BYTES_PER_PASS * world / float(t.item()) / 1e9
        e2e = {"value": round(e2e_val, 3), "unit": "GB/s", "h2d_bytes_per_step": BATCH * N_FFT * 8,
               "d2h_bytes_per_step": BATCH * N_FFT * 8, "ms_per_step": round(dt * 1e3, 3)}
        ctx_h.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": f"batched C2C forward, N={N_FFT} x {BATCH} transforms complex64 per GPU "
                                   f"(Stockham order), N(0,1) re/im from numpy default_rng(1 + rank), "
                                   f"device-resident",
                       "l2": "inputs larger than L2 (512 MiB in, 512 MiB out per pass)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": _profile_traffic(),
                         "peak_kind": f"{peak_kind} (hbm_gbs)", "kernel": "k_fft<Sched<12,4>,C2cIO>",
                         "kernel_ms": round(kern_avg, 4)},
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "legs": legs,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def measure_legs(ff, torch, stream, reps: int = 10):
    """Other legs of the configuration, device-resident, CUDA-event timed."""
    import numpy as np

    def timed(fn, nbytes):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / reps
        return {"ms": round(ms, 4), "GB/s": round(nbytes / (ms * 1e-3) / 1e9, 1)}

    legs = {}
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(BATCH, N_FFT, 2, device="cuda", generator=g)
    y = torch.empty_like(x)
    for name, kw in [("c2c_inverse_stockham", dict(kernel=2, inverse=1)),
                     ("c2c_forward_cooleytukey", dict(kernel=1)),
                     ("c2c_inverse_cooleytukey", dict(kernel=1, inverse=1))]:
        c = ff.FftContext.full_v2(N_FFT, **kw)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        legs[name] = timed(lambda: c.execute_c2c(x, y, BATCH), BYTES_PER_PASS)
        c.close()
    # R2C via fft_execute_batched, W = H = N = 4096, half spectrum, polar
    pcm = torch.rand(BATCH * N_FFT, device="cuda", generator=g) * 2 - 1
    bins = N_FFT // 2 + 1
    re = torch.empty(BATCH * bins, device="cuda"); im = torch.empty_like(re); mag = torch.empty_like(re)
    c = ff.FftContext.full_v2(N_FFT, kernel=2, window=N_FFT, hop=N_FFT, transform=1, half_spectrum=1, store_polar=1)
    c.set_stream(stream.cuda_stream)
    c.set_async(True)
    legs["r2c_stft_n4096_half_polar"] = timed(
        lambda: c.execute_batched(pcm, re, im, mag, pcm_len=BATCH * N_FFT),
        BATCH * N_FFT * 4 + 3 * BATCH * bins * 4)
    c.close()
    # C2R round trip leg: half spectrum, polar input, inverse
    out = torch.empty(BATCH * N_FFT, device="cuda")
    c = ff.FftContext.full_v2(N_FFT, kernel=0, inverse=1, transform=2, half_spectrum=1, store_polar=1)
    c.set_stream(stream.cuda_stream)
    c.set_async(True)
    legs["c2r_n4096_half_polar"] = timed(lambda: c.execute_complex_batched(re, im, BATCH, out),
                                         2 * BATCH * bins * 4 + BATCH * N_FFT * 4)
    c.close()
    # config 1 exactly: one call on one signal of 65,536 samples (U[-1,1),
    # seed 0) -> 253 frames x 513 bins; a synchronous call, so its latency is
    # host wall-clock per call (device buffers, and host buffers with the
    # copies inside)
    import time
    x1 = np.random.default_rng(0).uniform(-1, 1, 65536).astype(np.float32)
    c1 = ff.FftContext.full(1024, 1, 1, 0, 2, 4, None, 1, 1024, 256, 1, 1, 0, 1, 1, 0, 0, 0, 1)
    nb1 = 253 * 513
    hre1, him1, hmg1 = (np.zeros(nb1, np.float32) for _ in range(3))
    dx1 = torch.from_numpy(x1).cuda()
    dre1, dim1, dmg1 = (torch.empty(nb1, device="cuda") for _ in range(3))

    def latency_us(fn, n=300):
        for _ in range(20):
            fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / n * 1e6

    us_dev = latency_us(lambda: c1.execute_batched(dx1, dre1, dim1, dmg1, pcm_len=65536, pad_mode=1))
    us_host = latency_us(lambda: c1.execute_batched(x1, hre1, him1, hmg1, pad_mode=1))
    legs["stft_config1_single_call"] = {
        "frames": 253, "us_device_buffers": round(us_dev, 2), "us_host_buffers": round(us_host, 2),
        "frames_per_s_host_buffers": round(253 / (us_host * 1e-6), 1)}
    c1.close()
    # config-1 shape on a long signal: N=W=1024, H=256, half, magnitude
    L = 512 * 65536
    pcm1 = torch.rand(L, device="cuda", generator=g) * 2 - 1
    frames = 1 + (L - 1024) // 256
    b1 = 513
    re1 = torch.empty(frames * b1, device="cuda"); im1 = torch.empty_like(re1); mag1 = torch.empty_like(re1)
    c = ff.FftContext.full_v2(1024, kernel=2, radix=4, window=1024, hop=256, transform=1, reduce_magnitude=1,
                              half_spectrum=1)
    c.set_stream(stream.cuda_stream)
    c.set_async(True)
    legs["stft_r2c_n1024_h256_long_signal"] = timed(
        lambda: c.execute_batched(pcm1, re1, im1, mag1, pcm_len=L), L * 4 + 3 * frames * b1 * 4)
    legs["stft_r2c_n1024_h256_long_signal"]["frames_per_s"] = round(
        frames / (legs["stft_r2c_n1024_h256_long_signal"]["ms"] * 1e-3), 1)
    c.close()
    # 2-D: 4 column-major 4096 x 4096 complex64 matrices, forward on both
    # axes (columns by the batched kernel, rows by the strided one)
    R2, B2 = 4096, 4
    x2 = torch.randn(B2 * R2 * R2 * 2, device="cuda", generator=g)
    y2 = torch.empty_like(x2)
    c0 = ff.FftContext.full_v2(R2, kernel=2)
    c1 = ff.FftContext.full_v2(R2, kernel=2)
    c0.set_stream(stream.cuda_stream)
    c0.set_async(True)
    leg = timed(lambda: ff.execute_2d(c0, c1, x2, y2, R2, R2, B2), 2 * x2.numel() * 4)
    # two passes are the least any out-of-cache 2-D transform moves
    leg["two_pass_GB/s"] = round(4 * x2.numel() * 4 / (leg["ms"] * 1e-3) / 1e9, 1)
    legs["fft2d_c2c_4096x4096_b4"] = leg
    c0.close()
    c1.close()
    del x2, y2
    legs["griffin_lim_n1024_h256_f4096"] = measure_griffin_lim(ff, torch)
    legs["autograd_stft_magnitude"] = measure_autograd(torch, stream, timed)
    legs["ragged_r2c_4096"] = measure_ragged(ff, torch, stream, timed)
    legs["precision_c2c_n65536_b2048"] = measure_precision(ff, torch, stream, timed)
    return legs


def measure_griffin_lim(ff, torch, reps: int = 5):
    """fft_griffin_lim (fft_cffi.cpp:2176-2248) on 4096 frames x 513 bins
    (N=W=1024, H=256, Hann analysis), device magnitudes and outputs: host
    wall clock per synchronous call at 32 iterations, and the per-iteration
    cost from the 32- and 96-iteration calls.  Beside it the reference's own
    Griffin-Lim (oracle/_ref release build, host buffers, all host cores up
    to 16) on the same shape at 2 and 4 iterations, in a child process."""
    N, H, F = 1024, 256, 4096
    bins = N // 2 + 1
    g = torch.Generator(device="cuda").manual_seed(5)
    mag = torch.rand(F * bins, device="cuda", generator=g)
    re, im = torch.empty_like(mag), torch.empty_like(mag)
    fc = ff.FftContext.full_v2(N, kernel=2, window=N, hop=H, transform=1, half_spectrum=1, apply_windows=1,
                               analysis_kind=1)
    ic = ff.FftContext.full_v2(N, kernel=2, inverse=1, transform=2, half_spectrum=1, window=N, hop=H)
    L = ff.api.lib()

    def call_ms(iters):
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if L.fft_griffin_lim(fc.handle, ic.handle, ff.api._fp(mag), F, H, 1, iters, 1, 7, ff.api._fp(re),
                                 ff.api._fp(im)) != 1:
                raise RuntimeError("fft_griffin_lim failed")
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3)
        return statistics.median(ts)

    call_ms(2)
    ms32, ms96 = call_ms(32), call_ms(96)
    leg = {"frames": F, "bins": bins, "iterations": 32, "ms_per_call": round(ms32, 3),
           "us_per_iteration": round((ms96 - ms32) / 64 * 1e3, 2),
           "setup_ms": round(ms32 - 32 * (ms96 - ms32) / 64, 3)}
    fc.close()
    ic.close()
    ref = _in_child("_ref_griffin_lim", timeout_s=120.0, N=N, H=H, F=F)
    leg["cpu_baseline"] = ref if ref is not None else {
        "unavailable": "the reference's fft_griffin_lim crashed in every attempt (its WorkerPool)"}
    return leg


def _ref_griffin_lim(N: int, H: int, F: int):
    """The reference's own fft_griffin_lim (oracle/_ref release build, host
    buffers, all host cores up to 16) at 2 and 4 iterations on F frames of
    N/2 + 1 magnitudes U[0, 1) (numpy seed 5); run in a child process."""
    import numpy as np
    from oracle import reflib
    if not os.path.exists(reflib.release_path()):
        return {"unavailable": "the reference's release build is absent"}
    RL = reflib.release_lib()
    th = max(1, min(16, os.cpu_count() or 1))
    base = dict(n=N, threads=th, lanes=1, inverse=0, kernel=2, radix=0, radix_pattern=None, pad_mode=1,
                window=N, hop=H, transform=1, reduce_magnitude=0, store_polar=0, half_spectrum=1,
                allow_outer_parallel=1, allow_inner_parallel=0, inner_threads=0, save_crash_logs=0,
                silent_crash_reports=1, apply_windows=0, apply_ola=0, analysis_kind=0, analysis_p1=0.0,
                analysis_p2=0.0, synthesis_kind=0, synthesis_p1=0.0, synthesis_p2=0.0, norm_policy=0,
                cola_mode=0)
    rf = reflib.RefContext.full_v2(RL, **dict(base, apply_windows=1, analysis_kind=1))
    ri = reflib.RefContext.full_v2(RL, **dict(base, inverse=1, transform=2))
    hm = np.random.default_rng(5).random(F * (N // 2 + 1)).astype(np.float32)
    hr, hi = np.zeros_like(hm), np.zeros_like(hm)

    def ref_ms(iters):
        t0 = time.perf_counter()
        if RL.fft_griffin_lim(rf.h, ri.h, reflib.fp(hm), F, H, 1, iters, 1, 7, reflib.fp(hr), reflib.fp(hi)) != 1:
            raise RuntimeError("reference fft_griffin_lim failed")
        return (time.perf_counter() - t0) * 1e3

    r2, r4 = ref_ms(2), ref_ms(4)
    per = (r4 - r2) / 2
    rf.close()
    ri.close()
    return {"kind": "reference", "threads": th, "ms_per_iteration": round(per, 2), "setup_ms": round(r2 - 2 * per, 2),
            "ms_per_call_32_iterations_projected": round(r2 + 30 * per, 1),
            "sample": "2- and 4-iteration calls, same shape, magnitudes U[0, 1) (numpy seed 5)"}


def measure_precision(ff, torch, stream, timed):
    """C2C N=65536 (256 x 256 four-step) x 2048, re/im N(0,1) from seed 3:
    the FP32 CUDA-core path against the split-FP16 tensor-core radix-16
    variant (FFTFREE_TC16=1, mma.sync), each with its rel-L2 against an FP64
    DFT of 8 transforms; and C2C N=256 x 262,144 against the tcgen05 form
    (FFTFREE_TC16=2: tensor-memory accumulators), rel-L2 over 64 transforms."""
    import numpy as np

    N, B = 65536, 2048
    rng = np.random.default_rng(3)
    z = rng.standard_normal((B, N, 2)).astype(np.float32)
    x = torch.from_numpy(z).cuda()
    y = torch.empty_like(x)
    ref = np.fft.fft(z[:8, :, 0].astype(np.float64) + 1j * z[:8, :, 1].astype(np.float64), axis=1)
    out = {}
    for name, tc in (("fp32_cuda_core", "0"), ("split_fp16_tensor_core", "1")):
        os.environ["FFTFREE_TC16"] = tc
        c = ff.FftContext.full_v2(N, kernel=2)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        r = timed(lambda: c.execute_c2c(x, y, B), 16 * N * B)
        torch.cuda.synchronize()
        got = y[:8].cpu().numpy()
        got = got[..., 0].astype(np.float64) + 1j * got[..., 1].astype(np.float64)
        r["rel_l2_vs_fp64"] = float(f"{np.linalg.norm(got - ref) / np.linalg.norm(ref):.3e}")
        out[name] = r
        c.close()
    os.environ.pop("FFTFREE_TC16", None)
    out["kept"] = "split_fp16_tensor_core" if out["split_fp16_tensor_core"]["ms"] < out["fp32_cuda_core"]["ms"] \
        else "fp32_cuda_core"
    del x, y
    # 256-point transforms (one pass) x 262,144: the FP32 engine against the
    # tcgen05 split-FP16 kernel (FFTFREE_TC16=2, k_tc05.cu)
    N2, B2 = 256, 262144
    z2 = rng.standard_normal((B2, N2, 2)).astype(np.float32)
    x2 = torch.from_numpy(z2).cuda()
    y2 = torch.empty_like(x2)
    ref2 = np.fft.fft(z2[:64, :, 0].astype(np.float64) + 1j * z2[:64, :, 1].astype(np.float64), axis=1)
    n256 = {}
    for name, tc in (("fp32_cuda_core", "0"), ("split_fp16_tcgen05", "2")):
        os.environ["FFTFREE_TC16"] = tc
        c = ff.FftContext.full_v2(N2, kernel=2)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        r = timed(lambda: c.execute_c2c(x2, y2, B2), 16 * N2 * B2)
        torch.cuda.synchronize()
        got = y2[:64].cpu().numpy()
        got = got[..., 0].astype(np.float64) + 1j * got[..., 1].astype(np.float64)
        r["rel_l2_vs_fp64"] = float(f"{np.linalg.norm(got - ref2) / np.linalg.norm(ref2):.3e}")
        n256[name] = r
        c.close()
    os.environ.pop("FFTFREE_TC16", None)
    n256["kept"] = "split_fp16_tcgen05" if n256["split_fp16_tcgen05"]["ms"] < n256["fp32_cuda_core"]["ms"] \
        else "fp32_cuda_core"
    out["c2c_n256_b262144"] = n256
    return out


def measure_ragged(ff, torch, stream, timed):
    """Ragged batch: 4096 real signals, N = 2^e with e uniform in 6..16 drawn
    from seed 2, then each signal uniform[-1, 1) from the same generator; R2C
    half spectrum, planar re / im / mag outputs.  One persistent launch (a
    CUDA graph) against one fft_execute_batched call per signal on a context
    per size, the reference's usage (device buffers, enqueued back to back)."""
    import numpy as np

    rng = np.random.default_rng(2)
    e = rng.integers(6, 17, 4096)
    sizes = [1 << int(v) for v in e]
    pcm_h = np.concatenate([rng.uniform(-1, 1, n) for n in sizes]).astype(np.float32)
    plan = ff.RaggedPlan(sizes)
    plan.set_stream(stream.cuda_stream)
    pcm = torch.from_numpy(pcm_h).cuda()
    re, im, mag = (torch.empty(plan.bins, device="cuda") for _ in range(3))
    nbytes = plan.samples * 4 + 3 * plan.bins * 4
    one = timed(lambda: plan.execute(pcm, re, im, mag), nbytes)
    ctxs = {}
    for n in set(sizes):
        c = ff.FftContext.full_v2(n, kernel=2, pad_mode=1, window=n, hop=n, transform=1, half_spectrum=1)
        c.set_stream(stream.cuda_stream)
        c.set_async(True)
        ctxs[n] = c
    offs, po, ob = [], 0, 0
    for n in sizes:
        offs.append((n, po, ob))
        po += n
        ob += n // 2 + 1
    base_pcm, base_re, base_im, base_mg = pcm.data_ptr(), re.data_ptr(), im.data_ptr(), mag.data_ptr()

    def per_signal():
        for n, p0, o0 in offs:
            ctxs[n].execute_batched(base_pcm + 4 * p0, base_re + 4 * o0, base_im + 4 * o0, base_mg + 4 * o0,
                                    pcm_len=n)

    sep = timed(per_signal, nbytes)
    for c in ctxs.values():
        c.close()
    plan.close()
    return {"signals": len(sizes), "samples": int(pcm_h.size), "bytes": nbytes, "one_launch": one,
            "per_signal_launches": sep, "speedup": round(sep["ms"] / one["ms"], 2),
            "transforms_per_s": round(len(sizes) / (one["ms"] * 1e-3), 1)}


def measure_autograd(torch, stream, timed):
    """Differentiation workload: 64 signals x 262,144 samples (8 sinusoids,
    frequency U(0, fs/2), amplitude U[0.1, 1], phase U[0, 2 pi), plus N(0, 0.01)
    noise, seed 4), Hann W = N = 2048, H = 512 (509 frames x 1025 bins).
    Plain forward = the magnitude STFT kernel alone; fwd+bwd = the
    torch.autograd.Function forward and backward for a given upstream
    gradient; with_loss adds sum((|X| - T)^2) and its torch elementwise ops;
    loss_fused is the same loss through stft_magnitude_l2_loss (one fused
    forward kernel, one scaled adjoint kernel)."""
    from fftfree_b200 import autograd as ag

    S, L, N, H = 64, 262144, 2048, 512
    g = torch.Generator(device="cuda").manual_seed(4)
    t = torch.arange(L, device="cuda", dtype=torch.float32)
    x = torch.zeros(S, L, device="cuda")
    for _ in range(8):
        f = torch.rand(S, 1, device="cuda", generator=g) * 0.5
        a = torch.rand(S, 1, device="cuda", generator=g) * 0.9 + 0.1
        ph = torch.rand(S, 1, device="cuda", generator=g) * (2 * math.pi)
        x += a * torch.sin(2 * math.pi * f * t + ph)
    x += 0.1 * torch.randn(S, L, device="cuda", generator=g)
    plan = ag.StftPlan(N, H, N, "hann")
    F = plan.frames(L)
    bins = plan.bins
    target = plan.magnitude(x.roll(1, 0)).detach()
    upstream = torch.randn(S, F, bins, device="cuda", generator=g)
    in_b, mag_b = S * L * 4, S * F * bins * 4
    fwd = timed(lambda: plan.magnitude(x), in_b + mag_b)
    bwd = timed(lambda: plan.magnitude_backward(x, upstream), 2 * in_b + mag_b)
    xr = x.detach().clone().requires_grad_(True)

    def fwd_bwd():
        xr.grad = None
        ag.stft_magnitude(xr, plan).backward(upstream)

    def with_loss():
        xr.grad = None
        (ag.stft_magnitude(xr, plan) - target).square().sum().backward()

    def with_loss_fused():
        xr.grad = None
        ag.stft_magnitude_l2_loss(xr, target, plan).backward()

    # saved phasor (the default at this size): fwd writes |X| and X / |X|, bwd reads g and X / |X|
    assert plan.stores_phase(xr)
    fb = timed(fwd_bwd, in_b + 3 * mag_b + 3 * mag_b + in_b)
    fl = timed(with_loss, in_b + 3 * mag_b + 3 * mag_b + in_b)
    # fused loss: fwd reads x and T, writes the residual and the phasor; bwd
    # reads them and writes dL/dx
    flf = timed(with_loss_fused, in_b + 4 * mag_b + 3 * mag_b + in_b)
    _, ph = plan.magnitude_phasor(x)
    bwd_ph = timed(lambda: plan.magnitude_backward_phasor(ph, upstream, L), 3 * mag_b + in_b)
    plan.close()
    # recomputed spectrum (the path for signals whose phase exceeds the budget)
    plan = ag.StftPlan(N, H, N, "hann", phase_budget=0)
    assert not plan.stores_phase(xr)
    fb_rc = timed(fwd_bwd, 3 * in_b + 2 * mag_b)
    plan.close()
    return {"signals": S, "samples": L, "n_fft": N, "hop": H, "frames": F, "bins": bins,
            "fwd": fwd, "bwd_recompute": bwd, "bwd_saved_phasor": bwd_ph, "fwd_bwd": fb,
            "fwd_bwd_with_loss": fl, "fwd_bwd_loss_fused": flf, "fwd_bwd_recompute": fb_rc,
            "ratio_fwd_bwd_over_fwd": round(fb["ms"] / fwd["ms"], 3),
            "ratio_with_loss_over_fwd": round(fl["ms"] / fwd["ms"], 3),
            "ratio_loss_fused_over_fwd": round(flf["ms"] / fwd["ms"], 3),
            "ratio_recompute_over_fwd": round(fb_rc["ms"] / fwd["ms"], 3),
            "frames_per_s_fwd": round(S * F / (fwd["ms"] * 1e-3), 1)}


if __name__ == "__main__":
    sys.exit(main())
