"""CPU-only checks of the C-ABI library: it loads, it exports every symbol
that include/*.h declares, it refuses to run without a GPU instead of
falling back to the CPU, and the host-side recovery coordinator reproduces
the reference's dropout / restore / split decisions."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import fftfree_b200 as ff

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in sorted(os.listdir(os.path.join(REPO, "include"))):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(REPO, "include", h)).read()
        for m in re.finditer(r"FFT_CFFI_API\s+[\w\s\*]+?\b(\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    L = ff.lib()
    declared = _declared_symbols()
    assert len(declared) >= 38
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", ff.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert declared <= exported
    # nothing beyond the declared C ABI leaks out (C++ internals stay hidden)
    extra = {s for s in exported if not s.startswith("_") and s not in declared}
    assert not extra, sorted(extra)


def test_python_binding_covers_declarations():
    assert _declared_symbols() <= set(ff.EXPORTED)


def _declared_arity():
    out = {}
    for h in sorted(os.listdir(os.path.join(REPO, "include"))):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(REPO, "include", h)).read()
        for m in re.finditer(r"FFT_CFFI_API\s+[\w\s\*]+?\b(\w+)\s*\(([^)]*)\)", src):
            params = m.group(2).strip()
            out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_python_binding_arity_matches_header():
    from fftfree_b200.api import _SIGS
    arity = _declared_arity()
    for name, _, args in _SIGS:
        assert len(args) == arity[name], (name, len(args), arity[name])


def test_reference_symbol_set_present():
    # fft_cffi.hpp:26-346 -- the 33 C entry points of the reference header
    ref = """fft_pcm_to_channels fft_init fft_init_ex fft_init_full fft_init_full_v2 fft_execute
    fft_execute_batched fft_stft_execute fft_stream_reset fft_stream_push_pcm fft_stream_pending_frames
    fft_stream_backlog_samples fft_stream_push_spectrum fft_stream_pending_pcm fft_griffin_lim
    fft_execute_complex_batched fft_ctx_size fft_ctx_worker_threads fft_ctx_effective_threads
    fft_set_workerpool_debug_dropout fft_set_workerpool_dropout_pattern fft_set_workerpool_dropout_single
    fft_set_workerpool_dropout_persistent fft_clear_workerpool_dropout_history phase_init phase_infer_execute
    phase_free fft_free fft_register_restore_observer fft_config_window fft_config_window_custom""".split()
    L = ff.lib()
    for name in ref:
        assert hasattr(L, name), name


def test_constants_match_reference():
    # fft_cffi.hpp:62-81, 292-320
    assert (ff.FFT_KERNEL_COOLEYTUKEY, ff.FFT_KERNEL_STOCKHAM, ff.FFT_KERNEL_EXTERNAL) == (0, 1, 2)
    assert (ff.FFT_TRANSFORM_C2C, ff.FFT_TRANSFORM_R2C, ff.FFT_TRANSFORM_C2R, ff.FFT_TRANSFORM_R2R) == (0, 1, 2, 3)
    assert (ff.FFT_WINDOW_KAISER, ff.FFT_WINDOW_NORM_AREA, ff.FFT_COLA_NORMALIZE, ff.FFT_STREAM_FLUSH_FINAL) == \
        (5, 2, 1, 2)


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the behaviour without a CUDA device")
def test_init_without_gpu_fails_loudly_instead_of_cpu_fallback():
    code = ("import sys; sys.path.insert(0, %r); import fftfree_b200 as ff; L = ff.lib(); "
            "h = L.fft_init_full(1024,1,1,0,2,4,None,0,1,1024,256,1,1,0,1,1,0,0,0,1); "
            "print('HANDLE', h)" % REPO)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert "HANDLE None" in r.stdout
    assert "no CPU fallback" in r.stderr
    assert ff.lib().fftfree_device_available() == 0


def test_null_handles_are_safe():
    L = ff.lib()
    L.fft_free(None)
    assert L.fft_ctx_size(None) == 0
    assert L.fft_execute_batched(None, None, 0, None, None, None, 1, 0, 0) == 0
    assert L.fft_stream_pending_frames(None) == 0
    L.phase_free(None)


# -- recovery coordinator (fft_cffi.cpp:826-1027; eigen_fft.hpp:1196-1398) ----
class _Observer:
    def __init__(self):
        self.calls = []
        self.cb = ff.RESTORE_OBSERVER(lambda s, e: self.calls.append((s, e)))


@pytest.fixture
def observer():
    o = _Observer()
    L = ff.lib()
    L.fft_register_restore_observer(o.cb)
    yield o
    L.fft_register_restore_observer(ff.RESTORE_OBSERVER())
    L.fft_set_workerpool_dropout_pattern(0, 0, 0)
    L.fft_set_workerpool_dropout_single(-1)
    L.fft_set_workerpool_dropout_persistent(0)
    L.fft_set_workerpool_debug_dropout(0)
    L.fft_clear_workerpool_dropout_history()


def _plan(frames):
    raw = ctypes.create_string_buffer(frames)
    n = ff.lib().fftfree_debug_recovery_plan(frames, raw)
    return n, [b for b in raw.raw[:frames]]


def test_recovery_no_dropout(observer):
    n, raw = _plan(10)
    assert n == 0 and observer.calls == []


def test_recovery_stripe_one_shot(observer):
    # restore_test_cffi.cpp:100-112 default stripe: period 4, on 1, phase 0
    L = ff.lib()
    L.fft_clear_workerpool_dropout_history()
    L.fft_set_workerpool_dropout_pattern(4, 1, 0)
    n, raw = _plan(10)
    assert n == 0  # one-shot: each dropped range succeeds on retry
    assert sorted(observer.calls) == [(0, 1), (4, 5), (8, 9)]
    # history persists: a second pass over the same indices drops nothing
    observer.calls.clear()
    n, _ = _plan(10)
    assert n == 0 and observer.calls == []


def test_recovery_single_persistent_aborts(observer):
    L = ff.lib()
    L.fft_clear_workerpool_dropout_history()
    L.fft_set_workerpool_dropout_single(3)
    L.fft_set_workerpool_dropout_persistent(1)
    n, raw = _plan(6)
    # three failed attempts on range 3 (one restore each); the single-frame
    # persistent failure aborts the batch and frame 3 stays restored
    assert observer.calls == [(3, 4)] * 3
    assert n == 1 and raw[3] == 1 and sum(raw) == 1


def test_recovery_single_one_shot(observer):
    L = ff.lib()
    L.fft_clear_workerpool_dropout_history()
    L.fft_set_workerpool_dropout_single(2)
    n, raw = _plan(5)
    assert n == 0 and observer.calls == [(2, 3)]


def test_pattern_clamp_and_phase(observer):
    L = ff.lib()
    L.fft_clear_workerpool_dropout_history()
    L.fft_set_workerpool_dropout_pattern(3, 7, 1)  # on_len clamps to period
    n, _ = _plan(4)
    assert sorted(observer.calls) == [(0, 1), (1, 2), (2, 3), (3, 4)]
