"""ctypes wrapper over the reference's own C ABI, compiled unchanged from its
sources into oracle/_ref/ by ``make -C oracle ref REF=<reference tree>``.

TEST INFRASTRUCTURE ONLY: the checker that pins the oracle (and, where
present, the GPU results) to the reference itself.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs load
it; the product never does.

Two builds of the same sources:
  * ``libfftfree_ref.so`` -- IEEE arithmetic (-O2, no FMA contraction), the
    parity build the tests compare against;
  * ``libfftfree_ref_release_v{3,4}.so`` -- the reference's Release flags
    (-O3 -ffast-math, x86-64-v3 / v4 in place of -march=native), timed as the
    CPU baseline.

The library exports the 31 fft_* / phase_* symbols of fft_cffi.hpp, the two
ft_* pipelines of ft_tools_cffi.hpp and ref_plan_create / ref_plan_execute /
ref_plan_free (ref_driver.cpp: the C++ batched transform with metadata).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
PARITY_LIB = os.path.join(REF_DIR, "libfftfree_ref.so")

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int)
RESTORE_OBSERVER = ctypes.CFUNCTYPE(None, ctypes.c_size_t, ctypes.c_size_t)


class MetaReq(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("buf", c_float_p), ("count", ctypes.c_size_t)]


# fft_cffi.hpp:31-346 (argument types of the reference's declarations)
_I, _Z, _F = ctypes.c_int, ctypes.c_size_t, ctypes.c_float
_SIGS = [
    ("fft_pcm_to_channels", None, [c_float_p, c_float_p, c_float_p, c_float_p, _Z, _I]),
    ("fft_init", ctypes.c_void_p, [_Z, _I, _I, _I, _I, _I, c_int_p, _Z, _I]),
    ("fft_init_ex", ctypes.c_void_p, [_Z, _I, _I, _I, _I, _I, c_int_p, _Z, _I, _I, _I]),
    ("fft_init_full", ctypes.c_void_p, [_Z] + [_I] * 5 + [c_int_p, _Z] + [_I] * 12),
    ("fft_init_full_v2", ctypes.c_void_p, [_Z] + [_I] * 5 + [c_int_p, _Z] + [_I] * 15
     + [_F, _F, _I, _F, _F, _I, _I]),
    ("fft_execute", _I, [ctypes.c_void_p, c_float_p, c_float_p, c_float_p, c_float_p, _Z]),
    ("fft_execute_batched", _Z, [ctypes.c_void_p, c_float_p, _Z, c_float_p, c_float_p, c_float_p, _I, _I, _Z]),
    ("fft_stft_execute", _Z, [ctypes.c_void_p, c_float_p, _Z, c_float_p, c_float_p, c_float_p, _Z]),
    ("fft_execute_complex_batched", _Z, [ctypes.c_void_p, c_float_p, c_float_p, _Z, c_float_p, _I, _I, _Z]),
    ("fft_stream_reset", None, [ctypes.c_void_p]),
    ("fft_stream_push_pcm", _Z, [ctypes.c_void_p, c_float_p, _Z, c_float_p, c_float_p, c_float_p, _Z, _I]),
    ("fft_stream_pending_frames", _Z, [ctypes.c_void_p]),
    ("fft_stream_backlog_samples", _Z, [ctypes.c_void_p]),
    ("fft_stream_push_spectrum", _Z, [ctypes.c_void_p, c_float_p, c_float_p, _Z, c_float_p, _Z, _I]),
    ("fft_stream_pending_pcm", _Z, [ctypes.c_void_p]),
    ("fft_griffin_lim", _I, [ctypes.c_void_p, ctypes.c_void_p, c_float_p, _Z, _I, _I, _I, _I, ctypes.c_uint,
                             c_float_p, c_float_p]),
    ("fft_ctx_size", _Z, [ctypes.c_void_p]),
    ("fft_ctx_worker_threads", _Z, [ctypes.c_void_p]),
    ("fft_ctx_effective_threads", _Z, [ctypes.c_void_p]),
    ("fft_set_workerpool_debug_dropout", None, [_I]),
    ("fft_set_workerpool_dropout_pattern", None, [_I, _I, _I]),
    ("fft_set_workerpool_dropout_single", None, [ctypes.c_longlong]),
    ("fft_set_workerpool_dropout_persistent", None, [_I]),
    ("fft_clear_workerpool_dropout_history", None, []),
    ("phase_init", ctypes.c_void_p, [_I] * 5),
    ("phase_infer_execute", _Z, [ctypes.c_void_p, c_float_p, _Z, c_float_p, c_float_p]),
    ("phase_free", None, [ctypes.c_void_p]),
    ("fft_free", None, [ctypes.c_void_p]),
    ("fft_register_restore_observer", None, [RESTORE_OBSERVER]),
    ("fft_config_window", _I, [ctypes.c_void_p, _I, _I, _F, _F, _I, _I]),
    ("fft_config_window_custom", _I, [ctypes.c_void_p, c_float_p, _Z, c_float_p, _Z, _I, _I]),
    ("ft_apply_complex_pipeline", _I, [ctypes.c_void_p] * 4 + [c_float_p, c_float_p, _I, _I]),
    ("ft_apply_polar_pipeline", _I, [ctypes.c_void_p] * 4 + [c_float_p, c_float_p, _I, _I]),
    ("ref_plan_create", ctypes.c_void_p, [_I] * 8),
    ("ref_plan_execute", _I, [ctypes.c_void_p, c_float_p, _Z, ctypes.POINTER(MetaReq), _I]),
    ("ref_plan_free", None, [ctypes.c_void_p]),
    ("ref_observer_attach", None, []),
    ("ref_observer_calls", _Z, [ctypes.POINTER(ctypes.c_size_t), _Z]),
]
REFERENCE_SYMBOLS = [s[0] for s in _SIGS if not s[0].startswith("ref_")]

_libs: dict = {}


def available() -> bool:
    return os.path.exists(PARITY_LIB)


def _load(path: str) -> ctypes.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise OSError(f"{path} not built (make -C oracle ref REF=<reference tree>)")
        L = ctypes.CDLL(path)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _libs[path] = L
    return _libs[path]


def lib() -> ctypes.CDLL:
    """The parity build (IEEE arithmetic)."""
    return _load(PARITY_LIB)


def release_path() -> str:
    """The Release-flag build for this host: x86-64-v4 where the CPU has
    AVX-512 (F, BW, CD, DQ, VL), else x86-64-v3."""
    flags = set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        pass
    v4 = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags
    return os.path.join(REF_DIR, "libfftfree_ref_release_v4.so" if v4 else "libfftfree_ref_release_v3.so")


def release_lib() -> ctypes.CDLL:
    return _load(release_path())


def fp(a) -> c_float_p:
    if a is None:
        return None
    return a.ctypes.data_as(c_float_p)


def ip(seq):
    if not seq:
        return None, 0
    arr = (ctypes.c_int * len(seq))(*seq)
    return ctypes.cast(arr, c_int_p), len(seq)


def observer_attach(L=None):
    """Record the reference's restore-observer calls (in C, thread-safe)."""
    (L or lib()).ref_observer_attach()


def observer_calls(L=None):
    L = L or lib()
    n = int(L.ref_observer_calls(None, 0))
    buf = (ctypes.c_size_t * max(2 * n, 2))()
    n = int(L.ref_observer_calls(buf, n))
    return [(int(buf[2 * i]), int(buf[2 * i + 1])) for i in range(n)]


class RefContext:
    """One context of the reference's C ABI (host buffers, as the reference
    takes them)."""

    def __init__(self, handle, L=None):
        if not handle:
            raise RuntimeError("reference context initialisation failed (NULL)")
        self.L = L or lib()
        self.h = ctypes.c_void_p(handle)

    @classmethod
    def full_v2(cls, L=None, **kw):
        L = L or lib()
        p, plen = ip(kw.get("radix_pattern"))
        k = kw
        return cls(L.fft_init_full_v2(k["n"], k["threads"], k["lanes"], k["inverse"], k["kernel"], k["radix"], p,
                                      plen, k["pad_mode"], k["window"], k["hop"], k["transform"],
                                      k["reduce_magnitude"], k["store_polar"], k["half_spectrum"],
                                      k["allow_outer_parallel"], k["allow_inner_parallel"], k["inner_threads"],
                                      k["save_crash_logs"], k["silent_crash_reports"], k["apply_windows"],
                                      k["apply_ola"], k["analysis_kind"], k["analysis_p1"], k["analysis_p2"],
                                      k["synthesis_kind"], k["synthesis_p1"], k["synthesis_p2"], k["norm_policy"],
                                      k["cola_mode"]), L)

    def close(self):
        if self.h:
            self.L.fft_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def execute_batched(self, pcm, cap_frames, bins, pad_mode=1, enable_backup=0, max_frames=0):
        pcm = np.ascontiguousarray(pcm, np.float32)
        cap = max(cap_frames, 1) * bins
        re, im, mag = (np.zeros(cap, np.float32) for _ in range(3))
        n = int(self.L.fft_execute_batched(self.h, fp(pcm), pcm.size, fp(re), fp(im), fp(mag), pad_mode,
                                           enable_backup, max_frames))
        return n, re[: n * bins], im[: n * bins], mag[: n * bins]

    def execute_complex_batched(self, in_real, in_imag, frames, N, pad_mode=1, enable_backup=0, max_frames=0):
        in_real = np.ascontiguousarray(in_real, np.float32).ravel()
        in_imag = np.ascontiguousarray(in_imag, np.float32).ravel()
        out = np.zeros(max(frames, 1) * N, np.float32)
        n = int(self.L.fft_execute_complex_batched(self.h, fp(in_real), fp(in_imag), frames, fp(out), pad_mode,
                                                   enable_backup, max_frames))
        return n, out


class RefPlan:
    """The reference's C++ batched transform (eigfft::fft_inplace_batched_with_metadata)
    over rows of a (batch, N) complex64 array = columns of its N x batch
    column-major matrix."""

    def __init__(self, N, inverse=0, kernel=0, transform=0, reduce_magnitude=0, store_polar=0, half_spectrum=0,
                 threads=1, L=None):
        self.L = L or lib()
        self.N = N
        self.h = self.L.ref_plan_create(N, inverse, kernel, transform, reduce_magnitude, store_polar,
                                        half_spectrum, threads)
        if not self.h:
            raise RuntimeError("ref_plan_create failed")

    def execute(self, X: np.ndarray, metadata: dict | None = None):
        """In place on X (complex64, C-contiguous).  ``metadata`` maps
        eigfft::MetadataKind values to element counts; returns (ok, {kind: buf})."""
        assert X.dtype == np.complex64 and X.flags.c_contiguous
        bufs = {k: np.zeros(int(c), np.complex64) for k, c in (metadata or {}).items()}
        reqs = (MetaReq * max(1, len(bufs)))(*[MetaReq(int(k), fp(b.view(np.float32)), b.size)
                                                 for k, b in bufs.items()])
        batch = X.size // self.N
        ok = self.L.ref_plan_execute(self.h, fp(X.view(np.float32)), batch, reqs, len(bufs))
        return bool(ok), bufs

    def close(self):
        if self.h:
            self.L.ref_plan_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
