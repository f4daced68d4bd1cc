"""Python binding of libfft_cffi.so (the B200 build of the fftfree C ABI).

The reference's Python callers bind the library with ``cffi.dlopen`` and the
C declarations of fft_cffi.hpp (fft_to_png.py:14-114); this module does the
same with ctypes and adds a thin object wrapper, ``FftContext``, whose
methods keep the reference's argument meaning and return conventions
(frames produced, 0 on failure).  Buffers may be numpy arrays (host memory)
or CUDA tensors / raw device pointers; the library moves data as needed.

There is no CPU fallback: loading fails loudly when the shared library is
missing, and the init functions return NULL without a CUDA device.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfft_cffi.so")

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int)

# Constants of fft_cffi.hpp (same values)
FFT_KERNEL_COOLEYTUKEY, FFT_KERNEL_STOCKHAM, FFT_KERNEL_EXTERNAL = 0, 1, 2
FFT_TRANSFORM_C2C, FFT_TRANSFORM_R2C, FFT_TRANSFORM_C2R, FFT_TRANSFORM_R2R = 0, 1, 2, 3
FFT_WINDOW_RECT, FFT_WINDOW_HANN, FFT_WINDOW_HAMMING, FFT_WINDOW_BLACKMAN = 0, 1, 2, 3
FFT_WINDOW_TUKEY, FFT_WINDOW_KAISER = 4, 5
FFT_WINDOW_NORM_NONE, FFT_WINDOW_NORM_L2, FFT_WINDOW_NORM_AREA = 0, 1, 2
FFT_COLA_OFF, FFT_COLA_NORMALIZE = 0, 1
FFT_STREAM_FLUSH_NONE, FFT_STREAM_FLUSH_PARTIAL, FFT_STREAM_FLUSH_FINAL = 0, 1, 2

RESTORE_OBSERVER = ctypes.CFUNCTYPE(None, ctypes.c_size_t, ctypes.c_size_t)


class MetadataRequest(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("buffer", c_float_p), ("count", ctypes.c_size_t)]


# (name, restype, argtypes) for every exported symbol of include/*.h
_SIGS = [
    ("fft_pcm_to_channels", None, [c_float_p, c_float_p, c_float_p, c_float_p, ctypes.c_size_t, ctypes.c_int]),
    ("fft_init", ctypes.c_void_p, [ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, c_int_p, ctypes.c_size_t, ctypes.c_int]),
    ("fft_init_ex", ctypes.c_void_p, [ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, c_int_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int]),
    ("fft_init_full", ctypes.c_void_p, [ctypes.c_size_t] + [ctypes.c_int] * 5 + [c_int_p, ctypes.c_size_t]
     + [ctypes.c_int] * 12),
    ("fft_init_full_v2", ctypes.c_void_p, [ctypes.c_size_t] + [ctypes.c_int] * 5 + [c_int_p, ctypes.c_size_t]
     + [ctypes.c_int] * 15 + [ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                              ctypes.c_float, ctypes.c_int, ctypes.c_int]),
    ("fft_execute", ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p, c_float_p, c_float_p, ctypes.c_size_t]),
    ("fft_execute_batched", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t, c_float_p, c_float_p,
                                              c_float_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t]),
    ("fft_stft_execute", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t, c_float_p, c_float_p,
                                           c_float_p, ctypes.c_size_t]),
    ("fft_stream_reset", None, [ctypes.c_void_p]),
    ("fft_stream_push_pcm", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t, c_float_p, c_float_p,
                                              c_float_p, ctypes.c_size_t, ctypes.c_int]),
    ("fft_stream_pending_frames", ctypes.c_size_t, [ctypes.c_void_p]),
    ("fft_stream_backlog_samples", ctypes.c_size_t, [ctypes.c_void_p]),
    ("fft_stream_push_spectrum", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, c_float_p, ctypes.c_size_t,
                                                   c_float_p, ctypes.c_size_t, ctypes.c_int]),
    ("fft_stream_pending_pcm", ctypes.c_size_t, [ctypes.c_void_p]),
    ("fft_griffin_lim", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_float_p, ctypes.c_size_t, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint, c_float_p,
                                       c_float_p]),
    ("fft_execute_complex_batched", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, c_float_p, ctypes.c_size_t,
                                                      c_float_p, ctypes.c_int, ctypes.c_int, ctypes.c_size_t]),
    ("fft_ctx_size", ctypes.c_size_t, [ctypes.c_void_p]),
    ("fft_ctx_worker_threads", ctypes.c_size_t, [ctypes.c_void_p]),
    ("fft_ctx_effective_threads", ctypes.c_size_t, [ctypes.c_void_p]),
    ("fft_set_workerpool_debug_dropout", None, [ctypes.c_int]),
    ("fft_set_workerpool_dropout_pattern", None, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("fft_set_workerpool_dropout_single", None, [ctypes.c_longlong]),
    ("fft_set_workerpool_dropout_persistent", None, [ctypes.c_int]),
    ("fft_clear_workerpool_dropout_history", None, []),
    ("phase_init", ctypes.c_void_p, [ctypes.c_int] * 5),
    ("phase_infer_execute", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t, c_float_p, c_float_p]),
    ("phase_free", None, [ctypes.c_void_p]),
    ("fft_free", None, [ctypes.c_void_p]),
    ("fft_register_restore_observer", None, [RESTORE_OBSERVER]),
    ("fft_config_window", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                         ctypes.c_float, ctypes.c_int, ctypes.c_int]),
    ("fft_config_window_custom", ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_size_t, c_float_p,
                                                ctypes.c_size_t, ctypes.c_int, ctypes.c_int]),
    ("fftfree_execute_c2c", ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p, ctypes.c_size_t]),
    ("fftfree_execute_c2c_meta", ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p, ctypes.c_size_t,
                                                ctypes.POINTER(MetadataRequest), ctypes.c_int]),
    ("fftfree_set_stream", None, [ctypes.c_void_p, ctypes.c_void_p]),
    ("fftfree_ctx_stream", ctypes.c_void_p, [ctypes.c_void_p]),
    ("fftfree_set_async", None, [ctypes.c_void_p, ctypes.c_int]),
    ("fftfree_ctx_launch_count", ctypes.c_ulonglong, [ctypes.c_void_p]),
    ("fftfree_ctx_schedule", ctypes.c_int, [ctypes.c_void_p, c_int_p, ctypes.c_int]),
    ("fftfree_ctx_kernel", ctypes.c_int, [ctypes.c_void_p]),
    ("fftfree_frame_count", ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t]),
    ("fftfree_ctx_frame_shape", ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p]),
    ("fftfree_device_available", ctypes.c_int, []),
    ("fftfree_execute_complex_batched_noalloc", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, c_float_p,
                                                                   ctypes.c_size_t, c_float_p, ctypes.c_size_t]),
    ("ft_apply_complex_pipeline", ctypes.c_int, [ctypes.c_void_p] * 4 + [c_float_p, c_float_p, ctypes.c_int,
                                                                          ctypes.c_int]),
    ("ft_apply_polar_pipeline", ctypes.c_int, [ctypes.c_void_p] * 4 + [c_float_p, c_float_p, ctypes.c_int,
                                                                        ctypes.c_int]),
    ("fftfree_execute_2d", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_float_p, c_float_p, ctypes.c_size_t,
                                          ctypes.c_size_t, ctypes.c_size_t]),
    ("fftfree_stft_magnitude", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t, ctypes.c_size_t,
                                                 c_float_p, ctypes.c_size_t]),
    ("fftfree_stft_magnitude_backward", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t,
                                                          ctypes.c_size_t, c_float_p, c_float_p]),
    ("fftfree_stft_magnitude_phasor", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t,
                                                       ctypes.c_size_t, c_float_p, c_float_p, ctypes.c_size_t]),
    ("fftfree_stft_magnitude_backward_phasor", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t,
                                                                ctypes.c_size_t, c_float_p, c_float_p]),
    ("fftfree_stft_l2_partials", ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_size_t]),
    ("fftfree_stft_magnitude_l2", ctypes.c_size_t, [ctypes.c_void_p, c_float_p, ctypes.c_size_t, ctypes.c_size_t,
                                                    c_float_p, c_float_p, c_float_p, c_float_p, ctypes.c_size_t]),
    ("fftfree_stft_magnitude_backward_phasor_scaled", ctypes.c_size_t,
     [ctypes.c_void_p, c_float_p, ctypes.c_size_t, ctypes.c_size_t, c_float_p, c_float_p, c_float_p,
      ctypes.c_float]),
    ("fftfree_ragged_plan", ctypes.c_void_p, [ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t, ctypes.c_int,
                                              ctypes.c_int]),
    ("fftfree_ragged_plan_stft", ctypes.c_void_p, [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
                                                   c_int_p, c_int_p, c_int_p, c_float_p, ctypes.c_size_t,
                                                   ctypes.c_int, ctypes.c_int]),
    ("fftfree_ragged_frames", ctypes.c_size_t, [ctypes.c_void_p, ctypes.c_size_t]),
    ("fftfree_ragged_samples", ctypes.c_size_t, [ctypes.c_void_p]),
    ("fftfree_ragged_bins", ctypes.c_size_t, [ctypes.c_void_p]),
    ("fftfree_ragged_schedule", ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t]),
    ("fftfree_ragged_tile", ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t]),
    ("fftfree_ragged_set_stream", None, [ctypes.c_void_p, ctypes.c_void_p]),
    ("fftfree_ragged_execute", ctypes.c_int, [ctypes.c_void_p, c_float_p, c_float_p, c_float_p, c_float_p]),
    ("fftfree_ragged_launch_count", ctypes.c_ulonglong, [ctypes.c_void_p]),
    ("fftfree_ragged_free", None, [ctypes.c_void_p]),
    ("fftfree_debug_recovery_plan", ctypes.c_size_t, [ctypes.c_size_t, ctypes.c_char_p]),
]

EXPORTED = [s[0] for s in _SIGS]
_lib = None


def lib() -> ctypes.CDLL:
    """Load libfft_cffi.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        path = os.environ.get("FFTFREE_CFFI_LIB", LIB_PATH)
        if not os.path.exists(path):
            raise OSError(f"libfft_cffi.so not found at {path}; build it with "
                          "`python fftfree_b200/build.py` (there is no CPU fallback)")
        L = ctypes.CDLL(path)
        for name, res, args in _SIGS:
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def address(a) -> int:
    """The address of a numpy array, a torch tensor (host or CUDA) or an int."""
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return int(a.data_ptr())
    return int(a.ctypes.data)


def _fp(a) -> ctypes.POINTER(ctypes.c_float):
    """float* for a numpy array, a torch tensor (host or CUDA) or an int address."""
    if a is None:
        return None
    if isinstance(a, int):
        return ctypes.cast(ctypes.c_void_p(a), c_float_p)
    if hasattr(a, "data_ptr"):
        return ctypes.cast(ctypes.c_void_p(a.data_ptr()), c_float_p)
    return a.ctypes.data_as(c_float_p)


def _ip(seq):
    if not seq:
        return None, 0
    arr = (ctypes.c_int * len(seq))(*seq)
    return ctypes.cast(arr, c_int_p), len(seq)


class FftContext:
    """Owns one ``void*`` context of the C ABI."""

    def __init__(self, handle: int):
        if not handle:
            raise RuntimeError("fft context initialisation failed (NULL handle)")
        self.handle = ctypes.c_void_p(handle)

    # -- constructors with the reference argument lists ---------------------
    @classmethod
    def full(cls, n, threads=1, lanes=1, inverse=0, kernel=0, radix=0, radix_pattern=None, pad_mode=1,
             window=0, hop=0, transform=0, reduce_magnitude=0, store_polar=0, half_spectrum=0,
             allow_outer_parallel=0, allow_inner_parallel=0, inner_threads=0, save_crash_logs=0,
             silent_crash_reports=1):
        p, plen = _ip(radix_pattern)
        return cls(lib().fft_init_full(n, threads, lanes, inverse, kernel, radix, p, plen, pad_mode, window, hop,
                                       transform, reduce_magnitude, store_polar, half_spectrum,
                                       allow_outer_parallel, allow_inner_parallel, inner_threads,
                                       save_crash_logs, silent_crash_reports))

    @classmethod
    def full_v2(cls, n, threads=1, lanes=1, inverse=0, kernel=0, radix=0, radix_pattern=None, pad_mode=1,
                window=0, hop=0, transform=0, reduce_magnitude=0, store_polar=0, half_spectrum=0,
                allow_outer_parallel=0, allow_inner_parallel=0, inner_threads=0, save_crash_logs=0,
                silent_crash_reports=1, apply_windows=0, apply_ola=0, analysis_kind=0, analysis_p1=0.0,
                analysis_p2=0.0, synthesis_kind=0, synthesis_p1=0.0, synthesis_p2=0.0, norm_policy=0,
                cola_mode=0):
        p, plen = _ip(radix_pattern)
        return cls(lib().fft_init_full_v2(n, threads, lanes, inverse, kernel, radix, p, plen, pad_mode, window,
                                          hop, transform, reduce_magnitude, store_polar, half_spectrum,
                                          allow_outer_parallel, allow_inner_parallel, inner_threads,
                                          save_crash_logs, silent_crash_reports, apply_windows, apply_ola,
                                          analysis_kind, analysis_p1, analysis_p2, synthesis_kind, synthesis_p1,
                                          synthesis_p2, norm_policy, cola_mode))

    @classmethod
    def ex(cls, n, threads=0, lanes=0, inverse=0, kernel=0, radix=0, radix_pattern=None, pad_mode=0, window=0,
           hop=0):
        p, plen = _ip(radix_pattern)
        return cls(lib().fft_init_ex(n, threads, lanes, inverse, kernel, radix, p, plen, pad_mode, window, hop))

    def close(self):
        if self.handle:
            lib().fft_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- queries -------------------------------------------------------------
    @property
    def N(self) -> int:
        return int(lib().fft_ctx_size(self.handle))

    def schedule(self):
        buf = (ctypes.c_int * 32)()
        n = lib().fftfree_ctx_schedule(self.handle, buf, 32)
        return list(buf[:n])

    def frame_count(self, pcm_len: int, pad_mode: int = 1, max_frames: int = 0) -> int:
        return int(lib().fftfree_frame_count(self.handle, pcm_len, pad_mode, max_frames))

    def window_length(self) -> int:
        w, h = ctypes.c_int(0), ctypes.c_int(0)
        lib().fftfree_ctx_frame_shape(self.handle, ctypes.byref(w), ctypes.byref(h))
        return int(w.value)

    def hop_length(self) -> int:
        w, h = ctypes.c_int(0), ctypes.c_int(0)
        lib().fftfree_ctx_frame_shape(self.handle, ctypes.byref(w), ctypes.byref(h))
        return int(h.value)

    def kernel(self) -> int:
        """Executor code after the FFTFREE_DEFAULT_KERNEL override."""
        return int(lib().fftfree_ctx_kernel(self.handle))

    def launch_count(self) -> int:
        return int(lib().fftfree_ctx_launch_count(self.handle))

    def set_stream(self, stream_handle: Optional[int]):
        """Run on this cudaStream_t (an int handle, e.g. torch's
        ``stream.cuda_stream``; 0 is the legacy default stream)."""
        lib().fftfree_set_stream(self.handle, ctypes.c_void_p(stream_handle or 0))

    def stream(self) -> int:
        return int(lib().fftfree_ctx_stream(self.handle) or 0)

    def set_async(self, on: bool):
        lib().fftfree_set_async(self.handle, 1 if on else 0)

    # -- execution -----------------------------------------------------------
    def execute_batched(self, pcm, out_real, out_imag, out_mag, pcm_len=None, pad_mode=1, enable_backup=0,
                        max_frames=0) -> int:
        n = pcm_len if pcm_len is not None else (pcm.numel() if hasattr(pcm, "numel") else len(pcm))
        return int(lib().fft_execute_batched(self.handle, _fp(pcm), n, _fp(out_real), _fp(out_imag),
                                             _fp(out_mag), pad_mode, enable_backup, max_frames))

    def execute(self, pcm, out_real, out_imag, out_mag, n=None) -> int:
        n = n if n is not None else len(pcm)
        return int(lib().fft_execute(self.handle, _fp(pcm), _fp(out_real), _fp(out_imag), _fp(out_mag), n))

    def execute_complex_batched(self, in_real, in_imag, frames, out_pcm, pad_mode=1, enable_backup=0,
                                max_frames=0) -> int:
        return int(lib().fft_execute_complex_batched(self.handle, _fp(in_real), _fp(in_imag), frames,
                                                     _fp(out_pcm), pad_mode, enable_backup, max_frames))

    def execute_c2c(self, x, out, batch) -> int:
        return int(lib().fftfree_execute_c2c(self.handle, _fp(x), _fp(out), batch))

    def execute_c2c_meta(self, x, out, batch, requests) -> int:
        """requests: list of (kind, complex64 numpy buffer)."""
        arr = (MetadataRequest * max(1, len(requests)))()
        for i, (kind, buf) in enumerate(requests):
            arr[i].kind = kind
            arr[i].buffer = _fp(buf.view(np.float32)) if isinstance(buf, np.ndarray) else _fp(buf)
            if isinstance(buf, np.ndarray):
                arr[i].count = buf.size if np.iscomplexobj(buf) else buf.size // 2
            else:  # torch tensor: complex dtype, or interleaved floats
                arr[i].count = buf.numel() if buf.is_complex() else buf.numel() // 2
        return int(lib().fftfree_execute_c2c_meta(self.handle, _fp(x), _fp(out), batch, arr, len(requests)))


    def stft_magnitude(self, pcm, signals, length, out_mag, max_frames=0) -> int:
        return int(lib().fftfree_stft_magnitude(self.handle, _fp(pcm), signals, length, _fp(out_mag), max_frames))

    def stft_magnitude_phasor(self, pcm, signals, length, out_mag, out_phasor, max_frames=0) -> int:
        return int(lib().fftfree_stft_magnitude_phasor(self.handle, _fp(pcm), signals, length, _fp(out_mag),
                                                       _fp(out_phasor), max_frames))

    def stft_magnitude_backward_phasor(self, phasor, signals, length, grad_mag, grad_pcm) -> int:
        return int(lib().fftfree_stft_magnitude_backward_phasor(self.handle, _fp(phasor), signals, length,
                                                                _fp(grad_mag), _fp(grad_pcm)))

    def stft_l2_partials(self, frames_total) -> int:
        return int(lib().fftfree_stft_l2_partials(self.handle, frames_total))

    def stft_magnitude_l2(self, pcm, signals, length, target, out_residual, out_phasor, out_partials,
                          max_frames=0) -> int:
        return int(lib().fftfree_stft_magnitude_l2(self.handle, _fp(pcm), signals, length, _fp(target),
                                                   _fp(out_residual), _fp(out_phasor), _fp(out_partials),
                                                   max_frames))

    def stft_magnitude_backward_phasor_scaled(self, phasor, signals, length, grad_mag, grad_pcm, scale=None,
                                              factor=1.0) -> int:
        return int(lib().fftfree_stft_magnitude_backward_phasor_scaled(self.handle, _fp(phasor), signals, length,
                                                                       _fp(grad_mag), _fp(grad_pcm), _fp(scale),
                                                                       float(factor)))

    def stft_magnitude_backward(self, pcm, signals, length, grad_mag, grad_pcm) -> int:
        return int(lib().fftfree_stft_magnitude_backward(self.handle, _fp(pcm), signals, length, _fp(grad_mag),
                                                         _fp(grad_pcm)))


class RaggedPlan:
    """One persistent launch over real signals of mixed sizes (see
    fftfree_ragged_plan in include/fftfree_b200.h)."""

    def __init__(self, sizes, reduce_magnitude=0, store_polar=0, lengths=None, window=None, hop=None,
                 window_kind=None, window_param=None):
        """sizes: transform size N of each item.  With only sizes, item i is one
        frame of N samples; with ``lengths`` (samples per signal) and optional
        per-item ``window`` / ``hop`` / ``window_kind`` / ``window_param`` the
        items are framed signals (fftfree_ragged_plan_stft)."""
        self.sizes = [int(n) for n in sizes]
        cnt = len(self.sizes)
        arr = (ctypes.c_size_t * cnt)(*self.sizes)
        if lengths is None and window is None and hop is None and window_kind is None:
            self.handle = lib().fftfree_ragged_plan(arr, cnt, reduce_magnitude, store_polar)
        else:
            lens = (ctypes.c_size_t * cnt)(*[int(v) for v in (lengths if lengths is not None else self.sizes)])

            def ints(seq):
                return None if seq is None else ctypes.cast((ctypes.c_int * cnt)(*[int(v) for v in seq]), c_int_p)

            params = None if window_param is None else ctypes.cast(
                (ctypes.c_float * cnt)(*[float(v) for v in window_param]), c_float_p)
            self.handle = lib().fftfree_ragged_plan_stft(arr, lens, ints(window), ints(hop), ints(window_kind),
                                                         params, cnt, reduce_magnitude, store_polar)
        if not self.handle:
            raise RuntimeError("fftfree_ragged_plan failed")

    def frames(self, item: int) -> int:
        return int(lib().fftfree_ragged_frames(self.handle, item))

    @property
    def samples(self) -> int:
        return int(lib().fftfree_ragged_samples(self.handle))

    @property
    def bins(self) -> int:
        return int(lib().fftfree_ragged_bins(self.handle))

    def schedule(self, n) -> int:
        return int(lib().fftfree_ragged_schedule(self.handle, n))

    def tile(self, n) -> int:
        return int(lib().fftfree_ragged_tile(self.handle, n))

    def set_stream(self, stream_handle):
        lib().fftfree_ragged_set_stream(self.handle, ctypes.c_void_p(stream_handle or 0))

    def execute(self, pcm, out_real, out_imag, out_mag) -> int:
        return int(lib().fftfree_ragged_execute(self.handle, _fp(pcm), _fp(out_real), _fp(out_imag), _fp(out_mag)))

    def frame_count(self, pcm_len: int, pad_mode: int = 1, max_frames: int = 0) -> int:
        return int(lib().fftfree_frame_count(self.handle, pcm_len, pad_mode, max_frames))

    def window_length(self) -> int:
        w, h = ctypes.c_int(0), ctypes.c_int(0)
        lib().fftfree_ctx_frame_shape(self.handle, ctypes.byref(w), ctypes.byref(h))
        return int(w.value)

    def hop_length(self) -> int:
        w, h = ctypes.c_int(0), ctypes.c_int(0)
        lib().fftfree_ctx_frame_shape(self.handle, ctypes.byref(w), ctypes.byref(h))
        return int(h.value)

    def kernel(self) -> int:
        """Executor code after the FFTFREE_DEFAULT_KERNEL override."""
        return int(lib().fftfree_ctx_kernel(self.handle))

    def launch_count(self) -> int:
        return int(lib().fftfree_ragged_launch_count(self.handle))

    def close(self):
        if self.handle:
            lib().fftfree_ragged_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FtGridSpec(ctypes.Structure):
    """struct ft_grid_spec (ft_tools_cffi.hpp:9-14)."""
    _fields_ = [("time_origin", ctypes.c_double), ("freq_origin", ctypes.c_double),
                ("time_step", ctypes.c_double), ("freq_step", ctypes.c_double)]


class FtResamplePlan(ctypes.Structure):
    """struct ft_resample_plan_c (ft_tools_cffi.hpp:16-22)."""
    _fields_ = [("upsample_time", ctypes.c_int), ("upsample_freq", ctypes.c_int),
                ("downsample_time", ctypes.c_int), ("downsample_freq", ctypes.c_int),
                ("preserve_energy", ctypes.c_int)]


class FtQuantizerConfig(ctypes.Structure):
    """struct ft_quantizer_config (ft_tools_cffi.hpp:24-30)."""
    _fields_ = [("enabled", ctypes.c_int), ("base_frequency", ctypes.c_float), ("magnitude_step", ctypes.c_float),
                ("mix", ctypes.c_float), ("distance_decay", ctypes.c_float)]


class FtContrastConfig(ctypes.Structure):
    """struct ft_contrast_config (ft_tools_cffi.hpp:32-40)."""
    _fields_ = [("enabled", ctypes.c_int), ("kernel_time", ctypes.c_int), ("kernel_freq", ctypes.c_int),
                ("brightness", ctypes.c_float), ("contrast", ctypes.c_float), ("gamma", ctypes.c_float),
                ("clamp_zero", ctypes.c_int)]


def _byref(x):
    return ctypes.byref(x) if x is not None else None


def ft_apply_pipeline(a, b, time_bins: int, freq_bins: int, spec=None, plan=None, quant=None, contrast=None,
                      polar: bool = False) -> int:
    """ft_apply_complex_pipeline / ft_apply_polar_pipeline on planar float32
    grids (time_bins rows of freq_bins; host arrays or CUDA tensors), in
    place.  ``spec`` / ``plan`` / ``quant`` / ``contrast`` are the ctypes
    structs above or None."""
    fn = lib().ft_apply_polar_pipeline if polar else lib().ft_apply_complex_pipeline
    return int(fn(_byref(spec), _byref(plan), _byref(quant), _byref(contrast), _fp(a), _fp(b), time_bins, freq_bins))


def execute_2d(ctx_axis0: "FftContext", ctx_axis1: "FftContext", x, out, rows: int, cols: int,
               batch: int = 1) -> int:
    """2-D transform of ``batch`` column-major rows x cols complex matrices
    (eigen_fft.hpp:3177-3215): ctx_axis0 (N = rows) over the columns, then
    ctx_axis1 (N = cols) over the rows.  ``x`` / ``out`` hold interleaved
    complex float32 (host or CUDA), matrix after matrix; they may alias."""
    return int(lib().fftfree_execute_2d(ctx_axis0.handle, ctx_axis1.handle, _fp(x), _fp(out), rows, cols, batch))


def device_available() -> bool:
    return bool(lib().fftfree_device_available())
