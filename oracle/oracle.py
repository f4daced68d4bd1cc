"""ctypes wrapper over the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference leg import
this module.  See fftfree_oracle.h for the reference lines each routine
restates.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

META_KINDS = {
    "Twiddle": 0, "LayoutMap": 1, "StageSnapshot": 2, "StageParams": 3,
    "ButterflyPairs": 4, "StageInvariant": 5, "TwiddleIndexMap": 6, "Omega": 7,
    "StageSnapshotAll": 8, "ButterflyPairsAll": 9, "TwiddleIndexMapAll": 10,
}


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _Cfg(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("inverse", ctypes.c_int), ("kernel", ctypes.c_int),
        ("transform", ctypes.c_int), ("reduce_magnitude", ctypes.c_int),
        ("store_polar", ctypes.c_int), ("half_spectrum", ctypes.c_int),
        ("window", ctypes.c_int), ("hop", ctypes.c_int), ("pad_mode", ctypes.c_int),
        ("windows_enabled", ctypes.c_int), ("apply_ola", ctypes.c_int),
        ("cola_mode", ctypes.c_int),
        ("analysis_win", ctypes.POINTER(ctypes.c_float)),
        ("synthesis_win", ctypes.POINTER(ctypes.c_float)),
    ]


class _Req(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("buf", ctypes.POINTER(ctypes.c_float)),
                ("count", ctypes.c_size_t)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        fp = ctypes.POINTER(ctypes.c_float)
        L.oracle_plan_twiddles.argtypes = [ctypes.c_int, ctypes.c_int, fp]
        L.oracle_plan_twiddles.restype = ctypes.c_int
        L.oracle_build_window.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_int, fp]
        L.oracle_build_window.restype = None
        L.oracle_fft_columns.argtypes = [ctypes.POINTER(_Cfg), fp, ctypes.c_size_t,
                                         ctypes.POINTER(_Req), ctypes.c_int, ctypes.c_int]
        L.oracle_fft_columns.restype = ctypes.c_int
        L.oracle_execute_batched.argtypes = [ctypes.POINTER(_Cfg), fp, ctypes.c_size_t, fp, fp,
                                             fp, ctypes.c_int, ctypes.c_size_t, ctypes.c_int]
        L.oracle_execute_batched.restype = ctypes.c_size_t
        L.oracle_execute_complex_batched.argtypes = [ctypes.POINTER(_Cfg), fp, fp, ctypes.c_size_t,
                                                     fp, ctypes.c_size_t, ctypes.c_int]
        L.oracle_execute_complex_batched.restype = ctypes.c_size_t
        L.oracle_frame_count.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t]
        L.oracle_frame_count.restype = ctypes.c_size_t
        _lib = L
    return _lib


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def build_window(kind: int, W: int, p1: float = 0.0, p2: float = 0.0, norm: int = 0) -> np.ndarray:
    out = np.ones(max(W, 0), dtype=np.float32)
    if W > 0:
        lib().oracle_build_window(kind, W, p1, p2, norm, _fptr(out))
    return out


def plan_twiddles(N: int, inverse: bool = False) -> np.ndarray:
    out = np.zeros(2 * max(1, N // 2), dtype=np.float32)
    if not lib().oracle_plan_twiddles(N, int(inverse), _fptr(out)):
        raise ValueError("N must be a power of two")
    return out.view(np.complex64)


@dataclass
class OracleContext:
    """Mirror of the reference FftContext fields that shape results.

    ``windows`` follow ``fft_init_full_v2`` (fft_cffi.cpp:1893-1906): length N,
    the first W taps from the window builder and the rest 1.0.
    """
    N: int
    inverse: int = 0
    kernel: int = 0
    transform: int = 0
    reduce_magnitude: int = 0
    store_polar: int = 0
    half_spectrum: int = 0
    window: int = 0
    hop: int = 0
    pad_mode: int = 0
    apply_windows: int = 0
    apply_ola: int = 0
    analysis_kind: int = 0
    analysis_p1: float = 0.0
    analysis_p2: float = 0.0
    synthesis_kind: int = 0
    synthesis_p1: float = 0.0
    synthesis_p2: float = 0.0
    norm_policy: int = 0
    cola_mode: int = 0
    analysis_win: np.ndarray = field(default=None, repr=False)
    synthesis_win: np.ndarray = field(default=None, repr=False)

    def __post_init__(self):
        useW = self.window if self.window > 0 else self.N
        aw = build_window(self.analysis_kind, useW, self.analysis_p1, self.analysis_p2, self.norm_policy)
        sw = build_window(self.synthesis_kind, useW, self.synthesis_p1, self.synthesis_p2, self.norm_policy)
        self.analysis_win = np.ones(self.N, np.float32)
        self.synthesis_win = np.ones(self.N, np.float32)
        k = min(useW, self.N)
        self.analysis_win[:k] = aw[:k]
        self.synthesis_win[:k] = sw[:k]

    @property
    def bins(self) -> int:
        return self.N // 2 + 1 if self.half_spectrum else self.N

    def _cfg(self) -> _Cfg:
        c = _Cfg()
        c.N, c.inverse, c.kernel = self.N, self.inverse, self.kernel
        c.transform, c.reduce_magnitude = self.transform, self.reduce_magnitude
        c.store_polar, c.half_spectrum = self.store_polar, self.half_spectrum
        c.window, c.hop, c.pad_mode = self.window, self.hop, self.pad_mode
        c.windows_enabled, c.apply_ola, c.cola_mode = self.apply_windows, self.apply_ola, self.cola_mode
        c.analysis_win = _fptr(self.analysis_win)
        c.synthesis_win = _fptr(self.synthesis_win)
        return c

    def frame_count(self, pcm_len: int, pad_mode: int = 1, max_frames: int = 0) -> int:
        return int(lib().oracle_frame_count(self.N, self.window, self.hop, self.pad_mode,
                                            pcm_len, pad_mode, max_frames))

    def execute_batched(self, pcm: np.ndarray, pad_mode: int = 1, max_frames: int = 0,
                        threads: int = 1):
        pcm = np.ascontiguousarray(pcm, dtype=np.float32)
        frames = self.frame_count(len(pcm), pad_mode, max_frames)
        cap = max(frames, 1) * self.bins
        re = np.zeros(cap, np.float32); im = np.zeros(cap, np.float32); mag = np.zeros(cap, np.float32)
        c = self._cfg()
        n = lib().oracle_execute_batched(ctypes.byref(c), _fptr(pcm), len(pcm), _fptr(re), _fptr(im),
                                         _fptr(mag), pad_mode, max_frames, threads)
        n = int(n)
        shape = (n, self.bins)
        return n, re[: n * self.bins].reshape(shape), im[: n * self.bins].reshape(shape), \
            mag[: n * self.bins].reshape(shape)

    def execute_complex_batched(self, in_real: np.ndarray, in_imag: np.ndarray, frames: int,
                                max_frames: int = 0, threads: int = 1):
        in_real = np.ascontiguousarray(in_real, dtype=np.float32).ravel()
        in_imag = np.ascontiguousarray(in_imag, dtype=np.float32).ravel()
        out = np.zeros(max(frames, 1) * self.N, np.float32)
        c = self._cfg()
        n = lib().oracle_execute_complex_batched(ctypes.byref(c), _fptr(in_real), _fptr(in_imag),
                                                 frames, _fptr(out), max_frames, threads)
        return int(n), out[: frames * self.N].reshape(frames, self.N)

    def fft_columns(self, X: np.ndarray, metadata: dict | None = None, threads: int = 1):
        """Batched in-place transform of X (B, N) complex64 rows == columns of
        the reference's N x B column-major matrix.  ``metadata`` maps kind
        names to element counts; returns (ok, X_out, {kind: complex64 array})."""
        X = np.ascontiguousarray(X, dtype=np.complex64).copy()
        B = X.shape[0] if X.ndim == 2 else 1
        reqs = []
        bufs = {}
        for name, count in (metadata or {}).items():
            buf = np.zeros(int(count), np.complex64)
            bufs[name] = buf
            r = _Req()
            r.kind = META_KINDS[name]
            r.buf = buf.view(np.float32).ctypes.data_as(ctypes.POINTER(ctypes.c_float))
            r.count = int(count)
            reqs.append(r)
        arr = (_Req * max(1, len(reqs)))(*reqs) if reqs else None
        c = self._cfg()
        ok = lib().oracle_fft_columns(ctypes.byref(c), X.view(np.float32).ctypes.data_as(
            ctypes.POINTER(ctypes.c_float)), B, arr, len(reqs), threads)
        return bool(ok), X, bufs


def fft_2d(ctx_axis0: OracleContext, ctx_axis1: OracleContext, X: np.ndarray, threads: int = 1):
    """fft_inplace_2d (eigen_fft.hpp:3177-3215).  X: (batch, cols, rows)
    complex64 -- batch column-major rows x cols matrices, column c of matrix
    b is X[b, c].  The axis-0 plan runs over every column, the tiled transpose
    (eigen_fft.hpp:2448-2472, a pure data move) makes every row contiguous,
    the axis-1 plan runs over them and the transpose moves them back.
    Returns (ok, X_out) with X's shape."""
    X = np.ascontiguousarray(X, dtype=np.complex64)
    B, C, R = X.shape
    if ctx_axis0.N != R or ctx_axis1.N != C:
        return False, X
    ok0, Y, _ = ctx_axis0.fft_columns(X.reshape(B * C, R), threads=threads)
    Yt = np.ascontiguousarray(Y.reshape(B, C, R).transpose(0, 2, 1)).reshape(B * R, C)
    ok1, Z, _ = ctx_axis1.fft_columns(Yt, threads=threads)
    out = np.ascontiguousarray(Z.reshape(B, R, C).transpose(0, 2, 1))
    return bool(ok0 and ok1), out
