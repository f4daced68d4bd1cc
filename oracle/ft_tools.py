"""ctypes wrapper over the reference's own grid tools built as a checker: the
ft_apply_*_pipeline entry points of ft_tools_cffi.cpp, compiled unchanged into
oracle/_ref/libfftfree_ref.so by `make -C oracle ref REF=<reference tree>`.

TEST INFRASTRUCTURE ONLY: loaded by tests/ and by the fixture generator under
tests/golden/; never by the product.  The structs mirror ft_tools_cffi.hpp:9-40.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libfftfree_ref.so")


class GridSpec(ctypes.Structure):
    _fields_ = [("time_origin", ctypes.c_double), ("freq_origin", ctypes.c_double),
                ("time_step", ctypes.c_double), ("freq_step", ctypes.c_double)]


class ResamplePlan(ctypes.Structure):
    _fields_ = [("upsample_time", ctypes.c_int), ("upsample_freq", ctypes.c_int),
                ("downsample_time", ctypes.c_int), ("downsample_freq", ctypes.c_int),
                ("preserve_energy", ctypes.c_int)]


class QuantizerConfig(ctypes.Structure):
    _fields_ = [("enabled", ctypes.c_int), ("base_frequency", ctypes.c_float), ("magnitude_step", ctypes.c_float),
                ("mix", ctypes.c_float), ("distance_decay", ctypes.c_float)]


class ContrastConfig(ctypes.Structure):
    _fields_ = [("enabled", ctypes.c_int), ("kernel_time", ctypes.c_int), ("kernel_freq", ctypes.c_int),
                ("brightness", ctypes.c_float), ("contrast", ctypes.c_float), ("gamma", ctypes.c_float),
                ("clamp_zero", ctypes.c_int)]


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib():
    from oracle import reflib
    return reflib.lib()


def _ref(x):
    return ctypes.byref(x) if x is not None else None


def apply(a: np.ndarray, b: np.ndarray, T: int, F: int, spec=None, plan=None, quant=None, contrast=None,
          polar: bool = False):
    """Run the reference pipeline on copies of the planar grids; returns
    (ok, a_out, b_out)."""
    a = np.ascontiguousarray(a, np.float32).copy()
    b = np.ascontiguousarray(b, np.float32).copy()
    fn = lib().ft_apply_polar_pipeline if polar else lib().ft_apply_complex_pipeline
    fp = ctypes.POINTER(ctypes.c_float)
    ok = fn(_ref(spec), _ref(plan), _ref(quant), _ref(contrast), a.ctypes.data_as(fp), b.ctypes.data_as(fp), T, F)
    return int(ok), a, b
