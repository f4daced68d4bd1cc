"""Shared helpers for the parity tests: run a configuration through the CUDA
library (C ABI) and through the oracle, and compare with the tolerance the
path promises (rel-L2 <= 1e-5 * log2(N) against the reference float path)."""
from __future__ import annotations

import math

import numpy as np

from oracle.oracle import OracleContext


def tol_for(N: int) -> float:
    return 1e-5 * max(1.0, math.log2(max(N, 2)))


def rel_l2(got, ref) -> float:
    got = np.asarray(got, np.complex128 if np.iscomplexobj(got) or np.iscomplexobj(ref) else np.float64)
    ref = np.asarray(ref, got.dtype)
    den = np.linalg.norm(ref.ravel())
    num = np.linalg.norm((got - ref).ravel())
    if den < 1e-30:
        return float(num)
    return float(num / den)


def assert_close(got, ref, tol, what=""):
    e = rel_l2(got, ref)
    assert e <= tol, f"{what}: rel-L2 {e:.3e} > {tol:.3e}"
    return e


def polar_to_complex(mag, ph):
    return np.asarray(mag, np.float64) * np.exp(1j * np.asarray(ph, np.float64))


def ctx_kwargs(N, **kw):
    """fft_init_full_v2 keyword arguments (FftContext.full_v2) + matching oracle."""
    d = dict(n=N, threads=1, lanes=1, inverse=0, kernel=0, radix=0, radix_pattern=None, pad_mode=1,
             window=0, hop=0, transform=0, reduce_magnitude=0, store_polar=0, half_spectrum=0,
             allow_outer_parallel=0, allow_inner_parallel=0, inner_threads=0, save_crash_logs=0,
             silent_crash_reports=1, apply_windows=0, apply_ola=0, analysis_kind=0, analysis_p1=0.0,
             analysis_p2=0.0, synthesis_kind=0, synthesis_p1=0.0, synthesis_p2=0.0, norm_policy=0,
             cola_mode=0)
    d.update(kw)
    return d


def oracle_for(kw) -> OracleContext:
    return OracleContext(N=kw["n"], inverse=kw["inverse"], kernel=kw["kernel"], transform=kw["transform"],
                         reduce_magnitude=kw["reduce_magnitude"], store_polar=kw["store_polar"],
                         half_spectrum=kw["half_spectrum"], window=kw["window"], hop=kw["hop"],
                         pad_mode=kw["pad_mode"], apply_windows=kw["apply_windows"], apply_ola=kw["apply_ola"],
                         analysis_kind=kw["analysis_kind"], analysis_p1=kw["analysis_p1"],
                         analysis_p2=kw["analysis_p2"], synthesis_kind=kw["synthesis_kind"],
                         synthesis_p1=kw["synthesis_p1"], synthesis_p2=kw["synthesis_p2"],
                         norm_policy=kw["norm_policy"], cola_mode=kw["cola_mode"])


def compare_spectrum(kw, got, ref, tol):
    """got/ref: (re, im, mag) arrays of one execute_batched call."""
    gre, gim, gmag = (np.asarray(a, np.float64) for a in got)
    rre, rim, rmag = (np.asarray(a, np.float64) for a in ref)
    if kw["store_polar"]:
        assert_close(gre, rre, tol, "polar magnitude")
        assert_close(polar_to_complex(gre, gim), polar_to_complex(rre, rim), tol, "polar value")
    else:
        assert_close(gre + 1j * gim, rre + 1j * rim, tol, "complex")
    assert_close(gmag, rmag, tol, "mag")
