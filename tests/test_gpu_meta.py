"""Metadata capture through fftfree_execute_c2c_meta (the C++ API
fft_inplace_batched_with_metadata) against the oracle: integer kinds are
bit-exact, stage snapshots reproduce the reference's radix-2 arithmetic."""
import numpy as np
import pytest

import fftfree_b200 as ff
from oracle.oracle import META_KINDS, OracleContext
from tests.helpers import assert_close, tol_for

pytestmark = pytest.mark.gpu

INT_KINDS = ["LayoutMap", "StageParams", "ButterflyPairs", "TwiddleIndexMap", "ButterflyPairsAll",
             "TwiddleIndexMapAll"]


def _sizes(N, B, kinds):
    S = int(np.log2(N))
    tw = sum(1 << s for s in range(S))
    base = {"Twiddle": max(tw, 1), "LayoutMap": N, "StageSnapshot": N * S, "StageParams": S,
            "ButterflyPairs": N * S, "StageInvariant": S, "TwiddleIndexMap": N * S, "Omega": N,
            "StageSnapshotAll": N * S * B, "ButterflyPairsAll": N * S * B, "TwiddleIndexMapAll": N * S * B}
    return {k: max(base[k], 1) for k in kinds}


def run_both(N, B, kernel, kinds, inverse=0, transform=0, half=0, seed=0, x=None):
    rng = np.random.default_rng(seed)
    if x is None:
        x = (rng.standard_normal((B, N)) + 1j * rng.standard_normal((B, N))).astype(np.complex64)
    sizes = _sizes(N, B, kinds)
    ctx = ff.FftContext.full_v2(N, kernel=kernel, inverse=inverse, transform=transform, half_spectrum=half)
    bufs = {k: np.zeros(n, np.complex64) for k, n in sizes.items()}
    out = np.zeros_like(x)
    ok = ctx.execute_c2c_meta(x.view(np.float32), out.view(np.float32), B,
                              [(META_KINDS[k], bufs[k]) for k in kinds])
    ref_ok, ref_out, ref_bufs = OracleContext(N=N, kernel=kernel, inverse=inverse, transform=transform,
                                              half_spectrum=half).fft_columns(x, sizes)
    return ok, out, bufs, ref_ok, ref_out, ref_bufs


ALL = list(META_KINDS)


SINGLE = [k for k in ALL if not k.endswith("All")]
CT_ALL = ["Twiddle", "LayoutMap", "StageParams", "StageInvariant", "Omega", "StageSnapshotAll",
          "ButterflyPairsAll", "TwiddleIndexMapAll"]


@pytest.mark.parametrize("N", [1, 2, 4, 8, 16, 32, 256, 1024])
@pytest.mark.parametrize("B", [1, 3, 16])
@pytest.mark.parametrize("kernel,kinds", [(1, SINGLE), (1, CT_ALL), (2, SINGLE)], ids=["ct", "ct-all", "stockham"])
def test_metadata_all_kinds(N, B, kernel, kinds):
    ok, out, bufs, rok, rout, rbufs = run_both(N, B, kernel, kinds, seed=N * 7 + B)
    assert ok == 1 and rok
    assert_close(out, rout, tol_for(N), "spectrum")
    for k in kinds:
        g, r = bufs[k], rbufs[k]
        if k in INT_KINDS:
            assert np.array_equal(g, r), k
        elif k == "StageInvariant":
            # maxima of butterfly rounding noise: the energy term uses only
            # + - * and is bit-identical; the hypot term within one ulp
            assert np.array_equal(g.imag, r.imag), k
            assert np.allclose(g.real, r.real, rtol=2e-7, atol=0), k
        elif k.startswith("StageSnapshot"):
            assert np.array_equal(g.view(np.uint32), r.view(np.uint32)), k
        else:
            assert_close(g, r, 1e-6, k)


@pytest.mark.parametrize("kernel", [1, 2])
def test_snapshot_bitwise(kernel):
    # non-contracted float butterflies with the reference twiddle table:
    # the stage snapshots equal the oracle's bit for bit
    N, B = 64, 4
    kinds = ["StageSnapshot"]
    ok, out, bufs, rok, rout, rbufs = run_both(N, B, kernel, kinds, seed=11)
    assert ok == 1
    assert np.array_equal(bufs["StageSnapshot"].view(np.uint32), rbufs["StageSnapshot"].view(np.uint32))
    assert np.array_equal(out.view(np.uint32), rout.view(np.uint32))


def test_all_kinds_take_precedence_over_single():
    # eigen_fft.hpp:2981-3010: with both requested, only the *All buffer is written
    N, B = 16, 3
    kinds = ["StageSnapshot", "StageSnapshotAll", "ButterflyPairs", "ButterflyPairsAll"]
    ok, out, bufs, rok, _, rbufs = run_both(N, B, 1, kinds)
    assert ok == 1 and rok
    assert not np.any(bufs["StageSnapshot"]) and not np.any(bufs["ButterflyPairs"])
    assert np.array_equal(bufs["ButterflyPairsAll"], rbufs["ButterflyPairsAll"])


@pytest.mark.parametrize("kind", ["StageSnapshot", "ButterflyPairs", "TwiddleIndexMap", "LayoutMap",
                                  "StageParams", "StageInvariant", "Twiddle"])
def test_undersized_buffer_rejected(kind):
    N, B = 16, 2
    ctx = ff.FftContext.full_v2(N, kernel=1)
    x = np.zeros((B, N), np.complex64)
    out = np.zeros_like(x)
    short = np.zeros(max(_sizes(N, B, [kind])[kind] - 1, 0) or 0, np.complex64)
    if short.size == 0:
        short = np.zeros(0, np.complex64)
    r = ctx.execute_c2c_meta(x.view(np.float32), out.view(np.float32), B, [(META_KINDS[kind], short)])
    assert r == 0


def test_stockham_ignores_ct_only_kinds():
    # Stockham constructs no Omega / *All writers, so it neither validates nor writes them
    N, B = 8, 2
    ctx = ff.FftContext.full_v2(N, kernel=2)
    x = np.ones((B, N), np.complex64)
    out = np.zeros_like(x)
    om = np.zeros(1, np.complex64)
    sa = np.zeros(1, np.complex64)
    assert ctx.execute_c2c_meta(x.view(np.float32), out.view(np.float32), B,
                                [(META_KINDS["Omega"], om), (META_KINDS["StageSnapshotAll"], sa)]) == 1
    assert not np.any(om) and not np.any(sa)


def test_consensus_kat(kat):
    # tests/fftfree_tests.cpp:921-1086 through the GPU: both executors agree
    # within 20e-5, layout maps are permutations, twiddle metadata agrees.
    x = np.ascontiguousarray(kat["consensus_n8_b3__input"])
    kinds = ["Twiddle", "LayoutMap", "StageSnapshot", "StageParams", "ButterflyPairs", "StageInvariant",
             "TwiddleIndexMap"]
    r1 = run_both(8, 3, 1, kinds, x=x)
    r2 = run_both(8, 3, 2, kinds, x=x)
    tol = 20e-5
    assert np.max(np.abs(r1[1] - kat["consensus_n8_b3__expected"])) <= tol
    assert np.max(np.abs(r2[1] - kat["consensus_n8_b3__expected"])) <= tol
    assert np.max(np.abs(r1[1] - r2[1])) <= tol
    for r in (r1, r2):
        lay = np.rint(r[2]["LayoutMap"].real).astype(int)
        assert sorted(lay.tolist()) == list(range(8))
    assert np.max(np.abs(r1[2]["Twiddle"] - r2[2]["Twiddle"])) <= tol


def test_metadata_device_buffers():
    torch = pytest.importorskip("torch")
    N, B = 32, 5
    x = np.random.default_rng(2).standard_normal((B, N * 2)).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    dout = torch.zeros_like(dx)
    dpairs = torch.zeros(N * 5 * 2, device="cuda")
    ctx = ff.FftContext.full_v2(N, kernel=2)
    req = ff.MetadataRequest * 1
    arr = req()
    arr[0].kind = META_KINDS["ButterflyPairs"]
    arr[0].buffer = ff.api._fp(dpairs)
    arr[0].count = N * 5
    assert ff.lib().fftfree_execute_c2c_meta(ctx.handle, ff.api._fp(dx), ff.api._fp(dout), B, arr, 1) == 1
    _, _, rb = OracleContext(N=N, kernel=2).fft_columns(x.view(np.complex64), {"ButterflyPairs": N * 5})
    assert np.array_equal(dpairs.cpu().numpy().view(np.complex64), rb["ButterflyPairs"])
