"""2-D transforms (fftfree_execute_2d) against the oracle's fft_inplace_2d
restatement, and bit-identical to the same two axes run as contiguous
batched transforms with an explicit transpose."""
import numpy as np
import pytest
import torch

from oracle.oracle import fft_2d
from tests.helpers import assert_close, ctx_kwargs, oracle_for, tol_for

pytestmark = pytest.mark.gpu

api = pytest.importorskip("fftfree_b200.api")


def _mats(batch, rows, cols, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((batch, cols, rows)) + 1j * rng.standard_normal((batch, cols, rows))).astype(
        np.complex64)


def _pair(rows, cols, kw0=None, kw1=None):
    k0 = ctx_kwargs(rows, **(kw0 or {}))
    k1 = ctx_kwargs(cols, **(kw1 or {}))
    return api.FftContext.full_v2(**k0), api.FftContext.full_v2(**k1), oracle_for(k0), oracle_for(k1)


@pytest.mark.parametrize("rows,cols,batch", [(2, 2, 1), (16, 64, 3), (64, 16, 2), (256, 256, 2), (1024, 512, 1),
                                             (4096, 64, 1), (8, 8192, 2), (32, 2048, 1), (2, 4096, 5),
                                             (64, 16384, 1), (4, 65536, 1), (16384, 8, 1)])
@pytest.mark.parametrize("inverse", [0, 1])
def test_2d_matches_oracle(rows, cols, batch, inverse):
    c0, c1, o0, o1 = _pair(rows, cols, dict(inverse=inverse), dict(inverse=inverse))
    X = _mats(batch, rows, cols, rows + 3 * cols + inverse)
    out = np.zeros_like(X)
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), rows, cols, batch) == 1
    ok, ref = fft_2d(o0, o1, X)
    assert ok
    assert_close(out, ref, tol_for(rows * cols), "2-D")


@pytest.mark.parametrize("rows,cols", [(64, 128), (512, 1024), (16, 8192), (2048, 4)])
def test_2d_bit_identical_to_two_batched_passes(rows, cols):
    c0, c1, _, _ = _pair(rows, cols, dict(kernel=2), dict(kernel=2))
    batch = 2
    X = _mats(batch, rows, cols, 5)
    out = np.zeros_like(X)
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), rows, cols, batch) == 1
    y = np.zeros_like(X)
    assert c0.execute_c2c(X.view(np.float32), y.view(np.float32), batch * cols) == 1
    yt = np.ascontiguousarray(y.transpose(0, 2, 1))  # (batch, rows, cols): rows contiguous
    z = np.zeros_like(yt)
    assert c1.execute_c2c(yt.view(np.float32), z.view(np.float32), batch * rows) == 1
    want = np.ascontiguousarray(z.transpose(0, 2, 1))
    assert np.array_equal(out.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("kw0,kw1", [
    (dict(kernel=0, transform=1), dict(kernel=0, store_polar=1)),
    (dict(kernel=2, inverse=1, reduce_magnitude=1), dict(kernel=0, transform=2, half_spectrum=1, inverse=1)),
    (dict(kernel=0, transform=2, half_spectrum=1, inverse=1), dict(kernel=2)),
    (dict(kernel=2, store_polar=1), dict(kernel=0, transform=1)),
])
def test_2d_plan_hooks_match_oracle(kw0, kw1):
    rows, cols, batch = 128, 256, 2
    c0, c1, o0, o1 = _pair(rows, cols, kw0, kw1)
    # (A polar output of the first axis feeds its phases to the second one,
    # so only cases whose first-axis phases are well conditioned are used:
    # the phase of a real C2R output flips between -pi and pi with the sign of
    # a rounding-level imaginary part.)
    X = _mats(batch, rows, cols, 9)
    out = np.zeros_like(X)
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), rows, cols, batch) == 1
    ok, ref = fft_2d(o0, o1, X)
    assert ok
    if kw1.get("store_polar"):
        assert_close(out.real, ref.real, tol_for(rows * cols), "2-D polar magnitude")
        got = out.real * np.exp(1j * out.imag.astype(np.float64))
        want = ref.real * np.exp(1j * ref.imag.astype(np.float64))
        assert_close(got, want, tol_for(rows * cols), "2-D polar value")
    else:
        assert_close(out, ref, tol_for(rows * cols), "2-D")


@pytest.mark.parametrize("rows,cols", [(256, 512), (32, 16384)])
def test_2d_in_place_on_device(rows, cols):
    c0, c1, o0, o1 = _pair(rows, cols)
    X = _mats(3, rows, cols, 11)
    d = torch.from_numpy(X.view(np.float32).copy()).cuda()
    assert api.execute_2d(c0, c1, d, d, rows, cols, 3) == 1
    torch.cuda.synchronize()
    got = d.cpu().numpy().view(np.complex64).reshape(X.shape)
    ok, ref = fft_2d(o0, o1, X)
    assert_close(got, ref, tol_for(rows * cols), "2-D in place")


def test_2d_argument_checks():
    c0, c1, _, _ = _pair(16, 32)
    X = _mats(1, 16, 32, 0)
    out = np.zeros_like(X)
    L = api.lib()
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), 32, 16, 1) == 0
    assert api.execute_2d(c0, c1, X.view(np.float32), out.view(np.float32), 16, 32, 0) == 0
    assert L.fftfree_execute_2d(None, c1.handle, api._fp(X.view(np.float32)), api._fp(out.view(np.float32)), 16,
                                32, 1) == 0


def test_2d_row_pass_wait_that_gives_up_is_reported():
    """The TMA row pass bounds its wait for the input boxes; a block whose wait
    runs out leaves its lines unwritten and the call reports failure.  A
    test-only limit of 0 polls (FFTFREE_TEST_TMA_WAIT_LIMIT, read once per
    process, so this runs in a fresh interpreter) makes every block give up
    at once; the copies still land (the drain wait keeps its full limit).  A
    synchronous call returns 0; an asynchronous one makes the next call
    return 0; with the limit unset the same calls succeed."""
    import os
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, torch; sys.path.insert(0, %r)\n"
        "import fftfree_b200 as ff\n"
        "rows, cols, B = 256, 512, 2\n"
        "c0 = ff.FftContext.full_v2(rows); c1 = ff.FftContext.full_v2(cols)\n"
        "x = torch.randn(B * rows * cols * 2, device='cuda'); y = torch.empty_like(x)\n"
        "r_sync = ff.execute_2d(c0, c1, x, y, rows, cols, B)\n"
        "c0.set_async(True)\n"
        "r_a1 = ff.execute_2d(c0, c1, x, y, rows, cols, B); torch.cuda.synchronize()\n"
        "r_a2 = ff.execute_2d(c0, c1, x, y, rows, cols, B); torch.cuda.synchronize()\n"
        "print('RESULTS', r_sync, r_a1, r_a2)\n" % repo)
    outs = {}
    for limit in ("0", None):
        env = dict(os.environ)
        env.pop("FFTFREE_TEST_TMA_WAIT_LIMIT", None)
        if limit is not None:
            env["FFTFREE_TEST_TMA_WAIT_LIMIT"] = limit
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
        assert r.returncode == 0, r.stderr
        outs[limit] = r.stdout.split("RESULTS", 1)[1].split()
    assert outs["0"] == ["0", "1", "0"]
    assert outs[None] == ["1", "1", "1"]
