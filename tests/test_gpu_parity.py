"""GPU parity: the CUDA path through the C ABI against the FP64 oracle on
identical storage-rounded inputs.

Tolerances (rel-L2 = ||y - y_ref|| / ||y_ref||):
  plain FP16 form   <= 1e-3
  split hi+lo form  <= 2e-6
Outputs are NaN-poisoned before every run, so an element a kernel fails to
write shows up as an error.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from oracle import oracle  # noqa: E402
from tests.gpu_util import compare, rand_complex, rounded, run  # noqa: E402

PLAIN_TOL = 1e-3
SPLIT_TOL = 2e-6

SIZES_1D = [(16, 256), (32, 128), (64, 256), (128, 128), (256, 64), (512, 32), (1024, 16),
            (2048, 8), (4096, 256), (8192, 4), (8192, 33), (16384, 2), (32768, 2), (65536, 1),
            (1 << 20, 2), (1 << 22, 1)]


@pytest.mark.parametrize("n,batch", SIZES_1D)
def test_plain_1d(n, batch):
    x = rand_complex((batch, n), seed=n)
    with mc.Plan((n,), batch, mc.PREC_FP16) as p:
        y, sl = run(p, x, True)
    ref = oracle.fft1d(rounded(x, True)) * 2.0 ** sl
    rel, mx = compare(y, ref)
    assert rel < PLAIN_TOL, (rel, mx)


@pytest.mark.parametrize("n,batch", SIZES_1D)
def test_split_1d(n, batch):
    x = rand_complex((batch, n), seed=n + 1)
    with mc.Plan((n,), batch, mc.PREC_SPLIT) as p:
        y, sl = run(p, x, False)
    assert sl == 0
    ref = oracle.fft1d(rounded(x, False))
    rel, mx = compare(y, ref)
    assert rel < SPLIT_TOL, (rel, mx)


@pytest.mark.parametrize("n,batch", [(256, 8), (4096, 4), (1 << 16, 1)])
def test_split_1d_f16_input(n, batch):
    x = rand_complex((batch, n), seed=7)
    with mc.Plan((n,), batch, mc.PREC_SPLIT, mc.FLAG_INPUT_F16) as p:
        y, _ = run(p, x, True)
    ref = oracle.fft1d(rounded(x, True))
    rel, _ = compare(y, ref)
    assert rel < SPLIT_TOL, rel


@pytest.mark.parametrize("prec", [mc.PREC_FP16, mc.PREC_SPLIT])
@pytest.mark.parametrize("nx,ny,batch", [(16, 16, 4), (128, 256, 2), (256, 128, 2), (512, 512, 1),
                                         (1024, 1024, 1), (64, 2048, 1), (2048, 256, 1),
                                         (32, 4096, 2), (16, 1024, 3)])
def test_2d(prec, nx, ny, batch):
    f16 = prec == mc.PREC_FP16
    x = rand_complex((batch, nx, ny), seed=nx + ny)
    with mc.Plan((nx, ny), batch, prec) as p:
        y, sl = run(p, x, f16)
    ref = oracle.fftnd(rounded(x, f16), [nx, ny]) * 2.0 ** sl
    rel, _ = compare(y, ref)
    assert rel < (PLAIN_TOL if f16 else SPLIT_TOL), rel


def test_2d_wide_range_split():
    x = rand_complex((2, 256, 256), seed=2, dist="wide")
    with mc.Plan((256, 256), 2, mc.PREC_SPLIT) as p:
        y, _ = run(p, x, False)
    ref = oracle.fftnd(rounded(x, False), [256, 256])
    rel, _ = compare(y, ref)
    assert rel < SPLIT_TOL, rel


@pytest.mark.parametrize("prec", [mc.PREC_FP16, mc.PREC_SPLIT])
@pytest.mark.parametrize("dims", [(16, 16, 16), (32, 64, 128), (64, 64, 64), (256, 256, 32),
                                  (64, 16, 128)])
def test_3d(prec, dims):
    f16 = prec == mc.PREC_FP16
    x = rand_complex((1,) + dims, seed=3)
    with mc.Plan(dims, 1, prec) as p:
        y, sl = run(p, x, f16)
    ref = oracle.fftnd(rounded(x, f16), list(dims)) * 2.0 ** sl
    rel, _ = compare(y, ref)
    assert rel < (PLAIN_TOL if f16 else SPLIT_TOL), rel


@pytest.mark.parametrize("shape", [(4096,), (1 << 18,), (128, 512), (32, 32, 32)])
def test_split_inverse_roundtrip(shape):
    x = rand_complex((1,) + shape, seed=11)
    with mc.Plan(shape, 1, mc.PREC_SPLIT) as p:
        y, _ = run(p, x, False)
        # inverse of the forward output
        z, _ = run(p, y.reshape((1,) + shape), False, direction=mc.INVERSE)
    ntot = int(np.prod(shape))
    ref_inv = oracle.fftnd(rounded(y, False).reshape((1,) + shape), list(shape), sign=+1)
    rel_inv, _ = compare(z, ref_inv)
    assert rel_inv < SPLIT_TOL, rel_inv
    rel_rt, _ = compare(z / ntot, rounded(x, False))
    assert rel_rt < 4 * SPLIT_TOL, rel_rt


@pytest.mark.parametrize("shape,batch", [((1024,), 8), ((8192,), 6), ((1 << 24,), 1),
                                         ((16, 512), 4), ((256, 8192), 1)])
def test_plain_inverse(shape, batch):
    """Inverse transforms, plain form: one pass, the 8192-point pass with its
    computed radix-2 twiddles, three passes (2^24), a 16-point column pass,
    rows of 8192."""
    x = rand_complex((batch,) + shape, seed=5)
    with mc.Plan(shape, batch, mc.PREC_FP16) as p:
        y, sl = run(p, x, True, direction=mc.INVERSE)
    ref = oracle.fftnd(rounded(x, True), list(shape), sign=+1) * 2.0 ** sl
    rel, _ = compare(y, ref)
    assert rel < PLAIN_TOL, rel


def test_properties_delta_and_tone():
    """Delta -> constant; a single tone -> a delta at its bin (split form)."""
    n = 4096
    x = np.zeros((2, n), complex)
    x[0, 0] = 1.0
    k0 = 123
    x[1] = np.exp(2j * np.pi * k0 * np.arange(n) / n)
    with mc.Plan((n,), 2, mc.PREC_SPLIT) as p:
        y, _ = run(p, x, False)
    y = y.reshape(2, n)
    assert np.max(np.abs(y[0] - 1.0)) < 1e-6
    expect = np.zeros(n)
    expect[k0] = n
    assert np.max(np.abs(y[1] - expect)) < 1e-6 * n


def test_partial_tile_batch():
    """Batch not a multiple of the tile's column count (masked columns)."""
    n, batch = 256, 67
    x = rand_complex((batch, n), seed=67)
    with mc.Plan((n,), batch, mc.PREC_FP16) as p:
        y, sl = run(p, x, True)
    ref = oracle.fft1d(rounded(x, True)) * 2.0 ** sl
    rel, _ = compare(y, ref)
    assert rel < PLAIN_TOL, rel


@pytest.mark.parametrize("shape,batch", [((32,), 512), ((64,), 256), ((128,), 128), ((256,), 67),
                                         ((512,), 32), ((1024,), 16), ((2048,), 8), ((2048,), 5),
                                         ((4096,), 8), ((4096,), 3), ((1 << 20,), 1),
                                         ((512, 512), 1), ((64, 64, 64), 1)])
def test_plain_8k_tiles(shape, batch, monkeypatch):
    """The 8K-point tile variants, which the plan-time tuner takes where they
    are faster, forced for every pass (first choice 8K, tuning off).  Every
    pass here has an 8K layout; L = 4096 row passes take two columns per
    tile (batch 3: the last column block half empty)."""
    monkeypatch.setenv("MCFFT_TILE_POINTS", "8192")
    monkeypatch.setenv("MCFFT_AUTOTUNE", "0")
    x = rand_complex((batch,) + shape, seed=len(shape) * 1000 + batch)
    with mc.Plan(shape, batch, mc.PREC_FP16) as p:
        y, sl = run(p, x, True)
    ref = oracle.fftnd(rounded(x, True), shape) * 2.0 ** sl
    rel, mx = compare(y, ref)
    assert rel < PLAIN_TOL, (rel, mx)


@pytest.mark.parametrize("prec", [mc.PREC_FP16, mc.PREC_SPLIT])
def test_fourstep_twiddle_tables_switch(prec, monkeypatch):
    """The four-step twiddles from FP64-generated tables instead of the
    sine / cosine of the exact angle (MCFFT_FOURSTEP_TABLES=1): same bounds."""
    monkeypatch.setenv("MCFFT_FOURSTEP_TABLES", "1")
    n, batch = 1 << 20, 2
    x = rand_complex((batch, n), seed=77)
    f16 = prec == mc.PREC_FP16
    with mc.Plan((n,), batch, prec) as p:
        y, sl = run(p, x, f16)
    ref = oracle.fft1d(rounded(x, f16)) * 2.0 ** sl
    rel, _ = compare(y, ref)
    assert rel < (PLAIN_TOL if f16 else SPLIT_TOL), rel
