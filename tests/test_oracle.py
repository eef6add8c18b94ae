"""CPU tests of the oracle: the FP64 FFT against the reference's own golden
vectors (FFTW and rocFFT outputs printed in its dumps), the restated
reference algorithm against the FP64 FFT, the digit-reversal known-answer
test, and the error metric.  No GPU needed."""
import os

import numpy as np
import pytest

from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(name):
    return np.load(os.path.join(GOLDEN, name))


def test_fft_matches_numpy():
    rng = np.random.default_rng(0)
    for n in [16, 32, 256, 4096, 1 << 16]:
        x = rng.standard_normal((3, n)) + 1j * rng.standard_normal((3, n))
        y = oracle.fft1d(x)
        r = np.fft.fft(x)
        assert np.linalg.norm(y - r) / np.linalg.norm(r) < 1e-14


def test_fft_matches_direct_dft():
    rng = np.random.default_rng(1)
    for n in [16, 64, 128]:
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.allclose(oracle.fft1d(x[None])[0], oracle.dft_direct(x), rtol=0, atol=1e-12)


def test_fftnd_matches_numpy():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((2, 32, 64)) + 1j * rng.standard_normal((2, 32, 64))
    assert np.allclose(oracle.fftnd(x, [32, 64]), np.fft.fft2(x), atol=1e-10)
    x3 = rng.standard_normal((1, 16, 8, 32)) + 0j
    assert np.allclose(oracle.fftnd(x3, [16, 8, 32]), np.fft.fftn(x3, axes=(1, 2, 3)), atol=1e-10)


def test_inverse_roundtrip():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2, 1024)) + 1j * rng.standard_normal((2, 1024))
    z = oracle.fft1d(oracle.fft1d(x), sign=+1) / 1024
    assert np.allclose(z, x, atol=1e-13)


def test_generate_data_matches_reference_generator():
    """generate_data: srand(42), 1e-4f * rand() / RAND_MAX in float."""
    d = oracle.generate_data(4, 2, 42)
    assert d.shape == (2, 4)
    assert np.all(d.real >= 0) and np.all(d.real <= 1e-4)
    # the same draw twice
    assert np.array_equal(d, oracle.generate_data(4, 2, 42))


def test_golden_fftw_1d_262144():
    """2.txt's standard column: FFTW double of the seed-42 input, N=2^18."""
    std = _golden("fftw_1d_n262144_seed42_head.npy")
    x = oracle.generate_data(1 << 18, 1, 42)
    y = oracle.fft1d(x).reshape(-1).view(np.float64)[: std.size]
    # values are printed with 7 significant digits
    assert np.max(np.abs(y - std) / (np.abs(std) + 1e-9)) < 1e-6


def test_golden_rocfft_1d_256_b256():
    """3.txt: rocFFT (and the reference run of that revision) for N=256,
    batch 256, seed 42, first 128 transforms.  That run computed in single
    precision (absolute errors ~1e-10 on values of ~1e-4), so the check is
    relative to the largest output."""
    std = _golden("rocfft_1d_n256_b256_seed42_head.npy")
    tested = _golden("reference_tested_1d_n256_b256_seed42_head.npy")
    x = oracle.generate_data(256, 256, 42)
    y = oracle.fft1d(x).reshape(-1).view(np.float64)[: std.size]
    scale = np.max(np.abs(std))
    assert np.max(np.abs(y - std)) / scale < 2e-6
    assert np.max(np.abs(y - tested)) / scale < 2e-6
    assert np.median(np.abs(y - std) / (np.abs(std) + 1e-12)) < 1e-6


def test_golden_gen_rev_512():
    """1.log: the digit reversal the reference prints for N=512, radices
    {16, 16, 2} (its plan for 512, source/mcfft_1d_device.cpp:702-707)."""
    perm = _golden("gen_rev_512_16_16_2.npy")
    rad, _ = oracle.ref_plan_1d(512)
    assert rad == [16, 16, 2]
    assert np.array_equal(oracle.gen_rev(512, rad), perm)


def test_reference_plan_table():
    assert oracle.ref_plan_1d(4096) is None      # not in the reference's table
    assert oracle.ref_plan_1d(1 << 20) is None
    assert oracle.ref_plan_1d(256) == ([16, 16], [0])
    assert oracle.ref_plan_1d(1 << 17) == ([16, 16, 2, 16, 16], [1, 0])


@pytest.mark.parametrize("n", [256, 512, 1024, 1 << 17])
def test_restated_reference_1d(n):
    """The reference's own algorithm (digit-reversed input, DFT-16 matrix
    stages with float twiddles) computes the DFT to float-twiddle accuracy."""
    x = oracle.generate_data(n, 2, 7)
    y = oracle.ref_transform_1d(x)
    r = oracle.fft1d(x)
    rel, _ = oracle.error_norms(y, r)
    assert rel < 5e-6


@pytest.mark.parametrize("nx,ny", [(256, 256), (512, 256), (256, 512)])
def test_restated_reference_2d(nx, ny):
    x = oracle.generate_data(nx * ny, 1, 3).reshape(1, nx, ny)
    y = oracle.ref_transform_2d(x)
    r = oracle.fftnd(x, [nx, ny])
    rel, _ = oracle.error_norms(y, r)
    assert rel < 5e-6


def test_reference_2d_1024_unsupported():
    """Nx=1024 selects the never-assigned layer_1[2]
    (source/mcfft_2d_device.cpp:635-639, :652-656, :621)."""
    x = np.zeros((1, 1024, 256), complex)
    with pytest.raises(ValueError):
        oracle.ref_transform_2d(x)


def test_get_error_metric():
    a = np.array([[1 + 1j, 2 + 2j]])
    assert oracle.get_error(a, a) == 0.0
    b = np.array([[1.1 + 1j, 2 + 2j]])
    assert abs(oracle.get_error(b, a) - 0.1 / 2) < 1e-12
    c = np.array([[100 + 1j, 2 + 2j]])
    assert abs(oracle.get_error(c, a) - 1.0 / 2) < 1e-12   # min(1, |rel|)


def test_error_norms():
    ref = np.array([3 + 4j, 0j])
    rel, mx = oracle.error_norms(ref * (1 + 1e-3), ref)
    assert abs(rel - 1e-3) < 1e-12
    assert abs(mx - 1e-3) < 1e-12   # max|diff| = 4e-3 over max|ref| = 4
