"""The plan builder's size limits, at the limits.

The largest transforms a plan accepts run against the FP64 oracle in both
forms: 1D 2^25 and 2^26 (three passes of 256-512 points unless the plan-time
tuner measures a four-step pair with a direct-load 8192-point pass faster),
1D 2^27 (three passes of 512 points: the reference's largest 1D size), 2D
8192 x 8192, and a 3D side of 8192 on each axis in turn.  The first sizes
past the limits, and sizes that are not powers of two or are below 16, are
refused with MCFFT_UNSUPPORTED_SIZE (an error, never a fallback).

Both forms read the same FP16-rounded input (the split form with
MCFFT_FLAG_INPUT_F16), so one oracle transform per shape checks both.
Tolerances as in test_gpu_parity: plain rel-L2 <= 1e-3, split <= 2e-6.
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

BIG = [(1 << 25,), (1 << 26,), (1 << 27,), (8192, 8192)]
SIDES_3D = [(8192, 16, 16), (16, 8192, 16), (16, 16, 8192)]

_refs = {}


def _case(shape):
    """(input, oracle transform of its FP16 rounding), computed once per shape."""
    if shape not in _refs:
        _refs.clear()  # keep one 2^26-point case in host memory at a time
        x = rand_complex((1,) + shape, seed=int(np.prod(shape)) % 1000 + len(shape))
        _refs[shape] = (x, oracle.fftnd(rounded(x, True), shape))
    return _refs[shape]


@pytest.mark.parametrize("shape", BIG + SIDES_3D)
@pytest.mark.parametrize("prec", [mc.PREC_FP16, mc.PREC_SPLIT])
def test_largest_accepted_sizes(shape, prec):
    x, ref = _case(shape)
    flags = mc.FLAG_INPUT_F16 if prec == mc.PREC_SPLIT else mc.FLAG_NONE
    with mc.Plan(shape, 1, prec, flags) as p:
        y, sl = run(p, x, True)
    if prec == mc.PREC_FP16:
        assert sl == -int(np.log2(np.prod(shape)))
        rel, mx = compare(y, ref * 2.0 ** sl)
        assert rel < PLAIN_TOL, (rel, mx)
    else:
        rel, mx = compare(y, ref)
        assert rel < SPLIT_TOL, (rel, mx)


@pytest.mark.parametrize("shape", [(1 << 28,), (16384, 16), (16, 16384), (16384, 16, 16),
                                   (16, 16, 16384), (8,), (16, 8), (3000,), (1 << 20 | 16,),
                                   (48, 64)])
@pytest.mark.parametrize("prec", [mc.PREC_FP16, mc.PREC_SPLIT])
def test_sizes_past_the_limits_refused(shape, prec):
    with pytest.raises(mc.McfftError) as ei:
        mc.Plan(shape, 1, prec)
    assert ei.value.code == mc.UNSUPPORTED_SIZE


@pytest.mark.parametrize("n,batch", [(1 << 16, 3), (1 << 18, 5), (1 << 21, 2)])
@pytest.mark.parametrize("prec", [mc.PREC_FP16, mc.PREC_SPLIT])
def test_three_pass_plan_at_smaller_sizes(n, batch, prec, monkeypatch):
    """The three-pass 1D plan (taken for 2^27) forced at sizes with several
    transforms: its last pass runs once per transform."""
    monkeypatch.setenv("MCFFT_THREE_PASS", "1")
    x = rand_complex((batch, n), seed=n % 997 + batch)
    f16 = prec == mc.PREC_FP16
    with mc.Plan((n,), batch, prec) as p:
        assert p.info().num_passes == 2 + batch
        y, sl = run(p, x, f16)
    ref = oracle.fft1d(rounded(x, f16)) * 2.0 ** sl
    rel, mx = compare(y, ref)
    assert rel < (PLAIN_TOL if f16 else SPLIT_TOL), (rel, mx)
