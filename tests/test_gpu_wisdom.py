"""Autotuning on the GPU: a plan's tuner times its four-step split and its
tiled passes' tile shapes and records the choices; after export, forget and
import, a new plan of the same shape takes the recorded choices without
timing and computes bit-identical results.  Non-default four-step splits
(the tuner's other candidates) stay within the forms' tolerances and are
reported by mcfftPlanInfo."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from oracle import oracle  # noqa: E402
from tests.gpu_util import compare, rand_complex, rounded, run  # noqa: E402


def test_wisdom_skips_timing_and_keeps_results(tmp_path):
    n, batch = 1 << 20, 4
    x = rand_complex((batch, n), seed=31)
    mc.wisdom_forget()
    try:
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            info = p.info()
            # three four-step splits, then the chosen split's two passes
            assert info.timed_passes == 3 + info.num_passes, info.timed_passes
            assert info.fourstep_n1 in (512, 1024, 2048), info.fourstep_n1
            assert info.tile_points in (8192, 16384) and info.ctas > 0
            timed = info.timed_passes
            y1, _ = run(p, x, True)
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            assert p.info().timed_passes == 0  # records of this process
        path = str(tmp_path / "wisdom.txt")
        mc.wisdom_export(path)
        assert "fourstep n1048576" in open(path).read()
        mc.wisdom_forget()
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            assert p.info().timed_passes == timed  # forgotten: timed again
        mc.wisdom_forget()
        mc.wisdom_import(path)
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            assert p.info().timed_passes == 0
            y2, _ = run(p, x, True)
        assert np.array_equal(y1, y2)
    finally:
        mc.wisdom_forget()


@pytest.mark.parametrize("prec", [mc.PREC_FP16, mc.PREC_SPLIT])
@pytest.mark.parametrize("n1", [256, 512, 2048, 4096])
def test_non_default_fourstep_splits(prec, n1, monkeypatch):
    n, batch = 1 << 20, 2
    if prec == mc.PREC_SPLIT and n1 > 2048:
        pytest.skip("split tiles hold at most 2048 points per transform")
    monkeypatch.setenv("MCFFT_FOURSTEP_N1", str(n1))
    x = rand_complex((batch, n), seed=n1)
    f16 = prec == mc.PREC_FP16
    with mc.Plan((n,), batch, prec) as p:
        assert p.info().fourstep_n1 == n1
        y, sl = run(p, x, f16)
    ref = oracle.fft1d(rounded(x, f16)) * 2.0 ** sl
    rel, _ = compare(y, ref)
    assert rel < (1e-3 if f16 else 2e-6), rel


def test_three_pass_choice_from_wisdom(tmp_path):
    """From 2^21 points the tuner also times the three-pass plan; a record
    that names it (-1) makes a later plan take three passes without timing
    the decompositions, with results inside the plain form's tolerance."""
    n, batch = 1 << 22, 2
    x = rand_complex((batch, n), seed=41)
    mc.wisdom_forget()
    try:
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            info = p.info()
            # three four-step splits and the three-pass plan, then the
            # chosen plan's tiled passes
            assert info.timed_passes >= 4 + 2, info.timed_passes
        path = str(tmp_path / "wisdom.txt")
        mc.wisdom_export(path)
        lines = open(path).read().splitlines()
        fs = [ln for ln in lines if "\tfourstep n4194304 " in ln]
        assert len(fs) == 1, lines
        forced = [ln.rsplit("\t", 1)[0] + "\t-1" if ln in fs else ln for ln in lines]
        (tmp_path / "forced.txt").write_text("\n".join(forced) + "\n")
        mc.wisdom_forget()
        mc.wisdom_import(str(tmp_path / "forced.txt"))
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            info = p.info()
            assert info.num_passes == 2 + batch  # three passes, the last per transform
            assert info.fourstep_n1 == 1 << 7  # n = 2^7 * 2^7 * 2^8
            y, sl = run(p, x, True)
        ref = oracle.fft1d(rounded(x, True)) * 2.0 ** sl
        rel, _ = compare(y, ref)
        assert rel < 1e-3, rel
    finally:
        mc.wisdom_forget()


@pytest.mark.parametrize("n,n1,batch", [(1 << 22, 1024, 2), (1 << 23, 2048, 1)])
def test_split_four_step_with_4096_point_rows(n, n1, batch, monkeypatch):
    """Split form, four-step pairs whose second pass has 4096-point rows
    (two columns per 8K-point tile, FP32 column output): both passes on the
    tile kernels, within the split form's tolerance."""
    monkeypatch.setenv("MCFFT_FOURSTEP_N1", str(n1))
    x = rand_complex((batch, n), seed=n1 + batch)
    with mc.Plan((n,), batch, mc.PREC_SPLIT) as p:
        info = p.info()
        assert info.num_passes == 2 and info.fourstep_n1 == n1
        assert info.tile_points == 8192
        y, _ = run(p, x, False)
    ref = oracle.fft1d(rounded(x, False))
    rel, _ = compare(y, ref)
    assert rel < 2e-6, rel
