"""Autotuning records on the GPU: a plan's tuner times its tiled passes and
records the choices; after export, forget and import, a new plan of the same
shape takes the recorded shapes without timing and computes bit-identical
results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from tests.gpu_util import rand_complex, run  # noqa: E402


def test_wisdom_skips_timing_and_keeps_results(tmp_path):
    n, batch = 1 << 20, 4
    x = rand_complex((batch, n), seed=31)
    mc.wisdom_forget()
    try:
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            info = p.info()
            assert info.timed_passes == info.num_passes == 2
            y1, _ = run(p, x, True)
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            assert p.info().timed_passes == 0  # records of this process
        path = str(tmp_path / "wisdom.txt")
        mc.wisdom_export(path)
        mc.wisdom_forget()
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            assert p.info().timed_passes == 2  # forgotten: timed again
        mc.wisdom_forget()
        mc.wisdom_import(path)
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            assert p.info().timed_passes == 0
            y2, _ = run(p, x, True)
        assert np.array_equal(y1, y2)
    finally:
        mc.wisdom_forget()
