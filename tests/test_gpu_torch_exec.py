"""Plan.exec on torch CUDA tensors: the transform matches the FP64 oracle
(plain form, rel-L2 <= 1e-3), and tensors smaller than the plan's input or
output extents, or of the wrong element type, are refused before any
launch."""
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from oracle import oracle  # noqa: E402
from tests.gpu_util import compare, from_device, rand_complex, rounded, to_device  # noqa: E402


def test_torch_exec_matches_oracle_and_checks_sizes():
    n, batch = 1024, 4
    x = rand_complex((batch, n), seed=3)
    xd = to_device(x, True)
    with mc.Plan((n,), batch, mc.PREC_FP16) as p:
        y = p.exec(xd)
        torch.cuda.synchronize()
        p.check_status()
        ref = oracle.fft1d(rounded(x, True)) * 2.0 ** p.info().scale_log2
        rel, _ = compare(from_device(y), ref)
        assert rel < 1e-3, rel
        with pytest.raises(ValueError, match="bytes"):
            p.exec(xd[: n * batch // 2])
        with pytest.raises(ValueError, match="bytes"):
            p.exec(xd, out=torch.empty(16, dtype=torch.complex32, device="cuda"))
        # an FP32 tensor has enough bytes for this FP16 plan but the wrong type
        with pytest.raises(ValueError, match="needs"):
            p.exec(torch.zeros(n * batch, dtype=torch.complex64, device="cuda"))
        with pytest.raises(ValueError, match="needs"):
            p.exec(xd, out=torch.empty(n * batch, dtype=torch.complex64, device="cuda"))
    with mc.Plan((n,), batch, mc.PREC_SPLIT) as p:
        # the split form reads FP32 unless FLAG_INPUT_F16 and always writes FP32
        with pytest.raises(ValueError, match="needs"):
            p.exec(xd)
        xf = to_device(x, False)
        y = p.exec(xf)
        torch.cuda.synchronize()
        assert y.dtype == torch.complex64
        ref = oracle.fft1d(rounded(x, False))
        rel, _ = compare(from_device(y), ref)
        assert rel < 2e-6, rel
