"""Failure detection on the device.

Every wait in the kernels is bounded by one second of the GPU's global
timer; on expiry the kernel records a timeout in the plan's status word,
drains its own copies, frees its tensor memory and returns, and
mcfftPlanCheckStatus reports MCFFT_DEVICE_TIMEOUT.

The failure is made on the host: a plan built with MCFFT_INJECT_STALL
forges, in the batch kernel's pass table, a producer count that no
dependent tile ever sees reached (a dependency that never arrives).  The
exec must end by itself, report the timeout once (the status word is
cleared by the check), and leave the context usable: a plan built
afterwards on the same device transforms correctly.  Nothing traps,
faults or spins without a limit.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from oracle import oracle  # noqa: E402
from tests.gpu_util import compare, from_device, rand_complex, rounded, to_device  # noqa: E402

# single-pass lengths (no dependency) beside four-step and 2D transforms
# (second pass waits on the first)
SHAPES = [((256,), 3), ((4096,), 2), ((1 << 16,), 1), ((128, 256), 1)]
TOL = {mc.PREC_FP16: 1e-3, mc.PREC_SPLIT: 2e-6}


def _descs():
    descs, off = [], 0
    for shape, count in SHAPES:
        n = int(np.prod(shape))
        for _ in range(count):
            descs.append((shape, 1, off, off))
            off += n
    return descs, off


def _exec(p, xd, out):
    p.exec_ptr(xd.data_ptr(), out.data_ptr(), mc.FORWARD, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()


@pytest.mark.parametrize("precision", [mc.PREC_FP16, mc.PREC_SPLIT])
def test_unmet_dependency_times_out_and_context_survives(precision, monkeypatch):
    descs, total = _descs()
    flags = mc.FLAG_INPUT_F16 if precision == mc.PREC_SPLIT else mc.FLAG_NONE
    x = rand_complex((total,), seed=5)
    xd = to_device(x, True)
    odt = torch.complex64 if precision == mc.PREC_SPLIT else torch.complex32
    out = torch.empty(total, dtype=odt, device="cuda")

    monkeypatch.setenv("MCFFT_INJECT_STALL", "1")
    with mc.Plan(descs=descs, precision=precision, flags=flags) as p:
        assert p.info().launches == 1  # the batch kernel carries the dependencies
        t0 = time.monotonic()
        _exec(p, xd, out)
        waited = time.monotonic() - t0
        with pytest.raises(mc.McfftError) as ei:
            p.check_status()
        assert ei.value.code == mc.DEVICE_TIMEOUT
        p.check_status()  # reported once; the status word is cleared
    # one second of limit per wait, a few chained waits at most
    assert 0.5 < waited < 20.0, waited
    monkeypatch.delenv("MCFFT_INJECT_STALL")

    # the context is intact: the same batch, planned again, is correct
    out.view(torch.uint8).fill_(0xFF)
    with mc.Plan(descs=descs, precision=precision, flags=flags) as p:
        _exec(p, xd, out)
        p.check_status()
    y = from_device(out)
    xr = rounded(x, True)
    worst = 0.0
    for shape, batch, io, oo in descs:
        n = int(np.prod(shape))
        ref = oracle.fftnd(xr[io:io + n].reshape((1,) + tuple(shape)), shape)
        if precision == mc.PREC_FP16:
            ref = ref * 2.0 ** -int(np.log2(n))
        rel, _ = compare(y[oo:oo + n], ref)
        worst = max(worst, rel)
    assert worst < TOL[precision], worst
