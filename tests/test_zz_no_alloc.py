"""mcfftExec1dNoAlloc: the two-pass 1D transform for callers that cannot
allocate device memory where the transform runs (a framework's allocator
owns the device memory, allocation is forbidden after start-up, or the
synchronisation an allocation may imply is not affordable).  It keeps its
intermediate and tables in fixed device arrays inside the library.

Checked through the C ABI against the plan-based entry point (mcfftExec) on
the same input, within the plain FP16 form's tolerance, on two calls in a
row: the fixed arrays keep the previous call's contents, which must not leak
into the next result.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import mcfft_b200 as mc  # noqa: E402
from oracle import oracle  # noqa: E402
from tests.gpu_util import compare, from_device, rand_complex, rounded, run, to_device  # noqa: E402

PLAIN_TOL = 1e-3


def _no_alloc(x, n, batch, direction):
    xd = to_device(x, True)
    out = torch.empty(n * batch, dtype=torch.complex32, device="cuda")
    out.view(torch.uint8).fill_(0xFF)  # NaN poison
    rc = mc.lib().mcfftExec1dNoAlloc(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     n, batch, direction,
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == mc.SUCCESS, mc.error_string(rc)
    torch.cuda.synchronize()
    return from_device(out)


# The last two fill the scratch array exactly: the largest n (its tables
# fill the fixed arrays) and the smallest n with the largest batch.
@pytest.mark.parametrize("n,batch", [(1 << 16, 4), (1 << 20, 2), (1 << 15, 8), (1 << 22, 1),
                                     (1 << 14, 256)])
def test_no_alloc_matches_plan_two_calls(n, batch):
    for call, direction in enumerate((mc.FORWARD, mc.INVERSE)):
        x = rand_complex((batch, n), seed=1000 + call)
        y = _no_alloc(x, n, batch, direction)
        with mc.Plan((n,), batch, mc.PREC_FP16) as p:
            y_plan, sl = run(p, x, True, direction=direction)
        rel, _ = compare(y, y_plan)
        assert rel < PLAIN_TOL, (call, rel)
        ref = oracle.fft1d(rounded(x, True), sign=direction) * 2.0 ** sl
        rel_o, _ = compare(y, ref)
        assert rel_o < PLAIN_TOL, (call, rel_o)


def test_no_alloc_rejects_sizes_beyond_limits():
    L = mc.lib()
    dummy = ctypes.c_void_p(16)
    # too small / not a power of two: unsupported; too many points: invalid
    assert L.mcfftExec1dNoAlloc(dummy, dummy, 1 << 12, 1, mc.FORWARD, None) == mc.UNSUPPORTED_SIZE
    assert L.mcfftExec1dNoAlloc(dummy, dummy, 3 << 14, 1, mc.FORWARD, None) == mc.UNSUPPORTED_SIZE
    assert L.mcfftExec1dNoAlloc(dummy, dummy, 1 << 20, 5, mc.FORWARD, None) == mc.INVALID_VALUE
    # a batch whose product with n overflows 64 bits is refused too
    assert L.mcfftExec1dNoAlloc(dummy, dummy, 1 << 22, 1 << 42, mc.FORWARD, None) == mc.INVALID_VALUE
    assert L.mcfftExec1dNoAlloc(dummy, dummy, 1 << 14, (1 << 63) - 1, mc.FORWARD,
                                None) == mc.INVALID_VALUE
    assert L.mcfftExec1dNoAlloc(None, dummy, 1 << 16, 1, mc.FORWARD, None) == mc.INVALID_VALUE
