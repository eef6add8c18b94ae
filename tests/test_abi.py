"""CPU tests of the C ABI boundary: the library loads, exports every symbol
include/mcfft.h declares, reports errors without a device and refuses bad
arguments before touching one; the Python binding checks its tensors
before a launch.  No GPU compute."""
import ctypes
import os
import re

import pytest

import mcfft_b200 as mc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"MCFFT_API\s+[\w\s\*]+?\b(mcfft\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = mc.lib()
    names = _declared("mcfft.h")
    assert len(names) >= 10
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(mc.EXPORTS)


def test_version_and_error_strings():
    assert mc.version() >= 100
    assert mc.error_string(mc.SUCCESS) == "success"
    assert "unsupported" in mc.error_string(mc.UNSUPPORTED_SIZE)
    assert mc.error_string(9999) == "unknown error"


def test_invalid_arguments_rejected():
    L = mc.lib()
    h = ctypes.c_void_p()
    # null plan pointer / bad precision / bad counts fail before touching a device
    assert L.mcfftPlanCreateBatch(None, None, 0, 0, 0) == mc.INVALID_VALUE
    assert L.mcfftPlanCreate1d(ctypes.byref(h), 256, 1, 7, 0) != mc.SUCCESS
    assert L.mcfftExec(None, None, None, mc.FORWARD, None) == mc.INVALID_PLAN
    assert L.mcfftPlanDestroy(None) == mc.INVALID_PLAN
    assert L.mcfftPlanGetInfo(None, None) == mc.INVALID_PLAN
    # empty batches, impossible dimensionality and negative offsets too
    assert L.mcfftPlanCreate1d(ctypes.byref(h), 256, 0, mc.PREC_FP16, 0) == mc.INVALID_VALUE
    assert L.mcfftPlanCreate2d(ctypes.byref(h), 64, 64, -1, mc.PREC_SPLIT, 0) == mc.INVALID_VALUE
    for ndim, batch, ioff, ooff in ((0, 1, 0, 0), (4, 1, 0, 0), (1, 1, -16, 0), (1, 1, 0, -16)):
        d = mc.Desc(ndim, (ctypes.c_int64 * 3)(256, 1, 1), batch, ioff, ooff)
        assert L.mcfftPlanCreateBatch(ctypes.byref(h), ctypes.byref(d), 1, mc.PREC_FP16, 0) \
            == mc.INVALID_VALUE, (ndim, batch, ioff, ooff)
    assert not h.value  # nothing was created


def test_no_device_is_an_error_not_a_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(mc.McfftError) as ei:
        mc.Plan((256,), 4)
    assert ei.value.code == mc.NO_DEVICE


def test_header_declares_compat_entry_points():
    """The reference's harness signatures (include/mcfft_1d_utils.h:8-11)."""
    for h in ("mcfft_1d_utils.h", "mcfft_2d_utils.h", "mcfft_3d_utils.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        for fn in ("setup", "doit", "finalize", "generate_data"):
            assert re.search(r"\b%s\s*\(" % fn, src), (h, fn)


def test_torch_exec_refuses_unusable_tensors():
    """Plan.exec checks its tensors before any launch: a host tensor is
    refused (the plan shell here has no device plan; info() is stubbed)."""
    torch = pytest.importorskip("torch")
    p = mc.Plan.__new__(mc.Plan)
    p._h = ctypes.c_void_p()
    p.precision = mc.PREC_FP16
    p.flags = mc.FLAG_NONE
    p.device_index = None
    inf = mc.PlanInfo()
    inf.elements, inf.in_bytes, inf.out_bytes = 16, 64, 64
    p.info = lambda: inf
    with pytest.raises(ValueError, match="contiguous CUDA tensor"):
        p.exec(torch.zeros(32, dtype=torch.float16))
    with pytest.raises(ValueError, match="contiguous CUDA tensor"):
        p.exec(torch.zeros(64, dtype=torch.float16)[::2])


def test_error_norms_refuses_bad_segments():
    """mcfftErrorNorms checks its segment table before touching a device."""
    L = mc.lib()
    one = ctypes.c_void_p(256)
    out = (ctypes.c_double * 10)()
    offs = (ctypes.c_int64 * 3)(0, 8, 4)  # decreasing
    assert L.mcfftErrorNorms(one, 1, one, 2, offs, None, out, None) == mc.INVALID_VALUE
    offs = (ctypes.c_int64 * 2)(-4, 4)  # negative
    assert L.mcfftErrorNorms(one, 1, one, 1, offs, None, out, None) == mc.INVALID_VALUE
    offs = (ctypes.c_int64 * 2)(0, 4)
    assert L.mcfftErrorNorms(one, 1, one, 0, offs, None, out, None) == mc.INVALID_VALUE
    assert L.mcfftErrorNorms(None, 1, one, 1, offs, None, out, None) == mc.INVALID_VALUE
    with pytest.raises(ValueError):
        mc.error_norms(256, True, 256, [0])
