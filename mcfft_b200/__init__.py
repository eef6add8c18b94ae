"""mcfft_b200 -- batched complex-to-complex tensor-core FFT for B200 (sm_100a).

Python host side over the C ABI in include/mcfft.h (libmcfft.so, built in
tree by mcfft_b200/build.py).  The reference's plan-create/exec entry points
(include/mcfft_1d_device.h:37-38, include/mcfft_2d_device.h:37-38) map to
Plan(...) and Plan.exec(...); its harness functions setup/doit/finalize/
generate_data (include/mcfft_1d_utils.h:8-11) are mirrored in
mcfft_b200.harness.

There is no CPU fallback: if libmcfft.so is missing, or no CUDA device is
present when a plan is created, an exception is raised.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmcfft.so")

SUCCESS = 0
INVALID_PLAN = 1
ALLOC_FAILED = 2
INVALID_VALUE = 3
UNSUPPORTED_SIZE = 4
CUDA_ERROR = 5
DEVICE_TIMEOUT = 6
INTERNAL_ERROR = 7
NO_DEVICE = 8

PREC_FP16 = 0
PREC_SPLIT = 1
FORWARD = -1
INVERSE = 1
FLAG_NONE = 0
FLAG_INPUT_F16 = 1

# Every symbol include/mcfft.h declares.
EXPORTS = (
    "mcfftPlanCreate1d", "mcfftPlanCreate2d", "mcfftPlanCreate3d", "mcfftPlanCreateBatch",
    "mcfftExec", "mcfftPlanCheckStatus", "mcfftPlanGetInfo", "mcfftPlanDestroy",
    "mcfftGetErrorString", "mcfftGetVersion", "mcfftExec1dNoAlloc", "mcfftExecHost",
    "mcfftWisdomExport", "mcfftWisdomImport", "mcfftWisdomForget",
)


class McfftError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: {error_string(code)} (code {code})" if what else error_string(code))


class Desc(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("dims", ctypes.c_int64 * 3), ("batch", ctypes.c_int64),
                ("in_offset", ctypes.c_int64), ("out_offset", ctypes.c_int64)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int), ("dims", ctypes.c_int64 * 3), ("batch", ctypes.c_int64),
                ("precision", ctypes.c_int), ("num_passes", ctypes.c_int),
                ("scale_log2", ctypes.c_int), ("elements", ctypes.c_int64),
                ("in_bytes", ctypes.c_int64), ("out_bytes", ctypes.c_int64),
                ("workspace_bytes", ctypes.c_int64), ("num_descs", ctypes.c_int),
                ("launches", ctypes.c_int), ("timed_passes", ctypes.c_int)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libmcfft.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m mcfft_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        PP = ctypes.POINTER(ctypes.c_void_p)
        i64, u32, ci = ctypes.c_int64, ctypes.c_uint, ctypes.c_int
        L.mcfftPlanCreate1d.argtypes = [PP, i64, i64, ci, u32]
        L.mcfftPlanCreate2d.argtypes = [PP, i64, i64, i64, ci, u32]
        L.mcfftPlanCreate3d.argtypes = [PP, i64, i64, i64, i64, ci, u32]
        L.mcfftPlanCreateBatch.argtypes = [PP, ctypes.POINTER(Desc), ci, ci, u32]
        L.mcfftExec.argtypes = [P, P, P, ci, P]
        L.mcfftExecHost.argtypes = [P, P, P, ci, P]
        L.mcfftWisdomExport.argtypes = [ctypes.c_char_p]
        L.mcfftWisdomImport.argtypes = [ctypes.c_char_p]
        L.mcfftWisdomForget.argtypes = []
        for name in ("mcfftWisdomExport", "mcfftWisdomImport", "mcfftWisdomForget"):
            getattr(L, name).restype = ci
        L.mcfftPlanCheckStatus.argtypes = [P]
        L.mcfftPlanGetInfo.argtypes = [P, ctypes.POINTER(PlanInfo)]
        L.mcfftPlanDestroy.argtypes = [P]
        L.mcfftGetErrorString.argtypes = [ci]
        L.mcfftGetErrorString.restype = ctypes.c_char_p
        L.mcfftGetVersion.restype = ci
        L.mcfftExec1dNoAlloc.argtypes = [P, P, i64, i64, ci, P]
        L.mcfftExec1dNoAlloc.restype = ci
        for name in ("mcfftPlanCreate1d", "mcfftPlanCreate2d", "mcfftPlanCreate3d",
                     "mcfftPlanCreateBatch", "mcfftExec", "mcfftExecHost", "mcfftPlanCheckStatus",
                     "mcfftPlanGetInfo", "mcfftPlanDestroy"):
            getattr(L, name).restype = ci
        _lib = L
    return _lib


def error_string(code: int) -> str:
    return lib().mcfftGetErrorString(code).decode()


def _check(rc: int, what: str):
    if rc != SUCCESS:
        raise McfftError(rc, what)


class Plan:
    """A plan over one shape (or, with descs=..., many uneven shapes).

    Plan(shape=(n,), batch=B, precision=PREC_FP16)            1D
    Plan(shape=(nx, ny), ...) / Plan(shape=(nx, ny, nz), ...)  2D / 3D
    Plan(descs=[(shape, batch, in_offset, out_offset), ...])   uneven batch
    """

    def __init__(self, shape=None, batch: int = 1, precision: int = PREC_FP16,
                 flags: int = FLAG_NONE, descs=None):
        self._h = ctypes.c_void_p()
        L = lib()
        if descs is None:
            shape = tuple(int(s) for s in shape)
            descs = [(shape, batch, 0, 0)]
        arr = (Desc * len(descs))()
        for i, (shp, b, io, oo) in enumerate(descs):
            shp = tuple(int(s) for s in shp)
            arr[i].ndim = len(shp)
            for d in range(3):
                arr[i].dims[d] = shp[d] if d < len(shp) else 1
            arr[i].batch, arr[i].in_offset, arr[i].out_offset = int(b), int(io), int(oo)
        _check(L.mcfftPlanCreateBatch(ctypes.byref(self._h), arr, len(descs), precision, flags),
               "mcfftPlanCreateBatch")
        self.precision = precision
        self.flags = flags
        self.descs = descs

    @property
    def handle(self):
        return self._h

    def info(self) -> PlanInfo:
        inf = PlanInfo()
        _check(lib().mcfftPlanGetInfo(self._h, ctypes.byref(inf)), "mcfftPlanGetInfo")
        return inf

    def exec_ptr(self, in_ptr: int, out_ptr: int, direction: int = FORWARD, stream: int = 0):
        _check(lib().mcfftExec(self._h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr),
                               direction, ctypes.c_void_p(stream)), "mcfftExec")

    def exec_host_ptr(self, in_ptr: int, out_ptr: int, direction: int = FORWARD, stream: int = 0):
        """Host buffers in and out (page-locked for overlapped copies): copy
        in, transform and copy out in pipelined chunks on `stream`."""
        _check(lib().mcfftExecHost(self._h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr),
                                   direction, ctypes.c_void_p(stream)), "mcfftExecHost")

    def exec(self, x, out=None, direction: int = FORWARD):
        """Run on torch CUDA tensors (complex32 for the FP16 forms, complex64
        for FP32) on the current stream; returns `out`.  Both tensors must be
        contiguous and hold at least the plan's input / output bytes (the
        kernels read and write the extents the plan describes)."""
        import torch
        inf = self.info()

        def need(t, nbytes, what):
            if not (t.is_cuda and t.is_contiguous()):
                raise ValueError(f"{what} must be a contiguous CUDA tensor")
            have = t.numel() * t.element_size()
            if have < nbytes:
                raise ValueError(f"{what} holds {have} bytes; the plan needs {nbytes}")

        need(x, inf.in_bytes, "x")
        if out is None:
            dt = torch.complex64 if self.precision == PREC_SPLIT else torch.complex32
            out = torch.empty(inf.elements, dtype=dt, device=x.device)
        need(out, inf.out_bytes, "out")
        stream = torch.cuda.current_stream(x.device).cuda_stream
        self.exec_ptr(x.data_ptr(), out.data_ptr(), direction, stream)
        return out

    def check_status(self):
        _check(lib().mcfftPlanCheckStatus(self._h), "mcfftPlanCheckStatus")

    def close(self):
        if self._h:
            lib().mcfftPlanDestroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def exec_1d_no_alloc(in_ptr: int, out_ptr: int, n: int, batch: int,
                     direction: int = FORWARD, stream: int = 0):
    """Two-pass 1D FP16 transform without any device allocation (fixed
    device arrays inside the library; see include/mcfft.h)."""
    _check(lib().mcfftExec1dNoAlloc(ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), n, batch,
                                    direction, ctypes.c_void_p(stream)), "mcfftExec1dNoAlloc")


def wisdom_export(path: str):
    """Write this process's autotuning records to `path`."""
    _check(lib().mcfftWisdomExport(os.fsencode(path)), "mcfftWisdomExport")


def wisdom_import(path: str):
    """Read autotuning records; later plans reuse them instead of timing."""
    _check(lib().mcfftWisdomImport(os.fsencode(path)), "mcfftWisdomImport")


def wisdom_forget():
    _check(lib().mcfftWisdomForget(), "mcfftWisdomForget")


def version() -> int:
    return lib().mcfftGetVersion()
