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
    "mcfftWisdomExport", "mcfftWisdomImport", "mcfftWisdomForget", "mcfftErrorNorms",
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
                ("launches", ctypes.c_int), ("timed_passes", ctypes.c_int),
                ("fourstep_n1", ctypes.c_int64), ("tile_points", ctypes.c_int),
                ("ctas", ctypes.c_int)]


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
        L.mcfftErrorNorms.argtypes = [P, ci, P, ci, ctypes.POINTER(i64), ctypes.POINTER(ci),
                                      ctypes.POINTER(ctypes.c_double), P]
        L.mcfftErrorNorms.restype = ci
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
        # plans live on the device current at creation (cudaGetDevice)
        self.device_index = None
        try:
            import torch
            if torch.cuda.is_available():
                self.device_index = torch.cuda.current_device()
        except ImportError:
            pass

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
        """Run on torch CUDA tensors on the current stream; returns `out`.
        Element types: the input is complex32 (FP16) for the plain form and
        for the split form with FLAG_INPUT_F16, complex64 (FP32) otherwise;
        the output is complex32 for the plain form, complex64 for split.
        Both tensors must be contiguous, on the plan's device, and hold at
        least the plan's input / output bytes (the kernels read and write the
        extents the plan describes)."""
        import torch
        inf = self.info()
        split = self.precision == PREC_SPLIT
        in_dt = torch.complex64 if split and not (self.flags & FLAG_INPUT_F16) else torch.complex32
        out_dt = torch.complex64 if split else torch.complex32
        dev = None

        def need(t, dtype, nbytes, what):
            nonlocal dev
            if not (t.is_cuda and t.is_contiguous()):
                raise ValueError(f"{what} must be a contiguous CUDA tensor")
            if dev is None:
                dev = torch.device("cuda", self.device_index if self.device_index is not None
                                   else torch.cuda.current_device())
            if t.dtype != dtype:
                raise ValueError(f"{what} is {t.dtype}; this plan needs {dtype}")
            if t.device != dev:
                raise ValueError(f"{what} is on {t.device}; the plan was made on {dev}")
            have = t.numel() * t.element_size()
            if have < nbytes:
                raise ValueError(f"{what} holds {have} bytes; the plan needs {nbytes}")

        need(x, in_dt, inf.in_bytes, "x")
        if out is None:
            out = torch.empty(inf.elements, dtype=out_dt, device=dev)
        need(out, out_dt, inf.out_bytes, "out")
        stream = torch.cuda.current_stream(dev).cuda_stream
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


def error_norms(y_ptr: int, y_f16: bool, ref_ptr: int, seg_off, seg_scale_log2=None,
                stream: int = 0):
    """FP64 error norms on the GPU (see mcfftErrorNorms in include/mcfft.h).

    y_ptr: device result (complex FP16 if y_f16, else complex FP32); ref_ptr:
    device complex FP64 reference; seg_off: nseg + 1 element offsets;
    seg_scale_log2: per-segment power-of-two scale of y (or None).  Returns
    a list of per-segment dicts: rel_l2, max_rel (max |y - ref| / max |ref|)
    and get_error (the reference harness's metric)."""
    offs = [int(v) for v in seg_off]
    nseg = len(offs) - 1
    if nseg < 1:
        raise ValueError("need at least one segment")
    off_arr = (ctypes.c_int64 * len(offs))(*offs)
    sc_arr = None
    if seg_scale_log2 is not None:
        sc = [int(v) for v in seg_scale_log2]
        if len(sc) != nseg:
            raise ValueError("one scale per segment")
        sc_arr = (ctypes.c_int * nseg)(*sc)
    out = (ctypes.c_double * (5 * nseg))()
    _check(lib().mcfftErrorNorms(ctypes.c_void_p(y_ptr), int(bool(y_f16)), ctypes.c_void_p(ref_ptr),
                                 nseg, off_arr, sc_arr, out, ctypes.c_void_p(stream)),
           "mcfftErrorNorms")
    res = []
    for i in range(nseg):
        e2, r2, emax, rmax, rel = out[5 * i: 5 * i + 5]
        n = offs[i + 1] - offs[i]
        res.append({"rel_l2": (e2 / r2) ** 0.5 if r2 > 0 else float("inf"),
                    "max_rel": emax / rmax if rmax > 0 else float("inf"),
                    "get_error": rel / n if n else 0.0})
    return res


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
