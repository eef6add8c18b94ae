"""ctypes wrapper over oracle/fft64.c -- the CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline legs, as the checker.  The product library never
imports it.

Functions (all complex data is numpy complex128, natural order):
  fftnd(x, axes_dims, sign)      FP64 FFT (FFTW_FORWARD / unnormalised
                                 BACKWARD convention), stand-in for the FFTW
                                 double oracle of benchmark/accuracy_1d.cpp:12-24
  dft_direct(x, sign)            O(n^2) long-double DFT
  ref_transform_1d / _2d         restated reference pipeline
                                 (source/mcfft_1d_utils.cpp:37-86,
                                 source/mcfft_1d_device.cpp:58-790)
  gen_rev                        source/mcfft_1d_utils.cpp:8-35
  generate_data                  source/mcfft_1d_utils.cpp:88-100
  get_error                      benchmark/accuracy_1d.cpp:26-56
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile fft64.c with the committed Makefile (idempotent)."""
    src = os.path.join(_HERE, "fft64.c")
    if (not os.path.exists(_LIB_PATH)
            or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        dp, i64, ci = ctypes.POINTER(ctypes.c_double), ctypes.c_int64, ctypes.c_int
        ip = ctypes.POINTER(ctypes.c_int)
        L.oracle_fftnd.argtypes = [dp, ci, ctypes.POINTER(i64), i64, ci]
        L.oracle_fftnd.restype = ci
        L.oracle_dft_direct.argtypes = [dp, dp, i64, ci]
        L.oracle_generate_data.argtypes = [dp, i64, i64, ci]
        L.oracle_get_error.argtypes = [dp, dp, i64, i64]
        L.oracle_get_error.restype = ctypes.c_double
        L.oracle_error_norms.argtypes = [dp, dp, i64, dp, dp]
        L.ref_gen_rev.argtypes = [ci, ip, ip, ci]
        L.ref_plan_1d.argtypes = [ci, ip, ip, ip, ip]
        L.ref_plan_1d.restype = ci
        L.ref_transform_1d.argtypes = [dp, dp, ci, ci]
        L.ref_transform_1d.restype = ci
        L.ref_transform_2d.argtypes = [dp, dp, ci, ci, ci]
        L.ref_transform_2d.restype = ci
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fftnd(x: np.ndarray, dims, sign: int = -1) -> np.ndarray:
    """FFT over the trailing len(dims) axes of x (complex128), batched over
    the leading axes.  sign=-1 forward, +1 unnormalised backward."""
    dims = [int(d) for d in dims]
    y = np.ascontiguousarray(x, dtype=np.complex128).copy()
    tail = int(np.prod(dims))
    batch = y.size // tail
    d = (ctypes.c_int64 * len(dims))(*dims)
    rc = lib().oracle_fftnd(_dptr(y.view(np.float64)), len(dims), d, batch, sign)
    if rc != 0:
        raise MemoryError("oracle_fftnd failed")
    return y


def fft1d(x: np.ndarray, sign: int = -1) -> np.ndarray:
    return fftnd(x, [x.shape[-1]], sign)


def dft_direct(x: np.ndarray, sign: int = -1) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.empty_like(x)
    lib().oracle_dft_direct(_dptr(x.view(np.float64)), _dptr(y.view(np.float64)),
                            x.size, sign)
    return y


def generate_data(n: int, n_batch: int, seed: int = 42) -> np.ndarray:
    """The reference's generate_data: complex128 array of shape (n_batch, n)."""
    out = np.empty((n_batch, n), dtype=np.complex128)
    lib().oracle_generate_data(_dptr(out.view(np.float64)), n, n_batch, seed)
    return out


def get_error(tested: np.ndarray, standard: np.ndarray) -> float:
    t = np.ascontiguousarray(tested, dtype=np.complex128)
    s = np.ascontiguousarray(standard, dtype=np.complex128)
    n = t.shape[-1] if t.ndim > 1 else t.size
    nb = t.size // n
    return lib().oracle_get_error(_dptr(t.view(np.float64)), _dptr(s.view(np.float64)),
                                  n, nb)


def error_norms(y: np.ndarray, ref: np.ndarray):
    """(rel_l2, max_abs / max|ref|) reduced in long double."""
    a = np.ascontiguousarray(y, dtype=np.complex128)
    b = np.ascontiguousarray(ref, dtype=np.complex128)
    r1, r2 = ctypes.c_double(), ctypes.c_double()
    lib().oracle_error_norms(_dptr(a.view(np.float64)), _dptr(b.view(np.float64)),
                             a.size, ctypes.byref(r1), ctypes.byref(r2))
    return r1.value, r2.value


def gen_rev(n: int, radices) -> np.ndarray:
    r = (ctypes.c_int * len(radices))(*radices)
    out = (ctypes.c_int * n)()
    lib().ref_gen_rev(n, out, r, len(radices))
    return np.frombuffer(out, dtype=np.int32).copy()


def ref_plan_1d(n: int):
    """Returns (radices, mergings) of the reference's size table, or None."""
    rad = (ctypes.c_int * 9)()
    nr = ctypes.c_int()
    mer = (ctypes.c_int * 3)()
    nm = ctypes.c_int()
    if lib().ref_plan_1d(n, rad, ctypes.byref(nr), mer, ctypes.byref(nm)) != 0:
        return None
    return list(rad)[: nr.value], list(mer)[: nm.value]


def ref_transform_1d(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    n = x.shape[-1]
    nb = x.size // n
    y = np.empty_like(x)
    rc = lib().ref_transform_1d(_dptr(x.view(np.float64)), _dptr(y.view(np.float64)), n, nb)
    if rc != 0:
        raise ValueError(f"reference 1D algorithm does not support n={n} (rc={rc})")
    return y


def ref_transform_2d(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    nx, ny = x.shape[-2], x.shape[-1]
    nb = x.size // (nx * ny)
    y = np.empty_like(x)
    rc = lib().ref_transform_2d(_dptr(x.view(np.float64)), _dptr(y.view(np.float64)),
                                nx, ny, nb)
    if rc != 0:
        raise ValueError(f"reference 2D algorithm does not support {nx}x{ny} (rc={rc})")
    return y
