"""Build the native library mcfft_b200/libmcfft.so (sm_100a) in-tree, the
reference-signature harness libraries libmcfft_{1,2,3}d.so and the timing
drivers mcfft_perf_{1,2,3}d.

    python -m mcfft_b200.build            # or: python mcfft_b200/build.py

nvcc cross-compiles for sm_100a without a GPU.  Objects go to
mcfft_b200/_build/, the shared library next to this file so that it
travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmcfft.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
         "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr"]
SOURCES = ["tables.cu", "pass_kernels.cu", "tile_pass.cu", "tile_split.cu", "queue.cu",
           "queue_split.cu", "fused.cu", "layout.cpp", "mcfft_api.cu", "noalloc.cu", "norms.cu"]
HEADERS = ["sm100_ptx.cuh", "tail_layout.h", "fft_pass.cuh", "fft_pass_split.cuh", "fft_tile.cuh",
           "fft_tile_split.cuh", "fft_queue.cuh", "queue.h", "queue_order.h", "host_schedule.h",
           "tile_pass.h", "layout.h", "mcfft_internal.h"]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "mcfft.h"))
    if _stale(obj, deps):
        cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    return obj


def _compat(dim: int) -> str:
    """libmcfft_{dim}d.so: the reference's harness signatures over the C ABI."""
    out = os.path.join(HERE, f"libmcfft_{dim}d.so")
    src = os.path.join(CSRC, "compat.cu")
    deps = [src, LIB] + [os.path.join(HERE, "..", "include", h) for h in
                         ("mcfft.h", "common.h", f"mcfft_{dim}d_utils.h", f"mcfft_{dim}d_device.h")]
    if _stale(out, deps):
        obj = os.path.join(BUILD, f"compat_{dim}d.o")
        subprocess.run([NVCC, *ARCH, *FLAGS, f"-DMCFFT_COMPAT_DIM={dim}", "-c", src, "-o", obj],
                       check=True)
        subprocess.run([NVCC, *ARCH, "-shared", "-o", out, obj, "-L" + HERE, "-lmcfft",
                        "-Xlinker", "-rpath,$ORIGIN", "-cudart", "static"], check=True)
    return out


def _driver(dim: int) -> str:
    """mcfft_perf_{dim}d: the command-line timing driver (csrc/perf_driver.cpp)."""
    out = os.path.join(HERE, f"mcfft_perf_{dim}d")
    src = os.path.join(CSRC, "perf_driver.cpp")
    if _stale(out, [src, LIB, os.path.join(HERE, "..", "include", "mcfft.h")]):
        subprocess.run([NVCC, *ARCH, "-O2", "-std=c++17", f"-DMCFFT_PERF_DIM={dim}", src, "-o", out,
                        "-L" + HERE, "-lmcfft", "-Xlinker", "-rpath,$ORIGIN", "-cudart", "static"],
                       check=True)
    return out


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if _stale(LIB, objs):
        subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static"],
                       check=True)
    with cf.ThreadPoolExecutor(max_workers=6) as ex:
        list(ex.map(_compat, (1, 2, 3)))
        list(ex.map(_driver, (1, 2, 3)))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
