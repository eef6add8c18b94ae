"""The command-line timing drivers mcfft_perf_{1,2,3}d (the reference's
benchmark/test_{1,2,3}d.cpp options): without a GPU they must fail cleanly
(no CUDA device, exit 2) and reject unknown options with the usage text
(exit 1); on a GPU they print the reference's "@mcfft >" line (12 N log2 N
"tflops") and the 5 N log2 N line for plain, split, inverse and host-buffer
runs."""
import os
import re
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(HERE, "..", "mcfft_b200")


def driver(dim):
    path = os.path.join(PKG, f"mcfft_perf_{dim}d")
    if not os.path.exists(path):
        pytest.skip("timing drivers not built (python -m mcfft_b200.build)")
    return path


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.parametrize("dim,bad", [(1, "-x"), (2, "-n"), (3, "-q")])
def test_usage_on_unknown_option(dim, bad):
    r = subprocess.run([driver(dim), bad, "4"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "usage:" in r.stderr


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_no_device_fails_cleanly():
    r = subprocess.run([driver(1), "-n", "4096", "-b", "2"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 2
    assert "no CUDA device" in r.stderr


LINE = re.compile(r"@mcfft > .*iter: (\d+), time per iter: ([0-9.e+-]+), tflops: ([0-9.]+)")
LINE5 = re.compile(r"@mcfft5 > .*gflops\(5NlogN\): ([0-9.]+), hbm GB/s: ([0-9.]+)")


@pytest.mark.gpu
@pytest.mark.parametrize("dim,args", [
    (1, ["-n", "4096", "-b", "64"]),
    (1, ["-n", "65536", "-b", "8", "-p", "1", "-f"]),
    (1, ["-n", "1048576", "-b", "2", "-i"]),
    (2, ["-x", "256", "-y", "512", "-b", "4"]),
    (2, ["-x", "128", "-y", "128", "-b", "8", "-e"]),
    (3, ["-x", "64", "-y", "64", "-z", "64", "-p", "1"]),
])
def test_driver_runs_and_reports(dim, args):
    r = subprocess.run([driver(dim), *args, "-t", "0.05"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    m = LINE.search(r.stdout)
    m5 = LINE5.search(r.stdout)
    assert m and m5, r.stdout
    iters, per, tflops = int(m.group(1)), float(m.group(2)), float(m.group(3))
    assert iters >= 1 and per > 0 and tflops > 0
    gf5, gbs = float(m5.group(1)), float(m5.group(2))
    # the two conventions differ by the factor 12 / 5
    assert abs(tflops * 1e3 * 5 / 12 - gf5) <= 0.01 * gf5 + 0.01
    assert gbs > 0
