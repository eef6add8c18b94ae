"""The reference's own accuracy drivers (benchmark/accuracy_{1,2,3}d.cpp),
compiled unchanged against this project's compat libraries
(libmcfft_{1,2,3}d.so) and the FFTW-named FP64 oracle by
oracle/drivers.mk, run as child processes.  Each prints the reference's
get_error metric (mean over components of min(1, |relative error|)) of
the transform of its own seeded input against the FP64 FFT.

Also a caller of the device-level API compiled against the reference's own
include/mcfft_{1,2}d_device.h (oracle/handle_caller.cpp): its handle
struct, filled by mcfftCreate and passed to mcfftExec by value, runs the
transform (rel-L2 against the FP64 oracle at the split form's bound).

The drivers are built where the reference tree is mounted; the test skips
when they are absent."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

# The metric is dominated by near-zero outputs (relative error capped at
# 1); the split form keeps it near FP32 level.
METRIC_TOL = 1e-4


def _run(args):
    exe = os.path.join(REF, args[0])
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built")
    out = subprocess.run([exe] + args[1:], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    return float(out.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("args", [["accuracy_1d", "-n", "65536", "-b", "2", "-s", "42"],
                                  ["accuracy_1d", "-n", "4096", "-b", "16", "-s", "7"],
                                  ["accuracy_1d", "-n", "1048576", "-b", "1", "-s", "3"],
                                  ["accuracy_2d", "-x", "512", "-y", "512", "-b", "2"],
                                  ["accuracy_2d", "-x", "1024", "-y", "1024", "-b", "1"],
                                  ["accuracy_3d", "-x", "256", "-y", "256", "-b", "2"]])
def test_reference_accuracy_driver(args):
    err = _run(args)
    assert err < METRIC_TOL, (args, err)


@pytest.mark.parametrize("args,size", [(["handle_caller_1d", "4096", "16"], 144),
                                       (["handle_caller_1d", "1048576", "2"], 144),
                                       (["handle_caller_2d", "256", "512", "2"], 136)])
def test_reference_handle_by_value(args, size):
    exe = os.path.join(REF, args[0])
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built")
    out = subprocess.run([exe] + args[1:], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, (out.returncode, out.stderr)
    vals = dict(line.split() for line in out.stdout.strip().splitlines())
    assert int(vals["handle_bytes"]) == size
    assert float(vals["rel_l2"]) < 2e-6, vals
