"""The batch queue's item order (mcfft_b200/csrc/queue_order.h), checked on
the host on random synthetic plans (single-pass, four-step 1D, 2D and 3D
groups mixed): every item once, every dependency pointing backwards (so the
persistent kernel's queue always drains), and the lag of QC tiles per CTA
between a key's last producer and its consumers everywhere but in the final
flush.  Compiles tests/queue_order_check.cpp once.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path_factory.mktemp("queue_order") / "queue_order_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-Wall", "-Werror", "-o", exe,
                    os.path.join(HERE, "queue_order_check.cpp")], check=True)
    return exe


@pytest.mark.parametrize("grid,chunk", [(1, 1), (7, 4), (148, 16), (148, 4), (37, 16)])
def test_queue_order_properties(checker, grid, chunk):
    for seed in range(1, 121):
        r = subprocess.run([checker, str(seed), str(grid), str(chunk)], capture_output=True,
                           text=True, timeout=60)
        assert r.returncode == 0 and r.stdout.startswith("ok"), (seed, r.stdout, r.stderr)
