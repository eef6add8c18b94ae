"""The chunk schedule of mcfftExecHost (mcfft_b200/csrc/host_schedule.h),
checked on the host: the chunks cover the batch exactly, every chunk is a
power of two no larger than the largest chunk B, the lengths rise 1, 2, 4,
.. at the start and fall in the same steps at the end, and B is the
largest power of two whose input fits the byte target.  Compiles a small
driver against the header once.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "mcfft_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include "host_schedule.h"
int main(int argc, char** argv) {
  const long long batch = std::atoll(argv[1]), per = std::atoll(argv[2]), target = std::atoll(argv[3]);
  const long long big = mcfft::host_chunk_big(batch, per, target);
  std::printf("%lld", big);
  for (long long c : mcfft::host_schedule(batch, big)) std::printf(" %lld", c);
  std::printf("\n");
  return 0;
}
"""


@pytest.fixture(scope="module")
def schedule(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("host_schedule")
    src, exe = d / "drv.cpp", str(d / "drv")
    src.write_text(DRIVER)
    subprocess.run([cxx, "-O2", "-std=c++17", "-Wall", "-Werror", "-I", SRC, "-o", exe, str(src)],
                   check=True)

    def run(batch, per, target):
        out = subprocess.run([exe, str(batch), str(per), str(target)], capture_output=True,
                             text=True, check=True).stdout.split()
        return int(out[0]), [int(v) for v in out[1:]]
    return run


def test_bench_workload(schedule):
    # 1D 2^20 x 64 in FP16: 4 MiB per transform, 32 MiB target
    big, chunks = schedule(64, 4 << 20, 32 << 20)
    assert big == 8
    assert chunks == [1, 2, 4, 8, 8, 8, 8, 8, 8, 2, 4, 2, 1]


@pytest.mark.parametrize("per", [1 << 10, 1 << 20, 4 << 20, 48 << 20])
@pytest.mark.parametrize("target", [1, 8 << 20, 32 << 20])
def test_schedule_properties(schedule, per, target):
    for batch in list(range(1, 70)) + [127, 128, 1000, 4096, 65537]:
        big, chunks = schedule(batch, per, target)
        # B: largest power of two with B <= batch and B * per <= target (at least 1)
        assert big & (big - 1) == 0 and 1 <= big <= batch
        assert big == 1 or big * per <= target
        assert 2 * big > batch or 2 * big * per > target
        assert sum(chunks) == batch
        assert all(c & (c - 1) == 0 and 1 <= c <= big for c in chunks)
        # head 1, 2, .., 2^(h-1) (below B), the same lengths mirrored at the
        # end, and between them runs of B, then strictly falling powers of two
        def shaped(h):
            head = [1 << i for i in range(h)]
            if h and head[-1] >= big or 2 * h > len(chunks):
                return False
            if chunks[:h] != head or chunks[len(chunks) - h:] != head[::-1]:
                return False
            mid = chunks[h:len(chunks) - h]
            m = 0
            while m < len(mid) and mid[m] == big:
                m += 1
            rest = mid[m:]
            return all(a > b for a, b in zip(rest, rest[1:]))
        assert any(shaped(h) for h in range(len(chunks) // 2 + 1)), chunks
        if batch >= 4 and big >= 2:
            assert chunks[0] == 1 and chunks[-1] == 1, chunks
