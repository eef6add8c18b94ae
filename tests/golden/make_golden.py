"""Extract the golden vectors that the reference's own files hold.

Run where the reference is mounted:  python tests/golden/make_golden.py [REF_DIR]
Writes small fixtures next to this script; tests read only those.

Sources (paths within the reference project):
  1.log:2-513    gen_rev permutation printed by setup() for N=512,
                 radices {16,16,2} (source/mcfft_1d_utils.cpp:29-34)
  2.txt:1-131072 "tested ... standard" pairs; the standard column is FFTW
                 double (FFTW_ESTIMATE) of a 1D N=2^18 transform of the
                 seed-42 generate_data input (first 65536 complex values);
                 the tested column is the reference's failing run (error
                 1.345044, 2.txt:131073)
  3.txt:1-65536  "tested.....standard" of test_1d N=256 batch 256, seed 42
                 (first 128 transforms, interleaved re/im); both columns
                 agree at the printed precision
"""
import os
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
# The reference tree: the first argument, else $MCFFT_REF_DIR, else the
# directory named `reference` beside this repository.
REF = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MCFFT_REF_DIR")
       or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(OUT))), "reference"))
KEEP = 16384  # doubles kept from each dump (8192 complex values)


def main():
    lines = open(os.path.join(REF, "1.log")).read().split("\n")
    perm = np.array([int(s) for s in lines[1:513]], dtype=np.int32)
    assert sorted(perm.tolist()) == list(range(512))
    np.save(os.path.join(OUT, "gen_rev_512_16_16_2.npy"), perm)
    err_line = float(lines[514])

    std, tested = [], []
    with open(os.path.join(REF, "2.txt")) as f:
        for i, line in enumerate(f):
            if i >= KEEP:
                break
            a, _, b = line.split()
            tested.append(float(a))
            std.append(float(b))
    np.save(os.path.join(OUT, "fftw_1d_n262144_seed42_head.npy"), np.array(std))
    np.save(os.path.join(OUT, "reference_tested_1d_n262144_seed42_head.npy"),
            np.array(tested))

    t3, s3 = [], []
    with open(os.path.join(REF, "3.txt")) as f:
        for i, line in enumerate(f):
            if i >= KEEP:
                break
            a, b = line.strip().split(".....")
            t3.append(float(a))
            s3.append(float(b))
    np.save(os.path.join(OUT, "rocfft_1d_n256_b256_seed42_head.npy"), np.array(s3))
    np.save(os.path.join(OUT, "reference_tested_1d_n256_b256_seed42_head.npy"),
            np.array(t3))
    with open(os.path.join(OUT, "README.txt"), "w") as f:
        f.write(
            "Fixtures extracted by make_golden.py from the reference's dumps.\n"
            f"1.log error line (N=512 run): {err_line}\n"
            "gen_rev_512_16_16_2.npy: permutation for N=512, radices 16,16,2\n"
            "fftw_1d_n262144_seed42_head.npy: FFTW 1D N=2^18, first 8192 complex\n"
            "reference_tested_1d_n262144_seed42_head.npy: reference output, same run\n"
            "rocfft_1d_n256_b256_seed42_head.npy: rocFFT N=256 b=256, first 8192 complex\n"
            "reference_tested_1d_n256_b256_seed42_head.npy: reference output, same run\n"
            "Values are printed with 7 significant digits (%e).\n")


if __name__ == "__main__":
    main()
