// Host-side check of the pass layout engine (mcfft_b200/csrc/layout.cpp),
// compiled and run by tests/test_layout.py: for a pass shape given on the
// command line it builds the layout and prints its bank-conflict figures,
// the staging order and the twiddle-table mode, then verifies on the host
// that the tables are consistent -- every A-operand slot of stage 0 is
// written exactly once by the prologue, every staging slot is read once,
// and the column items' twiddle rows land on the physical rows the folded
// table stores them at, that paired row items share their rows, and that
// every stage's epilogue stores tile their destination buffer.
#include <cstdio>
#include <cstdlib>
#include <set>
#include <string>
#include <vector>

#include "../mcfft_b200/csrc/layout.h"

using namespace mcfft;
using namespace mcfft::layout;

int main(int argc, char** argv) {
  if (argc != 6 && argc != 8) {
    std::fprintf(stderr, "usage: layout_check L R C in(row|col) out(row|col) [in_elem out_elem]\n");
    return 2;
  }
  const int ie = argc == 8 ? std::atoi(argv[6]) : 4, oe = argc == 8 ? std::atoi(argv[7]) : 4;
  const int L = std::atoi(argv[1]), R = std::atoi(argv[2]), C = std::atoi(argv[3]);
  const Kind ik = std::string(argv[4]) == "col" ? COL : ROW;
  const Kind ok = std::string(argv[5]) == "col" ? COL : ROW;
  const int64_t nc = 1024, nouter = 16;
  // column layout: columns contiguous, points strided by nc; row layout: points contiguous
  const int64_t isp = ik == COL ? nc : 1, isc = ik == COL ? 1 : L, iso = (int64_t)L * nc;
  const int64_t osp = ok == COL ? nc : 1, osc = ok == COL ? 1 : L, oso = (int64_t)L * nc;
  PassLayout pl;
  std::string err;
  if (!build(&pl, L, R, C, ik, ok, ie, oe, isp, isc, iso, osp, osc, oso, nc, nouter, &err)) {
    std::printf("error %s\n", err.c_str());
    return 1;
  }
  std::printf("prologue_excess %.3f\nepilogue_excess %.3f\npmid %d\ntail_pm %d\nin_ndims %d\n",
              pl.prologue_excess, pl.epilogue_excess, pl.in.pmid, pl.tail_pm, pl.in.ndims);
  // staging slots read by the prologue loads: each 16-byte slot once
  std::set<uint32_t> loads, stores;
  bool ok_tabs = true;
  for (int it = 0; it < pl.items; ++it) {
    const uint32_t lb = (pl.item_tab[2 * it] & 0xFFFFu) << 2, sb = (pl.item_tab[2 * it] >> 16) << 2;
    for (uint32_t o : pl.lofs) ok_tabs &= loads.insert((lb ^ o) >> 4).second;
    for (uint32_t o : pl.sofs) ok_tabs &= stores.insert((sb ^ o) >> (R == 1 ? 4 : 2)).second;
  }
  // staging: L C elements of ie bytes; A operand (hi): L C FP16 complex
  const size_t in_slots = (size_t)L * C * ie / 16, a_slots = (size_t)L * C * 4 / 16;
  ok_tabs &= loads.size() == in_slots;
  ok_tabs &= stores.size() == (R == 1 ? a_slots : a_slots * 4);
  // column items: twiddle row = tail_row(v, tail_pm) of some v < L / R, all rows used
  if (R > 1 && ik == COL) {
    std::set<uint32_t> rows;
    for (int it = 0; it < pl.items; ++it) {
      const uint32_t w = pl.item_tab[2 * it + 1];
      ok_tabs &= (w >> 31) != 0;
      rows.insert(w & 0x7FFFFFFFu);
    }
    std::set<uint32_t> want;
    for (uint32_t v = 0; v < (uint32_t)(L / R); ++v) want.insert(tail_row(v, pl.tail_pm));
    ok_tabs &= rows == want;
  }
  // paired row items: items i and i + items / 2 read the same twiddle rows
  if (pl.tail_pm == kTailNaturalPaired)
    for (int it = 0; it < pl.items / 2; ++it)
      ok_tabs &= pl.item_tab[2 * it + 1] == pl.item_tab[2 * (it + pl.items / 2) + 1];
  std::printf("tables_consistent %d\n", ok_tabs ? 1 : 0);
  // epilogue: in every stage the 16 stores of each row (4-byte FP16
  // complex into the next stage's operand; after the last stage oe-byte
  // elements into the output staging) are aligned, inside the buffer, and
  // together write each of its L C slots exactly once
  bool ok_epi = (int)pl.epi_tab.size() == pl.NST * pl.NROWS && (int)pl.kofs.size() == pl.NST * 16 &&
                pl.NROWS * 16 == L * C;
  for (int s = 0; s < pl.NST && ok_epi; ++s) {
    const uint32_t eb = s == pl.NST - 1 ? (uint32_t)oe : 4u;
    const uint32_t nslots = (uint32_t)(L * C);
    std::set<uint32_t> slots;
    // the row's aux word: a stage-twiddle row of stage s (the kernel reads
    // row stage_tw_row0(s) + aux of its table, (L / R) / 16^(s+1) rows per
    // stage), or on the last stage v C + c (four-step twiddle of vector v,
    // column c)
    const uint32_t naux = s == pl.NST - 1 ? (uint32_t)(pl.NV * C)
                                          : (uint32_t)(((L / R) >> (4 * s)) / 16);
    for (int r = 0; r < pl.NROWS; ++r) {
      ok_epi &= (pl.epi_tab[(size_t)s * pl.NROWS + r] >> 16) < naux;
      const uint32_t dst = (pl.epi_tab[(size_t)s * pl.NROWS + r] & 0xFFFFu) << 2;
      for (int k = 0; k < 16; ++k) {
        const uint32_t o = dst ^ pl.kofs[(size_t)s * 16 + k];
        ok_epi &= o % eb == 0 && o / eb < nslots;
        ok_epi &= slots.insert(o / eb).second;
      }
    }
    ok_epi &= slots.size() == nslots;
  }
  // the kernel's compile-time table sizes (TileShape): items, rows, stages
  const int items = R == 1 ? L * C / 16 : L * C / (4 * R);
  ok_epi &= pl.items == items && (int)pl.item_tab.size() == 2 * items && pl.NROWS == L / 16 * C;
  std::printf("epilogue_consistent %d\n", ok_epi ? 1 : 0);
  return 0;
}
