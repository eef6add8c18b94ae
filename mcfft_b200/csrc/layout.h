// layout.h -- host-side layout engine for one FFT pass.
//
// Every index map the pass kernel needs is computed here, on the host, at
// plan time, and handed to the kernel as small tables:
//
//   staging     where TMA puts element (point pos, column c) of a tile in
//               shared memory (natural order, with the TMA swizzle applied)
//   A layout    the tcgen05 K-major SWIZZLE_64B operand: row r = one
//               16-point vector, K = 16 interleaved complex FP16 (64 bytes)
//   row maps    which vector (v, c) sits in A row r at each radix-16 stage
//   prologue    per work item: staging load offsets and A store offsets
//   epilogue    per A row and stage: destination base offset (next stage's A
//               row, or the output staging) and twiddle row; per output k an
//               XOR offset, so a lane's 16 stores are base ^ kofs[k]
//
// All maps are bit permutations plus XOR swizzles of power-of-two indices,
// hence GF(2)-linear; build() checks that property, so the kernel's
// "base XOR per-k constant" addressing is exact.  The row maps and the order
// of prologue items are chosen by a small search that minimises shared-
// memory bank conflicts, evaluated with the access model in conflicts().
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "tail_layout.h"

namespace mcfft {
namespace layout {

enum Kind { ROW = 0, COL = 1 };  // ROW: points contiguous in global; COL: columns contiguous

struct Staging {
  Kind kind = ROW;
  int L = 0, C = 0, elem = 4;  // elem: bytes per complex element (4 FP16, 8 FP32)
  int E = 0;                   // elements per 128-byte-or-less smem row (ROW: points, COL: columns)
  int row_bytes = 0;
  int swz = 0;                 // XOR mask applied to bits 4.. from bits 7.. (0, 1, 3, 7)
  // COL staging only: shared-memory row order of the points.  -1: natural;
  // t >= 1: point bits [t, t + 3) form the lowest three row bits, then bits
  // [0, t), then the rest (so that those bits select shared-memory banks).
  int pmid = -1;
  uint32_t bytes() const { return (uint32_t)L * C * elem; }
  // Bytes one TMA box moves (less than bytes() when the column blocks of a
  // column staging are clamped to a pass with fewer columns than C).
  uint32_t box_bytes() const {
    uint32_t v = (uint32_t)elem;
    for (int d = 0; d < ndims; ++d) v *= box[d];
    return v;
  }
  bool clamped() const { return box_bytes() != bytes(); }
  uint32_t offset(uint32_t pos, uint32_t c) const;
  // TMA box: dims innermost first.  For the kernel: coordinate of dim d for
  // tile (outer, cb) is cb * cmul[d] + outer * omul[d].
  int ndims = 0;
  uint64_t gdim[5]{}, gstride_bytes[5]{};  // gstride_bytes[0] unused (element stride)
  uint32_t box[5]{};
  int32_t cmul[5]{}, omul[5]{};
};

// noswz: no TMA swizzle (staging filled by row gathers, whose destinations
// are not aligned to the swizzle pattern's 1 KB period).
Staging make_staging(Kind kind, int L, int C, int elem, int64_t sp, int64_t sc, int64_t so,
                     int64_t ncols, int64_t nouter, int pmid = -1, bool noswz = false);

// A-operand byte offset of (row r, complex position n) in the SWIZZLE_64B
// K-major layout (8-row atoms of 512 bytes).
inline uint32_t a_offset(uint32_t r, uint32_t n) {
  return (r >> 3) * 512u + (r & 7u) * 64u + ((((n >> 2) ^ (r >> 1)) & 3u) << 4) + (n & 3u) * 4u;
}

struct PassLayout {
  // shape
  int L = 0, R = 1, C = 0, NV = 0, NST = 0, NROWS = 0;
  Kind in_kind = ROW, out_kind = ROW;
  Staging in, out;
  // row maps per stage: row -> (v, c) and (v, c) -> row
  std::vector<std::vector<uint32_t>> row_v, row_c, row_of;  // row_of[s][v * C + c]
  // prologue items
  int items = 0, item_loads = 0, item_stores = 0;
  std::vector<uint32_t> item_tab;   // per item: (lds_base >> 2) | (sts_base >> 2) << 16, plus
                                    // the tail twiddle row in a second word for R > 1
  std::vector<uint32_t> lofs;       // XOR offsets of the item's loads (bytes)
  std::vector<uint32_t> sofs;       // XOR offsets of the item's stores (bytes)
  // epilogue tables: per stage s, per row r: (dst_base >> 2) | (aux << 16)
  std::vector<uint32_t> epi_tab;    // [s][r]
  std::vector<uint32_t> kofs;       // [s][16] XOR offsets (bytes)
  // Radix-R twiddle table layout in shared memory (tail_layout.h): -1
  // natural (row items), t >= 0 folded with row order t (column items).
  int tail_pm = -1;
  // bank-conflict figures (wavefronts actually used / ideal), for reports
  double prologue_excess = 0, epilogue_excess = 0;
  std::string describe() const;
};

// Builds the layout of one pass.  out_elem: bytes of an output element.
// Returns false (with *err) if no layout satisfies the kernel's constraints.
// unsw: bit 0 / bit 1 -- the input / output staging without swizzle (see
// make_staging).
bool build(PassLayout* pl, int L, int R, int C, Kind in_kind, Kind out_kind, int in_elem,
           int out_elem, int64_t in_sp, int64_t in_sc, int64_t in_so, int64_t out_sp,
           int64_t out_sc, int64_t out_so, int64_t ncols, int64_t nouter, std::string* err,
           int unsw = 0);

}  // namespace layout
}  // namespace mcfft
