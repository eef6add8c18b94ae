// tail_layout.h -- shared-memory layout of the radix-R twiddle table of a
// tile pass, shared by the host layout engine (which writes the row of each
// column item into its table) and the kernels (which fill and read it).
//
// Natural layout (row-item passes, tail_pm < 0): entry (v, k), k < R, of 8
// bytes at 8 (R v + k); tail_pm = kTailNaturalPaired (-2) also says that the
// two prologue items of a thread (item indices i and i + items / 2) read the
// same rows.  Folded layout (column-item passes, tail_pm = t >= 0): row v
// at tail_row(v, t), which puts bits [t, t + 3) of v lowest (t = 0 keeps v),
// and within a row of R / 2 chunks of 16 bytes chunk k / 2 at
// (k / 2) ^ (row >> (3 - log2(R / 2)) & (R / 2 - 1)): the rows the eight
// lanes of a quarter warp read (bits [t, t + 3) of v varying) then fall in
// eight distinct 16-byte bank groups.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define MCFFT_HD __host__ __device__ __forceinline__
#else
#define MCFFT_HD inline
#endif

namespace mcfft {

constexpr int kTailNatural = -1;
constexpr int kTailNaturalPaired = -2;

MCFFT_HD uint32_t tail_row(uint32_t v, int t) {
  if (t <= 0) return v;
  const uint32_t lo = v & ((1u << t) - 1u), mid = (v >> t) & 7u;
  return mid | (lo << 3) | ((v >> (t + 3)) << (t + 3));
}

MCFFT_HD uint32_t tail_offset(uint32_t row, uint32_t k, int R) {
  const int cb = R >= 8 ? 2 : R >= 4 ? 1 : 0;  // log2(R / 2)
  const uint32_t chunk = (k >> 1) ^ ((row >> (3 - cb)) & ((1u << cb) - 1u));
  return row * (uint32_t)R * 8u + chunk * 16u + (k & 1u) * 8u;
}

// Byte offset of entry (v, k) for a pass with the given tail_pm.
MCFFT_HD uint32_t tail_entry(uint32_t v, uint32_t k, int R, int tail_pm) {
  return tail_pm < 0 ? 8u * ((uint32_t)R * v + k) : tail_offset(tail_row(v, tail_pm), k, R);
}

}  // namespace mcfft
