// tile_split.cu -- registry of the split-form tile kernel variants
// (fft_tile_split.cuh): 8K-point tiles, 16 consumer warps, one CTA per SM,
// FP16 or FP32 input staging, with and without the four-step twiddle.
// L = 4096 holds two columns per tile, which only row staging takes (the
// layout engine refuses it for column passes); the batch kernel has no
// such variant.  L = 16 (512 columns per tile) serves column passes only.
#include <vector>

#include "fft_tile_split.cuh"
#include "tile_pass.h"

namespace mcfft {

namespace {

template <int L, int R, bool PT, bool IN16>
TileKernel make_split() {
  constexpr int TP = 8192, NCW = 16;
  constexpr int C = TP / L;
  using T = TileSplit<L, R, C, PT, NCW, IN16>;
  using S = TileShape<L, R, C, NCW>;
  return TileKernel{reinterpret_cast<const void*>(&fft_tile_split<L, R, C, PT, NCW, IN16>),
                    L, R, C, PT, true, S::NT, T::SMEM_BYTES,
                    SplitTile<L, R, C, PT, NCW, IN16>::TMEM_COLS, TP, IN16};
}

#define MCFFT_SPLIT_VARIANTS(PT, IN16)                                                  \
  make_split<32, 2, PT, IN16>(), make_split<64, 4, PT, IN16>(),                         \
      make_split<128, 8, PT, IN16>(), make_split<256, 1, PT, IN16>(),                   \
      make_split<512, 2, PT, IN16>(), make_split<1024, 4, PT, IN16>(),                  \
      make_split<2048, 8, PT, IN16>(), make_split<4096, 1, PT, IN16>()

}  // namespace

const std::vector<TileKernel>& split_registry() {
  static const std::vector<TileKernel> v = {
      MCFFT_SPLIT_VARIANTS(false, false), MCFFT_SPLIT_VARIANTS(true, false),
      MCFFT_SPLIT_VARIANTS(false, true), MCFFT_SPLIT_VARIANTS(true, true),
      make_split<16, 1, false, false>(), make_split<16, 1, false, true>()};
  return v;
}

}  // namespace mcfft
