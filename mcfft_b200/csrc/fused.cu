// fused.cu -- registry of the fused four-step kernels (fft_fused in
// fft_queue.cuh): one persistent launch runs both passes of a 1D four-step
// transform group, for the length pairs (n1, n2) instantiated here.
#include <vector>

#define MCFFT_QUEUE_KERNEL
#include "fft_queue.cuh"
#include "queue.h"

namespace mcfft {

namespace {

// Pass 0: n1 points with the four-step twiddle (FP16 input in both forms'
// variants listed here: plain, and split with MCFFT_FLAG_INPUT_F16, or
// split with FP32 input); pass 1: n2 points.
template <bool SPLIT, int L1, bool ALT1, int L2, bool ALT2>
FusedKernel make_fused() {
  constexpr int V1 = queue::variant_of(L1, true, ALT1);
  constexpr int V2 = queue::variant_of(L2, false, ALT2);
  return FusedKernel{SPLIT, V1, V2, reinterpret_cast<const void*>(&fft_fused<SPLIT, V1, V2>),
                     FusedSmem<SPLIT, V1, V2>::SMEM_BYTES};
}

}  // namespace

const std::vector<FusedKernel>& fused_registry() {
  static const std::vector<FusedKernel> v = {
      // plain form, 16K-point tiles: 2^19, 2^20 (the tables of pairs with
      // 2048-point passes do not fit beside the three tile buffers)
      make_fused<false, 512, false, 1024, false>(),
      make_fused<false, 1024, false, 1024, false>(),
      // split form (8K-point tiles), FP16 or FP32 input: 2^20
      make_fused<true, 1024, true, 1024, false>(),
      make_fused<true, 1024, false, 1024, false>(),
  };
  return v;
}

const FusedKernel* find_fused(bool split, int v1, int v2) {
  for (const auto& k : fused_registry())
    if (k.split == split && k.v1 == v1 && k.v2 == v2) return &k;
  return nullptr;
}

}  // namespace mcfft
