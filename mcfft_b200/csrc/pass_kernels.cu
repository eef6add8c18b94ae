// pass_kernels.cu -- the instantiated pass-kernel variants and their launch.
//
// One variant per (L, tail radix R, columns per tile C, column-fast lane
// order, four-step post twiddle, precision form).  C is chosen so that one
// tile holds kTilePoints complex points (64 KiB of FP16 in shared memory for
// the plain form); the planner picks among these.
#include <cstdio>
#include <mutex>
#include <utility>
#include <vector>

#include "fft_pass.cuh"
#include "fft_pass_split.cuh"

namespace mcfft {

namespace {

constexpr int kTilePoints = 16384;
constexpr int kSplitTilePoints = 8192;

// Dynamic shared memory requested per CTA: at least the kernel's need, and
// enough that no more CTAs fit on an SM than its 512 TMEM columns can hold
// (a CTA whose tcgen05.alloc cannot be served would wait for a neighbour to
// finish its whole persistent loop).
constexpr int kSmemPerSM = 228 * 1024;
constexpr int smem_request(int need, int tmem_cols) {
  const int max_ctas = 512 / tmem_cols;
  const int floor_bytes = kSmemPerSM / (max_ctas + 1) + 1024;
  return need > floor_bytes ? need : floor_bytes;
}

template <int L, int R, int C, bool COLFAST, bool POSTTW>
PassKernel make_plain() {
  using S = PassShape<L, R, C, COLFAST>;
  return PassKernel{reinterpret_cast<const void*>(&fft_pass_f16<L, R, C, COLFAST, POSTTW>),
                    L, R, C, COLFAST, POSTTW, false,
                    smem_request(S::SMEM_BYTES, S::TMEM_COLS), S::TMEM_COLS};
}

template <int L, int R, int C, bool COLFAST, bool POSTTW>
PassKernel make_split() {
  using S = SplitShape<L, R, C, COLFAST>;
  return PassKernel{reinterpret_cast<const void*>(&fft_pass_split<L, R, C, COLFAST, POSTTW>),
                    L, R, C, COLFAST, POSTTW, true,
                    smem_request(S::SMEM_BYTES, S::TMEM_COLS), S::TMEM_COLS};
}

// All (L, R) with L = 16^a * R, 16 <= L <= 8192, instantiated for the
// given tile size, lane order and post-twiddle flag.
#define MCFFT_VARIANTS(MAKE, TP, CF, PT)                                   \
  MAKE<16, 1, (TP) / 16, CF, PT>(), MAKE<32, 2, (TP) / 32, CF, PT>(),       \
      MAKE<64, 4, (TP) / 64, CF, PT>(), MAKE<128, 8, (TP) / 128, CF, PT>(), \
      MAKE<256, 1, (TP) / 256, CF, PT>(), MAKE<512, 2, (TP) / 512, CF, PT>(), \
      MAKE<1024, 4, (TP) / 1024, CF, PT>(), MAKE<2048, 8, (TP) / 2048, CF, PT>(), \
      MAKE<4096, 1, (TP) / 4096, CF, PT>(), MAKE<8192, 2, (TP) / 8192, CF, PT>()

std::vector<PassKernel>& registry() {
  static std::vector<PassKernel> v = {
      MCFFT_VARIANTS(make_plain, kTilePoints, false, false),
      make_plain<16384, 4, 1, false, false>(),
      MCFFT_VARIANTS(make_plain, kTilePoints, true, false),
      make_plain<16384, 4, 1, true, false>(),
      MCFFT_VARIANTS(make_plain, kTilePoints, true, true),
      make_plain<16384, 4, 1, true, true>(),
      MCFFT_VARIANTS(make_split, kSplitTilePoints, false, false),
      MCFFT_VARIANTS(make_split, kSplitTilePoints, true, false),
      MCFFT_VARIANTS(make_split, kSplitTilePoints, true, true),
  };
  return v;
}

}  // namespace

const PassKernel* find_pass_kernel(int L, int R, int C, bool colfast, bool posttw, bool split) {
  for (const auto& k : registry())
    if (k.L == L && k.R == R && k.C == C && k.colfast == colfast && k.posttw == posttw &&
        k.split == split)
      return &k;
  return nullptr;
}

const PassKernel* pick_pass_kernel(int L, bool colfast, bool posttw, bool split,
                                   int64_t max_cols, int64_t tile_points) {
  const PassKernel* best = nullptr;
  for (const auto& k : registry()) {
    if (k.L != L || k.colfast != colfast || k.posttw != posttw || k.split != split) continue;
    if (tile_points > 0 && (int64_t)k.L * k.C > tile_points) continue;
    if (!best) { best = &k; continue; }
    const bool fits = k.C <= max_cols, best_fits = best->C <= max_cols;
    if (fits && (!best_fits || k.C > best->C)) best = &k;
    else if (!fits && !best_fits && k.C < best->C) best = &k;
  }
  return best;
}

cudaError_t launch_pass(const PassKernel& k, const PassArgs& a, int grid, cudaStream_t st) {
  // The shared-memory limit is a per-device attribute of the function: set
  // it once for every (device, kernel) pair this process launches.
  static std::mutex mu;
  static std::vector<std::pair<int, const void*>> configured;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cudaGetLastError();
    std::lock_guard<std::mutex> lock(mu);
    bool done = false;
    for (const auto& f : configured) done |= (f.first == dev && f.second == k.fn);
    if (!done) {
      cudaError_t e =
          cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem_bytes);
      if (e != cudaSuccess) return e;
      configured.push_back({dev, k.fn});
    }
  }
  void* args[] = {const_cast<PassArgs*>(&a)};
  return cudaLaunchKernel(k.fn, dim3(grid), dim3(kThreads), args, (size_t)k.smem_bytes, st);
}

}  // namespace mcfft
