// mcfft_internal.h -- types shared by the device kernels and the host plan
// code.  Not part of the public ABI (include/mcfft.h is).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace mcfft {

// Device status word values (written by kernels with atomicExch).
constexpr int kStatusOk = 0;
constexpr int kStatusTimeout = 1;
constexpr int kStatusLayout = 2;  // shared-memory window not where the kernel's addressing expects

// Arguments of one pass kernel launch.  All strides are in complex
// elements.  Element (tile, point p, column c) lives at
//   (tile / col_blocks) * so + (tile % col_blocks) * C * sc + p * sp + c * sc
struct PassArgs {
  const void* in;
  void* out;
  int64_t in_sp, in_sc, in_so;
  int64_t out_sp, out_sc, out_so;
  int64_t col_blocks;  // column blocks of C columns per outer index
  int64_t ntiles;      // outer count * col_blocks
  int64_t ncols;       // valid columns per outer index (last block may be partial)
  const float2* tw;       // radix-16 stage twiddles, stages concatenated, [R'][k]
  const float2* tail_tw;  // radix-R first-stage twiddles, [v][k]
  const uint4* bmat;      // DFT-16 real embedding (hi), tcgen05 K-major layout, 2 KB
  const uint4* bmat_lo;   // split form: low part of the same matrix
  const float2* post_lo;  // four-step twiddle W_N^e = lo[e & (2^shift-1)] * hi[e >> shift]
  const float2* post_hi;
  uint64_t post_mask;     // N - 1
  uint32_t post_shift;
  int inverse;            // 0 forward, 1 inverse (tail butterfly sign)
  float out_scale;        // plain form: applied after the last stage
  int split_in_f16;       // split form: input is FP16 (else FP32)
  int* status;            // device status word
};

// One kernel variant: a launchable function plus its static shape.
struct PassKernel {
  const void* fn;
  int L, R, C;
  bool colfast, posttw, split;
  int smem_bytes;
  int tmem_cols;
};

// Returns the kernel variant for (L, R, C, colfast, posttw, split), or
// nullptr if not instantiated.
const PassKernel* find_pass_kernel(int L, int R, int C, bool colfast, bool posttw, bool split);
// Largest-tile variant available for (L, colfast, posttw, split) whose C
// does not exceed max_cols (falls back to the smallest C available).
const PassKernel* pick_pass_kernel(int L, bool colfast, bool posttw, bool split,
                                   int64_t max_cols, int64_t tile_points);

cudaError_t launch_pass(const PassKernel& k, const PassArgs& a, int grid, cudaStream_t st);

// Table generation (FP64 on the GPU, rounded once).
// mode 0: entry i -> exponent (i / m1) * (i % m1);  mode 1: exponent i << shift
cudaError_t gen_twiddle_table(float2* dst, int64_t count, int mode, int64_t m1, int shift,
                              int64_t modulus, int sign, double scale, cudaStream_t st);
// DFT-16 real embedding in the tcgen05 canonical K-major layout; lo may be
// nullptr (plain form).
cudaError_t gen_dft16_embedding(void* hi, void* lo, int sign, cudaStream_t st);

}  // namespace mcfft
