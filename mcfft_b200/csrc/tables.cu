// tables.cu -- FP64 generation of twiddle tables and of the real-embedded
// 16-point DFT matrix, on the GPU, rounded once to their storage types.
//
// The reference builds its DFT matrix on the host with single-precision
// cosf/sinf (source/mcfft_1d_device.cpp:776-785) and advances twiddles by
// repeated complex multiplication (e.g. :119-123); here every entry is an
// independent FP64 sincospi of an exact rational angle.
#include <cuda_fp16.h>

#include "mcfft_internal.h"

namespace mcfft {

__global__ void k_gen_twiddles(float2* dst, int64_t count, int mode, int64_t m1, int shift,
                               int64_t modulus, int sign, double scale) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  int64_t e = mode == 0 ? (i / m1) * (i % m1) : (i << shift);
  e %= modulus;
  // angle = sign * 2*pi*e/modulus; sincospi takes it in units of pi.
  double x = (2.0 * (double)e) / (double)modulus;
  double s, c;
  sincospi(x, &s, &c);
  dst[i] = make_float2((float)(c * scale), (float)(sign * s * scale));
}

cudaError_t gen_twiddle_table(float2* dst, int64_t count, int mode, int64_t m1, int shift,
                              int64_t modulus, int sign, double scale, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  int threads = 256;
  int64_t blocks = (count + threads - 1) / threads;
  k_gen_twiddles<<<(unsigned)blocks, threads, 0, st>>>(dst, count, mode, m1, shift, modulus,
                                                       sign, scale);
  return cudaGetLastError();
}

// B[kk][j] with K index kk = 2n + ri (input point n, re/im) and N index
// j = 2k + rj (output point k, re/im):
//   rj = 0 (real out):  ri=0 -> cos,  ri=1 -> -sin
//   rj = 1 (imag out):  ri=0 -> sin,  ri=1 ->  cos
// where cos + i sin = exp(sign * 2 pi i k n / 16).  Stored N-row-major with
// K contiguous in 8-element chunks: byte (j&7)*16 + (j>>3)*512 + (kk>>3)*128
// + (kk&7)*2 -- the layout the stage kernels hand to tcgen05 as K-major B.
__global__ void k_gen_dft16(__half* hi, __half* lo, int sign) {
  int t = threadIdx.x;  // 0..1023
  int j = t >> 5, kk = t & 31;
  int k = j >> 1, rj = j & 1, n = kk >> 1, ri = kk & 1;
  double s, c;
  sincospi(2.0 * (double)((k * n) % 16) / 16.0, &s, &c);
  s *= sign;
  double val = ri == 0 ? (rj == 0 ? c : s) : (rj == 0 ? -s : c);
  int off = ((j & 7) * 16 + (j >> 3) * 512 + (kk >> 3) * 128 + (kk & 7) * 2) / 2;
  __half h = __double2half(val);
  hi[off] = h;
  if (lo) lo[off] = __double2half(val - (double)__half2float(h));
}

cudaError_t gen_dft16_embedding(void* hi, void* lo, int sign, cudaStream_t st) {
  k_gen_dft16<<<1, 1024, 0, st>>>(static_cast<__half*>(hi), static_cast<__half*>(lo), sign);
  return cudaGetLastError();
}

}  // namespace mcfft

namespace mcfft {

// Same matrix as k_gen_dft16 times `scale` (a power of two, so the FP16
// rounding is unchanged), with the N (output) index ordered by point pairs:
// j = 4p + 2 rj + (k & 1), p = k >> 1, so a TMEM row holds (re_2p, re_2p+1,
// im_2p, im_2p+1) for each pair p -- operands of the packed FP32x2
// epilogue.  Stored in the tcgen05 K-major 64-byte-swizzled layout: row j
// at (j>>3)*512 + (j&7)*64, 16-byte chunk q of the row at
// ((q ^ (j>>1)) & 3) * 16, element kk at (kk & 7) * 2 within it.
__global__ void k_gen_dft16_sw64(__half* hi, __half* lo, int sign, double scale) {
  int t = threadIdx.x;  // 0..1023
  int j = t >> 5, kk = t & 31;
  int k = 2 * (j >> 2) + (j & 1), rj = (j >> 1) & 1, n = kk >> 1, ri = kk & 1;
  double s, c;
  sincospi(2.0 * (double)((k * n) % 16) / 16.0, &s, &c);
  s *= sign;
  double val = scale * (ri == 0 ? (rj == 0 ? c : s) : (rj == 0 ? -s : c));
  const int q = kk >> 3;
  const int byte = (j >> 3) * 512 + (j & 7) * 64 + (((q ^ (j >> 1)) & 3) << 4) + (kk & 7) * 2;
  __half h = __double2half(val);
  hi[byte / 2] = h;
  if (lo) lo[byte / 2] = __double2half(val - (double)__half2float(h));
}

cudaError_t gen_dft16_sw64(void* hi, void* lo, int sign, double scale, cudaStream_t st) {
  k_gen_dft16_sw64<<<1, 1024, 0, st>>>(static_cast<__half*>(hi), static_cast<__half*>(lo), sign,
                                       scale);
  return cudaGetLastError();
}

// Stage twiddle rows of the tile kernel: for R' < rows, row R' holds
// scale * W^(k R'), W = exp(sign 2 pi i / modulus), k < 16, as eight chunks
// p = (re_2p, re_2p+1, im_2p, im_2p+1); chunk p is stored at position
// p ^ fold(R'), fold(r) = (r ^ r>>3 ^ r>>6 ^ r>>9) & 7 (the kernel's
// tw_fold).
__global__ void k_gen_stage_rows(float4* dst, int64_t rows, int64_t modulus, int sign,
                                 double scale) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= rows * 8) return;
  const int64_t r = t >> 3;
  const int p = (int)(t & 7);
  double c[2], s[2];
  for (int h = 0; h < 2; ++h) {
    const int64_t e = ((2 * p + h) * r) % modulus;
    sincospi(2.0 * (double)e / (double)modulus, &s[h], &c[h]);
  }
  const uint32_t ru = (uint32_t)r;
  const uint32_t fold = (ru ^ (ru >> 3) ^ (ru >> 6) ^ (ru >> 9)) & 7u;
  dst[r * 8 + (p ^ fold)] = make_float4((float)(scale * c[0]), (float)(scale * c[1]),
                                        (float)(scale * sign * s[0]), (float)(scale * sign * s[1]));
}

cudaError_t gen_stage_rows(float4* dst, int64_t rows, int64_t modulus, int sign, double scale,
                           cudaStream_t st) {
  if (rows <= 0) return cudaSuccess;
  const int threads = 256;
  const int64_t blocks = (rows * 8 + threads - 1) / threads;
  k_gen_stage_rows<<<(unsigned)blocks, threads, 0, st>>>(dst, rows, modulus, sign, scale);
  return cudaGetLastError();
}

}  // namespace mcfft
