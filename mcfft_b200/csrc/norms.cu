// norms.cu -- error norms of a transform result against an FP64 reference,
// reduced in FP64 on the GPU (mcfftErrorNorms).
//
// The reference's accuracy harness computes its error on the host, one
// element at a time (get_error, benchmark/accuracy_1d.cpp:26-56): the mean
// over components of min(1, |(tested - standard) / standard|).  Here the
// result never leaves the device: every block reduces a chunk of one
// segment (one transform, or any run of elements) in FP64 and merges its
// partials into the segment's five accumulators with atomics --
//   [0] sum |y s - r|^2     [1] sum |r|^2
//   [2] max |y s - r|       [3] max |r|   (over real and imaginary parts)
//   [4] sum over components of min(1, |(y s - r) / r|)  (get_error's sum)
// with s = 2^scale_log2 of the segment (the plain form's output scale).
// Maxima of non-negative doubles are merged as unsigned 64-bit integers,
// whose order is the same.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/mcfft.h"

namespace mcfft {
namespace {

constexpr int kNormThreads = 256;
constexpr int kNormPerThread = 16;
constexpr int64_t kNormChunk = (int64_t)kNormThreads * kNormPerThread;  // elements per block

struct NormAcc {
  double e2, r2, emax, rmax, rel;
};

__device__ __forceinline__ double rel_term(double e, double r) {
  // min(1, |e / r|); r == 0 gives 1 unless e == 0 too (0/0: the reference's
  // std::min(1.0, NaN) returns 1.0 as well, its first argument)
  const double q = fabs(e / r);
  return q < 1.0 ? q : 1.0;
}

template <bool F16>
__global__ void k_error_norms(const void* __restrict__ y, const double2* __restrict__ ref,
                              const int64_t* __restrict__ seg_off, const double* __restrict__ scale,
                              const int* __restrict__ block_seg,
                              const int64_t* __restrict__ block_start,
                              double* __restrict__ out) {
  const int seg = block_seg[blockIdx.x];
  const int64_t lo = block_start[blockIdx.x];
  const int64_t hi = min(lo + kNormChunk, seg_off[seg + 1]);
  const double s = scale[seg];
  NormAcc a{0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double yr, yi;
    if constexpr (F16) {
      const __half2 h = reinterpret_cast<const __half2*>(y)[i];
      yr = (double)__low2float(h);
      yi = (double)__high2float(h);
    } else {
      const float2 f = reinterpret_cast<const float2*>(y)[i];
      yr = (double)f.x;
      yi = (double)f.y;
    }
    const double2 r = ref[i];
    const double er = yr * s - r.x, ei = yi * s - r.y;
    const double e2 = er * er + ei * ei, r2 = r.x * r.x + r.y * r.y;
    a.e2 += e2;
    a.r2 += r2;
    a.emax = fmax(a.emax, fmax(fabs(er), fabs(ei)));
    a.rmax = fmax(a.rmax, fmax(fabs(r.x), fabs(r.y)));
    a.rel += rel_term(er, r.x) + rel_term(ei, r.y);
  }
  // warp, then block reduction
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a.e2 += __shfl_xor_sync(0xffffffffu, a.e2, o);
    a.r2 += __shfl_xor_sync(0xffffffffu, a.r2, o);
    a.emax = fmax(a.emax, __shfl_xor_sync(0xffffffffu, a.emax, o));
    a.rmax = fmax(a.rmax, __shfl_xor_sync(0xffffffffu, a.rmax, o));
    a.rel += __shfl_xor_sync(0xffffffffu, a.rel, o);
  }
  __shared__ NormAcc part[kNormThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) part[warp] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    NormAcc t = part[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      t.e2 += part[w].e2;
      t.r2 += part[w].r2;
      t.emax = fmax(t.emax, part[w].emax);
      t.rmax = fmax(t.rmax, part[w].rmax);
      t.rel += part[w].rel;
    }
    double* o = out + 5 * (int64_t)seg;
    atomicAdd(o + 0, t.e2);
    atomicAdd(o + 1, t.r2);
    atomicMax(reinterpret_cast<unsigned long long*>(o + 2), (unsigned long long)__double_as_longlong(t.emax));
    atomicMax(reinterpret_cast<unsigned long long*>(o + 3), (unsigned long long)__double_as_longlong(t.rmax));
    atomicAdd(o + 4, t.rel);
  }
}

}  // namespace
}  // namespace mcfft

using namespace mcfft;

extern "C" MCFFT_API mcfftResult mcfftErrorNorms(const void* y, int y_f16, const void* ref,
                                                 int nseg, const int64_t* seg_off,
                                                 const int* seg_scale_log2, double* out,
                                                 void* stream) {
  if (!y || !ref || !seg_off || !out || nseg < 1) return MCFFT_INVALID_VALUE;
  for (int i = 0; i < nseg; ++i)
    if (seg_off[i] < 0 || seg_off[i + 1] < seg_off[i]) return MCFFT_INVALID_VALUE;
  // block -> (segment, first element): every segment in chunks of kNormChunk
  std::vector<int> bseg;
  std::vector<int64_t> bstart;
  for (int i = 0; i < nseg; ++i)
    for (int64_t p = seg_off[i]; p < seg_off[i + 1]; p += kNormChunk) {
      bseg.push_back(i);
      bstart.push_back(p);
    }
  std::vector<double> scale(nseg);
  for (int i = 0; i < nseg; ++i)
    scale[i] = std::ldexp(1.0, seg_scale_log2 ? seg_scale_log2[i] : 0);
  const size_t nb = bseg.size();
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // one device block for the tables and the accumulators
  const size_t o_acc = 0, o_off = o_acc + sizeof(double) * 5 * nseg,
               o_scale = o_off + sizeof(int64_t) * (nseg + 1),
               o_bstart = o_scale + sizeof(double) * nseg,
               o_bseg = o_bstart + sizeof(int64_t) * std::max<size_t>(nb, 1),
               total = o_bseg + sizeof(int) * std::max<size_t>(nb, 1);
  char* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_ALLOC_FAILED;
  }
  cudaError_t e = cudaMemsetAsync(d + o_acc, 0, sizeof(double) * 5 * nseg, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d + o_off, seg_off, sizeof(int64_t) * (nseg + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d + o_scale, scale.data(), sizeof(double) * nseg, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nb) {
    e = cudaMemcpyAsync(d + o_bstart, bstart.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d + o_bseg, bseg.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st);
  }
  // one launch per 2^31 - 1 blocks (grid x limit)
  for (size_t b0 = 0; b0 < nb && e == cudaSuccess; b0 += 0x7fffffffu) {
    const unsigned g = (unsigned)std::min<size_t>(nb - b0, 0x7fffffffu);
    const int* bs = reinterpret_cast<const int*>(d + o_bseg) + b0;
    const int64_t* bst = reinterpret_cast<const int64_t*>(d + o_bstart) + b0;
    const int64_t* so = reinterpret_cast<const int64_t*>(d + o_off);
    const double* sc = reinterpret_cast<const double*>(d + o_scale);
    double* acc = reinterpret_cast<double*>(d + o_acc);
    const double2* r = static_cast<const double2*>(ref);
    if (y_f16)
      k_error_norms<true><<<g, kNormThreads, 0, st>>>(y, r, so, sc, bs, bst, acc);
    else
      k_error_norms<false><<<g, kNormThreads, 0, st>>>(y, r, so, sc, bs, bst, acc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, d + o_acc, sizeof(double) * 5 * nseg, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }
  return MCFFT_SUCCESS;
}
