// perf_driver.cpp -- command-line timing driver over the C ABI, in place of
// the reference's benchmark/test_{1,2,3}d.cpp (same options and defaults:
// 1D "-n N -b B", default n = 65536; 2D "-x -y -b", default 256 x 256; 3D
// "-x -y -z -b", default 256^3; batch 1).  Built three times with
// MCFFT_PERF_DIM = 1, 2, 3 into mcfft_perf_{1,2,3}d.
//
// Timing: a few warm-up execs, then batches of 1, 2, 4, .. execs timed with
// CUDA events on one stream until a batch takes at least -t seconds
// (benchmark/test_1d.cpp:175-191 doubles the same way against a wall clock,
// T_MIN = 4 s).  Output: the reference's line with its 12 N log2 N "tflops"
// (benchmark/test_1d.cpp:189), then the 5 N log2 N GFLOP/s convention and
// the HBM bytes per second of one read of the input and one write of the
// output.
//
// Extra options: -p 0|1 plain FP16 / split precision, -f FP16 input (split),
// -i inverse, -e end to end from page-locked host buffers (mcfftExecHost),
// -t seconds, -s seed.  Input: re, im uniform in [-1, 1).
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <getopt.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/mcfft.h"

#ifndef MCFFT_PERF_DIM
#define MCFFT_PERF_DIM 1
#endif

namespace {

int fail(const char* what, mcfftResult r) {
  std::fprintf(stderr, "mcfft_perf: %s: %s\n", what, mcfftGetErrorString(r));
  return 2;
}

int cuda_fail(const char* what, cudaError_t e) {
  std::fprintf(stderr, "mcfft_perf: %s: %s\n", what, cudaGetErrorString(e));
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  long long dims[3] = {MCFFT_PERF_DIM == 1 ? 65536 : 256, 256, 256};
  long long batch = 1;
  int prec = 0, f16in = 0, inverse = 0, e2e = 0;
  double tmin = 1.0;
  unsigned seed = 42;
  const char* opts = MCFFT_PERF_DIM == 1 ? "n:b:p:fiet:s:" : MCFFT_PERF_DIM == 2 ? "x:y:b:p:fiet:s:"
                                                                                : "x:y:z:b:p:fiet:s:";
  int c;
  while ((c = getopt(argc, argv, opts)) != -1) {
    switch (c) {
      case 'n': case 'x': dims[0] = std::atoll(optarg); break;
      case 'y': dims[1] = std::atoll(optarg); break;
      case 'z': dims[2] = std::atoll(optarg); break;
      case 'b': batch = std::atoll(optarg); break;
      case 'p': prec = std::atoi(optarg); break;
      case 'f': f16in = 1; break;
      case 'i': inverse = 1; break;
      case 'e': e2e = 1; break;
      case 't': tmin = std::atof(optarg); break;
      case 's': seed = (unsigned)std::strtoul(optarg, nullptr, 10); break;
      default:
        std::fprintf(stderr, "usage: %s %s\n", argv[0],
                     MCFFT_PERF_DIM == 1 ? "[-n N] [-b batch] [-p 0|1] [-f] [-i] [-e] [-t s] [-s seed]"
                     : MCFFT_PERF_DIM == 2 ? "[-x NX] [-y NY] [-b batch] [-p 0|1] [-f] [-i] [-e] [-t s] [-s seed]"
                                           : "[-x NX] [-y NY] [-z NZ] [-b batch] [-p 0|1] [-f] [-i] [-e] [-t s] [-s seed]");
        return 1;
    }
  }
  if (prec != 0 && prec != 1) return fail("-p", MCFFT_INVALID_VALUE);
  if (f16in && prec != 1) return fail("-f needs -p 1", MCFFT_INVALID_VALUE);

  mcfftPlan plan = nullptr;
  const mcfftPrecision pr = prec ? MCFFT_PREC_SPLIT : MCFFT_PREC_FP16;
  const unsigned flags = f16in ? MCFFT_FLAG_INPUT_F16 : MCFFT_FLAG_NONE;
  mcfftResult r = MCFFT_PERF_DIM == 1   ? mcfftPlanCreate1d(&plan, dims[0], batch, pr, flags)
                  : MCFFT_PERF_DIM == 2 ? mcfftPlanCreate2d(&plan, dims[0], dims[1], batch, pr, flags)
                                        : mcfftPlanCreate3d(&plan, dims[0], dims[1], dims[2], batch,
                                                            pr, flags);
  if (r) return fail("plan", r);
  mcfftPlanInfo info{};
  mcfftPlanGetInfo(plan, &info);

  // Input on the host, rounded once to the storage type.
  const size_t elems = (size_t)info.elements;
  const bool in_half = prec == 0 || f16in;
  std::vector<unsigned char> host_in(info.in_bytes);
  {
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    for (size_t i = 0; i < 2 * elems; ++i) {
      const double v = u(rng);
      if (in_half)
        reinterpret_cast<__half*>(host_in.data())[i] = __double2half(v);
      else
        reinterpret_cast<float*>(host_in.data())[i] = (float)v;
    }
  }
  cudaStream_t st;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e) return cuda_fail("stream", e);
  void *din = nullptr, *dout = nullptr, *hin = nullptr, *hout = nullptr;
  if (e2e) {
    e = cudaHostAlloc(&hin, info.in_bytes, cudaHostAllocDefault);
    if (!e) e = cudaHostAlloc(&hout, info.out_bytes, cudaHostAllocDefault);
    if (!e) std::memcpy(hin, host_in.data(), info.in_bytes);
  } else {
    e = cudaMalloc(&din, info.in_bytes);
    if (!e) e = cudaMalloc(&dout, info.out_bytes);
    if (!e) e = cudaMemcpy(din, host_in.data(), info.in_bytes, cudaMemcpyHostToDevice);
  }
  if (e) return cuda_fail("buffers", e);
  const int dir = inverse ? MCFFT_INVERSE : MCFFT_FORWARD;
  auto run = [&]() {
    return e2e ? mcfftExecHost(plan, hin, hout, dir, st) : mcfftExec(plan, din, dout, dir, st);
  };
  for (int w = 0; w < 3; ++w)
    if ((r = run())) return fail("exec", r);
  if ((e = cudaStreamSynchronize(st))) return cuda_fail("warm-up", e);
  if ((r = mcfftPlanCheckStatus(plan))) return fail("status", r);

  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  long long iter = 1;
  double secs = 0.0;
  for (;; iter *= 2) {
    cudaEventRecord(t0, st);
    for (long long k = 0; k < iter; ++k)
      if ((r = run())) return fail("exec", r);
    cudaEventRecord(t1, st);
    if ((e = cudaEventSynchronize(t1))) return cuda_fail("timing", e);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    secs = ms * 1e-3;
    if (secs >= tmin || iter >= (1ll << 30)) break;
  }
  if ((r = mcfftPlanCheckStatus(plan))) return fail("status", r);

  double n = (double)dims[0];
  for (int d = 1; d < MCFFT_PERF_DIM; ++d) n *= (double)dims[d];
  const double per = secs / (double)iter;
  const double tflops12 = 12.0 * n * std::log2(n) * (double)batch / per * 1e-12;
  const double gflops5 = 5.0 * n * std::log2(n) * (double)batch / per * 1e-9;
  const double gbs = (double)(info.in_bytes + info.out_bytes) / per * 1e-9;
  if (MCFFT_PERF_DIM == 1)
    std::printf("@mcfft > n: %lld, n_batch: %lld, iter: %lld, time per iter: %e, tflops: %lf \n",
                dims[0], batch, iter, per, tflops12);
  else if (MCFFT_PERF_DIM == 2)
    std::printf("@mcfft > x: %lld, y: %lld, n_batch: %lld, iter: %lld, time per iter: %e, tflops: %lf \n",
                dims[0], dims[1], batch, iter, per, tflops12);
  else
    std::printf("@mcfft > x: %lld, y: %lld, z: %lld, n_batch: %lld, iter: %lld, time per iter: %e, "
                "tflops: %lf \n",
                dims[0], dims[1], dims[2], batch, iter, per, tflops12);
  std::printf("@mcfft5 > %s %s%s, gflops(5NlogN): %.2f, hbm GB/s: %.1f, passes: %d, launches: %d\n",
              prec ? "split" : "plain", inverse ? "inverse" : "forward",
              e2e ? " (host buffers)" : "", gflops5, gbs, info.num_passes, info.launches);
  mcfftPlanDestroy(plan);
  if (e2e) {
    cudaFreeHost(hin);
    cudaFreeHost(hout);
  } else {
    cudaFree(din);
    cudaFree(dout);
  }
  cudaStreamDestroy(st);
  return 0;
}
