// compat.cu -- the reference's harness and device-level entry points over the
// C ABI (include/mcfft.h), compiled once per dimension (MCFFT_COMPAT_DIM =
// 1, 2 or 3) into libmcfft_{1,2,3}d.so, because the reference's 1D/2D/3D
// libraries export the same symbol names (source/mcfft_*_utils.cpp).
//
// The reference keeps one global plan and one device buffer per process
// (source/mcfft_1d_utils.cpp:3-6); so does this file.  Differences:
//   - no host digit reversal: data go to the device in natural order;
//   - FP64 <-> FP32 conversion happens on the device around a split-form
//     transform (FP32-level accuracy, unnormalised like FFTW_FORWARD);
//   - errors are reported on stderr and end the process (the reference
//     checks nothing and runs on into undefined behaviour);
//   - device memory is released at process exit.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>

#if MCFFT_COMPAT_DIM == 1
#include "../../include/mcfft_1d_utils.h"
#elif MCFFT_COMPAT_DIM == 2
#include "../../include/mcfft_2d_utils.h"
#else
#include "../../include/mcfft_3d_utils.h"
#endif

#define COMPAT_API __attribute__((visibility("default")))

namespace {

__global__ void k_d2f(const double* in, float* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}
__global__ void k_f2d(const float* in, double* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

void die(const char* what, int code) {
  std::fprintf(stderr, "mcfft compat: %s failed (%d: %s)\n", what, code,
               code >= 0 ? mcfftGetErrorString((mcfftResult)code) : "");
  std::exit(1);
}

int64_t elements(const mcfftHandle& h) {
#if MCFFT_COMPAT_DIM == 1
  return (int64_t)h.N * h.N_batch;
#else
  return (int64_t)h.Nx * h.Ny * h.N_batch;
#endif
}

void finish_create(mcfftHandle* h, mcfftResult r) {
  if (r != MCFFT_SUCCESS) die("plan creation", r);
  if (cudaMalloc(&h->work, (size_t)elements(*h) * 2 * sizeof(float) * 2) != cudaSuccess)
    die("cudaMalloc", -1);
}

mcfftHandle g_plan;
double* g_dev = nullptr;
bool g_registered = false;

void release_globals() {
  if (g_dev) cudaFree(g_dev);
  g_dev = nullptr;
  mcfftDestroy(&g_plan);
}

void setup_common(double* data) {
  const int64_t n = elements(g_plan) * 2;
  if (g_dev) cudaFree(g_dev);
  if (cudaMalloc(&g_dev, (size_t)n * sizeof(double)) != cudaSuccess) die("cudaMalloc", -1);
  if (cudaMemcpy(g_dev, data, (size_t)n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    die("cudaMemcpy", -1);
  if (!g_registered) {
    std::atexit(release_globals);
    g_registered = true;
  }
}

}  // namespace

COMPAT_API void mcfftExec(mcfftHandle h, MCTYPE* data) {
  const int64_t n = elements(h) * 2;
  float* w0 = static_cast<float*>(h.work);
  float* w1 = w0 + n;
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  k_d2f<<<blocks, 256>>>(data, w0, n);
  mcfftResult r = ::mcfftExec(h.plan, w0, w1, MCFFT_FORWARD, nullptr);
  if (r != MCFFT_SUCCESS) die("mcfftExec", r);
  k_f2d<<<blocks, 256>>>(w1, data, n);
}

#if MCFFT_COMPAT_DIM == 1
COMPAT_API void mcfftCreate(mcfftHandle* h, int n, int n_batch) {
  h->N = n;
  h->N_batch = n_batch;
  h->work = nullptr;
  finish_create(h, mcfftPlanCreate1d(&h->plan, n, n_batch, MCFFT_PREC_SPLIT, 0));
}
COMPAT_API void setup(double* data, int n, int n_batch) {
  mcfftCreate(&g_plan, n, n_batch);
  setup_common(data);
}
#else
COMPAT_API void mcfftCreate(mcfftHandle* h, int nx, int ny, int n_batch) {
  h->Nx = nx;
  h->Ny = ny;
  h->N_batch = n_batch;
  h->work = nullptr;
  finish_create(h, mcfftPlanCreate2d(&h->plan, nx, ny, n_batch, MCFFT_PREC_SPLIT, 0));
}
COMPAT_API void setup(double* data, int nx, int ny, int n_batch) {
  mcfftCreate(&g_plan, nx, ny, n_batch);
  setup_common(data);
}
#endif

#if MCFFT_COMPAT_DIM == 3
COMPAT_API void setup3d(double* data, int nx, int ny, int nz, int n_batch) {
  g_plan.Nx = nx;
  g_plan.Ny = ny * nz;  // elements() counts Nx * Ny * N_batch
  g_plan.N_batch = n_batch;
  g_plan.work = nullptr;
  finish_create(&g_plan, mcfftPlanCreate3d(&g_plan.plan, nx, ny, nz, n_batch, MCFFT_PREC_SPLIT, 0));
  setup_common(data);
}
#endif

COMPAT_API void mcfftDestroy(mcfftHandle* h) {
  if (h->plan) mcfftPlanDestroy(h->plan);
  if (h->work) cudaFree(h->work);
  h->plan = nullptr;
  h->work = nullptr;
}

COMPAT_API void doit(int iter) {
  for (int t = 0; t < iter; ++t) mcfftExec(g_plan, g_dev);
  if (cudaDeviceSynchronize() != cudaSuccess) die("cudaDeviceSynchronize", -1);
}

COMPAT_API void finalize(double* result) {
  const int64_t n = elements(g_plan) * 2;
  if (cudaMemcpy(result, g_dev, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    die("cudaMemcpy", -1);
}

// source/mcfft_1d_utils.cpp:88-100: glibc rand, 1e-4f * rand() / RAND_MAX
// in single precision, re then im, batch-major.
COMPAT_API void generate_data(double* data, int n, int n_batch, int seed) {
  srand((unsigned)seed);
  for (int i = 0; i < n_batch; ++i)
    for (int j = 0; j < n; ++j) {
      data[0 + j * 2 + (int64_t)i * n * 2] = 0.0001f * (float)rand() / (float)RAND_MAX;
      data[1 + j * 2 + (int64_t)i * n * 2] = 0.0001f * (float)rand() / (float)RAND_MAX;
    }
}
