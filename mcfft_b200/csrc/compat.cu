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

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

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

// The handle has the reference's layout (include/mcfft_*d_device.h:18-30
// there): callers built against that header pass it by value, so its size
// and field offsets must match.  The plan and the work buffers travel in
// the reference's two spare pointer fields.
#if MCFFT_COMPAT_DIM == 1
static_assert(sizeof(mcfftHandle) == 144, "reference 1D handle layout");
static_assert(offsetof(mcfftHandle, F_real_tmp) == 128, "reference 1D handle layout");
#else
static_assert(sizeof(mcfftHandle) == 136, "reference 2D/3D handle layout");
static_assert(offsetof(mcfftHandle, F_real_tmp) == 120, "reference 2D/3D handle layout");
#endif

mcfftPlan plan_of(const mcfftHandle& h) { return reinterpret_cast<mcfftPlan>(h.F_real_tmp); }
float* work_of(const mcfftHandle& h) { return reinterpret_cast<float*>(h.F_imag_tmp); }

// Radix factorisation 16^a * R of a power of two n (R first); returns the
// entry count, or 0 when it does not fit `cap` entries.
int factorise(int64_t n, int* out, int cap) {
  int lg = 0;
  while ((int64_t(1) << lg) < n) ++lg;
  int k = 0;
  if (lg % 4) {
    if (k < cap) out[k] = 1 << (lg % 4);
    ++k;
  }
  for (int i = 0; i < lg / 4; ++i) {
    if (k < cap) out[k] = 16;
    ++k;
  }
  if (k > cap) {
    for (int i = 0; i < cap; ++i) out[i] = 0;
    return 0;
  }
  return k;
}

void clear_handle(mcfftHandle* h) {
  std::memset(static_cast<void*>(h), 0, sizeof(*h));
}

void finish_create(mcfftHandle* h, mcfftPlan plan, mcfftResult r) {
  if (r != MCFFT_SUCCESS) die("plan creation", r);
  void* work = nullptr;
  if (cudaMalloc(&work, (size_t)elements(*h) * 2 * sizeof(float) * 2) != cudaSuccess)
    die("cudaMalloc", -1);
  h->F_real_tmp = reinterpret_cast<MCTYPE*>(plan);
  h->F_imag_tmp = reinterpret_cast<MCTYPE*>(work);
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
  if (!plan_of(h) || !work_of(h)) die("mcfftExec (handle not created by mcfftCreate)", -1);
  float* w0 = work_of(h);
  float* w1 = w0 + n;
  const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  k_d2f<<<blocks, 256>>>(data, w0, n);
  mcfftResult r = ::mcfftExec(plan_of(h), w0, w1, MCFFT_FORWARD, nullptr);
  if (r != MCFFT_SUCCESS) die("mcfftExec", r);
  k_f2d<<<blocks, 256>>>(w1, data, n);
}

#if MCFFT_COMPAT_DIM == 1
COMPAT_API void mcfftCreate(mcfftHandle* h, int n, int n_batch) {
  clear_handle(h);
  h->N = n;
  h->N_batch = n_batch;
  h->n_radices = factorise(n, h->radices, 9);
  mcfftPlan plan = nullptr;
  const mcfftResult r = mcfftPlanCreate1d(&plan, n, n_batch, MCFFT_PREC_SPLIT, 0);
  finish_create(h, plan, r);
}
COMPAT_API void setup(double* data, int n, int n_batch) {
  mcfftDestroy(&g_plan);
  mcfftCreate(&g_plan, n, n_batch);
  setup_common(data);
}
#else
COMPAT_API void mcfftCreate(mcfftHandle* h, int nx, int ny, int n_batch) {
  clear_handle(h);
  h->Nx = nx;
  h->Ny = ny;
  h->N_batch = n_batch;
  h->n_radices_x = factorise(nx, h->radices_x, 3);
  h->n_radices_y = factorise(ny, h->radices_y, 3);
  mcfftPlan plan = nullptr;
  const mcfftResult r = mcfftPlanCreate2d(&plan, nx, ny, n_batch, MCFFT_PREC_SPLIT, 0);
  finish_create(h, plan, r);
}
COMPAT_API void setup(double* data, int nx, int ny, int n_batch) {
  mcfftDestroy(&g_plan);
  mcfftCreate(&g_plan, nx, ny, n_batch);
  setup_common(data);
}
#endif

#if MCFFT_COMPAT_DIM == 3
COMPAT_API void setup3d(double* data, int nx, int ny, int nz, int n_batch) {
  mcfftDestroy(&g_plan);
  clear_handle(&g_plan);
  g_plan.Nx = nx;
  g_plan.Ny = ny * nz;  // elements() counts Nx * Ny * N_batch
  g_plan.N_batch = n_batch;
  mcfftPlan plan = nullptr;
  const mcfftResult r = mcfftPlanCreate3d(&plan, nx, ny, nz, n_batch, MCFFT_PREC_SPLIT, 0);
  finish_create(&g_plan, plan, r);
  setup_common(data);
}
#endif

COMPAT_API void mcfftDestroy(mcfftHandle* h) {
  if (plan_of(*h)) mcfftPlanDestroy(plan_of(*h));
  if (work_of(*h)) cudaFree(work_of(*h));
  h->F_real_tmp = nullptr;
  h->F_imag_tmp = nullptr;
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
