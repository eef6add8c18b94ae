// handle_caller.cpp -- TEST INFRASTRUCTURE: a caller of the reference's
// device-level API compiled against the REFERENCE's own header
// (include/mcfft_1d_device.h or include/mcfft_2d_device.h of the reference
// tree, with the HIP stand-ins of oracle/hip_stub), linked to this
// project's compat library.  It checks that a handle laid out by the
// reference's struct definition, filled by mcfftCreate and passed to
// mcfftExec BY VALUE, runs the transform: it prints the rel-L2 error of the
// in-place forward transform of the reference generator's data against the
// FP64 oracle (oracle/fft64.c), and the handle's size.
//
//   handle_caller_1d N BATCH        handle_caller_2d NX NY BATCH
//
// Built by oracle/drivers.mk (outputs in oracle/_ref/); run by
// tests/test_gpu_ref_drivers.py.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#if CALLER_DIM == 1
#include "mcfft_1d_device.h"
#else
#include "mcfft_2d_device.h"
#endif

// The compat library's generator (source/mcfft_1d_utils.cpp:88-100 there).
void generate_data(double* data, int n, int n_batch, int seed);

// CUDA runtime entry points, declared here so that no CUDA header (which
// defines its own double2) meets the reference's HIP stand-ins.
extern "C" int cudaMalloc(void** p, size_t bytes);
extern "C" int cudaFree(void* p);
extern "C" int cudaMemcpy(void* dst, const void* src, size_t bytes, int kind);
extern "C" int cudaDeviceSynchronize(void);
extern "C" int oracle_fftnd(double* data, int ndim, const int64_t* dims, int64_t batch, int sign);

int main(int argc, char** argv) {
#if CALLER_DIM == 1
  if (argc != 3) return 2;
  const int n = std::atoi(argv[1]), batch = std::atoi(argv[2]);
  const int64_t points = n;
  const int64_t dims[1] = {n};
#else
  if (argc != 4) return 2;
  const int nx = std::atoi(argv[1]), ny = std::atoi(argv[2]), batch = std::atoi(argv[3]);
  const int64_t points = (int64_t)nx * ny;
  const int64_t dims[2] = {nx, ny};
#endif
  const size_t count = (size_t)points * batch * 2;  // doubles
  std::vector<double> host(count), out(count);
  generate_data(host.data(), (int)points, batch, 42);
  void* dev = nullptr;
  if (cudaMalloc(&dev, count * sizeof(double)) != 0) return 3;
  if (cudaMemcpy(dev, host.data(), count * sizeof(double), 1 /* host to device */) != 0) return 3;

  mcfftHandle h;  // the reference's struct, with its default member values
#if CALLER_DIM == 1
  mcfftCreate(&h, n, batch);
  if (h.N != n || h.N_batch != batch) return 4;
#else
  mcfftCreate(&h, nx, ny, batch);
  if (h.Nx != nx || h.Ny != ny || h.N_batch != batch) return 4;
#endif
  mcfftHandle copy = h;  // by value, as the reference's harness passes it
  mcfftExec(copy, static_cast<MCTYPE*>(dev));
  if (cudaDeviceSynchronize() != 0) return 5;
  if (cudaMemcpy(out.data(), dev, count * sizeof(double), 2 /* device to host */) != 0) return 3;
  cudaFree(dev);

  if (oracle_fftnd(host.data(), CALLER_DIM, dims, batch, -1) != 0) return 6;
  long double num = 0, den = 0;
  for (size_t i = 0; i < count; ++i) {
    const long double d = (long double)out[i] - host[i];
    num += d * d;
    den += (long double)host[i] * host[i];
  }
  std::printf("handle_bytes %zu\n", sizeof(mcfftHandle));
  std::printf("rel_l2 %.6e\n", (double)std::sqrt((double)(num / den)));
  return 0;
}
