/* fftw_shim.c -- FFTW-named wrappers over oracle_fftnd (oracle/fft64.c).
 * TEST INFRASTRUCTURE ONLY; see fftw3.h. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fftw3.h"

int oracle_fftnd(double* data, int ndim, const int64_t* dims, int64_t batch, int sign);

struct fftw_plan_s {
  int ndim;
  int64_t dims[3];
  int64_t total;
  double* in;
  double* out;
  int sign;
};

void* fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void* p) { free(p); }

static fftw_plan make(int ndim, const int* d, fftw_complex* in, fftw_complex* out, int sign) {
  fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
  p->ndim = ndim;
  p->total = 1;
  for (int i = 0; i < ndim; ++i) {
    p->dims[i] = d[i];
    p->total *= d[i];
  }
  p->in = (double*)in;
  p->out = (double*)out;
  p->sign = sign;
  return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned f) {
  (void)f;
  return make(1, &n, in, out, sign);
}
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned f) {
  int d[2] = {n0, n1};
  (void)f;
  return make(2, d, in, out, sign);
}
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned f) {
  int d[3] = {n0, n1, n2};
  (void)f;
  return make(3, d, in, out, sign);
}

void fftw_execute(const fftw_plan p) {
  if (p->out != p->in) memcpy(p->out, p->in, sizeof(double) * 2 * (size_t)p->total);
  oracle_fftnd(p->out, p->ndim, p->dims, 1, p->sign);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
