/* fftw3.h -- FFTW's public double-precision complex interface over this
 * project's FP64 oracle FFT (oracle/fft64.c).  TEST INFRASTRUCTURE ONLY: FFTW
 * is not installed on these machines, and the reference's accuracy drivers
 * (benchmark/accuracy_1d.cpp:12-24, accuracy_2d.cpp:12-24) call
 * fftw_plan_dft_1d/2d(..., FFTW_FORWARD, FFTW_ESTIMATE), fftw_execute,
 * fftw_destroy_plan, fftw_malloc and fftw_free.  The names, types and
 * argument meanings are FFTW 3's documented API; the FFT behind them is the
 * oracle's own. */
#ifndef MCFFT_FFTW3_SHIM_H_
#define MCFFT_FFTW3_SHIM_H_
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct fftw_plan_s* fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#ifdef __cplusplus
}
#endif
#endif
