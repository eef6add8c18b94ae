/* mcfft_1d_device.h -- reference-compatible device-level entry points
 * (reference: include/mcfft_1d_device.h:18-38), implemented over the C ABI in
 * mcfft.h by libmcfft_1d.so.  No HIP or rocWMMA types.
 *
 * mcfftHandle has the reference's layout field for field
 * (include/mcfft_1d_device.h:18-30 there), so that a caller compiled
 * against the reference's header -- which passes the handle to mcfftExec
 * by value -- runs unchanged against this library.  The fields keep their
 * types' sizes; their use here:
 *   N, N_batch            transform length and count, as in the reference
 *   radices, n_radices    the length's radix factorisation 16^a * R (R
 *                         first), informational
 *   mergings, n_mergings  zero (no reference-style layer merging)
 *   layer_0, layer_1      NULL (no per-layer kernel pointers)
 *   F_real, F_imag        NULL (the DFT-16 matrix lives in the plan)
 *   F_real_tmp            this library's plan (an mcfftPlan)
 *   F_imag_tmp            its device FP32 work buffers
 *
 * Differences from the reference, all deliberate:
 *  - mcfftExec takes the data in natural order (the reference required the
 *    host digit reversal of source/mcfft_1d_utils.cpp:43-59 first);
 *  - every size the core supports is accepted (the reference's table has
 *    ten 1D sizes and three 2D sides);
 *  - the plan owns device memory; mcfftDestroy releases it.
 */
#ifndef MCFFT_1D_DEVICE_H_
#define MCFFT_1D_DEVICE_H_

#include "common.h"
#include "mcfft.h"

typedef struct {
  int N, N_batch;
  int radices[9];
  int n_radices;
  int mergings[3];
  int n_mergings;
  void (*layer_0[3])(void*, MCTYPE*, MCTYPE*);
  void (*layer_1[3])(int, void*, MCTYPE*, MCTYPE*);
  MCTYPE *F_real, *F_imag;
  MCTYPE *F_real_tmp, *F_imag_tmp;
} mcfftHandle;

/* In place on device FP64 interleaved complex data, forward transform,
 * unnormalised (FFTW_FORWARD convention), natural order in and out. */
void mcfftExec(mcfftHandle plan, MCTYPE* data);
void mcfftCreate(mcfftHandle* plan, int n, int n_batch);
void mcfftDestroy(mcfftHandle* plan);

#endif
