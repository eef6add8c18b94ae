/* mcfft_3d_device.h -- reference-compatible device-level entry points
 * (reference: include/mcfft_3d_device.h:37-38), implemented over the C ABI in mcfft.h by
 * libmcfft_3d.so.  No HIP or rocWMMA types.
 *
 * Differences from the reference, all deliberate:
 *  - mcfftExec takes the data in natural order (the reference required the
 *    host digit reversal of source/mcfft_1d_utils.cpp:43-59 first);
 *  - every size the core supports is accepted (the reference's table has
 *    ten 1D sizes and three 2D sides);
 *  - the plan owns device memory; mcfftDestroy releases it.
 */
#ifndef MCFFT_3D_DEVICE_H_
#define MCFFT_3D_DEVICE_H_

#include "common.h"
#include "mcfft.h"

typedef struct {
  int Nx, Ny, N_batch;
  mcfftPlan plan;   /* split-form plan (FP32 operands on the device) */
  void* work;       /* device FP32 staging, 2 buffers */
} mcfftHandle;

/* In place on device FP64 interleaved complex data, forward transform,
 * unnormalised (FFTW_FORWARD convention), natural order in and out. */
void mcfftExec(mcfftHandle plan, MCTYPE* data);
void mcfftCreate(mcfftHandle* plan, int nx, int ny, int n_batch);
void mcfftDestroy(mcfftHandle* plan);

#endif
