/* common.h -- element type of the reference-compatible harness
 * (reference: include/common.h:4-5, FP64 data).  The device transform runs
 * in the split hi+lo form (FP32-level accuracy); the harness converts on the
 * device. */
#ifndef MCFFT_COMMON_H_
#define MCFFT_COMMON_H_

typedef double MCTYPE;

#endif
