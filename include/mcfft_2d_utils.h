/* mcfft_2d_utils.h -- the reference's harness functions with their
 * signatures (reference: include/mcfft_2d_utils.h:8-11), so its drivers
 * (benchmark/accuracy_2d.cpp, benchmark/test_2d.cpp) link against
 * libmcfft_2d.so unchanged.
 *
 * setup copies the FP64 host data to the device in natural order (no host
 * permutation); doit runs the transform `iter` times in place; finalize
 * copies the result back; generate_data is the reference's glibc-rand
 * generator (source/mcfft_1d_utils.cpp:88-100).
 */
#ifndef MCFFT_2D_UTILS_H_
#define MCFFT_2D_UTILS_H_

#include "mcfft_2d_device.h"

void setup(double* data, int nx, int ny, int n_batch);
void doit(int iter);
void finalize(double* result);
void generate_data(double* data, int n, int n_batch, int seed = 42);

#endif
