/* mcfft_3d_utils.h -- the reference's harness functions with their
 * signatures (reference: include/mcfft_3d_utils.h:8-11), so its drivers
 * (benchmark/accuracy_3d.cpp, benchmark/test_3d.cpp) link against
 * libmcfft_3d.so unchanged.
 *
 * setup copies the FP64 host data to the device in natural order (no host
 * permutation); doit runs the transform `iter` times in place; finalize
 * copies the result back; generate_data is the reference's glibc-rand
 * generator (source/mcfft_1d_utils.cpp:88-100).
 *
 * The reference's 3D files are its 2D files under another name
 * (include/mcfft_3d_utils.h:8 keeps the 2-argument setup); this library
 * keeps that signature and behaviour, and adds setup3d for a true 3D
 * transform.
 */
#ifndef MCFFT_3D_UTILS_H_
#define MCFFT_3D_UTILS_H_

#include "mcfft_3d_device.h"

void setup(double* data, int nx, int ny, int n_batch);
void doit(int iter);
void finalize(double* result);
void generate_data(double* data, int n, int n_batch, int seed = 42);
void setup3d(double* data, int nx, int ny, int nz, int n_batch);

#endif
