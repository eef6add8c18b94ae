/* Minimal stand-in for <hip/hip_runtime.h>, TEST INFRASTRUCTURE ONLY: lets
 * the reference's unchanged drivers (benchmark/accuracy_*.cpp) compile with
 * g++ against its own headers (include/mcfft_*_device.h includes this
 * file), so they can be linked to this project's compat libraries.  Only
 * the vector type the reference's common.h names is provided. */
#ifndef MCFFT_HIP_STUB_RUNTIME_H_
#define MCFFT_HIP_STUB_RUNTIME_H_
struct double2 { double x, y; };
#endif
