// queue.h -- host interface of the persistent batch kernel.
#pragma once
#include <cuda_runtime.h>

#include "fft_queue.cuh"
#include "tile_pass.h"

namespace mcfft {

// Variant index of a tile pass in the batch kernel, or -1 if it has none.
int queue_variant(const TileKernel& k);
// Queue entry of a tile pass for one exec: tensor maps over in/out, tables
// for direction `dir`; dependencies unset.  False if encoding fails.
bool fill_qpass(const TilePass& tp, int dir, const void* in, void* out, QPass* q);
// Cooperative launch (queue_max_grid has configured the kernel).
cudaError_t launch_queue(const QArgs& a, int grid, bool split, cudaStream_t st);
// CTAs of the batch kernel that can be resident at once (0 on error); also
// sets the kernel's shared-memory limit.
int queue_max_grid(int sms, bool split);

// A fused four-step kernel (both passes of one 1D transform group in one
// launch) for passes on tile variants v1 (with the four-step twiddle) and v2.
struct FusedKernel {
  bool split;
  int v1, v2;
  const void* fn;
  int smem_bytes;
};
const FusedKernel* find_fused(bool split, int v1, int v2);
// The same launch and occupancy query for any kernel over a QArgs block.
cudaError_t launch_queue_fn(const void* fn, int smem_bytes, const QArgs& a, int grid,
                            cudaStream_t st);
int queue_max_grid_fn(const void* fn, int smem_bytes, int sms);

}  // namespace mcfft
