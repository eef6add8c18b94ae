// tile_pass.h -- host interface of the TMA-fed pass kernel.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fft_tile.cuh"
#include "layout.h"

namespace mcfft {

struct TileKernel {
  const void* fn;
  int L, R, C;
  bool posttw, split;
  int nthreads;
  int smem_bytes;
  int tmem_cols;
  int tile_points;
  bool in16;  // split form: FP16 input staging (FP32 otherwise); plain: always
};

// Split-form variants (tile_split.cu).
const std::vector<TileKernel>& split_registry();

// One pass of a plan executed by the TMA-fed kernel.
struct TilePass {
  const TileKernel* k = nullptr;
  layout::PassLayout lay;
  TileArgs args{};  // everything except tensor maps and per-direction tables
  int grid = 1;
  const float4* tw[2] = {nullptr, nullptr};
  const float2* tail[2] = {nullptr, nullptr};
  const float2* post_a[2] = {nullptr, nullptr};
  const float2* post_b[2] = {nullptr, nullptr};
  const uint4* bmat[2] = {nullptr, nullptr};
  const uint4* bmat_lo[2] = {nullptr, nullptr};
};

const TileKernel* find_tile_kernel(int L, bool posttw, bool split, int tile_points, bool in16);
// unsw: bit 0 / bit 1 -- input / output staging without TMA swizzle (filled
// by row gathers, see layout::make_staging).
bool tile_layout(layout::PassLayout* out, int L, int R, int C, layout::Kind ik, layout::Kind ok,
                 int in_elem, int out_elem, int64_t isp, int64_t isc, int64_t iso, int64_t osp,
                 int64_t osc, int64_t oso, int64_t ncols, int64_t nouter, std::string* err,
                 int unsw = 0);
bool tile_check_encode(const layout::Staging& s, const void* probe);
bool tile_encode(CUtensorMap* map, const layout::Staging& s, const void* base);
void fill_tile_args(TilePass* tp);
// pdl: launch with programmatic stream serialization (the kernel's setup
// may overlap the previous kernel on the stream; it waits for that kernel's
// completion before touching `in` or `out`).
cudaError_t launch_tile_pass(const TilePass& tp, const void* in, void* out, int dir,
                             cudaStream_t st, bool pdl = false);

// DFT-16 embedding times `scale` (a power of two) in the 64-byte-swizzled
// K-major layout the tile kernel reads (row j = output component, K = 16
// interleaved complex inputs).
cudaError_t gen_dft16_sw64(void* hi, void* lo, int sign, double scale, cudaStream_t st);
// Stage twiddle rows (scale * W^(k R'), k < 16, chunked and swizzled for
// the tile kernel), W = exp(sign 2 pi i / modulus), R' < rows.
cudaError_t gen_stage_rows(float4* dst, int64_t rows, int64_t modulus, int sign, double scale,
                           cudaStream_t st);

}  // namespace mcfft
