// mcfft_api.cu -- plan construction and execution behind include/mcfft.h.
//
// Replaces the reference's mcfftCreate / mcfftExec
// (source/mcfft_1d_device.cpp:596-790, source/mcfft_2d_device.cpp:594-695):
// instead of a fixed size->schedule switch (ten 1D sizes, three 2D sides)
// the plan decomposes any power-of-two shape into HBM passes, each a
// length-L transform (L = 16^a * R) along one axis, and picks a tile shape
// for each pass from the instantiated kernel variants.
//
//   1D, n <= 8192        one row pass
//   1D, n > 8192         four-step: n = n1 * n2; pass 1 = n1-point column
//                        transforms (stride n2) with the W_n^(k1 n2)
//                        twiddle fused into their epilogue, into a scratch
//                        buffer; pass 2 = n2-point row transforms written
//                        with stride n1 (natural order output)
//   2D (nx, ny)          row pass (ny), then in-place column pass (nx)
//   3D (nx, ny, nz)      row pass (nz), column passes (ny, then nx)
//
// All tables (stage twiddles, tail twiddles, four-step twiddles, the DFT-16
// embedding) are generated in FP64 on the GPU at plan time for both
// directions.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/mcfft.h"
#include "mcfft_internal.h"
#include "tile_pass.h"

namespace mcfft {
namespace {

constexpr int kVersion = 100;  // 0.1.0

enum Buf { kUserIn = 0, kUserOut = 1, kScratch = 2 };

struct Pass {
  bool tiled = false;  // TMA-fed kernel (tile_pass) instead of the direct one
  TilePass tp;
  const PassKernel* k = nullptr;
  PassArgs a{};
  int in_buf = kUserIn, out_buf = kUserOut;
  int in_f16 = 1, out_f16 = 1;   // element types at this pass's ends
  int64_t in_off = 0, out_off = 0;  // element offsets into the buffers
  int grid = 0;
  const float2* tw[2] = {nullptr, nullptr};
  const float2* tail[2] = {nullptr, nullptr};
  const float2* plo[2] = {nullptr, nullptr};
  const float2* phi[2] = {nullptr, nullptr};
};

}  // namespace
}  // namespace mcfft

struct mcfftPlan_st {
  int device = 0;
  int sms = 148;
  bool split = false;
  unsigned flags = 0;
  std::vector<mcfft::Pass> passes;
  std::vector<void*> allocs;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  const uint4* bmat[2] = {nullptr, nullptr};
  const uint4* bmat_lo[2] = {nullptr, nullptr};
  const uint4* bsw64[2] = {nullptr, nullptr};     // same matrices, 64B-swizzled layout
  const uint4* bsw64_lo[2] = {nullptr, nullptr};
  int* status = nullptr;
  cudaStream_t last_stream = nullptr;
  mcfftPlanInfo info{};
};

namespace mcfft {
namespace {

bool is_pow2(int64_t x) { return x > 0 && (x & (x - 1)) == 0; }
int ilog2(int64_t x) {
  int r = 0;
  while ((int64_t(1) << r) < x) ++r;
  return r;
}

mcfftResult cuda_fail(cudaError_t e) {
  if (e == cudaErrorMemoryAllocation) return MCFFT_ALLOC_FAILED;
  return e == cudaSuccess ? MCFFT_SUCCESS : MCFFT_CUDA_ERROR;
}

template <class T>
mcfftResult plan_alloc(mcfftPlan p, T** out, size_t bytes) {
  void* d = nullptr;
  cudaError_t e = cudaMalloc(&d, bytes < 16 ? 16 : bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_ALLOC_FAILED;
  }
  p->allocs.push_back(d);
  *out = static_cast<T*>(d);
  return MCFFT_SUCCESS;
}

int ctas_per_sm(const PassKernel& k) {
  int occ = 0;
  cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k.smem_bytes);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k.fn, 256, k.smem_bytes) != cudaSuccess) {
    cudaGetLastError();
    occ = 1;
  }
  int tmem_limit = 512 / k.tmem_cols;
  return std::max(1, std::min(occ, tmem_limit));
}

// Tile-size override for experiments: MCFFT_TILE_POINTS (0 = default).
int64_t tile_points_env() {
  const char* s = std::getenv("MCFFT_TILE_POINTS");
  return s ? std::atoll(s) : 0;
}

struct PassSpec {
  int64_t L;
  bool colfast, posttw;
  int64_t in_sp, in_sc, in_so, out_sp, out_sc, out_so;
  int64_t ncols, nouter;
  int in_buf, out_buf;
  int64_t postN;
  int in_f16, out_f16;
  int64_t in_off, out_off;
};

// Tables shared by both kernel families: stage twiddles [R'][k] (1/16 per
// stage; skipped when tw is null) and radix-R twiddles [v][k] (1/R), for
// both directions.
mcfftResult make_stage_tables(mcfftPlan p, int L, int R, const float2* tw[2],
                              const float2* tail[2]) {
  int nst = 0;
  for (int64_t t = L / R; t > 1; t >>= 4) ++nst;
  int64_t tw_count = 0;
  {
    int64_t Ls = L / R;
    for (int st = 0; st < nst - 1; ++st) { tw_count += Ls; Ls >>= 4; }
  }
  for (int dir = 0; dir < 2; ++dir) {
    const int sign = dir == 0 ? -1 : 1;
    if (tw_count > 0 && tw) {
      float2* t;
      mcfftResult r = plan_alloc(p, &t, sizeof(float2) * tw_count);
      if (r) return r;
      int64_t off = 0, Ls = L / R;
      for (int st = 0; st < nst - 1; ++st) {
        cudaError_t e = gen_twiddle_table(t + off, Ls, 0, 16, 0, Ls, sign, 1.0 / 16.0, 0);
        if (e != cudaSuccess) return cuda_fail(e);
        off += Ls;
        Ls >>= 4;
      }
      tw[dir] = t;
    }
    if (R > 1) {
      float2* t;
      mcfftResult r = plan_alloc(p, &t, sizeof(float2) * L);
      if (r) return r;
      cudaError_t e = gen_twiddle_table(t, L, 0, R, 0, L, sign, 1.0 / R, 0);
      if (e != cudaSuccess) return cuda_fail(e);
      tail[dir] = t;
    }
  }
  return MCFFT_SUCCESS;
}

// Stage twiddle rows of the tile kernel, both directions: for every stage
// but the last, W^(k R') with W = exp(-+2 pi i / L_s), R' < L_s/16, k < 16.
mcfftResult make_stage_rows(mcfftPlan p, int L, int R, double scale, const float4* tw[2]) {
  int nst = 0;
  for (int64_t t = L / R; t > 1; t >>= 4) ++nst;
  int64_t count = 0;
  {
    int64_t Ls = L / R;
    for (int st = 0; st < nst - 1; ++st) { count += Ls / 16; Ls >>= 4; }
  }
  if (count == 0) return MCFFT_SUCCESS;
  for (int dir = 0; dir < 2; ++dir) {
    float4* t;
    mcfftResult r = plan_alloc(p, &t, sizeof(float4) * 8 * count);
    if (r) return r;
    int64_t off = 0, Ls = L / R;
    for (int st = 0; st < nst - 1; ++st) {
      cudaError_t e = gen_stage_rows(t + 8 * off, Ls / 16, Ls, dir == 0 ? -1 : 1, scale, 0);
      if (e != cudaSuccess) return cuda_fail(e);
      off += Ls / 16;
      Ls >>= 4;
    }
    tw[dir] = t;
  }
  return MCFFT_SUCCESS;
}

// Builds a pass on the TMA-fed kernel.  Returns MCFFT_UNSUPPORTED_SIZE when
// the shape is outside what that kernel handles (the caller falls back).
mcfftResult add_tile_pass(mcfftPlan p, const PassSpec& s) {
  if (std::getenv("MCFFT_NO_TILE")) return MCFFT_UNSUPPORTED_SIZE;
  layout::Kind ik, ok;
  if (s.in_sp == 1) ik = layout::ROW;
  else if (s.in_sc == 1) ik = layout::COL;
  else return MCFFT_UNSUPPORTED_SIZE;
  if (s.out_sp == 1) ok = layout::ROW;
  else if (s.out_sc == 1) ok = layout::COL;
  else return MCFFT_UNSUPPORTED_SIZE;
  // Tile size: plain form 16K points (one CTA per SM) first unless
  // MCFFT_TILE_POINTS says otherwise, the other size if that variant or its
  // layout is missing; split form 8K points (its FP32 staging is twice as
  // large per point).
  int first = 16384;
  if (const char* e = std::getenv("MCFFT_TILE_POINTS")) first = std::atoi(e);
  const int order[2] = {p->split ? 8192 : first,
                        p->split ? 8192 : (first == 16384 ? 8192 : 16384)};
  const int in_elem = s.in_f16 ? 4 : 8, out_elem = s.out_f16 ? 4 : 8;
  Pass ps;
  ps.tiled = true;
  TilePass& tp = ps.tp;
  const TileKernel* k = nullptr;
  for (int oi = 0; oi < 2 && !k; ++oi) {
    const TileKernel* cand =
        find_tile_kernel((int)s.L, s.posttw, p->split, order[oi], s.in_f16 != 0);
    if (!cand) continue;
    if (!p->split && (in_elem != 4 || out_elem != 4)) continue;
    std::string err;
    if (!tile_layout(&tp.lay, cand->L, cand->R, cand->C, ik, ok, in_elem, out_elem, s.in_sp,
                     s.in_sc, s.in_so, s.out_sp, s.out_sc, s.out_so, s.ncols, s.nouter, &err))
      continue;
    if (!tile_check_encode(tp.lay.in, p->status) || !tile_check_encode(tp.lay.out, p->status))
      continue;
    k = cand;
  }
  if (!k) return MCFFT_UNSUPPORTED_SIZE;
  tp.k = k;
  fill_tile_args(&tp);
  TileArgs& a = tp.args;
  a.col_blocks = (s.ncols + k->C - 1) / k->C;
  a.ntiles = a.col_blocks * s.nouter;
  a.out_scale = 1.0f;  // unused: the plain form's last 1/16 is in the DFT-16 matrix,
                       // the split form derives its output factor per tile
  a.status = p->status;
  // tables
  uint2* items;
  uint32_t* epi;
  mcfftResult r = plan_alloc(p, &items, tp.lay.item_tab.size() * sizeof(uint32_t));
  if (!r) r = plan_alloc(p, &epi, tp.lay.epi_tab.size() * sizeof(uint32_t));
  if (r) return r;
  cudaError_t e = cudaMemcpy(items, tp.lay.item_tab.data(), tp.lay.item_tab.size() * 4,
                             cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(epi, tp.lay.epi_tab.data(), tp.lay.epi_tab.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e);
  a.item_tab = items;
  a.epi_tab = epi;
  r = make_stage_tables(p, k->L, k->R, nullptr, tp.tail);
  if (r) return r;
  // stage rows: the plain form's 1/16 is in its DFT-16 matrix, the split
  // form's in the rows
  r = make_stage_rows(p, k->L, k->R, p->split ? 1.0 / 16.0 : 1.0, tp.tw);
  if (r) return r;
  if (s.posttw) {
    // two-level table for W_N^e: lo[e & (2^sh - 1)] * hi[e >> sh]
    const int lg = ilog2(s.postN), sh = (lg + 1) / 2;
    const int64_t nlo = int64_t(1) << sh, nhi = s.postN >> sh;
    for (int dir = 0; dir < 2; ++dir) {
      const int sign = dir == 0 ? -1 : 1;
      float2 *lo, *hi;
      r = plan_alloc(p, &lo, sizeof(float2) * nlo);
      if (!r) r = plan_alloc(p, &hi, sizeof(float2) * nhi);
      if (r) return r;
      cudaError_t e2 = gen_twiddle_table(lo, nlo, 1, 0, 0, s.postN, sign, 1.0, 0);
      if (e2 == cudaSuccess) e2 = gen_twiddle_table(hi, nhi, 1, 0, sh, s.postN, sign, 1.0, 0);
      if (e2 != cudaSuccess) return cuda_fail(e2);
      tp.post_a[dir] = lo;
      tp.post_b[dir] = hi;
    }
    a.post_mask = (uint64_t)s.postN - 1;
    a.post_shift = (uint32_t)sh;
  }
  for (int dir = 0; dir < 2; ++dir) {
    tp.bmat[dir] = p->bsw64[dir];
    tp.bmat_lo[dir] = p->bsw64_lo[dir];
  }
  int occ = 1;
  cudaFuncSetAttribute(k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k->smem_bytes);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k->fn, k->nthreads, k->smem_bytes) !=
      cudaSuccess) {
    cudaGetLastError();
    occ = 1;
  }
  occ = std::max(1, std::min(occ, 512 / k->tmem_cols));
  tp.grid = (int)std::min<int64_t>(a.ntiles, (int64_t)p->sms * occ);
  ps.in_buf = s.in_buf; ps.out_buf = s.out_buf;
  ps.in_f16 = s.in_f16; ps.out_f16 = s.out_f16;
  ps.in_off = s.in_off; ps.out_off = s.out_off;
  p->passes.push_back(ps);
  return MCFFT_SUCCESS;
}

mcfftResult add_pass(mcfftPlan p, const PassSpec& s) {
  {
    mcfftResult tr = add_tile_pass(p, s);
    if (tr != MCFFT_UNSUPPORTED_SIZE) return tr;
  }
  const PassKernel* k =
      pick_pass_kernel((int)s.L, s.colfast, s.posttw, p->split, s.ncols, tile_points_env());
  if (!k) return MCFFT_UNSUPPORTED_SIZE;
  Pass ps;
  ps.k = k;
  PassArgs& a = ps.a;
  a.in_sp = s.in_sp; a.in_sc = s.in_sc; a.in_so = s.in_so;
  a.out_sp = s.out_sp; a.out_sc = s.out_sc; a.out_so = s.out_so;
  a.ncols = s.ncols;
  a.col_blocks = (s.ncols + k->C - 1) / k->C;
  a.ntiles = a.col_blocks * s.nouter;
  a.out_scale = 1.0f / 16.0f;
  a.split_in_f16 = s.in_f16;
  a.status = p->status;
  ps.in_buf = s.in_buf; ps.out_buf = s.out_buf;
  ps.in_f16 = s.in_f16; ps.out_f16 = s.out_f16;
  ps.in_off = s.in_off; ps.out_off = s.out_off;
  ps.grid = (int)std::min<int64_t>(a.ntiles, (int64_t)p->sms * ctas_per_sm(*k));
  if (ps.grid < 1) ps.grid = 1;

  const int L = k->L, R = k->R;
  int nst = 0;
  for (int64_t t = L / R; t > 1; t >>= 4) ++nst;
  // stage tables for stages 0..nst-2 (the last stage has R' = 0)
  int64_t tw_count = 0;
  {
    int64_t Ls = L / R;
    for (int st = 0; st < nst - 1; ++st) { tw_count += Ls; Ls >>= 4; }
  }
  for (int dir = 0; dir < 2; ++dir) {
    const int sign = dir == 0 ? -1 : 1;
    if (tw_count > 0) {
      float2* t;
      mcfftResult r = plan_alloc(p, &t, sizeof(float2) * tw_count);
      if (r) return r;
      int64_t off = 0, Ls = L / R;
      for (int st = 0; st < nst - 1; ++st) {
        cudaError_t e = gen_twiddle_table(t + off, Ls, 0, 16, 0, Ls, sign, 1.0 / 16.0, 0);
        if (e != cudaSuccess) return cuda_fail(e);
        off += Ls;
        Ls >>= 4;
      }
      ps.tw[dir] = t;
    }
    if (R > 1) {
      float2* t;
      mcfftResult r = plan_alloc(p, &t, sizeof(float2) * L);
      if (r) return r;
      cudaError_t e = gen_twiddle_table(t, L, 0, R, 0, L, sign, 1.0 / R, 0);
      if (e != cudaSuccess) return cuda_fail(e);
      ps.tail[dir] = t;
    }
    if (s.posttw) {
      const int lg = ilog2(s.postN), sh = lg / 2;
      const int64_t nlo = int64_t(1) << sh, nhi = s.postN >> sh;
      float2 *lo, *hi;
      mcfftResult r = plan_alloc(p, &lo, sizeof(float2) * nlo);
      if (r) return r;
      r = plan_alloc(p, &hi, sizeof(float2) * nhi);
      if (r) return r;
      cudaError_t e = gen_twiddle_table(lo, nlo, 1, 0, 0, s.postN, sign, 1.0, 0);
      if (e == cudaSuccess) e = gen_twiddle_table(hi, nhi, 1, 0, sh, s.postN, sign, 1.0, 0);
      if (e != cudaSuccess) return cuda_fail(e);
      ps.plo[dir] = lo;
      ps.phi[dir] = hi;
      a.post_shift = (uint32_t)sh;
      a.post_mask = (uint64_t)s.postN - 1;
    }
  }
  p->passes.push_back(ps);
  return MCFFT_SUCCESS;
}

constexpr int64_t kMaxSinglePass = 8192;

// Appends the passes of one transform group.  `in_buf/out_buf` and offsets
// locate it inside the user's buffers; the first pass reads in_buf, the
// last writes out_buf.
mcfftResult build_group(mcfftPlan p, int ndim, const int64_t* dims, int64_t batch,
                        int64_t in_off, int64_t out_off, int* scale_log2) {
  const bool split = p->split;
  const int in_f16 = split ? ((p->flags & MCFFT_FLAG_INPUT_F16) ? 1 : 0) : 1;
  const int mid_f16 = split ? 0 : 1;
  int64_t total = 1;
  for (int d = 0; d < ndim; ++d) {
    if (!is_pow2(dims[d]) || dims[d] < 16) return MCFFT_UNSUPPORTED_SIZE;
    total *= dims[d];
  }
  *scale_log2 = split ? 0 : -ilog2(total);
  if (ndim == 1) {
    const int64_t n = dims[0];
    if (n <= kMaxSinglePass) {
      PassSpec s{n, false, false, 1, n, 0, 1, n, 0, batch, 1, kUserIn, kUserOut, 0,
                 in_f16, split ? 0 : 1, in_off, out_off};
      return add_pass(p, s);
    }
    if (n > kMaxSinglePass * kMaxSinglePass) return MCFFT_UNSUPPORTED_SIZE;
    const int lg = ilog2(n);
    int lg1 = lg / 2;
    if (const char* e = std::getenv("MCFFT_FOURSTEP_N1")) lg1 = ilog2(std::atoll(e));
    const int64_t n1 = int64_t(1) << lg1, n2 = n >> lg1;
    if (n1 < 16 || n2 < 16 || n1 > kMaxSinglePass || n2 > kMaxSinglePass)
      return MCFFT_UNSUPPORTED_SIZE;
    // pass 1: columns n2, points n1 at stride n2, four-step twiddle
    PassSpec s1{n1, true, true, n2, 1, n, n2, 1, n, n2, batch, kUserIn, kScratch, n,
                in_f16, mid_f16, in_off, 0};
    mcfftResult r = add_pass(p, s1);
    if (r) return r;
    // pass 2: rows k1 (stride n2) of n2 points; output X[k1 + n1 k2]
    PassSpec s2{n2, false, false, 1, n2, n, n1, 1, n, n1, batch, kScratch, kUserOut, 0,
                mid_f16, split ? 0 : 1, 0, out_off};
    r = add_pass(p, s2);
    if (r) return r;
    const size_t need = (size_t)n * batch * (split ? 8 : 4);
    p->scratch_bytes = std::max(p->scratch_bytes, need);
    return MCFFT_SUCCESS;
  }
  for (int d = 0; d < ndim; ++d)
    if (dims[d] > kMaxSinglePass) return MCFFT_UNSUPPORTED_SIZE;
  if (ndim == 2) {
    const int64_t nx = dims[0], ny = dims[1];
    PassSpec s1{ny, false, false, 1, ny, 0, 1, ny, 0, nx * batch, 1, kUserIn, kUserOut, 0,
                in_f16, mid_f16, in_off, out_off};
    mcfftResult r = add_pass(p, s1);
    if (r) return r;
    PassSpec s2{nx, true, false, ny, 1, nx * ny, ny, 1, nx * ny, ny, batch, kUserOut, kUserOut,
                0, mid_f16, mid_f16, out_off, out_off};
    return add_pass(p, s2);
  }
  if (ndim == 3) {
    const int64_t nx = dims[0], ny = dims[1], nz = dims[2];
    PassSpec s1{nz, false, false, 1, nz, 0, 1, nz, 0, nx * ny * batch, 1, kUserIn, kUserOut, 0,
                in_f16, mid_f16, in_off, out_off};
    mcfftResult r = add_pass(p, s1);
    if (r) return r;
    PassSpec s2{ny, true, false, nz, 1, ny * nz, nz, 1, ny * nz, nz, nx * batch, kUserOut,
                kUserOut, 0, mid_f16, mid_f16, out_off, out_off};
    r = add_pass(p, s2);
    if (r) return r;
    PassSpec s3{nx, true, false, ny * nz, 1, total, ny * nz, 1, total, ny * nz, batch, kUserOut,
                kUserOut, 0, mid_f16, mid_f16, out_off, out_off};
    return add_pass(p, s3);
  }
  return MCFFT_INVALID_VALUE;
}

mcfftResult plan_begin(mcfftPlan* out, mcfftPrecision prec, unsigned flags, mcfftPlan* made) {
  if (!out) return MCFFT_INVALID_VALUE;
  *out = nullptr;
  if (prec != MCFFT_PREC_FP16 && prec != MCFFT_PREC_SPLIT) return MCFFT_INVALID_VALUE;
  if ((flags & MCFFT_FLAG_INPUT_F16) && prec != MCFFT_PREC_SPLIT) return MCFFT_INVALID_VALUE;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return MCFFT_NO_DEVICE;
  }
  mcfftPlan p = new (std::nothrow) mcfftPlan_st();
  if (!p) return MCFFT_ALLOC_FAILED;
  cudaGetDevice(&p->device);
  cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, p->device);
  p->split = prec == MCFFT_PREC_SPLIT;
  p->flags = flags;
  p->info.precision = (int)prec;
  mcfftResult r = plan_alloc(p, &p->status, sizeof(int));
  if (!r) r = cuda_fail(cudaMemset(p->status, 0, sizeof(int)));
  for (int dir = 0; dir < 2 && !r; ++dir) {
    uint4 *hi = nullptr, *lo = nullptr;
    r = plan_alloc(p, &hi, 2048);
    if (!r && p->split) r = plan_alloc(p, &lo, 2048);
    if (!r) r = cuda_fail(gen_dft16_embedding(hi, lo, dir == 0 ? -1 : 1, 0));
    p->bmat[dir] = hi;
    p->bmat_lo[dir] = lo;
    uint4 *hs = nullptr, *ls = nullptr;
    if (!r) r = plan_alloc(p, &hs, 2048);
    if (!r && p->split) r = plan_alloc(p, &ls, 2048);
    // The tile kernel's plain form folds the 1/16 stage scale into the
    // matrix (exact: a power of two); the split form keeps it unscaled so
    // the low part stays in FP16's normal range.
    if (!r) r = cuda_fail(gen_dft16_sw64(hs, ls, dir == 0 ? -1 : 1, p->split ? 1.0 : 1.0 / 16.0, 0));
    p->bsw64[dir] = hs;
    p->bsw64_lo[dir] = ls;
  }
  if (r) {
    mcfftPlanDestroy(p);
    return r;
  }
  *made = p;
  return MCFFT_SUCCESS;
}

mcfftResult plan_finish(mcfftPlan p, mcfftPlan* out) {
  mcfftResult r = MCFFT_SUCCESS;
  if (p->scratch_bytes) r = plan_alloc(p, &p->scratch, p->scratch_bytes);
  if (!r) r = cuda_fail(cudaDeviceSynchronize());
  if (r) {
    mcfftPlanDestroy(p);
    return r;
  }
  p->info.num_passes = (int)p->passes.size();
  p->info.workspace_bytes = (int64_t)p->scratch_bytes;
  *out = p;
  return MCFFT_SUCCESS;
}

}  // namespace
}  // namespace mcfft

using namespace mcfft;

extern "C" {

mcfftResult mcfftPlanCreateBatch(mcfftPlan* plan, const mcfftDesc* descs, int count,
                                 mcfftPrecision precision, unsigned flags) {
  if (!plan || !descs || count <= 0) return MCFFT_INVALID_VALUE;
  for (int i = 0; i < count; ++i)
    if (descs[i].ndim < 1 || descs[i].ndim > 3 || descs[i].batch < 1 || descs[i].in_offset < 0 ||
        descs[i].out_offset < 0)
      return MCFFT_INVALID_VALUE;
  mcfftPlan p = nullptr;
  mcfftResult r = plan_begin(plan, precision, flags, &p);
  if (r) return r;
  int64_t elements = 0;
  for (int i = 0; i < count && !r; ++i) {
    int sl = 0;
    r = build_group(p, descs[i].ndim, descs[i].dims, descs[i].batch, descs[i].in_offset,
                    descs[i].out_offset, &sl);
    int64_t t = descs[i].batch;
    for (int d = 0; d < descs[i].ndim; ++d) t *= descs[i].dims[d];
    elements += t;
    if (i == 0) {
      p->info.ndim = descs[0].ndim;
      for (int d = 0; d < 3; ++d) p->info.dims[d] = d < descs[0].ndim ? descs[0].dims[d] : 1;
      p->info.batch = descs[0].batch;
      p->info.scale_log2 = sl;
    } else if (sl != p->info.scale_log2) {
      p->info.scale_log2 = 1;  // mixed scales: 1 flags "per transform"
    }
  }
  if (r) {
    mcfftPlanDestroy(p);
    return r;
  }
  p->info.num_descs = count;
  p->info.elements = elements;
  const int in_b = p->split ? ((flags & MCFFT_FLAG_INPUT_F16) ? 4 : 8) : 4;
  p->info.in_bytes = elements * in_b;
  p->info.out_bytes = elements * (p->split ? 8 : 4);
  return plan_finish(p, plan);
}

mcfftResult mcfftPlanCreate1d(mcfftPlan* plan, int64_t n, int64_t batch, mcfftPrecision precision,
                              unsigned flags) {
  mcfftDesc d{1, {n, 1, 1}, batch, 0, 0};
  return mcfftPlanCreateBatch(plan, &d, 1, precision, flags);
}

mcfftResult mcfftPlanCreate2d(mcfftPlan* plan, int64_t nx, int64_t ny, int64_t batch,
                              mcfftPrecision precision, unsigned flags) {
  mcfftDesc d{2, {nx, ny, 1}, batch, 0, 0};
  return mcfftPlanCreateBatch(plan, &d, 1, precision, flags);
}

mcfftResult mcfftPlanCreate3d(mcfftPlan* plan, int64_t nx, int64_t ny, int64_t nz, int64_t batch,
                              mcfftPrecision precision, unsigned flags) {
  mcfftDesc d{3, {nx, ny, nz}, batch, 0, 0};
  return mcfftPlanCreateBatch(plan, &d, 1, precision, flags);
}

mcfftResult mcfftExec(mcfftPlan p, const void* in, void* out, int direction, void* stream) {
  if (!p) return MCFFT_INVALID_PLAN;
  if (!in || !out) return MCFFT_INVALID_VALUE;
  if (direction != MCFFT_FORWARD && direction != MCFFT_INVERSE) return MCFFT_INVALID_VALUE;
  const int dir = direction == MCFFT_FORWARD ? 0 : 1;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (auto& ps : p->passes) {
    PassArgs a = ps.a;
    auto base = [&](int b) -> char* {
      return b == kUserIn ? (char*)const_cast<void*>(in) : b == kUserOut ? (char*)out : (char*)p->scratch;
    };
    const int ib = p->split ? (ps.in_f16 ? 4 : 8) : 4;
    const int ob = p->split ? (ps.out_f16 ? 4 : 8) : 4;
    a.in = base(ps.in_buf) + ps.in_off * ib;
    a.out = base(ps.out_buf) + ps.out_off * ob;
    if (ps.tiled) {
      cudaError_t e = launch_tile_pass(ps.tp, a.in, a.out, dir, st);
      if (e == cudaSuccess && std::getenv("MCFFT_DEBUG_SYNC")) {
        e = cudaStreamSynchronize(st);
        fprintf(stderr, "[mcfft] tile pass L=%d R=%d C=%d grid=%d tiles=%lld: %s\n", ps.tp.k->L,
                ps.tp.k->R, ps.tp.k->C, ps.tp.grid, (long long)ps.tp.args.ntiles,
                cudaGetErrorString(e));
      }
      if (e != cudaSuccess) {
        cudaGetLastError();
        return MCFFT_CUDA_ERROR;
      }
      continue;
    }
    a.tw = ps.tw[dir];
    a.tail_tw = ps.tail[dir];
    a.post_lo = ps.plo[dir];
    a.post_hi = ps.phi[dir];
    a.bmat = p->bmat[dir];
    a.bmat_lo = p->bmat_lo[dir];
    a.inverse = dir;
    cudaError_t e = launch_pass(*ps.k, a, ps.grid, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return MCFFT_CUDA_ERROR;
    }
  }
  p->last_stream = st;
  return MCFFT_SUCCESS;
}

mcfftResult mcfftPlanCheckStatus(mcfftPlan p) {
  if (!p) return MCFFT_INVALID_PLAN;
  int h = 0;
  if (cudaStreamSynchronize(p->last_stream) != cudaSuccess) return MCFFT_CUDA_ERROR;
  if (cudaMemcpy(&h, p->status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return MCFFT_CUDA_ERROR;
  if (h != kStatusOk) {
    cudaMemset(p->status, 0, sizeof(int));
    return h == kStatusTimeout ? MCFFT_DEVICE_TIMEOUT : MCFFT_INTERNAL_ERROR;
  }
  return MCFFT_SUCCESS;
}

mcfftResult mcfftPlanGetInfo(mcfftPlan p, mcfftPlanInfo* info) {
  if (!p) return MCFFT_INVALID_PLAN;
  if (!info) return MCFFT_INVALID_VALUE;
  *info = p->info;
  return MCFFT_SUCCESS;
}

mcfftResult mcfftPlanDestroy(mcfftPlan p) {
  if (!p) return MCFFT_INVALID_PLAN;
  for (void* d : p->allocs) cudaFree(d);
  delete p;
  return MCFFT_SUCCESS;
}

const char* mcfftGetErrorString(mcfftResult r) {
  switch (r) {
    case MCFFT_SUCCESS: return "success";
    case MCFFT_INVALID_PLAN: return "invalid plan handle";
    case MCFFT_ALLOC_FAILED: return "device allocation failed";
    case MCFFT_INVALID_VALUE: return "invalid argument";
    case MCFFT_UNSUPPORTED_SIZE: return "unsupported transform size";
    case MCFFT_CUDA_ERROR: return "CUDA error";
    case MCFFT_DEVICE_TIMEOUT: return "device wait timed out";
    case MCFFT_INTERNAL_ERROR: return "internal error";
    case MCFFT_NO_DEVICE: return "no CUDA device";
  }
  return "unknown error";
}

int mcfftGetVersion(void) { return kVersion; }

}  // extern "C"
