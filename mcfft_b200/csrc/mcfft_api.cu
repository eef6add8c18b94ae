// mcfft_api.cu -- plan construction and execution behind include/mcfft.h.
//
// Replaces the reference's mcfftCreate / mcfftExec
// (source/mcfft_1d_device.cpp:596-790, source/mcfft_2d_device.cpp:594-695):
// instead of a fixed size->schedule switch (ten 1D sizes, three 2D sides)
// the plan decomposes any power-of-two shape into HBM passes, each a
// length-L transform (L = 16^a * R) along one axis, and picks a tile shape
// for each pass from the instantiated kernel variants.
//
//   1D, n <= 8192        one row pass (split form: n <= 4096; a plan bound
//                        for the batch kernel: 4096, split 2048)
//   1D, larger n         four-step: n = n1 * n2; pass 1 = n1-point column
//                        transforms (stride n2) with the W_n^(k1 n2)
//                        twiddle fused into their epilogue, into a scratch
//                        buffer; pass 2 = n2-point row transforms written
//                        with stride n1 (natural order output)
//   2D (nx, ny)          row pass (ny), then in-place column pass (nx)
//   3D (nx, ny, nz)      row pass (nz), column passes (ny, then nx)
//
// All tables (stage twiddles, tail twiddles, four-step twiddles, the DFT-16
// embedding) are generated in FP64 on the GPU at plan time for both
// directions; the plain form's four-step twiddles and the radix-2 twiddles
// of 8192-point passes are instead computed in the kernel from their exact
// angle.  A plan of several transform groups (mcfftPlanCreateBatch) whose
// passes all run on tile kernels the batch kernel holds executes as one
// launch of the persistent batch kernel (fft_queue.cuh) over a queue of
// (pass, tile) items built here; otherwise one launch per pass.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/mcfft.h"
#include "mcfft_internal.h"
#include "queue.h"
#include "host_schedule.h"
#include "queue_order.h"
#include "tile_pass.h"

namespace mcfft {
namespace {

constexpr int kVersion = 200;  // 0.2.0

enum Buf { kUserIn = 0, kUserOut = 1, kScratch = 2 };

struct PassSpec {
  int64_t L;
  bool colfast, posttw;
  int64_t in_sp, in_sc, in_so, out_sp, out_sc, out_so;
  int64_t ncols, nouter;
  int in_buf, out_buf;
  int64_t postN;
  int in_f16, out_f16;
  int64_t in_off, out_off;
  // Transforms at unrelated offsets of the user's buffers (an indexed
  // group): the element offset of each outer index (in_so / out_so unused),
  // or, for a gathered one-pass 1D group (columns = transforms, one outer
  // index), of each column.  Empty: affine addressing.
  std::vector<int64_t> in_idx = {}, out_idx = {};
  bool gather = false;
};

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
  // Place in its transform group (one descriptor) and dependency data for
  // the batch queue: a pass at level > 0 reads what the previous pass of its
  // group wrote.  Producer side: tile t completes keys [t sig_mul / sig_div,
  // ((t + 1) sig_mul - 1) / sig_div]; consumer side: tile (cb, outer) needs
  // key `outer` complete, i.e. wait_count producer tiles; `keys` = nouter.
  int grp = -1, level = 0;
  PassSpec spec{};  // what the pass computes (kept for plan-time retuning)
  int64_t sig_mul = 1, sig_div = 1;
  int wait_count = 0;
  int64_t keys = 0;
  // Indexed / gathered addressing (PassSpec::in_idx): device tables and the
  // staging-row geometry the batch kernel reads (QPassAux).
  const int32_t* in_tab = nullptr;
  const int32_t* out_tab = nullptr;
  int gin_rows = 0, gout_rows = 0, g_row_bytes = 0;
};

// The batch queue of a plan: every pass in one persistent launch.
struct Queue {
  bool on = false;
  QItem* items = nullptr;  // device
  int64_t nitems = 0;
  int* counters = nullptr;  // device
  int64_t ncounters = 0;
  std::vector<int> wait_base, sig_base;  // per pass
  int grid = 0;
  QArgs* args = nullptr;  // host staging of the parameter block
  std::vector<const QPassAux*> aux;  // per pass, device (or null)
  // The kernel: the general batch kernel, or a fused four-step kernel for a
  // single 1D transform group (fused.cu).
  const void* fn = nullptr;
  int smem = 0;
  bool fused = false;
  // Fault injection for the failure-detection tests (MCFFT_INJECT_STALL at
  // plan time): every dependent pass waits for a producer count that can
  // never be reached, so its tiles time out on the device and the exec
  // reports MCFFT_DEVICE_TIMEOUT.  Host-side only; nothing faults.
  bool stall = false;
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
  mcfft::Queue q;
  int ngroups = 0;
  // The plan is meant for the batch queue (several transform groups, or
  // MCFFT_QUEUE=1): its passes take only tile shapes the batch kernel holds.
  bool queue_planned = false;
  // A group the batch queue cannot run (three-pass 1D lengths).
  bool no_queue = false;
  // An indexed transform group (per-transform offsets), which only the
  // batch queue can run.
  bool indexed = false;
  // Four-step split n1 = 2^fs_lg1 of the 1D group being built (0: default).
  int fs_lg1 = 0;
  // Programmatic dependent launch of the second and later tile passes of
  // an exec (their setup overlaps the previous pass's last tiles);
  // MCFFT_PDL=0 at plan creation launches every pass in plain stream order.
  bool pdl = true;
  // Executable graphs of recent execs, keyed by (in, out, direction): an
  // exec repeated on the same buffers replays its captured launches.
  struct GraphEntry {
    const void* in = nullptr;
    void* out = nullptr;
    int dir = -1;
    int uses = 0;  // execs seen with this key (captured on the second)
    cudaGraphExec_t exec = nullptr;
    uint64_t stamp = 0;
  };
  GraphEntry graphs[4];
  uint64_t graph_clock = 0;
  bool graphs_on = true;
  cudaStream_t capture_stream = nullptr;
  std::mutex graph_mu;
  // Creation arguments, for the chunk plan of mcfftExecHost.
  mcfftPrecision prec = MCFFT_PREC_FP16;
  mcfftDesc desc0{};
  int ndesc = 0;
  int64_t in_extent = 0, out_extent = 0;  // bytes of the input / output buffers an exec touches
  // mcfftExecHost state, made on its first call: the chunk schedule (runs of
  // whole transforms) with a plan per chunk length (the plan itself when the
  // whole batch is one chunk), a ring of device buffers per side, copy
  // streams and the events that order the pipeline.
  static constexpr int kHostRing = 4;
  struct HostChunk {
    int64_t first, count;  // transforms [first, first + count)
    mcfftPlan plan;
  };
  struct HostPipe {
    bool ready = false;
    std::vector<std::pair<int64_t, mcfftPlan>> plans;  // chunk plans by transform count
    std::vector<HostChunk> chunks;
    int nbuf = 1;
    size_t in_per = 0, out_per = 0;  // bytes per transform (one chunk: per whole buffer)
    void* din[kHostRing] = {};
    void* dout[kHostRing] = {};
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t start = nullptr, done = nullptr;
    cudaEvent_t loaded[kHostRing] = {}, computed[kHostRing] = {}, stored[kHostRing] = {};
  } host;
  std::mutex host_mu;
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

// Largest power of two dividing every offset (at most 2^20).
int64_t offsets_unit(const std::vector<int64_t>& v) {
  int64_t u = int64_t(1) << 20;
  for (int64_t x : v)
    while (x % u) u >>= 1;
  return u;
}

// Indexed outer dimension of a staging's tensor map (PassSpec::in_idx):
// stride = the offsets' common unit, extent = the largest offset / unit + 1;
// `tab` receives offset / unit per outer index.  False if impossible.
bool index_outer(layout::Staging* st, const std::vector<int64_t>& offs, std::vector<int32_t>* tab) {
  const int64_t unit = offsets_unit(offs);
  if ((unit * st->elem) % 16) return false;
  int d = -1;
  for (int i = 0; i < st->ndims; ++i)
    if (st->omul[i] == 1) d = i;
  if (d < 1) return false;
  int64_t mx = 0;
  tab->clear();
  for (int64_t o : offs) {
    if (o < 0 || o / unit >= (int64_t(1) << 31)) return false;
    tab->push_back((int32_t)(o / unit));
    mx = std::max(mx, o / unit);
  }
  st->gdim[d] = (uint64_t)mx + 1;
  st->gstride_bytes[d] = (uint64_t)(unit * st->elem);
  return true;
}

// Row map of a gathered side: rows of the tile staging's E points over the
// whole buffer (extent: the last transform's end), box E x 1, no swizzle;
// `tab` receives each column's first row (columns padded to a multiple of
// C with the last one).  False if an offset is not a whole row.
bool gather_rows(const layout::Staging& tile_st, int64_t L, int64_t C,
                 const std::vector<int64_t>& offs, layout::Staging* out, std::vector<int32_t>* tab) {
  const int64_t E = tile_st.E;
  if (tile_st.kind != layout::ROW || E * tile_st.elem != 128 || L % E) return false;
  int64_t end = 0;
  tab->clear();
  for (int64_t o : offs) {
    if (o < 0 || o % E || (o + L) / E >= (int64_t(1) << 31)) return false;
    tab->push_back((int32_t)(o / E));
    end = std::max(end, o + L);
  }
  while ((int64_t)tab->size() % C) tab->push_back(tab->back());
  layout::Staging g;
  g.kind = layout::ROW;
  g.L = (int)L;
  g.C = (int)C;
  g.elem = tile_st.elem;
  g.E = (int)E;
  g.row_bytes = 128;
  g.swz = 0;
  g.ndims = 2;
  g.gdim[0] = (uint64_t)E;
  g.box[0] = (uint32_t)E;
  g.gdim[1] = (uint64_t)(end / E);
  g.box[1] = 1;
  g.gstride_bytes[1] = 128;
  *out = g;
  return true;
}

// Builds a pass on the TMA-fed kernel.  Returns MCFFT_UNSUPPORTED_SIZE when
// the shape is outside what that kernel handles (the caller falls back).
mcfftResult add_tile_pass(mcfftPlan p, const PassSpec& s, int only_tile_points = 0) {
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
  int order[2] = {p->split ? 8192 : first, p->split ? 8192 : (first == 16384 ? 8192 : 16384)};
  if (only_tile_points) order[0] = order[1] = only_tile_points;
  const int in_elem = s.in_f16 ? 4 : 8, out_elem = s.out_f16 ? 4 : 8;
  Pass ps;
  ps.tiled = true;
  TilePass& tp = ps.tp;
  const TileKernel* k = nullptr;
  std::vector<int32_t> in_tab, out_tab;
  const bool indexed = s.gather || !s.in_idx.empty() || !s.out_idx.empty();
  for (int oi = 0; oi < 2 && !k; ++oi) {
    const TileKernel* cand =
        find_tile_kernel((int)s.L, s.posttw, p->split, order[oi], s.in_f16 != 0);
    if (!cand) continue;
    if (!p->split && (in_elem != 4 || out_elem != 4)) continue;
    // a plan meant for the batch queue takes only tile shapes the batch
    // kernel holds (not L = 4096 in 8K-point tiles); indexed passes run
    // only there, gathered ones with four columns per gather
    if ((p->queue_planned || indexed) && queue_variant(*cand) < 0) continue;
    if (s.gather && (cand->C < 4 || ik != layout::ROW || ok != layout::ROW)) continue;
    std::string err;
    if (!tile_layout(&tp.lay, cand->L, cand->R, cand->C, ik, ok, in_elem, out_elem, s.in_sp,
                     s.in_sc, s.in_so, s.out_sp, s.out_sc, s.out_so, s.ncols, s.nouter, &err,
                     s.gather ? 3 : 0))
      continue;
    if (s.gather) {
      layout::Staging gi, go;
      if (!gather_rows(tp.lay.in, s.L, cand->C, s.in_idx, &gi, &in_tab) ||
          !gather_rows(tp.lay.out, s.L, cand->C, s.out_idx, &go, &out_tab))
        continue;
      ps.gin_rows = (int)(s.L / tp.lay.in.E);
      ps.gout_rows = (int)(s.L / tp.lay.out.E);
      ps.g_row_bytes = 128;
      tp.lay.in = gi;
      tp.lay.out = go;
    } else {
      if (!s.in_idx.empty() && !index_outer(&tp.lay.in, s.in_idx, &in_tab)) continue;
      if (!s.out_idx.empty() && !index_outer(&tp.lay.out, s.out_idx, &out_tab)) continue;
    }
    if (!tile_check_encode(tp.lay.in, p->status) || !tile_check_encode(tp.lay.out, p->status))
      continue;
    k = cand;
  }
  if (!k) return MCFFT_UNSUPPORTED_SIZE;
  tp.k = k;
  fill_tile_args(&tp);
  TileArgs& a = tp.args;
  if (s.gather) a.in_tile_bytes = (uint32_t)(k->L * k->C * in_elem);
  for (int side = 0; side < 2; ++side) {
    const std::vector<int32_t>& t = side ? out_tab : in_tab;
    if (t.empty()) continue;
    int32_t* d = nullptr;
    mcfftResult r = plan_alloc(p, &d, t.size() * sizeof(int32_t));
    if (r) return r;
    if (cudaMemcpy(d, t.data(), t.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
      return MCFFT_CUDA_ERROR;
    (side ? ps.out_tab : ps.in_tab) = d;
  }
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
    // W_N^e from the exact angle e (2 / N) (sine / cosine in the kernel) up to
    // N = 2^24, else from the FP64-generated two-level table;
    // MCFFT_FOURSTEP_TABLES=1 takes the tables for every N (to measure the
    // angle path's error against them)
    const char* ft = std::getenv("MCFFT_FOURSTEP_TABLES");
    const bool tables = (ft && std::atoi(ft) != 0) || s.postN > (int64_t(1) << 24);
    a.post_scale = tables ? 0.f : (float)(2.0 / (double)s.postN);
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
  ps.spec = s;
  p->passes.push_back(ps);
  return MCFFT_SUCCESS;
}

// Median CUDA-event time (ms) of one tile pass on the given buffers.
float time_tile_pass(const TilePass& tp, void* a, void* b, cudaStream_t st) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return -1.f;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return -1.f;
  }
  float t[5] = {0};
  bool ok = launch_tile_pass(tp, a, b, 0, st) == cudaSuccess &&
            launch_tile_pass(tp, a, b, 0, st) == cudaSuccess;
  for (int r = 0; r < 5 && ok; ++r) {
    ok = cudaEventRecord(e0, st) == cudaSuccess && launch_tile_pass(tp, a, b, 0, st) == cudaSuccess &&
         cudaEventRecord(e1, st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
         cudaEventElapsedTime(&t[r], e0, e1) == cudaSuccess;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!ok) {
    cudaGetLastError();
    return -1.f;
  }
  std::sort(t, t + 5);
  return t[2];
}

// Autotuning records ("wisdom"): the tile shape the plan-time tuner chose
// for a pass, keyed by the GPU (name and SM count) and everything the
// choice depends on (the pass's length, layout, strides and extents).  The
// records of this process can be written to a text file and read back by a
// later process, whose plans then take the recorded shapes without timing.
// File format: the line "mcfft-wisdom 1", then one record per line:
// "<gpu name>\t<sms>\t<pass key>\t<tile points>".
struct Wisdom {
  std::mutex mu;
  std::vector<std::pair<std::string, int>> recs;  // key (gpu + pass) -> tile points
};
Wisdom& wisdom() {
  static Wisdom w;
  return w;
}

std::string gpu_key(const mcfftPlan p) {
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, p->device) != cudaSuccess) {
    cudaGetLastError();
    prop.name[0] = 0;
  }
  std::string name(prop.name);
  for (char& c : name)
    if (c == '\t' || c == '\n') c = ' ';
  return name + "\t" + std::to_string(p->sms);
}

std::string pass_key(const PassSpec& s) {
  char b[512];
  std::snprintf(b, sizeof b, "L%lld c%d t%d i%lld,%lld,%lld o%lld,%lld,%lld n%lld,%lld h%d,%d N%lld",
                (long long)s.L, (int)s.colfast, (int)s.posttw, (long long)s.in_sp, (long long)s.in_sc,
                (long long)s.in_so, (long long)s.out_sp, (long long)s.out_sc, (long long)s.out_so,
                (long long)s.ncols, (long long)s.nouter, s.in_f16, s.out_f16, (long long)s.postN);
  return b;
}

int wisdom_find(const std::string& key) {
  Wisdom& w = wisdom();
  std::lock_guard<std::mutex> lk(w.mu);
  for (auto& r : w.recs)
    if (r.first == key) return r.second;
  return 0;
}

void wisdom_put(const std::string& key, int tile_points) {
  Wisdom& w = wisdom();
  std::lock_guard<std::mutex> lk(w.mu);
  for (auto& r : w.recs)
    if (r.first == key) {
      r.second = tile_points;
      return;
    }
  w.recs.push_back({key, tile_points});
}

// Plan-time tuning of the tile shape of the plain-form passes [first, end)
// of one transform group (`points` complex elements): each pass takes the
// shape recorded for it, or is timed with 16K- and 8K-point tiles on
// scratch buffers and keeps the faster (by more than 3 %), which is then
// recorded.  MCFFT_AUTOTUNE=0 keeps the default shapes.
mcfftResult autotune_group(mcfftPlan p, size_t first, int64_t points) {
  if (p->split) return MCFFT_SUCCESS;
  if (const char* e = std::getenv("MCFFT_AUTOTUNE"))
    if (std::atoi(e) == 0) return MCFFT_SUCCESS;
  const std::string gk = gpu_key(p);
  std::vector<size_t> todo;
  for (size_t i = first; i < p->passes.size(); ++i) {
    // indexed passes keep the default shape (they run only in the batch
    // queue, which the tuner's single-pass timing does not model)
    if (!p->passes[i].tiled || p->passes[i].in_tab || p->passes[i].out_tab) continue;
    const int rec = wisdom_find(gk + "\t" + pass_key(p->passes[i].spec));
    if (!rec) {
      todo.push_back(i);
      continue;
    }
    if (rec == p->passes[i].tp.k->tile_points) continue;
    if (add_tile_pass(p, p->passes[i].spec, rec) != MCFFT_SUCCESS) continue;
    Pass cand = p->passes.back();
    p->passes.pop_back();
    cand.grp = p->passes[i].grp;
    cand.level = p->passes[i].level;
    p->passes[i] = cand;
  }
  if (todo.empty()) return MCFFT_SUCCESS;
  void *a = nullptr, *b = nullptr;
  const size_t bytes = (size_t)points * 8;
  if (cudaMalloc(&a, bytes) != cudaSuccess || cudaMalloc(&b, bytes) != cudaSuccess ||
      cudaMemset(a, 0, bytes) != cudaSuccess || cudaMemset(b, 0, bytes) != cudaSuccess) {
    cudaGetLastError();
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    return MCFFT_SUCCESS;  // no room to tune: keep the default shapes
  }
  for (size_t i : todo) {
    const int alt = p->passes[i].tp.k->tile_points == 16384 ? 8192 : 16384;
    if (add_tile_pass(p, p->passes[i].spec, alt) != MCFFT_SUCCESS) continue;
    Pass cand = p->passes.back();
    p->passes.pop_back();
    const float t0 = time_tile_pass(p->passes[i].tp, a, b, 0);
    const float t1 = time_tile_pass(cand.tp, a, b, 0);
    ++p->info.timed_passes;
    if (std::getenv("MCFFT_DEBUG_PLAN"))
      fprintf(stderr, "[mcfft] tune pass L=%d: %d-point tiles %.4f ms, %d-point tiles %.4f ms\n",
              p->passes[i].tp.k->L, p->passes[i].tp.k->tile_points, t0, alt, t1);
    if (t0 > 0.f && t1 > 0.f && t1 < 0.97f * t0) {
      cand.grp = p->passes[i].grp;
      cand.level = p->passes[i].level;
      p->passes[i] = cand;
    }
    if (t0 > 0.f && t1 > 0.f)
      wisdom_put(gk + "\t" + pass_key(p->passes[i].spec), p->passes[i].tp.k->tile_points);
  }
  cudaFree(a);
  cudaFree(b);
  return MCFFT_SUCCESS;
}

mcfftResult add_pass(mcfftPlan p, const PassSpec& s) {
  {
    mcfftResult tr = add_tile_pass(p, s);
    if (tr != MCFFT_UNSUPPORTED_SIZE) return tr;
    // the direct-load kernels address only affine layouts
    if (s.gather || !s.in_idx.empty() || !s.out_idx.empty()) return tr;
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
constexpr int64_t kMaxTilePass = 4096;  // longest column of the four-column tiles

// The longest 1D transform one pass takes: 8192 points in the plain form
// (two per 16K-point tile) and 4096 in the split form (two per 8K-point
// tile), outside the batch queue; a plan bound for it takes only the tile
// shapes the batch kernel holds (4096, split 2048) and runs longer lengths
// as four-step pairs.
int64_t max_one_pass(const mcfftPlan p) {
  if (p->queue_planned) return p->split ? kMaxTilePass / 2 : kMaxTilePass;
  return p->split ? kMaxTilePass : 2 * kMaxTilePass;
}

constexpr int64_t kMaxLength1d = int64_t(1) << 27;

// The three-pass decomposition, and the single pass of two columns per tile
// (plain 8192, split 4096 points), as choices of the four-step tuner (in
// mcfftPlan_st::fs_lg1 and in "fourstep" wisdom records).
constexpr int kThreePass = -1;
constexpr int kOnePass = -2;

// The longest 1D transform of the four-column tiles (one pass, no choice).
int64_t max_four_column(const mcfftPlan p) { return p->split ? kMaxTilePass / 2 : kMaxTilePass; }

// The untuned decomposition of a 1D length past the four-column tiles: one
// pass of two columns per tile where the form has it (plain 8192, split
// 4096, outside the batch queue), the four-step split n1 = 2^floor(lg n /
// 2), or three passes from 2^24 points (plain form) and 2^23 (split form).  Measured on a B200, 2^26 points in all per
// exec: the split form's tile kernels hold at most 2048 points per column,
// so its four-step pairs past 2^22 run a direct-load pass (2^23: 1.44 ms
// against 0.80 ms in three passes); the plain form's pair of 4096-point
// passes at 2^24 takes 0.65 ms against 0.41 ms in three, and past 2^24 its
// pairs run a direct-load pass (2^26: 2.68 ms against 0.42 ms).
int default_lg1(const mcfftPlan p, int64_t n) {
  if (n <= max_one_pass(p)) return kOnePass;
  if (n >= (p->split ? (int64_t(1) << 23) : (int64_t(1) << 24))) return kThreePass;
  return ilog2(n) / 2;
}

// 1D lengths of 2^27 (the reference plans 2^27 in three passes,
// source/mcfft_1d_device.cpp:762-771): n = n1 * n2 * n3, m = n2 * n3, the
// four-step split applied twice --
//   pass 1  n1-point columns j < m (stride m), times W_n^(k1 j), into the
//           scratch as A[k1][j]
//   pass 2  in place in the scratch, per row k1: n2-point columns j3 < n3
//           (stride n3), times W_m^(k2 j3): B[k1][k2][j3]
//   pass 3  per transform, per k2: n3-point rows of B, columns k1 (stride m
//           in the scratch), written to X[k1 + n1 k2 + n1 n2 k3] (stride
//           n1 n2, columns contiguous)
// Pass 3's outer index (k2) would need a second stride across transforms,
// so it is one pass per transform.  Such a group never runs in the batch
// queue.
mcfftResult build_three_pass(mcfftPlan p, int64_t n, int64_t batch, int64_t in_off,
                             int64_t out_off) {
  if (n > kMaxLength1d) return MCFFT_UNSUPPORTED_SIZE;
  const bool split = p->split;
  const int in_f16 = split ? ((p->flags & MCFFT_FLAG_INPUT_F16) ? 1 : 0) : 1;
  const int mid_f16 = split ? 0 : 1;
  const int lg = ilog2(n), lg1 = lg / 3, lg2 = (lg - lg1) / 2;
  const int64_t n1 = int64_t(1) << lg1, n2 = int64_t(1) << lg2, n3 = n >> (lg1 + lg2);
  const int64_t m = n2 * n3;
  const size_t ebytes = split ? 8 : 4;
  const int64_t soff = (int64_t)(p->scratch_bytes / ebytes);
  PassSpec s1{n1, true, true, m, 1, n, m, 1, n, m, batch, kUserIn, kScratch, n,
              in_f16, mid_f16, in_off, soff};
  mcfftResult r = add_pass(p, s1);
  if (r) return r;
  PassSpec s2{n2, true, true, n3, 1, m, n3, 1, m, n3, batch * n1, kScratch, kScratch, m,
              mid_f16, mid_f16, soff, soff};
  r = add_pass(p, s2);
  if (r) return r;
  for (int64_t b = 0; b < batch && !r; ++b) {
    PassSpec s3{n3, false, false, 1, m, n3, n1 * n2, 1, n1, n1, n2, kScratch, kUserOut, 0,
                mid_f16, split ? 0 : 1, soff + b * n, out_off + b * n};
    r = add_pass(p, s3);
  }
  if (r) return r;
  p->scratch_bytes += (size_t)n * batch * ebytes;
  p->no_queue = true;
  return MCFFT_SUCCESS;
}

// Appends the passes of one transform group.  `in_buf/out_buf` and offsets
// locate it inside the user's buffers; the first pass reads in_buf, the
// last writes out_buf.
mcfftResult build_group_passes(mcfftPlan p, int ndim, const int64_t* dims, int64_t batch,
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
    PassSpec one{n, false, false, 1, n, 0, 1, n, 0, batch, 1, kUserIn, kUserOut, 0,
                 in_f16, split ? 0 : 1, in_off, out_off};
    if (n <= max_four_column(p)) return add_pass(p, one);
    // MCFFT_THREE_PASS=1 takes the three-pass plan for every length past one
    // pass (a test switch: the same code path at sizes that test quickly)
    // MCFFT_FOURSTEP_N1 forces a four-step split
    const char* three = std::getenv("MCFFT_THREE_PASS");
    int lg1 = default_lg1(p, n);
    if (const char* e = std::getenv("MCFFT_FOURSTEP_N1")) lg1 = ilog2(std::atoll(e));
    if (p->fs_lg1 != 0) lg1 = p->fs_lg1;  // the plan-time tuner's choice or candidate
    if (lg1 == kOnePass && n <= max_one_pass(p)) return add_pass(p, one);
    if (lg1 == kOnePass) lg1 = ilog2(n) / 2;
    if (n > kMaxSinglePass * kMaxSinglePass || (three && std::atoi(three) != 0 && n >= 4096 * 16) ||
        lg1 == kThreePass)
      return build_three_pass(p, n, batch, in_off, out_off);
    const int64_t n1 = int64_t(1) << lg1, n2 = n >> lg1;
    if (n1 < 16 || n2 < 16 || n1 > kMaxSinglePass || n2 > kMaxSinglePass)
      return MCFFT_UNSUPPORTED_SIZE;
    // Every four-step group has its own scratch region (groups of one plan
    // may run concurrently in the batch queue).
    const size_t ebytes = split ? 8 : 4;
    const int64_t soff = (int64_t)(p->scratch_bytes / ebytes);
    // pass 1: columns n2, points n1 at stride n2, four-step twiddle
    PassSpec s1{n1, true, true, n2, 1, n, n2, 1, n, n2, batch, kUserIn, kScratch, n,
                in_f16, mid_f16, in_off, soff};
    mcfftResult r = add_pass(p, s1);
    if (r) return r;
    // pass 2: rows k1 (stride n2) of n2 points; output X[k1 + n1 k2]
    PassSpec s2{n2, false, false, 1, n2, n, n1, 1, n, n1, batch, kScratch, kUserOut, 0,
                mid_f16, split ? 0 : 1, soff, out_off};
    r = add_pass(p, s2);
    if (r) return r;
    p->scratch_bytes += (size_t)n * batch * ebytes;
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
  p->prec = prec;
  if (const char* e = std::getenv("MCFFT_GRAPH")) p->graphs_on = std::atoi(e) != 0;
  if (std::getenv("MCFFT_DEBUG_SYNC")) p->graphs_on = false;
  if (const char* e = std::getenv("MCFFT_PDL")) p->pdl = std::atoi(e) != 0;
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

// Group index, level and batch-queue dependency data of the passes
// [first, end) of one transform group.
void link_group(mcfftPlan p, size_t first, int ndim, const int64_t* dims, int64_t batch) {
  const int g = p->ngroups++;
  for (size_t i = first; i < p->passes.size(); ++i) {
    p->passes[i].grp = g;
    p->passes[i].level = (int)(i - first);
  }
  if (p->passes.size() - first < 2) return;
  if (ndim == 1 && p->passes.size() - first != 2) return;  // three-pass: never queued
  for (size_t i = first; i < p->passes.size(); ++i)
    if (!p->passes[i].tiled) return;  // the queue only runs tile passes
  auto C = [&](size_t i) -> int64_t { return p->passes[i].tp.k->C; };
  auto CB = [&](size_t i) -> int64_t { return p->passes[i].tp.args.col_blocks; };
  Pass& P0 = p->passes[first];
  Pass& P1 = p->passes[first + 1];
  if (ndim == 1) {  // four-step: key = transform
    P0.sig_mul = 1;
    P0.sig_div = CB(first);
    P1.wait_count = (int)CB(first);
    P1.keys = batch;
  } else if (ndim == 2) {  // rows, then columns: key = 2D transform
    const int64_t nx = dims[0], c = C(first);
    P0.sig_mul = c;
    P0.sig_div = nx;
    P1.wait_count = (int)std::max<int64_t>(1, nx / c);
    P1.keys = batch;
  } else {  // z rows, y columns (key = x slab), x columns (key = 3D transform)
    const int64_t nx = dims[0], ny = dims[1], c = C(first);
    Pass& P2 = p->passes[first + 2];
    P0.sig_mul = c;
    P0.sig_div = ny;
    P1.wait_count = (int)std::max<int64_t>(1, ny / c);
    P1.keys = nx * batch;
    P1.sig_mul = 1;
    P1.sig_div = CB(first + 1) * nx;
    P2.wait_count = (int)(CB(first + 1) * nx);
    P2.keys = batch;
  }
}

cudaError_t launch_one(mcfftPlan p, const Pass& ps, const void* src, void* dst, int dir,
                       cudaStream_t st, bool follows);
int in_elem(const mcfftPlan p, const Pass& ps);
int out_elem(const mcfftPlan p, const Pass& ps);

// Median CUDA-event time (ms) of the passes [first, end) of the group being
// built, launched as an exec would, on scratch buffers: `a` stands for the
// user's input, `b` for the output and `c` for the plan's scratch (element
// offsets taken relative to the group's own: in_off, out_off, soff0).
float time_group(mcfftPlan p, size_t first, void* a, void* b, void* c, int64_t in_off,
                 int64_t out_off, int64_t soff0) {
  auto ptr = [&](int buf, int64_t off, int eb) -> char* {
    if (buf == kUserIn) return (char*)a + (off - in_off) * eb;
    if (buf == kUserOut) return (char*)b + (off - out_off) * eb;
    return (char*)c + (off - soff0) * eb;
  };
  auto run = [&]() -> bool {
    for (size_t i = first; i < p->passes.size(); ++i) {
      const Pass& ps = p->passes[i];
      if (launch_one(p, ps, ptr(ps.in_buf, ps.in_off, in_elem(p, ps)),
                     ptr(ps.out_buf, ps.out_off, out_elem(p, ps)), 0, 0, i > first) != cudaSuccess)
        return false;
    }
    return true;
  };
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return -1.f;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return -1.f;
  }
  float t[5] = {0};
  bool ok = run() && run();
  for (int r = 0; r < 5 && ok; ++r)
    ok = cudaEventRecord(e0, 0) == cudaSuccess && run() && cudaEventRecord(e1, 0) == cudaSuccess &&
         cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&t[r], e0, e1) == cudaSuccess;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!ok) {
    cudaGetLastError();
    return -1.f;
  }
  std::sort(t, t + 5);
  return t[2];
}

// Plan-time choice of a 1D group's decomposition past one pass.  The
// candidates are the untuned default (default_lg1), the four-step splits
// n = n1 * n2 with n1 = 2^floor(lg n / 2) and its neighbours n1 / 2 and
// 2 n1, and, from n = 2^21 on, the three-pass plan n = n1 * n2 * n3.  Each is built and timed on scratch
// buffers as an exec runs it (median CUDA-event time of the whole group);
// the fastest wins when it beats the default by more than 3 %.  A split
// whose factor exceeds the tile kernels' range runs a direct-load pass, and
// the timing decides between it and three tile passes: the four-step pair
// of 2^25 and 2^26 points has such a factor (8192), the three-pass plan
// does not.  Where the form has a pass of two columns per tile (plain 8192,
// split 4096) that single pass is the default and the splits are timed
// against it.  The choice is recorded as wisdom ("fourstep" records: lg n1,
// -1 for three passes, -2 for one pass) and reported in
// mcfftPlanInfo.fourstep_n1 (0 for one pass).
// MCFFT_AUTOTUNE=0, MCFFT_FOURSTEP_N1 or MCFFT_THREE_PASS keep the default
// (or the forced plan).
int tune_fourstep(mcfftPlan p, int64_t n, int64_t batch, int64_t in_off, int64_t out_off) {
  const int lg = ilog2(n), def = default_lg1(p, n);
  if (n <= max_four_column(p) || n > kMaxSinglePass * kMaxSinglePass) return 0;
  if (std::getenv("MCFFT_FOURSTEP_N1") || std::getenv("MCFFT_THREE_PASS")) return 0;
  if (const char* e = std::getenv("MCFFT_AUTOTUNE"))
    if (std::atoi(e) == 0) return 0;
  char kb[160];
  std::snprintf(kb, sizeof kb, "fourstep n%lld b%lld p%d f%u", (long long)n, (long long)batch,
                (int)p->prec, p->flags);
  const std::string key = gpu_key(p) + "\t" + kb;
  if (const int rec = wisdom_find(key)) return rec;
  // each candidate's passes are built, timed, then removed again
  const size_t first = p->passes.size();
  const size_t scratch0 = p->scratch_bytes;
  const bool no_queue0 = p->no_queue;
  const size_t eb = p->split ? 8 : 4;
  const int64_t soff0 = (int64_t)(scratch0 / eb);
  void *a = nullptr, *b = nullptr, *c = nullptr;
  const size_t bytes = (size_t)n * batch * eb;
  if (cudaMalloc(&a, bytes) != cudaSuccess || cudaMalloc(&b, bytes) != cudaSuccess ||
      cudaMalloc(&c, bytes) != cudaSuccess || cudaMemset(a, 0, bytes) != cudaSuccess ||
      cudaMemset(b, 0, bytes) != cudaSuccess || cudaMemset(c, 0, bytes) != cudaSuccess) {
    cudaGetLastError();
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    if (c) cudaFree(c);
    return 0;
  }
  std::vector<int> cands = {def};
  for (int lg1 : {lg / 2, lg / 2 - 1, lg / 2 + 1}) {
    const int64_t n1 = int64_t(1) << lg1, n2 = n >> lg1;
    if (lg1 != def && n1 >= 32 && n2 >= 32 && n1 <= kMaxSinglePass && n2 <= kMaxSinglePass)
      cands.push_back(lg1);
  }
  if (lg >= 21 && def != kThreePass) cands.push_back(kThreePass);
  if (n <= max_one_pass(p) && def != kOnePass) cands.push_back(kOnePass);
  float best_t = -1.f, def_t = -1.f;
  int best = def;
  for (int cand : cands) {
    p->fs_lg1 = cand;
    int sl = 0;
    const mcfftResult r = build_group_passes(p, 1, &n, batch, in_off, out_off, &sl);
    const float t = r == MCFFT_SUCCESS ? time_group(p, first, a, b, c, in_off, out_off, soff0) : -1.f;
    const size_t npasses = p->passes.size() - first;
    int tiled = 0;
    for (size_t i = first; i < p->passes.size(); ++i) tiled += p->passes[i].tiled ? 1 : 0;
    p->passes.resize(first);
    p->scratch_bytes = scratch0;
    p->no_queue = no_queue0;
    p->fs_lg1 = 0;
    if (t <= 0.f) continue;
    ++p->info.timed_passes;
    if (std::getenv("MCFFT_DEBUG_PLAN")) {
      if (cand == kThreePass)
        fprintf(stderr, "[mcfft] tune 1D n=%lld: three passes (%zu launches) %.4f ms\n",
                (long long)n, npasses, t);
      else if (cand == kOnePass)
        fprintf(stderr, "[mcfft] tune 1D n=%lld: one pass (%d tiled) %.4f ms\n", (long long)n,
                tiled, t);
      else
        fprintf(stderr, "[mcfft] tune 1D n=%lld: n1=%lld (%d of 2 passes tiled) %.4f ms\n",
                (long long)n, (long long)(int64_t(1) << cand), tiled, t);
    }
    if (cand == def) def_t = t;
    if (best_t < 0.f || t < best_t) {
      best_t = t;
      best = cand;
    }
  }
  cudaFree(a);
  cudaFree(b);
  cudaFree(c);
  if (def_t > 0.f && best != def && best_t >= 0.97f * def_t) best = def;
  if (best_t > 0.f) wisdom_put(key, best);
  return best;
}

mcfftResult build_group(mcfftPlan p, int ndim, const int64_t* dims, int64_t batch,
                        int64_t in_off, int64_t out_off, int* scale_log2) {
  const size_t first = p->passes.size();
  p->fs_lg1 = ndim == 1 ? tune_fourstep(p, dims[0], batch, in_off, out_off) : 0;
  mcfftResult r = build_group_passes(p, ndim, dims, batch, in_off, out_off, scale_log2);
  if (!r && ndim == 1 && first == 0 && p->passes.size() >= 2)
    p->info.fourstep_n1 = p->passes[0].spec.L;
  p->fs_lg1 = 0;
  int64_t points = batch;
  for (int d = 0; d < ndim; ++d) points *= dims[d];
  if (!r) r = autotune_group(p, first, points);
  if (!r) link_group(p, first, ndim, dims, batch);
  return r;
}

// An indexed transform group: B transforms of one shape at the element
// offsets ioff[b] of the input and ooff[b] of the output, in no particular
// order (descriptors of one shape that do not follow each other).  The same
// passes as build_group_passes, with per-transform coordinate tables: a
// one-pass 1D group gathers its tiles' columns (transforms) row by row, the
// other passes look their outer (transform) coordinate up.  Such a group
// runs only in the batch kernel.
mcfftResult build_indexed_group(mcfftPlan p, int ndim, const int64_t* dims,
                                const std::vector<int64_t>& ioff, const std::vector<int64_t>& ooff,
                                int* scale_log2) {
  const size_t first = p->passes.size();
  const bool split = p->split;
  const int in_f16 = split ? ((p->flags & MCFFT_FLAG_INPUT_F16) ? 1 : 0) : 1;
  const int mid_f16 = split ? 0 : 1, out_f16 = split ? 0 : 1;
  const int64_t B = (int64_t)ioff.size();
  int64_t total = 1;
  for (int d = 0; d < ndim; ++d) {
    if (!is_pow2(dims[d]) || dims[d] < 16) return MCFFT_UNSUPPORTED_SIZE;
    total *= dims[d];
  }
  *scale_log2 = split ? 0 : -ilog2(total);
  mcfftResult r = MCFFT_SUCCESS;
  if (ndim == 1) {
    const int64_t n = dims[0];
    if (n <= (split ? kMaxTilePass / 2 : kMaxTilePass)) {
      PassSpec sp{n, false, false, 1, n, 0, 1, n, 0, B, 1, kUserIn, kUserOut, 0,
                  in_f16, out_f16, 0, 0};
      sp.in_idx = ioff;
      sp.out_idx = ooff;
      sp.gather = true;
      r = add_pass(p, sp);
    } else if (n <= kMaxSinglePass * kMaxSinglePass) {
      const int lg = ilog2(n), lg1 = lg / 2;
      const int64_t n1 = int64_t(1) << lg1, n2 = n >> lg1;
      if (n1 < 16 || n2 < 16 || n1 > kMaxSinglePass || n2 > kMaxSinglePass)
        return MCFFT_UNSUPPORTED_SIZE;
      const size_t ebytes = split ? 8 : 4;
      const int64_t soff = (int64_t)(p->scratch_bytes / ebytes);
      PassSpec s1{n1, true, true, n2, 1, n, n2, 1, n, n2, B, kUserIn, kScratch, n,
                  in_f16, mid_f16, 0, soff};
      s1.in_idx = ioff;
      r = add_pass(p, s1);
      if (r) return r;
      PassSpec s2{n2, false, false, 1, n2, n, n1, 1, n, n1, B, kScratch, kUserOut, 0,
                  mid_f16, out_f16, soff, 0};
      s2.out_idx = ooff;
      r = add_pass(p, s2);
      if (r) return r;
      p->scratch_bytes += (size_t)n * B * ebytes;
    } else {
      return MCFFT_UNSUPPORTED_SIZE;
    }
  } else {
    for (int d = 0; d < ndim; ++d)
      if (dims[d] > kMaxSinglePass) return MCFFT_UNSUPPORTED_SIZE;
    if (ndim == 2) {
      const int64_t nx = dims[0], ny = dims[1];
      PassSpec s1{ny, false, false, 1, ny, 0, 1, ny, 0, nx, B, kUserIn, kUserOut, 0,
                  in_f16, mid_f16, 0, 0};
      s1.in_idx = ioff;
      s1.out_idx = ooff;
      r = add_pass(p, s1);
      if (r) return r;
      PassSpec s2{nx, true, false, ny, 1, 0, ny, 1, 0, ny, B, kUserOut, kUserOut, 0,
                  mid_f16, mid_f16, 0, 0};
      s2.in_idx = ooff;
      s2.out_idx = ooff;
      r = add_pass(p, s2);
    } else if (ndim == 3) {
      const int64_t nx = dims[0], ny = dims[1], nz = dims[2];
      PassSpec s1{nz, false, false, 1, nz, 0, 1, nz, 0, nx * ny, B, kUserIn, kUserOut, 0,
                  in_f16, mid_f16, 0, 0};
      s1.in_idx = ioff;
      s1.out_idx = ooff;
      r = add_pass(p, s1);
      if (r) return r;
      std::vector<int64_t> slabs;  // outer (b, x): the x-th slab of transform b
      for (int64_t b = 0; b < B; ++b)
        for (int64_t x = 0; x < nx; ++x) slabs.push_back(ooff[b] + x * ny * nz);
      PassSpec s2{ny, true, false, nz, 1, 0, nz, 1, 0, nz, nx * B, kUserOut, kUserOut, 0,
                  mid_f16, mid_f16, 0, 0};
      s2.in_idx = slabs;
      s2.out_idx = slabs;
      r = add_pass(p, s2);
      if (r) return r;
      PassSpec s3{nx, true, false, ny * nz, 1, 0, ny * nz, 1, 0, ny * nz, B, kUserOut, kUserOut,
                  0, mid_f16, mid_f16, 0, 0};
      s3.in_idx = ooff;
      s3.out_idx = ooff;
      r = add_pass(p, s3);
    } else {
      return MCFFT_INVALID_VALUE;
    }
    // the first pass's tiles must not straddle transforms (its dependency
    // keys count whole tiles per transform)
    if (!r && p->passes[first].spec.ncols % p->passes[first].tp.k->C != 0)
      return MCFFT_UNSUPPORTED_SIZE;
  }
  if (r) return r;
  link_group(p, first, ndim, dims, B);
  p->indexed = true;
  return MCFFT_SUCCESS;
}

// L2 use of pass i in the batch kernels (MCFFT_L2_HINTS=1; off by default:
// measured slower on the four-step pair, whose column tiles read half
// lines that the neighbouring tile reads again): an intermediate another
// pass reads (the plan's scratch, or the output read again in place) is
// stored with evict-last priority; data read or written once streams with
// evict-first.
bool l2_hints_on() {
  static const bool on = [] {
    const char* e = std::getenv("MCFFT_L2_HINTS");
    return e && std::atoi(e) != 0;
  }();
  return on;
}
// Scratch lines dropped from L2 after their last read (MCFFT_L2_DISCARD=1).
// Off by default: the discard instructions cost more than the write-backs
// they save (uneven batch 0.353 against 0.344 ms, fused four-step pair
// 0.304 against 0.295 ms).
bool l2_discard_on() {
  static const bool on = [] {
    const char* e = std::getenv("MCFFT_L2_DISCARD");
    return e && std::atoi(e) != 0;
  }();
  return on;
}

void set_l2_use(mcfftPlan p, size_t i, QPass* Q) {
  if (!l2_hints_on()) return;
  const Pass& ps = p->passes[i];
  const bool read_later = i + 1 < p->passes.size() && p->passes[i + 1].grp == ps.grp &&
                          p->passes[i + 1].level > 0;
  Q->l2_out = read_later ? kL2EvictLast : kL2EvictFirst;
  if (ps.in_buf == kUserIn || ps.in_buf == kScratch) Q->l2_in = kL2EvictFirst;
}

// Plan-time per-pass features of the batch kernels (QPassAux): a row-input
// pass reading the scratch drops each tile's source lines from L2 once the
// tile is loaded (no write-back of a dead intermediate), when its tiles
// cover whole rows.  Returns the host copy; `any` tells whether it holds
// anything.
QPassAux make_aux(mcfftPlan p, size_t i, bool* any) {
  QPassAux x;
  std::memset(&x, 0, sizeof(x));
  *any = false;
  const Pass& ps = p->passes[i];
  if (l2_discard_on() && ps.in_buf == kScratch) {
    const PassSpec& sp = ps.spec;
    const int64_t C = ps.tp.k->C, eb = ps.in_f16 ? 4 : 8;
    const int64_t row = sp.L * eb;
    const char* in_base = static_cast<const char*>(p->scratch) + ps.in_off * eb;
    if (sp.in_sp == 1 && sp.ncols % C == 0 && row % 128 == 0 && (row & (row - 1)) == 0 &&
        (sp.in_sc * eb) % 128 == 0 &&
        (sp.in_so * eb) % 128 == 0 && (reinterpret_cast<uintptr_t>(in_base) & 127) == 0) {
      x.disc_base = in_base;
      x.disc_sc = sp.in_sc * eb;
      x.disc_so = sp.in_so * eb;
      x.disc_row_bytes = (uint32_t)row;
      x.disc_C = (int32_t)C;
      *any = true;
    }
  }
  if (ps.in_tab || ps.out_tab) {
    const bool g = ps.spec.gather;
    x.in_otab = g ? nullptr : ps.in_tab;
    x.out_otab = g ? nullptr : ps.out_tab;
    x.in_gtab = g ? ps.in_tab : nullptr;
    x.out_gtab = g ? ps.out_tab : nullptr;
    x.gin_rows = ps.gin_rows;
    x.gout_rows = ps.gout_rows;
    x.g_C = ps.tp.k->C;
    x.g_row_bytes = ps.g_row_bytes;
    *any = true;
  }
  return x;
}

// With MCFFT_FUSED=1, a single 1D four-step transform group whose pair of
// tile variants has a fused kernel runs both passes in one launch of it,
// its items ordered in chunks of two tiles per CTA (a transform's second
// pass follows its first within a few tiles per CTA, while its
// intermediate is still in L2).  Off by default: on the 2^20 x 64 workload
// the two pass launches measured faster (0.258 against 0.294 ms).
const FusedKernel* fused_for(mcfftPlan p) {
  const char* e = std::getenv("MCFFT_FUSED");
  if (!e || std::atoi(e) == 0) return nullptr;
  if (p->ngroups != 1 || p->passes.size() != 2 || p->no_queue) return nullptr;
  const Pass &a = p->passes[0], &b = p->passes[1];
  if (!a.tiled || !b.tiled || !a.spec.posttw || b.spec.posttw || a.out_buf != kScratch ||
      b.in_buf != kScratch)
    return nullptr;
  const int v1 = queue_variant(*a.tp.k), v2 = queue_variant(*b.tp.k);
  if (v1 < 0 || v2 < 0) return nullptr;
  return find_fused(p->split, v1, v2);
}

// Builds the batch queue (every pass of the plan in one persistent launch)
// for plans of several transform groups (uneven batches) -- or any plan
// with MCFFT_QUEUE=1; MCFFT_QUEUE=0 disables it -- when every pass runs on
// a tile-kernel variant the batch kernel holds and the passes fit its
// parameter block; otherwise the plan launches pass by pass (one transform
// shape is faster that way: each pass kernel keeps its tables in its
// parameter block).
// Queue order (queue_order.h): first passes in chunks of QC (sixteen) tiles
// per CTA, group after group; after each chunk, every later-pass tile whose
// key was completed at least QC tiles per CTA earlier, across all groups.
// Every dependency points backwards, a CTA runs several tiles of one pass in
// a row (its tables stay in shared memory), and the tail of one group's
// later pass runs beside the next group's first pass instead of waiting on
// the tiles queued just before it.
mcfftResult build_queue(mcfftPlan p) {
  const FusedKernel* fk = fused_for(p);
  bool want = p->ngroups > 1 || fk || p->indexed;
  if (const char* e = std::getenv("MCFFT_QUEUE")) want = std::atoi(e) != 0 || fk || p->indexed;
  if (!want || p->no_queue) return MCFFT_SUCCESS;
  const size_t np = p->passes.size();
  if (np > (size_t)kQueueMaxPasses) return MCFFT_SUCCESS;
  for (const auto& ps : p->passes)
    if (!ps.tiled || queue_variant(*ps.tp.k) < 0) {
      if (std::getenv("MCFFT_DEBUG_PLAN"))
        fprintf(stderr, "[mcfft] no batch queue: pass L=%lld not on a queue tile variant\n",
                (long long)(ps.tiled ? ps.tp.k->L : ps.k->L));
      return MCFFT_SUCCESS;
    }
  Queue& q0 = p->q;
  q0.fused = fk != nullptr;
  q0.fn = fk ? fk->fn : nullptr;
  q0.smem = fk ? fk->smem_bytes : 0;
  const int maxg = fk ? queue_max_grid_fn(fk->fn, fk->smem_bytes, p->sms)
                      : queue_max_grid(p->sms, p->split);
  if (maxg <= 0) {
    q0.fused = false;
    q0.fn = nullptr;
    return MCFFT_SUCCESS;
  }
  Queue& q = p->q;
  q.wait_base.assign(np, -1);
  q.sig_base.assign(np, -1);
  int64_t nc = 0;
  for (size_t i = 0; i < np; ++i)
    if (p->passes[i].level > 0) {
      q.wait_base[i] = (int)nc;
      q.sig_base[i - 1] = (int)nc;
      nc += p->passes[i].keys;
    }
  const int64_t G = maxg;
  // first-pass tiles per CTA queued at a time (a CTA reloads a pass's tables when its
  // consecutive items switch pass)
  int64_t QC = fk ? 2 : 16;
  if (const char* e = std::getenv("MCFFT_QUEUE_CHUNK")) QC = std::max<int64_t>(1, std::atoll(e));
  std::vector<QOrderPass> qo(np);
  for (size_t i = 0; i < np; ++i) {
    const Pass& ps = p->passes[i];
    qo[i].ntiles = ps.tp.args.ntiles;
    qo[i].col_blocks = ps.tp.args.col_blocks;
    qo[i].sig_mul = ps.sig_mul;
    qo[i].sig_div = ps.sig_div;
    qo[i].keys = ps.level > 0 ? ps.keys : 0;
    qo[i].grp = ps.grp;
  }
  int64_t QLAG = 0;  // lag between a key's completion and its readers (0: QC)
  if (const char* e = std::getenv("MCFFT_QUEUE_LAG")) QLAG = std::max<int64_t>(0, std::atoll(e));
  const std::vector<QOrderItem> order = queue_order(qo, G, QC, QLAG);
  if (order.empty()) return MCFFT_SUCCESS;  // no consistent order: pass by pass
  std::vector<QItem> items(order.size());
  for (size_t i = 0; i < order.size(); ++i) items[i] = {order[i].pass, order[i].tile};
  if (std::getenv("MCFFT_DEBUG_PLAN")) {
    // runs: stretches of one CTA's items (i, i + G, ..) on one pass; each
    // run reloads the pass's tables
    int64_t runs = 0;
    for (int64_t b = 0; b < G; ++b)
      for (int64_t i = b; i < (int64_t)items.size(); i += G)
        runs += (i < G || items[i].pass != items[i - G].pass) ? 1 : 0;
    fprintf(stderr, "[mcfft] queue: %zu passes, %zu items on %lld CTAs, %lld runs (%.2f items per run)\n",
            np, items.size(), (long long)G, (long long)runs,
            runs ? (double)items.size() / (double)runs : 0.0);
  }
  mcfftResult r = plan_alloc(p, &q.items, items.size() * sizeof(QItem));
  if (!r) r = plan_alloc(p, &q.counters, (size_t)std::max<int64_t>(nc, 1) * sizeof(int));
  if (r) return r;
  cudaError_t e = cudaMemcpy(q.items, items.data(), items.size() * sizeof(QItem),
                             cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e);
  q.aux.assign(np, nullptr);
  for (size_t i = 0; i < np; ++i) {
    bool any = false;
    const QPassAux x = make_aux(p, i, &any);
    if (!any) continue;
    QPassAux* d = nullptr;
    r = plan_alloc(p, &d, sizeof(QPassAux));
    if (r) return r;
    e = cudaMemcpy(d, &x, sizeof(x), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e);
    q.aux[i] = d;
  }
  q.nitems = (int64_t)items.size();
  q.ncounters = nc;
  q.grid = (int)std::min<int64_t>(G, q.nitems);
  q.args = new (std::nothrow) QArgs();
  if (!q.args) return MCFFT_ALLOC_FAILED;
  q.stall = std::getenv("MCFFT_INJECT_STALL") != nullptr;
  q.on = true;
  return MCFFT_SUCCESS;
}

mcfftResult exec_queue(mcfftPlan p, const void* in, void* out, int dir, cudaStream_t st) {
  Queue& q = p->q;
  QArgs& A = *q.args;
  A.items = q.items;
  A.nitems = q.nitems;
  A.counters = q.counters;
  A.status = p->status;
  A.bmat = p->bsw64[dir];
  A.bmat_lo = p->bsw64_lo[dir];
  A.npass = (int)p->passes.size();
  auto base = [&](int b) -> char* {
    return b == kUserIn ? (char*)const_cast<void*>(in) : b == kUserOut ? (char*)out : (char*)p->scratch;
  };
  for (size_t i = 0; i < p->passes.size(); ++i) {
    const Pass& ps = p->passes[i];
    QPass& Q = A.pass[i];
    const int ib = ps.in_f16 ? 4 : 8, ob = ps.out_f16 ? 4 : 8;
    if (!fill_qpass(ps.tp, dir, base(ps.in_buf) + ps.in_off * ib, base(ps.out_buf) + ps.out_off * ob,
                    &Q))
      return MCFFT_CUDA_ERROR;
    Q.wait_base = q.wait_base[i];
    Q.wait_count = q.stall && Q.wait_base >= 0 ? INT32_MAX : ps.wait_count;
    Q.sig_base = q.sig_base[i];
    Q.sig_mul = ps.sig_mul;
    Q.sig_div = ps.sig_div;
    Q.sig_kmax = q.sig_base[i] >= 0 ? p->passes[i + 1].keys - 1 : 0;
    set_l2_use(p, i, &Q);
    Q.aux = q.aux[i];
  }
  cudaError_t e = q.ncounters ? cudaMemsetAsync(q.counters, 0, q.ncounters * sizeof(int), st)
                              : cudaSuccess;
  if (e == cudaSuccess)
    e = q.fused ? launch_queue_fn(q.fn, q.smem, A, q.grid, st) : launch_queue(A, q.grid, p->split, st);
  if (e == cudaSuccess && std::getenv("MCFFT_DEBUG_SYNC")) {
    e = cudaStreamSynchronize(st);
    fprintf(stderr, "[mcfft] queue: %d passes, %lld items, grid %d: %s\n", A.npass,
            (long long)q.nitems, q.grid, cudaGetErrorString(e));
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }
  p->last_stream = st;
  return MCFFT_SUCCESS;
}

mcfftResult plan_finish(mcfftPlan p, mcfftPlan* out) {
  mcfftResult r = MCFFT_SUCCESS;
  if (p->scratch_bytes) r = plan_alloc(p, &p->scratch, p->scratch_bytes);
  if (!r) r = build_queue(p);
  if (!r && p->indexed && !p->q.on) r = MCFFT_UNSUPPORTED_SIZE;
  if (!r) r = cuda_fail(cudaDeviceSynchronize());
  if (r) {
    mcfftPlanDestroy(p);
    return r;
  }
  p->info.num_passes = (int)p->passes.size();
  p->info.launches = p->q.on ? 1 : (int)p->passes.size();
  if (!p->passes.empty()) {
    const Pass& f = p->passes[0];
    p->info.tile_points = f.tiled ? f.tp.k->tile_points : 0;
    p->info.ctas = p->q.on ? p->q.grid : (f.tiled ? f.tp.grid : f.grid);
  }
  p->info.workspace_bytes = (int64_t)p->scratch_bytes;
  *out = p;
  return MCFFT_SUCCESS;
}

mcfftResult exec_launches(mcfftPlan p, const void* in, void* out, int dir, cudaStream_t st);

// Replays the launches of an exec from a CUDA graph captured on the second
// exec with the same buffers and direction (the first runs them directly,
// which also completes any one-time kernel configuration).  Returns
// MCFFT_UNSUPPORTED_SIZE when the exec should run directly instead.
mcfftResult exec_graph(mcfftPlan p, const void* in, void* out, int dir, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(p->graph_mu);
  if (!p->graphs_on) return MCFFT_UNSUPPORTED_SIZE;
  mcfftPlan_st::GraphEntry* e = nullptr;
  for (auto& g : p->graphs)
    if (g.in == in && g.out == out && g.dir == dir) e = &g;
  if (!e) {
    e = &p->graphs[0];
    for (auto& g : p->graphs)
      if (g.stamp < e->stamp) e = &g;
    if (e->exec) cudaGraphExecDestroy(e->exec);
    *e = mcfftPlan_st::GraphEntry();
    e->in = in;
    e->out = out;
    e->dir = dir;
  }
  e->stamp = ++p->graph_clock;
  if (!e->exec && e->uses++ == 0) return MCFFT_UNSUPPORTED_SIZE;
  if (!e->exec) {
    if (!p->capture_stream &&
        cudaStreamCreateWithFlags(&p->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      p->graphs_on = false;
      return MCFFT_UNSUPPORTED_SIZE;
    }
    cudaGraph_t g = nullptr;
    mcfftResult r = MCFFT_CUDA_ERROR;
    if (cudaStreamBeginCapture(p->capture_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      r = exec_launches(p, in, out, dir, p->capture_stream);
      if (cudaStreamEndCapture(p->capture_stream, &g) != cudaSuccess) r = MCFFT_CUDA_ERROR;
    }
    if (r == MCFFT_SUCCESS && g && cudaGraphInstantiate(&e->exec, g, 0) != cudaSuccess) {
      e->exec = nullptr;
      r = MCFFT_CUDA_ERROR;
    }
    if (g) cudaGraphDestroy(g);
    if (r != MCFFT_SUCCESS) {
      // not capturable here: run this plan's execs directly from now on
      cudaGetLastError();
      p->graphs_on = false;
      return MCFFT_UNSUPPORTED_SIZE;
    }
  }
  if (cudaGraphLaunch(e->exec, st) != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }
  p->last_stream = st;
  return MCFFT_SUCCESS;
}

// One pass on the stream: `src` and `dst` are its input and output with
// the pass's element offsets already applied.  `follows`: a pass of the
// same exec ran just before on the stream.
cudaError_t launch_one(mcfftPlan p, const Pass& ps, const void* src, void* dst, int dir,
                       cudaStream_t st, bool follows) {
  if (ps.tiled) {
    cudaError_t e = launch_tile_pass(ps.tp, src, dst, dir, st, follows && p->pdl);
    if (e == cudaSuccess && std::getenv("MCFFT_DEBUG_SYNC")) {
      e = cudaStreamSynchronize(st);
      fprintf(stderr, "[mcfft] tile pass L=%d R=%d C=%d grid=%d tiles=%lld: %s\n", ps.tp.k->L,
              ps.tp.k->R, ps.tp.k->C, ps.tp.grid, (long long)ps.tp.args.ntiles,
              cudaGetErrorString(e));
    }
    return e;
  }
  PassArgs a = ps.a;
  a.in = src;
  a.out = dst;
  a.tw = ps.tw[dir];
  a.tail_tw = ps.tail[dir];
  a.post_lo = ps.plo[dir];
  a.post_hi = ps.phi[dir];
  a.bmat = p->bmat[dir];
  a.bmat_lo = p->bmat_lo[dir];
  a.inverse = dir;
  return launch_pass(*ps.k, a, ps.grid, st);
}

// Element size (bytes) at the input / output end of a pass.
int in_elem(const mcfftPlan p, const Pass& ps) { return p->split ? (ps.in_f16 ? 4 : 8) : 4; }
int out_elem(const mcfftPlan p, const Pass& ps) { return p->split ? (ps.out_f16 ? 4 : 8) : 4; }

mcfftResult exec_launches(mcfftPlan p, const void* in, void* out, int dir, cudaStream_t st) {
  if (p->q.on) return exec_queue(p, in, out, dir, st);
  for (size_t i = 0; i < p->passes.size(); ++i) {
    const Pass& ps = p->passes[i];
    auto base = [&](int b) -> char* {
      return b == kUserIn ? (char*)const_cast<void*>(in) : b == kUserOut ? (char*)out : (char*)p->scratch;
    };
    cudaError_t e = launch_one(p, ps, base(ps.in_buf) + ps.in_off * in_elem(p, ps),
                               base(ps.out_buf) + ps.out_off * out_elem(p, ps), dir, st, i > 0);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return MCFFT_CUDA_ERROR;
    }
  }
  p->last_stream = st;
  return MCFFT_SUCCESS;
}

// Chunks and device buffers of mcfftExecHost.  A single-shape plan (one
// descriptor, no offsets) follows the chunk schedule of host_schedule.h,
// with one plan per chunk length; anything else is one chunk run by the
// plan itself.
mcfftResult host_pipe_setup(mcfftPlan p) {
  auto& h = p->host;
  const mcfftDesc& d = p->desc0;
  const bool single = p->ndesc == 1 && d.in_offset == 0 && d.out_offset == 0 && d.batch > 1;
  size_t max_in = (size_t)p->in_extent, max_out = (size_t)p->out_extent;
  if (single) {
    int64_t target = int64_t(32) << 20;
    if (const char* e = std::getenv("MCFFT_HOST_CHUNK_BYTES")) target = std::max<int64_t>(1, std::atoll(e));
    h.in_per = (size_t)(p->info.in_bytes / d.batch);
    h.out_per = (size_t)(p->info.out_bytes / d.batch);
    const int64_t big = host_chunk_big(d.batch, (int64_t)h.in_per, target);
    int64_t first = 0;
    for (int64_t c : host_schedule(d.batch, big)) {
      mcfftPlan x = nullptr;
      if (c == d.batch) x = p;
      for (auto& pr : h.plans)
        if (pr.first == c) x = pr.second;
      if (!x) {
        mcfftDesc cd = d;
        cd.batch = c;
        mcfftResult r = mcfftPlanCreateBatch(&x, &cd, 1, p->prec, p->flags);
        if (r) return r;
        h.plans.push_back({c, x});
      }
      h.chunks.push_back({first, c, x});
      first += c;
    }
    max_in = (size_t)big * h.in_per;
    max_out = (size_t)big * h.out_per;
  } else {
    h.in_per = max_in;
    h.out_per = max_out;
    h.chunks.push_back({0, 1, p});
  }
  h.nbuf = (int)std::min<size_t>(mcfftPlan_st::kHostRing, h.chunks.size());
  for (int b = 0; b < h.nbuf; ++b) {
    mcfftResult r = plan_alloc(p, &h.din[b], max_in);
    if (!r) r = plan_alloc(p, &h.dout[b], max_out);
    if (r) return r;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&h.s_in, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h.s_out, cudaStreamNonBlocking);
  std::vector<cudaEvent_t*> evs = {&h.start, &h.done};
  for (int b = 0; b < h.nbuf; ++b) {
    evs.push_back(&h.loaded[b]);
    evs.push_back(&h.computed[b]);
    evs.push_back(&h.stored[b]);
  }
  for (cudaEvent_t* ev : evs)
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  if (e != cudaSuccess) return cuda_fail(e);
  h.ready = true;
  return MCFFT_SUCCESS;
}

void host_pipe_release(mcfftPlan p) {
  auto& h = p->host;
  for (auto& pr : h.plans) mcfftPlanDestroy(pr.second);
  if (h.s_in) cudaStreamDestroy(h.s_in);
  if (h.s_out) cudaStreamDestroy(h.s_out);
  std::vector<cudaEvent_t> evs = {h.start, h.done};
  for (int b = 0; b < mcfftPlan_st::kHostRing; ++b) {
    evs.push_back(h.loaded[b]);
    evs.push_back(h.computed[b]);
    evs.push_back(h.stored[b]);
  }
  for (cudaEvent_t ev : evs)
    if (ev) cudaEventDestroy(ev);
  h = mcfftPlan_st::HostPipe();
}

// Chunk i, ring slot b = i % nbuf: copy in on s_in into din[b] once the
// transform of chunk i - nbuf has read it; transform on the caller's stream
// once chunk i is in and the copy out of chunk i - nbuf has drained dout[b];
// copy out on s_out.  The caller's stream waits for the last copy out.
mcfftResult exec_host(mcfftPlan p, const char* hin, char* hout, int direction, cudaStream_t st) {
  auto& h = p->host;
  cudaError_t e = cudaEventRecord(h.start, st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h.s_in, h.start, 0);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h.s_out, h.start, 0);
  const int64_t n = (int64_t)h.chunks.size();
  for (int64_t i = 0; i < n && e == cudaSuccess; ++i) {
    const mcfftPlan_st::HostChunk& c = h.chunks[i];
    const int b = (int)(i % h.nbuf);
    if (i >= h.nbuf) e = cudaStreamWaitEvent(h.s_in, h.computed[b], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h.din[b], hin + c.first * h.in_per, c.count * h.in_per,
                          cudaMemcpyHostToDevice, h.s_in);
    if (e == cudaSuccess) e = cudaEventRecord(h.loaded[b], h.s_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h.loaded[b], 0);
    if (e == cudaSuccess && i >= h.nbuf) e = cudaStreamWaitEvent(st, h.stored[b], 0);
    if (e != cudaSuccess) break;
    const mcfftResult r = mcfftExec(c.plan, h.din[b], h.dout[b], direction, st);
    if (r) return r;
    e = cudaEventRecord(h.computed[b], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h.s_out, h.computed[b], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hout + c.first * h.out_per, h.dout[b], c.count * h.out_per,
                          cudaMemcpyDeviceToHost, h.s_out);
    if (e == cudaSuccess) e = cudaEventRecord(h.stored[b], h.s_out);
  }
  if (e == cudaSuccess) e = cudaEventRecord(h.done, h.s_out);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(st, h.done, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }
  p->last_stream = st;
  return MCFFT_SUCCESS;
}

}  // namespace
}  // namespace mcfft

using namespace mcfft;

extern "C" {

}  // extern "C"

namespace mcfft {
namespace {

// The plan of a batch of descriptors.  by_shape: one group per shape
// (indexed where its transforms are not contiguous and in order; *indexed
// tells whether any was); else one group per run of consecutive
// descriptors of one shape whose data follow each other in both buffers.
mcfftResult create_batch(mcfftPlan* plan, const mcfftDesc* descs, int count,
                         mcfftPrecision precision, unsigned flags, bool by_shape, bool* indexed) {
  mcfftPlan p = nullptr;
  mcfftResult r = plan_begin(plan, precision, flags, &p);
  if (r) return r;
  int64_t elements = 0;
  auto points = [](const mcfftDesc& d) {
    int64_t t = 1;
    for (int k = 0; k < d.ndim; ++k) t *= d.dims[k];
    return t;
  };
  // group boundaries: i starts a group unless it continues the previous one
  auto continues = [&](int i, const mcfftDesc& g) {
    const mcfftDesc& d = descs[i];
    bool same = d.ndim == g.ndim;
    for (int k = 0; k < g.ndim && same; ++k) same = d.dims[k] == g.dims[k];
    const int64_t len = g.batch * points(g);
    return same && d.in_offset == g.in_offset + len && d.out_offset == g.out_offset + len;
  };
  // Groups: (shape, per-transform input and output offsets) in order of
  // first appearance.
  struct Group {
    mcfftDesc shape;
    std::vector<int64_t> in, out;
  };
  std::vector<Group> groups;
  if (by_shape) {
    for (int i = 0; i < count; ++i) {
      const mcfftDesc& d = descs[i];
      Group* g = nullptr;
      for (auto& x : groups) {
        bool same = x.shape.ndim == d.ndim;
        for (int k = 0; k < d.ndim && same; ++k) same = x.shape.dims[k] == d.dims[k];
        if (same) g = &x;
      }
      if (!g) {
        groups.push_back(Group{d, {}, {}});
        g = &groups.back();
      }
      const int64_t n = points(d);
      for (int64_t b = 0; b < d.batch; ++b) {
        g->in.push_back(d.in_offset + b * n);
        g->out.push_back(d.out_offset + b * n);
      }
    }
    // groups are independent: queue them by dimensionality, then shape
    std::stable_sort(groups.begin(), groups.end(), [](const Group& a, const Group& b) {
      if (a.shape.ndim != b.shape.ndim) return a.shape.ndim < b.shape.ndim;
      for (int k = 0; k < a.shape.ndim; ++k)
        if (a.shape.dims[k] != b.shape.dims[k]) return a.shape.dims[k] < b.shape.dims[k];
      return false;
    });
  } else {
    for (int i = 0; i < count;) {
      mcfftDesc g = descs[i];
      for (++i; i < count && continues(i, g); ++i) g.batch += descs[i].batch;
      const int64_t n = points(g);
      Group x{g, {}, {}};
      for (int64_t b = 0; b < g.batch; ++b) {
        x.in.push_back(g.in_offset + b * n);
        x.out.push_back(g.out_offset + b * n);
      }
      groups.push_back(x);
    }
  }
  p->queue_planned = groups.size() > 1;
  if (const char* e = std::getenv("MCFFT_QUEUE")) p->queue_planned = std::atoi(e) != 0;
  for (size_t gi = 0; gi < groups.size() && !r; ++gi) {
    const Group& g = groups[gi];
    const int64_t n = points(g.shape), B = (int64_t)g.in.size();
    bool affine = true;
    for (int64_t b = 0; b < B && affine; ++b)
      affine = g.in[b] == g.in[0] + b * n && g.out[b] == g.out[0] + b * n;
    int sl = 0;
    if (affine) {
      r = build_group(p, g.shape.ndim, g.shape.dims, B, g.in[0], g.out[0], &sl);
    } else {
      *indexed = true;
      r = build_indexed_group(p, g.shape.ndim, g.shape.dims, g.in, g.out, &sl);
    }
    elements += B * n;
    if (gi == 0) {
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
  const int out_b = p->split ? 8 : 4;
  p->info.in_bytes = elements * in_b;
  p->info.out_bytes = elements * out_b;
  p->desc0 = descs[0];
  p->ndesc = count;
  for (int i = 0; i < count; ++i) {
    const int64_t len = descs[i].batch * points(descs[i]);
    p->in_extent = std::max(p->in_extent, (descs[i].in_offset + len) * in_b);
    p->out_extent = std::max(p->out_extent, (descs[i].out_offset + len) * out_b);
  }
  return plan_finish(p, plan);
}

}  // namespace
}  // namespace mcfft

extern "C" {

mcfftResult mcfftPlanCreateBatch(mcfftPlan* plan, const mcfftDesc* descs, int count,
                                 mcfftPrecision precision, unsigned flags) {
  if (!plan || !descs || count <= 0) return MCFFT_INVALID_VALUE;
  for (int i = 0; i < count; ++i)
    if (descs[i].ndim < 1 || descs[i].ndim > 3 || descs[i].batch < 1 || descs[i].in_offset < 0 ||
        descs[i].out_offset < 0)
      return MCFFT_INVALID_VALUE;
  // Transforms of one shape form one group, wherever they lie (descriptors
  // in any order); if that plan cannot run (an indexed group the batch
  // kernel cannot take), groups of consecutive contiguous descriptors
  // instead (MCFFT_GROUPING=adjacent forces that).
  bool by_shape = true;
  if (const char* e = std::getenv("MCFFT_GROUPING")) by_shape = std::strcmp(e, "adjacent") != 0;
  if (by_shape) {
    bool indexed = false;
    const mcfftResult r = create_batch(plan, descs, count, precision, flags, true, &indexed);
    if (r != MCFFT_UNSUPPORTED_SIZE || !indexed) return r;
  }
  bool unused = false;
  return create_batch(plan, descs, count, precision, flags, false, &unused);
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
  const mcfftResult r = exec_graph(p, in, out, dir, st);
  if (r != MCFFT_UNSUPPORTED_SIZE) return r;
  return exec_launches(p, in, out, dir, st);
}

mcfftResult mcfftExecHost(mcfftPlan p, const void* host_in, void* host_out, int direction,
                          void* stream) {
  if (!p) return MCFFT_INVALID_PLAN;
  if (!host_in || !host_out) return MCFFT_INVALID_VALUE;
  if (direction != MCFFT_FORWARD && direction != MCFFT_INVERSE) return MCFFT_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(p->host_mu);
  if (!p->host.ready) {
    const mcfftResult r = host_pipe_setup(p);
    if (r) {
      host_pipe_release(p);
      return r;
    }
  }
  // The copy out of one chunk may not overwrite input a later chunk has
  // still to copy in: the buffers must be disjoint, or identical with
  // chunks of equal size on both sides.
  const char* a = static_cast<const char*>(host_in);
  const char* b = static_cast<const char*>(host_out);
  const bool overlap = a < b + p->out_extent && b < a + p->in_extent;
  if (overlap && (a != b || p->host.in_per != p->host.out_per)) return MCFFT_INVALID_VALUE;
  return exec_host(p, a, static_cast<char*>(host_out), direction, static_cast<cudaStream_t>(stream));
}

mcfftResult mcfftPlanCheckStatus(mcfftPlan p) {
  if (!p) return MCFFT_INVALID_PLAN;
  for (auto& pr : p->host.plans) {
    const mcfftResult r = mcfftPlanCheckStatus(pr.second);
    if (r) return r;
  }
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
  host_pipe_release(p);
  for (auto& g : p->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (p->capture_stream) cudaStreamDestroy(p->capture_stream);
  for (void* d : p->allocs) cudaFree(d);
  delete p->q.args;
  delete p;
  return MCFFT_SUCCESS;
}

mcfftResult mcfftWisdomExport(const char* path) {
  if (!path) return MCFFT_INVALID_VALUE;
  FILE* f = std::fopen(path, "w");
  if (!f) return MCFFT_INVALID_VALUE;
  Wisdom& w = wisdom();
  std::lock_guard<std::mutex> lk(w.mu);
  bool ok = std::fprintf(f, "mcfft-wisdom 1\n") > 0;
  for (auto& r : w.recs) ok = ok && std::fprintf(f, "%s\t%d\n", r.first.c_str(), r.second) > 0;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? MCFFT_SUCCESS : MCFFT_INVALID_VALUE;
}

mcfftResult mcfftWisdomImport(const char* path) {
  if (!path) return MCFFT_INVALID_VALUE;
  FILE* f = std::fopen(path, "r");
  if (!f) return MCFFT_INVALID_VALUE;
  std::vector<std::pair<std::string, int>> got;
  char line[1024];
  bool ok = std::fgets(line, sizeof line, f) && std::strcmp(line, "mcfft-wisdom 1\n") == 0;
  while (ok && std::fgets(line, sizeof line, f)) {
    std::string l(line);
    if (!l.empty() && l.back() == '\n') {
      l.pop_back();
    } else if (!std::feof(f)) {
      ok = false;  // a line longer than the buffer
      break;
    }
    if (l.empty()) continue;
    // four tab-separated fields; the value is a supported tile size
    const size_t t3 = l.rfind('\t');
    size_t tabs = 0;
    for (char c : l) tabs += c == '\t';
    if (tabs != 3 || t3 == std::string::npos) { ok = false; break; }
    const std::string v = l.substr(t3 + 1);
    char* end = nullptr;
    const long tp = std::strtol(v.c_str(), &end, 10);
    // tile-shape records hold 8192 or 16384 points; four-step records lg n1
    // (4..13), -1 (three passes) or -2 (one two-column pass)
    const bool fs = l.find("\tfourstep ") != std::string::npos;
    const bool fs_ok = (tp >= 4 && tp <= 13) || tp == kThreePass || tp == kOnePass;
    if (v.empty() || *end || (fs ? !fs_ok : (tp != 8192 && tp != 16384))) {
      ok = false;
      break;
    }
    got.push_back({l.substr(0, t3), (int)tp});
  }
  std::fclose(f);
  if (!ok) return MCFFT_INVALID_VALUE;
  for (auto& r : got) wisdom_put(r.first, r.second);
  return MCFFT_SUCCESS;
}

mcfftResult mcfftWisdomForget(void) {
  Wisdom& w = wisdom();
  std::lock_guard<std::mutex> lk(w.mu);
  w.recs.clear();
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
