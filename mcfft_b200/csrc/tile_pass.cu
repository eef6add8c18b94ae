// tile_pass.cu -- host side of the TMA-fed pass kernel (fft_tile.cuh):
// variant registry, plan-time table construction and exec-time tensor-map
// encoding and launch.
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <utility>
#include <string>
#include <vector>

#include "fft_tile.cuh"
#include "layout.h"
#include "tile_pass.h"

namespace mcfft {

namespace {

// Two tile sizes, both with 16 consumer warps at one CTA per SM: 16K points
// (the default), and 8K points, half the work per thread and so about half
// the latency per tile, which the plan-time tuner takes where a pass has
// too few tiles to fill the SMs (small batches).  8K tiles need at least
// four columns (L <= 2048).  These 8K routines are the ones the batch
// kernel runs for a pass tuned to 8K.
template <int L, int R, bool PT, int TP, int NCW>
TileKernel make_f16() {
  constexpr int C = TP / L;
  using T = TileF16<L, R, C, PT, NCW>;
  using S = TileShape<L, R, C, NCW>;
  return TileKernel{reinterpret_cast<const void*>(&fft_tile_f16<L, R, C, PT, NCW>),
                    L, R, C, PT, false, S::NT, T::SMEM_BYTES, F16Tile<L, R, C, PT, NCW>::TMEM_COLS,
                    TP, true};
}

#define MCFFT_TILE_VARIANTS(PT, TP, NCW)                                                  \
  make_f16<32, 2, PT, TP, NCW>(), make_f16<64, 4, PT, TP, NCW>(),                         \
      make_f16<128, 8, PT, TP, NCW>(), make_f16<256, 1, PT, TP, NCW>(),                   \
      make_f16<512, 2, PT, TP, NCW>(), make_f16<1024, 4, PT, TP, NCW>(),                  \
      make_f16<2048, 8, PT, TP, NCW>(), make_f16<4096, 1, PT, TP, NCW>()

// L = 16 (one radix-16 stage, 1024 or 512 columns per tile): column passes
// only (the layout engine has no row staging for it), never with the
// four-step twiddle; the sides of 16 of 2D and 3D transforms.  L = 8192
// (two columns per 16K-point tile, radix-2 twiddles computed): row-in /
// row-out passes only (1D 8192 in one pass, rows of 8192).
const std::vector<TileKernel>& registry() {
  static const std::vector<TileKernel> v = {
      MCFFT_TILE_VARIANTS(false, 16384, 16), MCFFT_TILE_VARIANTS(true, 16384, 16),
      MCFFT_TILE_VARIANTS(false, 8192, 16), MCFFT_TILE_VARIANTS(true, 8192, 16),
      make_f16<16, 1, false, 16384, 16>(), make_f16<16, 1, false, 8192, 16>(),
      make_f16<8192, 2, false, 16384, 16>()};
  return v;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

bool encode(CUtensorMap* map, const layout::Staging& s, const void* base) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t gdim[5], gstr[4];
  cuuint32_t box[5], estr[5];
  for (int d = 0; d < s.ndims; ++d) {
    gdim[d] = s.gdim[d];
    box[d] = s.box[d];
    estr[d] = 1;
    if (d > 0) gstr[d - 1] = s.gstride_bytes[d];
  }
  const CUtensorMapSwizzle sw = s.swz == 7 ? CU_TENSOR_MAP_SWIZZLE_128B
                                : s.swz == 3 ? CU_TENSOR_MAP_SWIZZLE_64B
                                : s.swz == 1 ? CU_TENSOR_MAP_SWIZZLE_32B
                                             : CU_TENSOR_MAP_SWIZZLE_NONE;
  const CUtensorMapDataType dt =
      s.elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32;
  CUresult r = fn(map, dt, (cuuint32_t)s.ndims, const_cast<void*>(base), gdim, gstr, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// Layouts are pure functions of their parameters; memoise them per process.
// Layouts already built, by pass shape (the search takes up to seconds).
// Bounded: past kLayoutCacheMax entries the oldest is dropped, so a process
// that plans many batch sizes does not grow without limit.
constexpr size_t kLayoutCacheMax = 256;
std::mutex g_lay_mu;
std::map<std::string, layout::PassLayout> g_lay_cache;
std::deque<std::string> g_lay_order;  // insertion order of g_lay_cache's keys

}  // namespace

const TileKernel* find_tile_kernel(int L, bool posttw, bool split, int tile_points, bool in16) {
  for (const auto& k : split ? split_registry() : registry())
    if (k.L == L && k.posttw == posttw && k.tile_points == tile_points && (!split || k.in16 == in16))
      return &k;
  return nullptr;
}

bool tile_layout(layout::PassLayout* out, int L, int R, int C, layout::Kind ik, layout::Kind ok,
                 int in_elem, int out_elem, int64_t isp, int64_t isc, int64_t iso, int64_t osp,
                 int64_t osc, int64_t oso, int64_t ncols, int64_t nouter, std::string* err,
                 int unsw) {
  char key[512];
  snprintf(key, sizeof key, "%d %d %d %d %d %d %d %lld %lld %lld %lld %lld %lld %lld %lld %d", L,
           R, C, (int)ik, (int)ok, in_elem, out_elem, (long long)isp, (long long)isc,
           (long long)iso, (long long)osp, (long long)osc, (long long)oso, (long long)ncols,
           (long long)nouter, unsw);
  {
    std::lock_guard<std::mutex> lk(g_lay_mu);
    auto it = g_lay_cache.find(key);
    if (it != g_lay_cache.end()) {
      *out = it->second;
      return true;
    }
  }
  if (!layout::build(out, L, R, C, ik, ok, in_elem, out_elem, isp, isc, iso, osp, osc, oso, ncols,
                     nouter, err, unsw))
    return false;
  // The kernels size their table reads at compile time (TileShape): items,
  // epilogue rows and stages must be exactly what the layout holds.
  const int items = R == 1 ? L * C / 16 : L * C / (4 * R);
  if (out->items != items || out->NROWS != L / 16 * C ||
      (int)out->item_tab.size() != 2 * items ||
      out->epi_tab.size() != (size_t)out->NST * out->NROWS || out->kofs.size() != (size_t)out->NST * 16) {
    *err = "layout tables do not match the kernel's tile shape";
    return false;
  }
  std::lock_guard<std::mutex> lk(g_lay_mu);
  if (g_lay_cache.emplace(key, *out).second) {
    g_lay_order.push_back(key);
    while (g_lay_order.size() > kLayoutCacheMax) {
      g_lay_cache.erase(g_lay_order.front());
      g_lay_order.pop_front();
    }
  }
  return true;
}

bool tile_encode(CUtensorMap* map, const layout::Staging& s, const void* base) {
  return encode(map, s, base);
}

bool tile_check_encode(const layout::Staging& s, const void* probe) {
  CUtensorMap m;
  return encode(&m, s, probe);
}

cudaError_t launch_tile_pass(const TilePass& tp, const void* in, void* out, int dir,
                             cudaStream_t st, bool pdl) {
  TileArgs a = tp.args;
  if (!encode(&a.tmap_in, tp.lay.in, in) || !encode(&a.tmap_out, tp.lay.out, out))
    return cudaErrorInvalidValue;
  a.tw = tp.tw[dir];
  a.tail_tw = tp.tail[dir];
  a.post_a = tp.post_a[dir];
  a.post_b = tp.post_b[dir];
  a.bmat = tp.bmat[dir];
  a.bmat_lo = tp.bmat_lo[dir];
  a.inverse = dir;
  // The shared-memory limit is a per-device attribute of the function.
  static std::mutex mu;
  static std::vector<std::pair<int, const void*>> configured;
  {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cudaGetLastError();
    std::lock_guard<std::mutex> lock(mu);
    bool done = false;
    for (const auto& f : configured) done |= (f.first == dev && f.second == tp.k->fn);
    if (!done) {
      cudaError_t e = cudaFuncSetAttribute(tp.k->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           tp.k->smem_bytes);
      if (e != cudaSuccess) return e;
      configured.push_back({dev, tp.k->fn});
    }
  }
  void* args[] = {&a};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tp.grid);
  cfg.blockDim = dim3(tp.k->nthreads);
  cfg.dynamicSmemBytes = (size_t)tp.k->smem_bytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelExC(&cfg, tp.k->fn, args);
}

void fill_tile_args(TilePass* tp) {
  const layout::PassLayout& l = tp->lay;
  TileArgs& a = tp->args;
  std::memset(&a, 0, sizeof(a));
  a.in_ndims = l.in.ndims;
  a.out_ndims = l.out.ndims;
  for (int d = 0; d < 5; ++d) {
    a.in_cmul[d] = l.in.cmul[d];
    a.in_omul[d] = l.in.omul[d];
    a.out_cmul[d] = l.out.cmul[d];
    a.out_omul[d] = l.out.omul[d];
  }
  a.in_tile_bytes = l.in.box_bytes();
  a.tail_pm = l.tail_pm;
  for (size_t i = 0; i < l.lofs.size() && i < 16; ++i) a.lofs[i] = l.lofs[i];
  for (size_t i = 0; i < l.sofs.size() && i < 32; ++i) a.sofs[i] = l.sofs[i];
  for (int s = 0; s < l.NST && s < kMaxStages; ++s)
    for (int k = 0; k < 16; ++k) a.kofs[s][k] = l.kofs[(size_t)s * 16 + k];
}

}  // namespace mcfft
