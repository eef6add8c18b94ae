// fft_tile.cuh -- warp-specialised, TMA-fed FFT pass kernel (sm_100a).
//
// One persistent CTA per SM processes tiles of C columns x L points
// (L = 16^a * R, R in {1,2,4,8}) of one pass of a batched C2C FFT:
//
//   producer warp   TMA bulk-tensor load of tile i+2 into staging buffer
//                   b = i % 2 once tile i's output has left it; TMA bulk-
//                   tensor store of tile i's output from the same buffer
//   consumer warps  prologue: staging -> registers -> [radix-R stage in
//                   FP32] -> FP16 -> tcgen05 A operand (K-major, 64-byte
//                   swizzle); per radix-16 stage: one thread issues the
//                   tcgen05.mma (D = A * DFT16, FP32 in TMEM), every warp
//                   drains its TMEM sub-partition with tcgen05.ld, applies
//                   twiddle and scale, and stores into the next stage's A
//                   rows -- or, after the last stage, into the staging
//                   buffer in natural order for the TMA store.
//
// All addressing comes from host-built tables (layout.cpp): per prologue
// item a load/store base, per A row and stage a destination base; the
// per-element offsets are XOR constants passed as kernel parameters, so a
// stored element costs one XOR and one st.shared.  The layouts are chosen
// on the host to be free of shared-memory bank conflicts.
//
// Synchronisation: mbarriers for TMA completion (full[b]), for "output
// staged" (outrdy[b]) and for MMA completion (dfull, via tcgen05.commit);
// named barrier 1 among consumer warps.  Every wait is bounded; on timeout
// the kernel records kStatusTimeout in the status word and winds down.
#pragma once
#include <cuda.h>
#include <cstdint>
#include <cuda_fp16.h>

#include "fft_pass.cuh"
#include "mcfft_internal.h"
#include "sm100_ptx.cuh"
#include "tail_layout.h"

namespace mcfft {

constexpr int kMaxStages = 4;

struct alignas(64) TileArgs {
  CUtensorMap tmap_in;
  CUtensorMap tmap_out;
  int32_t in_cmul[5], in_omul[5], out_cmul[5], out_omul[5];
  int32_t in_ndims, out_ndims;
  int64_t col_blocks, ntiles;
  uint32_t in_tile_bytes;
  const uint2* item_tab;   // per prologue item: {lds_base>>2 | sts_base>>2 << 16, tail twiddle row}
  const uint32_t* epi_tab; // [stage][row]: dst_base>>2 | aux << 16
  uint32_t lofs[16];       // XOR offsets of an item's loads
  uint32_t sofs[32];       // XOR offsets of an item's stores
  uint32_t kofs[kMaxStages][16];
  const float4* tw;        // stage twiddle rows (8 chunks of 16 B per R'), stages concatenated
  const float2* tail_tw;   // radix-R twiddles (scaled by 1/R), [v][k]
  const uint4* bmat;       // DFT-16 embedding (hi), 64B-swizzled K-major, 2 KB
  const uint4* bmat_lo;    // split form: low part
  const float2* post_a;    // four-step: W_N^e low table, e in [0, 2^post_shift)
  const float2* post_b;    // four-step: W_N^(e << post_shift) high table
  uint64_t post_mask;      // N - 1
  uint32_t post_shift;
  float post_scale;        // 2 / N when N <= 2^24 (four-step twiddles by sincospif), else 0
  float out_scale;         // split form: applied after the last stage (the plain form keeps its 1/16 per stage in the DFT-16 matrix)
  int inverse;
  int split_in_f16;
  int32_t tail_pm;         // radix-R table layout (tail_layout.h): -1 natural, t >= 0 folded
  int* status;
};

namespace tile {

__device__ __forceinline__ void named_bar(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(sm100::smem_u32(bar)) : "memory");
}
__device__ __forceinline__ uint4 lds128(uint32_t addr) {
  uint4 v;
  asm volatile("ld.shared.v4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(addr));
  return v;
}
__device__ __forceinline__ void sts128(uint32_t addr, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z),
               "r"(v.w)
               : "memory");
}
__device__ __forceinline__ uint2 lds64(uint32_t addr) {
  uint2 v;
  asm volatile("ld.shared.v2.b32 {%0,%1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(addr));
  return v;
}
__device__ __forceinline__ void sts32(uint32_t addr, uint32_t v) {
  asm volatile("st.shared.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ void sts64(uint32_t addr, float2 v) {
  asm volatile("st.shared.v2.f32 [%0], {%1,%2};" ::"r"(addr), "f"(v.x), "f"(v.y) : "memory");
}

// Brings a tensor map (a kernel parameter's generic address) into the
// descriptor cache ahead of the copy that uses it.
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// TMA bulk-tensor load / store of one tile; coordinates from the recipe.
__device__ __forceinline__ void tma_load(const CUtensorMap* map, int nd, const int32_t* crd,
                                         uint32_t dst, uint64_t* bar) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  const uint32_t mb = sm100::smem_u32(bar);
  if (nd == 3)
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(m), "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(mb)
        : "memory");
  else if (nd == 4)
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(m), "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(crd[3]), "r"(mb)
        : "memory");
  else
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(m), "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(crd[3]), "r"(crd[4]), "r"(mb)
        : "memory");
}
__device__ __forceinline__ void tma_store(const CUtensorMap* map, int nd, const int32_t* crd,
                                          uint32_t src) {
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  if (nd == 3)
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(m),
                 "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(src)
                 : "memory");
  else if (nd == 4)
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(m),
                 "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(crd[3]), "r"(src)
                 : "memory");
  else
    asm volatile(
        "cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(m),
        "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(crd[3]), "r"(crd[4]), "r"(src)
        : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// The same with an L2 cache policy (createpolicy) attached: `pol` 0 means
// none.  Used by the batch kernels to keep an intermediate resident in L2
// while the input and output stream through it.
__device__ __forceinline__ void tma_load_pol(const CUtensorMap* map, int nd, const int32_t* crd,
                                             uint32_t dst, uint64_t* bar, uint64_t pol) {
  if (!pol) {
    tma_load(map, nd, crd, dst, bar);
    return;
  }
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  const uint32_t mb = sm100::smem_u32(bar);
  if (nd == 3)
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(dst),
        "l"(m), "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(mb), "l"(pol)
        : "memory");
  else if (nd == 4)
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3, %4, %5}], [%6], %7;" ::"r"(dst),
        "l"(m), "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(crd[3]), "r"(mb), "l"(pol)
        : "memory");
  else
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7], %8;" ::"r"(dst),
        "l"(m), "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(crd[3]), "r"(crd[4]), "r"(mb), "l"(pol)
        : "memory");
}
__device__ __forceinline__ void tma_store_pol(const CUtensorMap* map, int nd, const int32_t* crd,
                                              uint32_t src, uint64_t pol) {
  if (!pol) {
    tma_store(map, nd, crd, src);
    return;
  }
  const uint64_t m = reinterpret_cast<uint64_t>(map);
  if (nd == 3)
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%1, %2, %3}], [%4], %5;" ::"l"(m),
        "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(src), "l"(pol)
        : "memory");
  else if (nd == 4)
    asm volatile(
        "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%1, %2, %3, %4}], [%5], %6;" ::"l"(m),
        "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(crd[3]), "r"(src), "l"(pol)
        : "memory");
  else
    asm volatile(
        "cp.async.bulk.tensor.5d.global.shared::cta.bulk_group.L2::cache_hint [%0, {%1, %2, %3, %4, %5}], [%6], %7;" ::"l"(m),
        "r"(crd[0]), "r"(crd[1]), "r"(crd[2]), "r"(crd[3]), "r"(crd[4]), "r"(src), "l"(pol)
        : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Row gathers and scatters of a 2D tensor map whose rows hold E points
// (box: E x 1): four rows at the given row coordinates, placed one after
// another (4 x row bytes) at dst / read from src.  For passes whose
// columns (transforms) lie at unrelated offsets of the buffer.
__device__ __forceinline__ void tma_gather4(const CUtensorMap* map, uint32_t dst, uint64_t* bar,
                                            int32_t r0, int32_t r1, int32_t r2, int32_t r3) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3),
      "r"(sm100::smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_scatter4(const CUtensorMap* map, uint32_t src, int32_t r0,
                                             int32_t r1, int32_t r2, int32_t r3) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.tile::scatter4.bulk_group"
      " [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(reinterpret_cast<uint64_t>(map)),
      "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(src)
      : "memory");
}
// L2 policies for all accesses of an instruction: evict first (streamed
// data) or evict last (data read again soon).
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// Drops one 128-byte line from L2 without writing it back (its contents
// become undefined): for an intermediate that has been read for the last
// time.
__device__ __forceinline__ void discard_l2_line(const void* p) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}
__device__ __forceinline__ void tma_store_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void tma_store_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// K-major, 64-byte-swizzled shared-memory matrix descriptor (8-row atoms of
// 512 bytes; `sbo` = 512 between atoms).
__device__ __forceinline__ uint64_t sdesc_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
  d |= static_cast<uint64_t>(1) << 16;                 // LBO (unused for swizzled K-major)
  d |= static_cast<uint64_t>(512u >> 4) << 32;         // SBO
  d |= static_cast<uint64_t>(1) << 46;                 // sm_100 descriptor version
  d |= static_cast<uint64_t>(4) << 61;                 // SWIZZLE_64B
  return d;
}

__device__ __forceinline__ void tile_coords(const int32_t* cm, const int32_t* om, int64_t cb,
                                            int64_t outer, int32_t* crd) {
#pragma unroll
  for (int d = 0; d < 5; ++d) crd[d] = (int32_t)(cb * cm[d] + outer * om[d]);
}

}  // namespace tile

template <int L, int R, int C, int NCW>
struct TileShape {
  static constexpr int NV = L / 16;
  static constexpr int NROWS = NV * C;
  static constexpr int NMT = NROWS / 128;
  static constexpr int NST = ilog2c(L / R) / 4;
  static constexpr int NCT = NCW * 32;
  static constexpr int NT = NCT + 32;
  static constexpr int TMEM_COLS = pow2ceil(NMT * 32 < 32 ? 32 : NMT * 32);
  static constexpr int ITEMS = R == 1 ? L * C / 16 : L * C / (4 * R);
  static_assert(NROWS % 128 == 0, "tile must hold a multiple of 128 vectors");
  static_assert(NMT * 32 <= 512, "tile exceeds tensor memory");
  static_assert(NST >= 1 && NST <= kMaxStages, "stage count");
};

// Stage twiddle rows: one 128-byte row per R' < L_s / 16 for every stage
// but the last, stages concatenated.  Row R' holds W_(L_s)^(k R'), k < 16,
// as eight 16-byte chunks p = (re_2p, re_2p+1, im_2p, im_2p+1), chunk p
// stored at position p ^ tw_fold(R') so that the few rows the lanes of a
// warp share fall into distinct banks.
template <int L, int R>
constexpr int stage_tw_rows() {
  int n = 0, Ls = L / R, nst = ilog2c(L / R) / 4;
  for (int s = 0; s < nst - 1; ++s) { n += Ls / 16; Ls >>= 4; }
  return n;
}
template <int L, int R>
__device__ __forceinline__ uint32_t stage_tw_row0(int s) {
  uint32_t off = 0, Ls = L / R;
  for (int i = 0; i < s; ++i) { off += Ls / 16; Ls >>= 4; }
  return off;
}
__host__ __device__ __forceinline__ uint32_t tw_fold(uint32_t r) {
  return (r ^ (r >> 3) ^ (r >> 6) ^ (r >> 9)) & 7u;
}

// Packed FP32x2 arithmetic (sm_100 f32x2 instructions) on 64-bit register
// pairs (lo, hi).
__device__ __forceinline__ uint64_t f2p(float lo, float hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2u(uint64_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
// Two complex products at once: (re, im) pairs of points 2p, 2p+1 times
// the twiddle pair (wr, wi):  yr = re wr - im wi,  yi = re wi + im wr.
__device__ __forceinline__ void cmul2(uint64_t re, uint64_t im, uint64_t wr, uint64_t wi,
                                      uint64_t& yr, uint64_t& yi) {
  yr = sub2(mul2(re, wr), mul2(im, wi));
  yi = fma2(re, wi, mul2(im, wr));
}

// Plain FP16 form.  Staging holds FP16 complex (4 bytes) in and out.

template <int L, int R, int C, bool POSTTW, int NCW>
struct TileF16 {
  using S = TileShape<L, R, C, NCW>;
  static constexpr int STAGE_BYTES = L * C * 4;
  static constexpr int A_BYTES = S::NROWS * 64;
  // Twiddle tables that are constant for the whole launch live in shared
  // memory: the radix-R table, and the stage rows when they take at most
  // 16 KB (all L but 4096 with R = 1, whose rows are read through L1).
  static constexpr int TW_ROWS = stage_tw_rows<L, R>();
  static constexpr bool TW_SMEM = TW_ROWS <= 128;
  // L = 8192 (R = 2, two columns per 16K-point tile): the radix-2 table
  // (64 KB) does not fit beside the tile; its twiddles are computed.
  static constexpr bool TAIL_CALC = R == 2 && L >= 8192;
  static constexpr int TAIL_BYTES = R > 1 && !TAIL_CALC ? L * 8 : 0;
  static constexpr int TWS_BYTES = TW_SMEM ? TW_ROWS * 128 : 0;
  static constexpr int OFF_S0 = 0;
  static constexpr int OFF_S1 = STAGE_BYTES;
  static constexpr int OFF_A = 2 * STAGE_BYTES;
  static constexpr int OFF_B = OFF_A + A_BYTES;
  static constexpr int OFF_TAIL = OFF_B + 2048;
  static constexpr int OFF_TWS = OFF_TAIL + TAIL_BYTES;
  static constexpr int OFF_BAR = OFF_TWS + TWS_BYTES;
  static constexpr int SMEM_BYTES = OFF_BAR + 256 + 1024;  // + alignment slack
  static_assert(SMEM_BYTES <= 232448, "shared memory budget");
};

__device__ __forceinline__ float2 lds64f(uint32_t addr) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}
__device__ __forceinline__ float4 lds128f(uint32_t addr) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(addr));
  return v;
}

// W_N^e from the two-level table: lo[e & (2^sh - 1)] * hi[e >> sh].
__device__ __forceinline__ float2 twiddle2(const float2* lo, const float2* hi, uint64_t e, uint32_t sh) {
  return cmulf(__ldg(lo + (e & ((1ull << sh) - 1))), __ldg(hi + (e >> sh)));
}

// Operand-buffer addressing.  Offsets inside a buffer are XOR-linear
// (off ^ k).  The dynamic shared window starts after the 1 KB the hardware
// reserves for the system (kWinBase), and every buffer sits at kWinBase + a
// multiple of its own power-of-two size, so with bb = buffer - kWinBase the
// address is ((off ^ k) | bb) + kWinBase: one LOP3, with kWinBase folded
// into the access's immediate offset.  The kernel checks the window base
// at entry and fails with a status code if it differs.
constexpr uint32_t kWinBase = 1024;
__device__ __forceinline__ uint32_t xo(uint32_t off, uint32_t k, uint32_t bb) {
  uint32_t r;
  asm("lop3.b32 %0, %1, %2, %3, 0xBE;" : "=r"(r) : "r"(off), "r"(k), "r"(bb));  // (a ^ b) | c
  return r;
}
__device__ __forceinline__ void sts32w(uint32_t a, uint32_t v) {
  asm volatile("st.shared.b32 [%0+1024], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void sts128w(uint32_t a, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0+1024], {%1,%2,%3,%4};" ::"r"(a), "r"(v.x), "r"(v.y), "r"(v.z),
               "r"(v.w)
               : "memory");
}
__device__ __forceinline__ uint4 lds128w(uint32_t a) {
  uint4 v;
  asm volatile("ld.shared.v4.b32 {%0,%1,%2,%3}, [%4+1024];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(a));
  return v;
}

// Packed-FP16 complex helpers for the plain form's radix-R stage: a __half2
// holds (re, im).
__device__ __forceinline__ __half2 h2swap(__half2 z) { return __lowhigh2highlow(z); }
// z * (s i), s = +-1: (-s im, s re)
__device__ __forceinline__ __half2 h2muli(__half2 z, __half2 negpos) {
  return __hmul2(h2swap(z), negpos);
}
// z * w with w given as (wr, wr) and (-wi, wi)
__device__ __forceinline__ __half2 h2cmul(__half2 z, __half2 wrr, __half2 wni) {
  return __hfma2(h2swap(z), wni, __hmul2(z, wrr));
}

// The radix-2 prologue twiddle W_L^v / 2 (v < L / 2; sgn -1 forward, +1
// inverse) as the packed pair {(wr, wr), (-wi, wi)} that h2cmul takes, for
// the lengths whose table is not kept in shared memory: the angle
// pi * v * (2 / L) is exact in FP32 before the product with pi and lies in
// [0, pi), where the hardware sine and cosine are accurate to ~1e-6
// absolute, far below the FP16 rounding of the pair.
template <int L>
__device__ __forceinline__ uint2 tail_tw_calc(uint32_t v, float sgn) {
  float sn, cs;
  __sincosf((float)v * (2.f / (float)L) * 3.14159265358979f, &sn, &cs);
  const float wr = 0.5f * cs, wi = 0.5f * sgn * sn;
  const __half2 wrr = __float2half2_rn(wr);
  const __half2 wni = __floats2half2_rn(-wi, wi);
  return make_uint2(*reinterpret_cast<const uint32_t*>(&wrr),
                    *reinterpret_cast<const uint32_t*>(&wni));
}

template <int R>
__device__ __forceinline__ void small_dft_h2(__half2 (&x)[R], float sgn) {
  // (-s, s) for multiplying by s*i
  const __half2 np = __floats2half2_rn(-sgn, sgn);
  if constexpr (R == 2) {
    const __half2 a = x[0], b = x[1];
    x[0] = __hadd2(a, b);
    x[1] = __hsub2(a, b);
  } else if constexpr (R == 4) {
    const __half2 a0 = __hadd2(x[0], x[2]), a1 = __hsub2(x[0], x[2]);
    const __half2 b0 = __hadd2(x[1], x[3]), b1 = h2muli(__hsub2(x[1], x[3]), np);
    x[0] = __hadd2(a0, b0);
    x[2] = __hsub2(a0, b0);
    x[1] = __hadd2(a1, b1);
    x[3] = __hsub2(a1, b1);
  } else {
    static_assert(R == 8, "tail radix must be 2, 4 or 8");
    const __half2 hh = __float2half2_rn(0.70710678118654752440f);
    __half2 e[4], o[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      e[n] = __hadd2(x[n], x[n + 4]);
      o[n] = __hsub2(x[n], x[n + 4]);
    }
    // o[n] *= W8^n, W8 = exp(s 2 pi i / 8) = h (1 + s i)
    o[1] = __hmul2(__hadd2(o[1], h2muli(o[1], np)), hh);
    o[2] = h2muli(o[2], np);
    o[3] = __hmul2(__hsub2(h2muli(o[3], np), o[3]), hh);
    small_dft_h2<4>(e, sgn);
    small_dft_h2<4>(o, sgn);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x[2 * k] = e[k];
      x[2 * k + 1] = o[k];
    }
  }
}

// Four-step twiddles of this thread's epilogue rows, w[j] = {W_N^(v g),
// W_N^(NV g)} for row j (vector v of column g), computed before the MMA
// wait so that their cost overlaps it.  N <= 2^24: the exact angle
// x = e (2 / N) (e / N is exact in FP32) -- FAST (plain form): x reduced to
// [-1, 1) and the hardware sine / cosine of pi x (__sincosf, absolute error
// below 1e-6, three orders of magnitude under the FP16 rounding of the
// output); otherwise FP32 sincospif (split form).  Larger N: the two-level
// table product lo[e & (2^sh - 1)] * hi[e >> sh].
template <int C, int NV, bool FAST, int NIT_E, int NST, class A>
__device__ __forceinline__ void post_twiddles(const A& a, int64_t cb, int s,
                                              const uint32_t (&eent)[NST][NIT_E],
                                              float2 (&w)[NIT_E][2]) {
  const float sgn = a.inverse ? 1.f : -1.f;
  const uint64_t lmask = (1ull << a.post_shift) - 1;
#pragma unroll
  for (int j = 0; j < NIT_E; ++j) {
    const uint32_t aux = eent[s][j] >> 16;
    const uint64_t g = (uint64_t)(cb * C + aux % C);
    const uint64_t e[2] = {((uint64_t)(aux / C) * g) & a.post_mask, ((uint64_t)NV * g) & a.post_mask};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (a.post_scale != 0.f) {
        float sn, cs;
        if constexpr (FAST) {
          float xr = (float)e[h] * a.post_scale;  // [0, 2)
          xr = xr >= 1.f ? xr - 2.f : xr;
          __sincosf(xr * 3.14159265358979f, &sn, &cs);  // pi x
        } else {
          sincospif((float)e[h] * a.post_scale, &sn, &cs);
        }
        w[j][h] = make_float2(cs, sgn * sn);
      } else {
        w[j][h] = cmulf(__ldg(a.post_a + (e[h] & lmask)), __ldg(a.post_b + (e[h] >> a.post_shift)));
      }
    }
  }
}

// Per-CTA shared-memory and tensor-memory handles of the tile routines.
struct TileCtx {
  uint32_t sS0, sS1, sA, sB, sTail, sTws;  // shared addresses
  uint32_t bS0, bS1, bA;                   // the same, relative to the window base
  uint32_t tmem;                           // TMEM accumulator base
  uint64_t* mmab;                          // per-M-tile MMA completion barriers
  volatile int* abort_flag;
};

// One tile of one pass, plain FP16 form: prologue, radix-16 stages on
// tcgen05 and their epilogues, run by the NCW consumer warps once the
// tile's staging buffer b holds its input.  `A` is any argument block with
// the pass's layout tables and twiddle pointers (the per-pass kernel's
// TileArgs, or one pass of the batch queue).
template <int L, int R, int C, bool POSTTW, int NCW>
struct F16Tile {
  using S = TileShape<L, R, C, NCW>;
  using T = TileF16<L, R, C, POSTTW, NCW>;
  static constexpr int NCT = S::NCT;
  static constexpr int NIT_P = (S::ITEMS + NCT - 1) / NCT;  // prologue items per consumer thread
  static constexpr int NIT_E = S::NMT * 4 / NCW;            // 32-row blocks per warp per stage
  static constexpr int NMT = S::NMT;
  static constexpr int NST = S::NST;
  static_assert(S::NMT * 4 % NCW == 0, "row blocks per warp");
  static_assert(NMT <= 16, "per-M-tile barriers");
  // Operand buffers alternate between the A buffer and the tile's staging
  // buffer so that every stage's epilogue writes a buffer its MMAs do not
  // read, and the last stage writes the staging buffer (the TMA store
  // source).  X[s] = A when NST - s is odd, staging otherwise; with an even
  // stage count the prologue transposes the staging buffer in place.
  static constexpr bool INPLACE_PROLOGUE = (S::NST % 2) == 0;
  static constexpr int TMEM_COLS = S::TMEM_COLS;

  // This thread's prologue items and epilogue rows (the same for every tile
  // of a pass).
  template <class A>
  static __device__ __forceinline__ void entries(const A& a, int ctid, uint2 (&ient)[NIT_P],
                                                 uint32_t (&eent)[NST][NIT_E]) {
    const int warp = ctid >> 5, lane = ctid & 31, sp = warp & 3;
#pragma unroll
    for (int j = 0; j < NIT_P; ++j) {
      const int it = ctid + j * NCT;
      ient[j] = it < S::ITEMS ? __ldg(a.item_tab + it) : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int s = 0; s < NST; ++s)
#pragma unroll
      for (int j = 0; j < NIT_E; ++j) {
        const uint32_t m = (warp >> 2) + j * (NCW / 4);
        eent[s][j] = __ldg(a.epi_tab + s * S::NROWS + m * 128 + sp * 32 + lane);
      }
  }

  // Radix-R twiddles (as packed-FP16 pairs {(wr, wr), (-wi, wi)}, laid out
  // as a.tail_pm says) and stage twiddle rows into shared memory; consumer
  // threads only.
  template <class A>
  static __device__ __forceinline__ void tables(const A& a, uint8_t* tail, uint8_t* tws, int ctid) {
    if constexpr (R > 1 && !T::TAIL_CALC) {
      for (int i = ctid; i < L; i += NCT) {
        const float2 w = __ldg(a.tail_tw + i);
        const __half2 wrr = __float2half2_rn(w.x);
        const __half2 wni = __floats2half2_rn(-w.y, w.y);
        uint2 v;
        v.x = *reinterpret_cast<const uint32_t*>(&wrr);
        v.y = *reinterpret_cast<const uint32_t*>(&wni);
        *reinterpret_cast<uint2*>(tail + tail_entry(i / R, i % R, R, a.tail_pm)) = v;
      }
    }
    if constexpr (T::TW_SMEM && T::TW_ROWS > 0) {
      for (int i = ctid; i < T::TW_ROWS * 8; i += NCT)
        *reinterpret_cast<float4*>(tws + 16 * i) = __ldg(a.tw + i);
    }
  }

  // Prologue of the tile in staging buffer b (ends with the consumer
  // barrier).
  template <class A>
  static __device__ __forceinline__ void prologue(const A& a, const TileCtx& x, int ctid, int b,
                                                  const uint2 (&ient)[NIT_P]) {
    const float tsgn = a.inverse ? 1.f : -1.f;
    // ---------------------------------------------------------- prologue
    // Offsets are XOR-linear relative to their buffer.
    const uint32_t bb = b ? x.bS1 : x.bS0;
    const uint32_t x0 = INPLACE_PROLOGUE ? bb : x.bA;  // stage-0 operand buffer
    if constexpr (R == 1) {
      uint4 q[NIT_P][4];
#pragma unroll
      for (int j = 0; j < NIT_P; ++j) {
        const uint32_t lb = (ient[j].x & 0xFFFFu) << 2;
#pragma unroll
        for (int n = 0; n < 4; ++n) q[j][n] = lds128w(xo(lb, a.lofs[n], bb));
      }
      if (INPLACE_PROLOGUE) tile::named_bar(1, NCT);
#pragma unroll
      for (int j = 0; j < NIT_P; ++j) {
        if (S::ITEMS % NCT != 0 && ctid + j * NCT >= S::ITEMS) break;
        const uint32_t st = (ient[j].x >> 16) << 2;
        sts128w(xo(st, a.sofs[0], x0), make_uint4(q[j][0].x, q[j][1].x, q[j][2].x, q[j][3].x));
        sts128w(xo(st, a.sofs[1], x0), make_uint4(q[j][0].y, q[j][1].y, q[j][2].y, q[j][3].y));
        sts128w(xo(st, a.sofs[2], x0), make_uint4(q[j][0].z, q[j][1].z, q[j][2].z, q[j][3].z));
        sts128w(xo(st, a.sofs[3], x0), make_uint4(q[j][0].w, q[j][1].w, q[j][2].w, q[j][3].w));
      }
    } else {
      uint4 q[NIT_P][R];
#pragma unroll
      for (int j = 0; j < NIT_P; ++j) {
        const uint32_t lb = (ient[j].x & 0xFFFFu) << 2;
#pragma unroll
        for (int n = 0; n < R; ++n) q[j][n] = lds128w(xo(lb, a.lofs[n], bb));
      }
      if (INPLACE_PROLOGUE) tile::named_bar(1, NCT);
      // Sub-vector jj of item j: radix-R butterflies, twiddles W^(k v) / R
      // (k = 0 is exactly 1 / R, a power of two: output 0 is only scaled,
      // and only entry 1 of the row's first chunk is read: tw1 = entry 1,
      // tw_of(k2) = chunk k2), stores.
      auto subvec = [&](int j, int jj, uint2 tw1, auto tw_of) {
        const uint32_t st = (ient[j].x >> 16) << 2;
        __half2 hv[R];
#pragma unroll
        for (int n = 0; n < R; ++n) {
          const uint32_t w = jj == 0 ? q[j][n].x : jj == 1 ? q[j][n].y : jj == 2 ? q[j][n].z : q[j][n].w;
          hv[n] = *reinterpret_cast<const __half2*>(&w);
        }
        small_dft_h2<R>(hv, tsgn);
        const __half2 y1 = h2cmul(hv[1], *reinterpret_cast<const __half2*>(&tw1.x),
                                  *reinterpret_cast<const __half2*>(&tw1.y));
        const __half2 y0 = __hmul2(hv[0], __float2half2_rn(1.f / R));
        sts32w(xo(st, a.sofs[jj * R], x0), *reinterpret_cast<const uint32_t*>(&y0));
        sts32w(xo(st, a.sofs[jj * R + 1], x0), *reinterpret_cast<const uint32_t*>(&y1));
#pragma unroll
        for (int k2 = 1; k2 < R / 2; ++k2) {
          const uint4 tw = tw_of(k2);
          const __half2 z0 = h2cmul(hv[2 * k2], *reinterpret_cast<const __half2*>(&tw.x),
                                    *reinterpret_cast<const __half2*>(&tw.y));
          const __half2 z1 = h2cmul(hv[2 * k2 + 1], *reinterpret_cast<const __half2*>(&tw.z),
                                    *reinterpret_cast<const __half2*>(&tw.w));
          sts32w(xo(st, a.sofs[jj * R + 2 * k2], x0), *reinterpret_cast<const uint32_t*>(&z0));
          sts32w(xo(st, a.sofs[jj * R + 2 * k2 + 1], x0), *reinterpret_cast<const uint32_t*>(&z1));
        }
      };
      constexpr int HP = NIT_P / 2;
      if constexpr (T::TAIL_CALC) {
        // row items only (two-column tiles take row staging): sub-vector jj
        // of item j has tail row v = trow + jj
#pragma unroll
        for (int j = 0; j < NIT_P; ++j) {
          if (S::ITEMS % NCT != 0 && ctid + j * NCT >= S::ITEMS) break;
          const uint32_t trow = ient[j].y & 0x7FFFFFFFu;
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
            subvec(j, jj, tail_tw_calc<L>(trow + jj, tsgn), [&](int) { return make_uint4(0u, 0u, 0u, 0u); });
        }
      } else if (NIT_P % 2 == 0 && S::ITEMS % NCT == 0 && a.tail_pm == kTailNaturalPaired) {
        // Row items whose pairs (j, j + NIT_P / 2) read the same twiddle
        // rows (the layout guarantees it): each row is loaded once.
#pragma unroll
        for (int j = 0; j < HP; ++j) {
          const uint32_t trow = ient[j].y & 0x7FFFFFFFu;
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            const uint32_t row = x.sTail + (trow + jj) * (R * 8);
            const uint2 tw1 = tile::lds64(row + 8);
            uint4 twr[R / 2];
#pragma unroll
            for (int k2 = 1; k2 < R / 2; ++k2) twr[k2] = tile::lds128(row + 16 * k2);
            subvec(j, jj, tw1, [&](int k2) { return twr[k2]; });
            subvec(j + HP, jj, tw1, [&](int k2) { return twr[k2]; });
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < NIT_P; ++j) {
          if (S::ITEMS % NCT != 0 && ctid + j * NCT >= S::ITEMS) break;
          // item word 1: tail twiddle row of sub-vector 0; bit 31 set for
          // column items (all four sub-vectors share the row)
          const uint32_t trow = ient[j].y & 0x7FFFFFFFu;
          const bool colitem = (ient[j].y >> 31) != 0;
          if (colitem) {
            // column items (folded table): the four sub-vectors share one
            // twiddle row
            const uint2 tc1 = tile::lds64(x.sTail + tail_offset(trow, 1, R));
            uint4 twc[R / 2];
#pragma unroll
            for (int k2 = 1; k2 < R / 2; ++k2)
              twc[k2] = tile::lds128(x.sTail + tail_offset(trow, 2 * k2, R));
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) subvec(j, jj, tc1, [&](int k2) { return twc[k2]; });
          } else {
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
              const uint32_t row = x.sTail + (trow + jj) * (R * 8);
              subvec(j, jj, tile::lds64(row + 8), [&](int k2) { return tile::lds128(row + 16 * k2); });
            }
          }
        }
      }
    }
    sm100::fence_proxy_async_smem();
    sm100::tc_fence_before();
    tile::named_bar(1, NCT);
    sm100::tc_fence_after();

  }

  // MMAs of stage s of the tile in buffer b: accumulators in TMEM columns
  // tm + [0, 32 NMT), completion of M-tile m on bars[m].
  static __device__ __forceinline__ void issue(const TileCtx& x, int s, int b, int ctid, uint32_t tm,
                                               uint64_t* bars) {
    const int warp = ctid >> 5, lane = ctid & 31, sp = warp & 3;
    constexpr uint32_t IDESC = sm100::idesc_f16_f32(128, 32);
    const uint32_t sb = b ? x.sS1 : x.sS0;
    const uint32_t xs = ((S::NST - s) & 1) ? x.sA : sb;  // this stage's operand
    // Each M-tile's two MMAs and its commit are issued by lane 0 of one of
    // the four warps that drain that M-tile -- the one on sub-partition
    // (warp / 4) % 4, so that the issuing warps sit on all four SM
    // sub-partitions and issue in parallel (one thread serialises its
    // tcgen05.mma instructions).  tcgen05.commit tracks the issuing thread's
    // MMAs.
    if (sp == ((warp >> 2) & 3) && lane == 0) {
#pragma unroll
      for (int j = 0; j < NIT_E; ++j) {
        const uint32_t m = (warp >> 2) + j * (NCW / 4);
#pragma unroll
        for (int ks = 0; ks < 2; ++ks)
          sm100::umma_f16(tm + 32u * m, tile::sdesc_sw64(xs + m * 8192u + ks * 32u),
                          tile::sdesc_sw64(x.sB + ks * 32u), IDESC, ks);
        sm100::umma_commit(&bars[m]);
      }
    }
  }

  // Epilogue of stage s of the tile in buffer b: waits for bars[m] (phase
  // bit m of `phase`, toggled here), reads TMEM columns tm + .., writes the
  // next stage's operand or, after the last stage, the output staging
  // (ends with the consumer barrier).
  template <int s, class A>
  static __device__ __forceinline__ void epilogue(const A& a, const TileCtx& x, int ctid, int b,
                                                  int64_t cb, uint32_t tm, uint64_t* bars,
                                                  uint32_t& phase,
                                                  const uint32_t (&eent)[NST][NIT_E]) {
    const int warp = ctid >> 5, sp = warp & 3;
    const uint32_t bb = b ? x.bS1 : x.bS0;
    const uint32_t xn = ((S::NST - s) & 1) ? bb : x.bA;  // next stage's operand (window-relative)
    const bool last = s == S::NST - 1;
    const uint32_t row0 = stage_tw_row0<L, R>(s);
    float2 pt[NIT_E][2];
    if constexpr (POSTTW && s == S::NST - 1) post_twiddles<C, S::NV, true>(a, cb, s, eent, pt);
#pragma unroll
    for (int j = 0; j < NIT_E; ++j) {
      const uint32_t m = (warp >> 2) + j * (NCW / 4);
      const uint32_t e = eent[s][j];
      const uint32_t aux = e >> 16;
      const uint32_t dst = (e & 0xFFFFu) << 2;
      // TMEM columns per lane (the DFT-16 matrix's N order): for point
      // pair p, d[4p..4p+3] = (re_2p, re_2p+1, im_2p, im_2p+1).  The 1/16
      // stage scale is in the matrix.
      float4 wg[8];
      if (!last && !T::TW_SMEM) {
        const float4* t4 = a.tw + (size_t)(row0 + aux) * 8;
#pragma unroll
        for (int p = 0; p < 8; ++p) wg[p] = __ldg(t4 + (p ^ tw_fold(aux)));
      }
      if (!sm100::mbar_wait_bounded(&bars[m], (phase >> m) & 1u, kWaitLimit)) *x.abort_flag = 1;
      sm100::tc_fence_after();
      uint32_t d[32];
      sm100::tmem_ld32(tm + ((uint32_t)(32 * sp) << 16) + 32u * m, d);
      if (!last) {
        const uint32_t trow = x.sTws + (row0 + aux) * 128u;
        const uint32_t fold = tw_fold(aux);
        sm100::tmem_wait_ld();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float4 w[4];
#pragma unroll
          for (int pp = 0; pp < 4; ++pp)
            w[pp] = T::TW_SMEM ? lds128f(trow + (((4 * h + pp) ^ fold) << 4)) : wg[4 * h + pp];
#pragma unroll
          for (int pp = 0; pp < 4; ++pp) {
            const int p = 4 * h + pp;
            uint64_t yr, yi;
            cmul2(f2p(__uint_as_float(d[4 * p]), __uint_as_float(d[4 * p + 1])),
                  f2p(__uint_as_float(d[4 * p + 2]), __uint_as_float(d[4 * p + 3])),
                  f2p(w[pp].x, w[pp].y), f2p(w[pp].z, w[pp].w), yr, yi);
            float r0, r1, i0, i1;
            f2u(yr, r0, r1);
            f2u(yi, i0, i1);
            sts32w(xo(dst, a.kofs[s][2 * p], xn), sm100::pack_half2(r0, i0));
            sts32w(xo(dst, a.kofs[s][2 * p + 1], xn), sm100::pack_half2(r1, i1));
          }
        }
      } else if (POSTTW) {
        // Four-step twiddle W_N^((v + NV k) g): pairs (w_2p, w_2p+1)
        // from w_0 = W_N^(v g) and ws = W_N^(NV g), advanced by ws^2
        // (FP32 recurrence, 7 steps, far below the FP16 output rounding).
        const float2 w0 = pt[j][0];
        const float2 ws = pt[j][1];
        const float2 w1 = cmulf(w0, ws);
        const float2 s2 = cmulf(ws, ws);
        uint64_t wr = f2p(w0.x, w1.x), wi = f2p(w0.y, w1.y);
        const uint64_t s2r = f2p(s2.x, s2.x), s2i = f2p(s2.y, s2.y);
        sm100::tmem_wait_ld();
#pragma unroll
        for (int p = 0; p < 8; ++p) {
          uint64_t yr, yi;
          cmul2(f2p(__uint_as_float(d[4 * p]), __uint_as_float(d[4 * p + 1])),
                f2p(__uint_as_float(d[4 * p + 2]), __uint_as_float(d[4 * p + 3])), wr, wi, yr,
                yi);
          float r0, r1, i0, i1;
          f2u(yr, r0, r1);
          f2u(yi, i0, i1);
          sts32w(xo(dst, a.kofs[s][2 * p], bb), sm100::pack_half2(r0, i0));
          sts32w(xo(dst, a.kofs[s][2 * p + 1], bb), sm100::pack_half2(r1, i1));
          if (p < 7) {
            uint64_t nr, ni;
            cmul2(wr, wi, s2r, s2i, nr, ni);
            wr = nr;
            wi = ni;
          }
        }
      } else {
        sm100::tmem_wait_ld();
#pragma unroll
        for (int p = 0; p < 8; ++p) {
          sts32w(xo(dst, a.kofs[s][2 * p], bb),
                 sm100::pack_half2(__uint_as_float(d[4 * p]), __uint_as_float(d[4 * p + 2])));
          sts32w(xo(dst, a.kofs[s][2 * p + 1], bb),
                 sm100::pack_half2(__uint_as_float(d[4 * p + 1]), __uint_as_float(d[4 * p + 3])));
        }
      }
    }
    phase ^= (1u << NMT) - 1u;
    sm100::fence_proxy_async_smem();
    sm100::tc_fence_before();
    tile::named_bar(1, NCT);
    sm100::tc_fence_after();
  }

  // The whole tile, stage after stage (mphase: phase bits of x.mmab).
  template <class A>
  static __device__ __forceinline__ void run(const A& a, const TileCtx& x, int ctid, int b,
                                             int64_t cb, uint32_t& mphase,
                                             const uint2 (&ient)[NIT_P],
                                             const uint32_t (&eent)[NST][NIT_E]) {
    prologue(a, x, ctid, b, ient);
    issue(x, 0, b, ctid, x.tmem, x.mmab);
    epilogue<0>(a, x, ctid, b, cb, x.tmem, x.mmab, mphase, eent);
    if constexpr (NST > 1) {
      if (*x.abort_flag) return;
      issue(x, 1, b, ctid, x.tmem, x.mmab);
      epilogue<1 < NST ? 1 : 0>(a, x, ctid, b, cb, x.tmem, x.mmab, mphase, eent);
    }
    if constexpr (NST > 2) {
      if (*x.abort_flag) return;
      issue(x, 2, b, ctid, x.tmem, x.mmab);
      epilogue<2 < NST ? 2 : 0>(a, x, ctid, b, cb, x.tmem, x.mmab, mphase, eent);
    }
  }
};

template <int L, int R, int C, bool POSTTW, int NCW>
// Registers are granted per block in units of four warps: 17 warps (16
// consumers + producer) count as 20, so 65536 / 640 -> 96 per thread; the
// 9-warp variants count as 12 warps and run two CTAs per SM -> 80.
__global__ void __maxnreg__(NCW <= 8 ? 80 : 96) fft_tile_f16(const __grid_constant__ TileArgs a) {
  using S = TileShape<L, R, C, NCW>;
  using T = TileF16<L, R, C, POSTTW, NCW>;
  using TL = F16Tile<L, R, C, POSTTW, NCW>;
  constexpr int NCT = S::NCT;
  constexpr int NMT = S::NMT;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_u = sm100::smem_u32(smem_raw);
  const uint32_t base_u = (raw_u + 1023u) & ~1023u;
  uint8_t* smem = smem_raw + (base_u - raw_u);
  const uint32_t sS0 = base_u + T::OFF_S0, sS1 = base_u + T::OFF_S1;
  const uint32_t sA = base_u + T::OFF_A;
  const uint32_t sB = base_u + T::OFF_B;
  const uint32_t sTail = base_u + T::OFF_TAIL;
  const uint32_t sTws = base_u + T::OFF_TWS;
  // buffer bases relative to the window base (see xo)
  const uint32_t bS0 = sS0 - kWinBase, bS1 = sS1 - kWinBase, bA = sA - kWinBase;
  if (((bS0 | bS1 | bA) & (uint32_t)(T::STAGE_BYTES - 1)) != 0) {
    // a different shared-window layout than the one the addressing assumes
    if (threadIdx.x == 0 && a.status) atomicExch(a.status, kStatusLayout);
    return;
  }
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + T::OFF_BAR);      // [2]
  uint64_t* outrdy = full + 2;                                          // [2]
  uint64_t* mmab = full + 4;                                            // [NMT]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(full + 4 + 16);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(full + 4 + 17);

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const bool producer = warp == NCW;

  if (producer) {
    if (lane == 0) {
      sm100::mbar_init(&full[0], 1);
      sm100::mbar_init(&full[1], 1);
      sm100::mbar_init(&outrdy[0], 1);
      sm100::mbar_init(&outrdy[1], 1);
      for (int m = 0; m < NMT; ++m) sm100::mbar_init(&mmab[m], 1);
      *abort_flag = 0;
      sm100::fence_mbar_init();
    }
    __syncwarp();
    sm100::tmem_alloc(tmem_slot, TL::TMEM_COLS);
    sm100::tmem_relinquish();
  } else {
    for (int i = tid; i < 128; i += NCT)
      *reinterpret_cast<uint4*>(smem + T::OFF_B + 16 * i) = __ldg(a.bmat + i);
    TL::tables(a, smem + T::OFF_TAIL, smem + T::OFF_TWS, tid);
  }
  sm100::fence_proxy_async_smem();
  sm100::tc_fence_before();
  __syncthreads();
  sm100::tc_fence_after();
  // The setup above reads only this launch's constant tables, so under a
  // programmatic dependent launch it overlaps the previous pass's last
  // tiles; the buffers the passes share are touched only from here on.
  sm100::grid_dep_wait();
  sm100::grid_dep_launch();
  const uint32_t tmem_base = *tmem_slot;
  const TileCtx x{sS0, sS1, sA, sB, sTail, sTws, bS0, bS1, bA, tmem_base, mmab, abort_flag};

  if (producer) {
    // ------------------------------------------------------------- producer
    if (lane == 0) {
      bool pending[2] = {false, false};
      uint32_t pend_par[2] = {0u, 0u};
      for (int j = 0; j < 2; ++j) {
        const int64_t t = blockIdx.x + (int64_t)j * gridDim.x;
        if (t < a.ntiles) {
          int32_t crd[5];
          tile::tile_coords(a.in_cmul, a.in_omul, t % a.col_blocks, t / a.col_blocks, crd);
          sm100::mbar_arrive_expect_tx(&full[j], a.in_tile_bytes);
          tile::tma_load(&a.tmap_in, a.in_ndims, crd, j ? sS1 : sS0, &full[j]);
          pending[j] = true;
          pend_par[j] = 0;
        }
      }
      int i = 0;
      for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++i) {
        const int b = i & 1;
        const uint32_t sb = b ? sS1 : sS0;
        if (!sm100::mbar_wait_bounded(&outrdy[b], (i >> 1) & 1, kWaitLimit) || *abort_flag) {
          *abort_flag = 1;
          break;
        }
        pending[b] = false;  // the consumers waited on full[b] for this tile
        int32_t crd[5];
        tile::tile_coords(a.out_cmul, a.out_omul, t % a.col_blocks, t / a.col_blocks, crd);
        tile::tma_store(&a.tmap_out, a.out_ndims, crd, sb);
        tile::tma_store_wait_read();
        const int64_t t2 = t + 2 * (int64_t)gridDim.x;
        if (t2 < a.ntiles) {
          tile::tile_coords(a.in_cmul, a.in_omul, t2 % a.col_blocks, t2 / a.col_blocks, crd);
          sm100::mbar_arrive_expect_tx(&full[b], a.in_tile_bytes);
          tile::tma_load(&a.tmap_in, a.in_ndims, crd, sb, &full[b]);
          pending[b] = true;
          pend_par[b] = ((i + 2) >> 1) & 1;
        }
      }
      tile::tma_store_wait_all();
      // Loads issued but never consumed (abort path) must land before the
      // CTA's shared memory is released.
      for (int b = 0; b < 2; ++b)
        if (pending[b]) sm100::mbar_wait_bounded(&full[b], pend_par[b], kWaitLimit);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ consumers
    // The tables are the same for every tile: keep this thread's entries in
    // registers for the whole launch.
    uint2 ient[TL::NIT_P];
    uint32_t eent[TL::NST][TL::NIT_E];
    TL::entries(a, tid, ient, eent);
    uint32_t mphase = 0;  // bit m: completions of M-tile barrier m so far, mod 2
    int i = 0;
    for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++i) {
      const int b = i & 1;
      if (!sm100::mbar_wait_bounded(&full[b], (i >> 1) & 1, kWaitLimit)) *abort_flag = 1;
      if (*abort_flag) break;
      TL::run(a, x, tid, b, t % a.col_blocks, mphase, ient, eent);
      if (*abort_flag) break;
      if (tid == 0) tile::mbar_arrive(&outrdy[b]);
    }
  }
  __syncthreads();
  if (tid == 0 && *abort_flag && a.status) atomicExch(a.status, kStatusTimeout);
  if (producer) sm100::tmem_dealloc(tmem_base, TL::TMEM_COLS);
}

}  // namespace mcfft
