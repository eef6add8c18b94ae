// fft_pass.cuh -- one HBM pass of a batched C2C FFT on sm_100a.
//
// A pass computes length-L DFTs along one axis of a tile of C "columns"
// (independent lines that share the tile), L = 16^a * R with R in {1,2,4,8}.
// It replaces the reference's layer kernels (source/mcfft_1d_device.cpp:
// 58-593): the radix-16 stages are still products with the 16-point DFT
// matrix, but the data never leaves the SM between stages and the input is
// taken in natural order (the reference scatters it through a host digit
// reversal, source/mcfft_1d_utils.cpp:43-59).
//
// Algorithm (Stockham DIF, natural in -> natural out).  With radices
// r_0..r_{m-1} (R first when R > 1, then 16s), stage t has done-digit
// count P_t = r_0...r_{t-1} and sub-length L_t = L / P_t.  Its vector v
// (0 <= v < L / r_t) = R' * P_t + K takes the r_t points at pos = n*(L/r_t) + v,
// and output k goes to pos' = K + P_t * (k + r_t * R') after the twiddle
// W_{L_t}^{k R'}.  After the last stage pos' is the natural output index.
//
// Data path of one tile (one CTA, persistent over tiles):
//   prologue   global -> registers -> [radix-R SIMT stage] -> shared memory
//              in the tcgen05 K-major layout of the first radix-16 stage
//              (row = one 16-point vector, K = 16 interleaved complex FP16)
//   stage s    one thread issues, per 128-row M-tile, two
//              tcgen05.mma.kind::f16 (K = 16 each, N = 32): D = A * B with
//              B the 32x32 real embedding of DFT-16; FP32 accumulators in
//              TMEM.  Then every warp reads its TMEM sub-partition
//              (tcgen05.ld 32x32b.x32: one lane = one vector, 16 complex
//              outputs), applies the stage twiddle and the 1/16 scale in
//              FP32, rounds to FP16 and stores each output into the next
//              stage's A row (shared memory), or, after the last stage,
//              to global memory in natural order.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>

#include "mcfft_internal.h"
#include "sm100_ptx.cuh"

namespace mcfft {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Time limit, in nanoseconds of the global timer, for every wait in the
// kernels (mbarrier phases, dependency counters): far above any legitimate
// wait (microseconds for a load or an MMA, milliseconds for the largest
// producing pass of a queued transform), short enough that a lost arrival
// or an unmet dependency ends the kernel with an error status after about
// one second instead of hanging the GPU.
constexpr uint32_t kWaitLimit = 1000000000u;

__host__ __device__ constexpr int ilog2c(int x) { return x <= 1 ? 0 : 1 + ilog2c(x >> 1); }
__host__ __device__ constexpr int pow2ceil(int x) { return x <= 1 ? 1 : 2 * pow2ceil((x + 1) >> 1); }

// Byte offset of (row p, complex position n) in the K-major no-swizzle
// layout: 8-row core matrices of 16 bytes (4 complex FP16) per row; the four
// K chunks of an 8-row group are 128 bytes apart (LBO), groups 512 bytes
// apart (SBO).
__device__ __forceinline__ uint32_t a_off(uint32_t p, uint32_t n) {
  return (p & 7u) * 16u + (p >> 3) * 512u + (n >> 2) * 128u + (n & 3u) * 4u;
}
// Row swizzle: physical row of logical row u.  XOR of bits 4..6 into 0..2
// spreads the epilogue's scattered 4-byte stores over more banks.  It is an
// involution, so it also maps a physical row back to its logical row.
__device__ __forceinline__ uint32_t row_swz(uint32_t u) { return u ^ ((u >> 4) & 7u); }

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Small DFT of size R (2, 4 or 8) in registers, sign = -1 forward, +1 inverse.
template <int R>
__device__ __forceinline__ void small_dft(float2 (&x)[R], float sgn) {
  if constexpr (R == 2) {
    float2 a = x[0], b = x[1];
    x[0] = make_float2(a.x + b.x, a.y + b.y);
    x[1] = make_float2(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 4) {
    float2 a0 = make_float2(x[0].x + x[2].x, x[0].y + x[2].y);
    float2 a1 = make_float2(x[0].x - x[2].x, x[0].y - x[2].y);
    float2 b0 = make_float2(x[1].x + x[3].x, x[1].y + x[3].y);
    float2 b1 = make_float2(x[1].x - x[3].x, x[1].y - x[3].y);
    // b1 * (sgn * i)
    float2 jb1 = make_float2(-sgn * b1.y, sgn * b1.x);
    x[0] = make_float2(a0.x + b0.x, a0.y + b0.y);
    x[2] = make_float2(a0.x - b0.x, a0.y - b0.y);
    x[1] = make_float2(a1.x + jb1.x, a1.y + jb1.y);
    x[3] = make_float2(a1.x - jb1.x, a1.y - jb1.y);
  } else {
    static_assert(R == 8, "tail radix must be 2, 4 or 8");
    // radix-2 over (n, n+4), twiddle, then two radix-4.
    const float h = 0.70710678118654752440f;
    float2 e[4], o[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      e[n] = make_float2(x[n].x + x[n + 4].x, x[n].y + x[n + 4].y);
      o[n] = make_float2(x[n].x - x[n + 4].x, x[n].y - x[n + 4].y);
    }
    // o[n] *= W8^(n) with W8 = exp(sgn * 2 pi i / 8)
    o[1] = make_float2(h * (o[1].x - sgn * o[1].y), h * (o[1].y + sgn * o[1].x));
    o[2] = make_float2(-sgn * o[2].y, sgn * o[2].x);
    o[3] = make_float2(h * (-o[3].x - sgn * o[3].y), h * (-o[3].y + sgn * o[3].x));
    small_dft<4>(e, sgn);
    small_dft<4>(o, sgn);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      x[2 * k] = e[k];
      x[2 * k + 1] = o[k];
    }
  }
}

template <int L, int R, int C, bool COLFAST>
struct PassShape {
  static constexpr int NV = L / 16;        // radix-16 vectors per column
  static constexpr int NVR = L / R;        // tail vectors per column
  static constexpr int NROWS = NV * C;     // A rows per tile
  static constexpr int NMT = NROWS / 128;  // 128-row M-tiles
  static constexpr int NST = ilog2c(L / R) / 4;  // radix-16 stages
  static constexpr int TMEM_COLS = pow2ceil(NMT * 32 < 32 ? 32 : NMT * 32);
  static constexpr int A_BYTES = NROWS * 64;
  static constexpr int SMEM_BYTES = A_BYTES + 2048 + 64;
  static_assert((L & (L - 1)) == 0 && L >= 16, "L must be a power of two");
  static_assert(R == 1 || R == 2 || R == 4 || R == 8, "bad tail radix");
  static_assert(NST >= 1 && (1 << (4 * NST)) * R == L, "L must be 16^a * R");
  static_assert(NROWS % 128 == 0, "tile must hold a multiple of 128 vectors");
  static_assert(NMT * 32 <= 512, "tile exceeds tensor memory");
  __device__ static __forceinline__ uint32_t row_of(uint32_t v, uint32_t c) {
    return COLFAST ? c + C * v : v + NV * c;
  }
  __device__ static __forceinline__ void vec_of(uint32_t u, uint32_t& v, uint32_t& c) {
    if (COLFAST) { c = u % C; v = u / C; } else { v = u % NV; c = u / NV; }
  }
};

// Offset (in float2) of stage s's twiddle table inside PassArgs::tw: stage
// s holds L_s = L / P_s entries, laid out [R'][k].
template <int L, int R>
__device__ __forceinline__ uint32_t stage_tw_offset(int s) {
  uint32_t off = 0, Ls = L / R;
  for (int i = 0; i < s; ++i) { off += Ls; Ls >>= 4; }
  return off;
}

template <int L, int R, int C, bool COLFAST, bool POSTTW>
__global__ void __launch_bounds__(kThreads, 2) fft_pass_f16(const __grid_constant__ PassArgs a) {
  using S = PassShape<L, R, C, COLFAST>;
  constexpr int NV = S::NV;
  constexpr int LOG_NV = ilog2c(NV);
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sA = smem;
  uint8_t* sB = smem + S::A_BYTES;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + 2048);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sB + 2048 + 8);
  int* abort_flag = reinterpret_cast<int*>(sB + 2048 + 16);

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const __half2* gin = static_cast<const __half2*>(a.in);
  __half2* gout = static_cast<__half2*>(a.out);

  if (tid == 0) {
    sm100::mbar_init(mbar, 1);
    sm100::fence_mbar_init();
    *abort_flag = 0;
  }
  if (warp == 0) {
    sm100::tmem_alloc(tmem_slot, S::TMEM_COLS);
    sm100::tmem_relinquish();
  }
  // The DFT-16 embedding (forward or inverse), already in canonical layout.
  for (int i = tid; i < 128; i += kThreads)
    reinterpret_cast<uint4*>(sB)[i] = __ldg(a.bmat + i);
  sm100::fence_proxy_async_smem();
  sm100::tc_fence_before();
  __syncthreads();
  sm100::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t sA_u32 = sm100::smem_u32(sA);
  const uint32_t sB_u32 = sm100::smem_u32(sB);
  constexpr uint32_t IDESC = sm100::idesc_f16_f32(128, 32);
  uint32_t phase = 0;
  const float tsgn = a.inverse ? 1.f : -1.f;

  for (int64_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int64_t outer = tile / a.col_blocks;
    const int64_t cb = tile - outer * a.col_blocks;
    const int64_t in_base = outer * a.in_so + cb * C * a.in_sc;
    const int64_t out_base = outer * a.out_so + cb * C * a.out_sc;

    // ---------------------------------------------------------- prologue
    if constexpr (R == 1) {
      // Transpose into stage-0 rows: vector v of column c, chunk j holds
      // points n = 4j..4j+3 at pos = n*NV + v.
      for (int i = tid; i < S::NROWS * 4; i += kThreads) {
        const uint32_t j = i / S::NROWS, u = i % S::NROWS;
        uint32_t v, c;
        S::vec_of(u, v, c);
        uint32_t h[4] = {0u, 0u, 0u, 0u};
        if (cb * C + c < a.ncols) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int64_t pos = (int64_t)(4 * j + q) * NV + v;
            h[q] = __ldg(reinterpret_cast<const unsigned int*>(gin + in_base + pos * a.in_sp +
                                                                (int64_t)c * a.in_sc));
          }
        }
        *reinterpret_cast<uint4*>(sA + a_off(row_swz(u), 4 * j)) = make_uint4(h[0], h[1], h[2], h[3]);
      }
    } else {
      // Radix-R first stage in FP32 registers: vector vr takes the R points
      // pos = n*(L/R) + vr; output k goes to pos' = k + R*vr after the
      // twiddle W_L^(k vr) / R, i.e. to stage-1 row (pos' % NV), K (pos' / NV).
      constexpr int NVR = S::NVR;
      for (int i = tid; i < NVR * C; i += kThreads) {
        uint32_t vr, c;
        if (COLFAST) { c = i % C; vr = i / C; } else { vr = i % NVR; c = i / NVR; }
        float2 x[R];
        const bool valid = cb * C + c < a.ncols;
#pragma unroll
        for (int n = 0; n < R; ++n) {
          const int64_t pos = (int64_t)n * NVR + vr;
          const uint32_t w = valid ? __ldg(reinterpret_cast<const unsigned int*>(
                                         gin + in_base + pos * a.in_sp + (int64_t)c * a.in_sc))
                                   : 0u;
          x[n] = sm100::unpack_half2(w);
        }
        small_dft<R>(x, tsgn);
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const float2 t = __ldg(a.tail_tw + vr * R + k);
          const float2 y = cmulf(x[k], t);
          const uint32_t pos1 = k + R * vr;
          const uint32_t n1 = pos1 >> LOG_NV, v1 = pos1 & (NV - 1);
          *reinterpret_cast<uint32_t*>(sA + a_off(row_swz(S::row_of(v1, c)), n1)) =
              sm100::pack_half2(y.x, y.y);
        }
      }
    }
    sm100::fence_proxy_async_smem();
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();

    // ------------------------------------------------------------ stages
    for (int s = 0; s < S::NST; ++s) {
      if (tid == 0) {
#pragma unroll 1
        for (int m = 0; m < S::NMT; ++m) {
          const uint32_t d = tmem_base + 32u * m;
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            const uint64_t ad = sm100::sdesc_kmajor(sA_u32 + m * 8192u + ks * 256u, 128u, 512u);
            const uint64_t bd = sm100::sdesc_kmajor(sB_u32 + ks * 256u, 128u, 512u);
            sm100::umma_f16(d, ad, bd, IDESC, ks);
          }
        }
        sm100::umma_commit(mbar);
      }
      if (!sm100::mbar_wait_bounded(mbar, phase, kWaitLimit)) {
        *abort_flag = 1;  // benign race: every writer stores 1
      }
      phase ^= 1u;
      sm100::tc_fence_after();

      const bool last = (s == S::NST - 1);
      const uint32_t P = (uint32_t)R << (4 * s);  // done-digit count
      const float2* tws = a.tw + stage_tw_offset<L, R>(s);
      const int sp = warp & 3;
      for (int m = warp >> 2; m < S::NMT; m += kWarps / 4) {
        uint32_t r[32];
        sm100::tmem_ld32(tmem_base + ((uint32_t)(32 * sp) << 16) + 32u * m, r);
        sm100::tmem_wait_ld();
        const uint32_t prow = m * 128 + sp * 32 + lane;
        uint32_t v, c;
        S::vec_of(row_swz(prow), v, c);
        if (!last) {
          const uint32_t K = v % P, Rp = v / P;
          const float4* t4 = reinterpret_cast<const float4*>(tws + Rp * 16);
#pragma unroll
          for (int k2 = 0; k2 < 8; ++k2) {
            const float4 w = __ldg(t4 + k2);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int k = 2 * k2 + h;
              const float2 x = make_float2(__uint_as_float(r[2 * k]), __uint_as_float(r[2 * k + 1]));
              const float2 y = cmulf(x, h ? make_float2(w.z, w.w) : make_float2(w.x, w.y));
              const uint32_t pos1 = K + P * (k + 16 * Rp);
              const uint32_t n1 = pos1 >> LOG_NV, v1 = pos1 & (NV - 1);
              *reinterpret_cast<uint32_t*>(sA + a_off(row_swz(S::row_of(v1, c)), n1)) =
                  sm100::pack_half2(y.x, y.y);
            }
          }
        } else {
          const int64_t g = cb * C + c;  // global column index (four-step twiddle)
          if (g >= a.ncols) continue;
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            float2 y = make_float2(__uint_as_float(r[2 * k]) * a.out_scale,
                                   __uint_as_float(r[2 * k + 1]) * a.out_scale);
            const uint32_t pos1 = v + NV * k;
            if constexpr (POSTTW) {
              const uint64_t e = ((uint64_t)pos1 * (uint64_t)g) & a.post_mask;
              const float2 w = cmulf(__ldg(a.post_lo + (e & ((1ull << a.post_shift) - 1))),
                                     __ldg(a.post_hi + (e >> a.post_shift)));
              y = cmulf(y, w);
            }
            __half2 hv = __floats2half2_rn(y.x, y.y);
            gout[out_base + (int64_t)pos1 * a.out_sp + (int64_t)c * a.out_sc] = hv;
          }
        }
      }
      sm100::fence_proxy_async_smem();
      sm100::tc_fence_before();
      __syncthreads();
      sm100::tc_fence_after();
      if (*abort_flag) break;
    }
    if (*abort_flag) break;
  }

  __syncthreads();
  if (tid == 0 && *abort_flag && a.status) atomicExch(a.status, kStatusTimeout);
  if (warp == 0) sm100::tmem_dealloc(tmem_base, S::TMEM_COLS);
}

}  // namespace mcfft
