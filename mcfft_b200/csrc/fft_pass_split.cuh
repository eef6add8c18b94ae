// fft_pass_split.cuh -- the split-precision form of one FFT pass.
//
// Same Stockham schedule and tile organisation as fft_pass.cuh, but every
// tensor-core operand is carried as a pair of FP16 values, x = hi + lo with
// hi = fp16(x) and lo = fp16(x - hi), and each radix-16 stage accumulates
// three products in FP32:
//     D = A_hi * B_hi + A_lo * B_hi + A_hi * B_lo
// (six tcgen05.mma per 128-row M-tile, K = 16 each).  The dropped
// A_lo * B_lo term is ~2^-22 relative.  Twiddles are FP32 and applied to the
// FP32 accumulators in the epilogue, which re-splits the result for the
// next stage.
//
// Range: the prologue scales the whole tile by one power of two so that its
// largest component lies in [2^13, 2^14), which keeps hi finite and lo
// normal for every value within 2^-16 of the tile maximum; each stage then
// scales by 1/16 (1/R for the tail) so magnitudes never grow.  The last
// stage multiplies by L / (16 * scale), an exact power of two, so the output
// is the unnormalised DFT (the FFTW_FORWARD / FFTW_BACKWARD convention the
// reference's accuracy harness compares against, benchmark/accuracy_1d.cpp:15).
#pragma once
#include "fft_pass.cuh"

namespace mcfft {

template <int L, int R, int C, bool COLFAST>
struct SplitShape : PassShape<L, R, C, COLFAST> {
  using B = PassShape<L, R, C, COLFAST>;
  static constexpr int A_BYTES = B::NROWS * 64;                    // per part (hi or lo)
  static constexpr int SMEM_BYTES = 2 * A_BYTES + 4096 + 128;
  // work items of the prologue per thread (each item = 4 points for R = 1,
  // R points for R > 1)
  static constexpr int ITEMS = (R == 1 ? B::NROWS * 4 : B::NVR * C) / kThreads;
  static constexpr int PTS = (R == 1 ? 4 : R);
  static_assert((R == 1 ? B::NROWS * 4 : B::NVR * C) % kThreads == 0, "uneven prologue");
  static_assert(ITEMS * PTS * 2 <= 64, "prologue would not fit in registers");
};

__device__ __forceinline__ void split2(float2 y, uint32_t& hi, uint32_t& lo) {
  const __half2 h = __floats2half2_rn(y.x, y.y);
  const float2 hf = __half22float2(h);
  const __half2 l = __floats2half2_rn(y.x - hf.x, y.y - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// 2^e as a float for e in [-126, 127].
__device__ __forceinline__ float exp2i(int e) {
  e = e < -126 ? -126 : (e > 127 ? 127 : e);
  return __int_as_float((127 + e) << 23);
}

template <int L, int R, int C, bool COLFAST, bool POSTTW>
__global__ void __launch_bounds__(kThreads, 2) fft_pass_split(const __grid_constant__ PassArgs a) {
  using S = SplitShape<L, R, C, COLFAST>;
  constexpr int NV = S::NV;
  constexpr int LOG_NV = ilog2c(NV);
  constexpr int NROWS = S::NROWS;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t* sAh = smem;
  uint8_t* sAl = smem + S::A_BYTES;
  uint8_t* sBh = smem + 2 * S::A_BYTES;
  uint8_t* sBl = sBh + 2048;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sBl + 2048);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sBl + 2048 + 8);
  int* abort_flag = reinterpret_cast<int*>(sBl + 2048 + 16);
  uint32_t* red = reinterpret_cast<uint32_t*>(sBl + 2048 + 32);  // kWarps words

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  float2* gout = static_cast<float2*>(a.out);

  if (tid == 0) {
    sm100::mbar_init(mbar, 1);
    sm100::fence_mbar_init();
    *abort_flag = 0;
  }
  if (warp == 0) {
    sm100::tmem_alloc(tmem_slot, S::TMEM_COLS);
    sm100::tmem_relinquish();
  }
  for (int i = tid; i < 128; i += kThreads) {
    reinterpret_cast<uint4*>(sBh)[i] = __ldg(a.bmat + i);
    reinterpret_cast<uint4*>(sBl)[i] = __ldg(a.bmat_lo + i);
  }
  sm100::fence_proxy_async_smem();
  sm100::tc_fence_before();
  __syncthreads();
  sm100::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t sAh_u = sm100::smem_u32(sAh), sAl_u = sm100::smem_u32(sAl);
  const uint32_t sBh_u = sm100::smem_u32(sBh), sBl_u = sm100::smem_u32(sBl);
  constexpr uint32_t IDESC = sm100::idesc_f16_f32(128, 32);
  uint32_t phase = 0;
  const float tsgn = a.inverse ? 1.f : -1.f;

  for (int64_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int64_t outer = tile / a.col_blocks;
    const int64_t cb = tile - outer * a.col_blocks;
    const int64_t in_base = outer * a.in_so + cb * C * a.in_sc;
    const int64_t out_base = outer * a.out_so + cb * C * a.out_sc;

    // ------------------------------------------------ prologue: load + max
    float2 x[S::ITEMS][S::PTS];
    uint32_t amax = 0;
#pragma unroll
    for (int it = 0; it < S::ITEMS; ++it) {
      const int i = tid + it * kThreads;
      uint32_t v, c, j = 0;
      if constexpr (R == 1) {
        j = i / NROWS;
        S::vec_of(i % NROWS, v, c);
      } else {
        if (COLFAST) { c = i % C; v = i / C; } else { v = i % S::NVR; c = i / S::NVR; }
      }
      const bool valid = cb * C + c < a.ncols;
#pragma unroll
      for (int q = 0; q < S::PTS; ++q) {
        const int64_t pos = R == 1 ? (int64_t)(4 * j + q) * NV + v : (int64_t)q * S::NVR + v;
        const int64_t gi = in_base + pos * a.in_sp + (int64_t)c * a.in_sc;
        float2 val = make_float2(0.f, 0.f);
        if (valid) {
          if (a.split_in_f16)
            val = sm100::unpack_half2(
                __ldg(reinterpret_cast<const unsigned int*>(static_cast<const __half2*>(a.in) + gi)));
          else
            val = __ldg(static_cast<const float2*>(a.in) + gi);
        }
        x[it][q] = val;
      }
      if constexpr (R > 1) {
        small_dft<R>(x[it], tsgn);
#pragma unroll
        for (int k = 0; k < R; ++k) x[it][k] = cmulf(x[it][k], __ldg(a.tail_tw + v * R + k));
      }
#pragma unroll
      for (int q = 0; q < S::PTS; ++q) {
        amax = max(amax, __float_as_uint(fabsf(x[it][q].x)));
        amax = max(amax, __float_as_uint(fabsf(x[it][q].y)));
      }
    }
    amax = __reduce_max_sync(0xffffffffu, amax);
    if (lane == 0) red[warp] = amax;
    __syncthreads();
    uint32_t tmax = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) tmax = max(tmax, red[w]);
    // scale = 2^(13 - floor(log2 max)) puts the tile maximum in [2^13, 2^14)
    const int e = tmax == 0 ? 0 : (int)((tmax >> 23) & 0xff) - 127;
    const int sexp = tmax == 0 ? 0 : 13 - e;
    const float sc = exp2i(sexp);
    // L/(16 * scale): undoes the stage scalings (1/L in total) and the tile scale
    const float fm = exp2i(ilog2c(L) - 4 - sexp);

#pragma unroll
    for (int it = 0; it < S::ITEMS; ++it) {
      const int i = tid + it * kThreads;
      if constexpr (R == 1) {
        const uint32_t j = i / NROWS, u = i % NROWS;
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
          split2(make_float2(x[it][q].x * sc, x[it][q].y * sc), hi[q], lo[q]);
        const uint32_t off = a_off(row_swz(u), 4 * j);
        *reinterpret_cast<uint4*>(sAh + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(sAl + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
      } else {
        uint32_t v, c;
        if (COLFAST) { c = i % C; v = i / C; } else { v = i % S::NVR; c = i / S::NVR; }
#pragma unroll
        for (int k = 0; k < R; ++k) {
          const uint32_t pos1 = k + R * v;
          const uint32_t n1 = pos1 >> LOG_NV, v1 = pos1 & (NV - 1);
          const uint32_t off = a_off(row_swz(S::row_of(v1, c)), n1);
          uint32_t hi, lo;
          split2(make_float2(x[it][k].x * sc, x[it][k].y * sc), hi, lo);
          *reinterpret_cast<uint32_t*>(sAh + off) = hi;
          *reinterpret_cast<uint32_t*>(sAl + off) = lo;
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
            const uint32_t ao = m * 8192u + ks * 256u, bo = ks * 256u;
            const uint64_t ah = sm100::sdesc_kmajor(sAh_u + ao, 128u, 512u);
            const uint64_t al = sm100::sdesc_kmajor(sAl_u + ao, 128u, 512u);
            const uint64_t bh = sm100::sdesc_kmajor(sBh_u + bo, 128u, 512u);
            const uint64_t bl = sm100::sdesc_kmajor(sBl_u + bo, 128u, 512u);
            sm100::umma_f16(d, ah, bh, IDESC, ks);
            sm100::umma_f16(d, al, bh, IDESC, 1);
            sm100::umma_f16(d, ah, bl, IDESC, 1);
          }
        }
        sm100::umma_commit(mbar);
      }
      if (!sm100::mbar_wait_bounded(mbar, phase, kWaitLimit)) *abort_flag = 1;
      phase ^= 1u;
      sm100::tc_fence_after();

      const bool last = (s == S::NST - 1);
      const uint32_t P = (uint32_t)R << (4 * s);
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
              const float2 xv = make_float2(__uint_as_float(r[2 * k]), __uint_as_float(r[2 * k + 1]));
              const float2 y = cmulf(xv, h ? make_float2(w.z, w.w) : make_float2(w.x, w.y));
              const uint32_t pos1 = K + P * (k + 16 * Rp);
              const uint32_t n1 = pos1 >> LOG_NV, v1 = pos1 & (NV - 1);
              const uint32_t off = a_off(row_swz(S::row_of(v1, c)), n1);
              uint32_t hi, lo;
              split2(y, hi, lo);
              *reinterpret_cast<uint32_t*>(sAh + off) = hi;
              *reinterpret_cast<uint32_t*>(sAl + off) = lo;
            }
          }
        } else {
          const int64_t g = cb * C + c;
          if (g >= a.ncols) continue;
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            float2 y = make_float2(__uint_as_float(r[2 * k]) * fm, __uint_as_float(r[2 * k + 1]) * fm);
            const uint32_t pos1 = v + NV * k;
            if constexpr (POSTTW) {
              const uint64_t e2 = ((uint64_t)pos1 * (uint64_t)g) & a.post_mask;
              const float2 w = cmulf(__ldg(a.post_lo + (e2 & ((1ull << a.post_shift) - 1))),
                                     __ldg(a.post_hi + (e2 >> a.post_shift)));
              y = cmulf(y, w);
            }
            gout[out_base + (int64_t)pos1 * a.out_sp + (int64_t)c * a.out_sc] = y;
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
