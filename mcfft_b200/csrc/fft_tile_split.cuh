// fft_tile_split.cuh -- split hi+lo form of the TMA-fed pass kernel (sm_100a).
//
// Same organisation as fft_tile_f16 (fft_tile.cuh): one persistent CTA per
// SM, a TMA producer warp double-buffering tiles, consumer warps running the
// prologue, the radix-16 stages on tcgen05 and their epilogues, all shared
// addressing from the host layout tables.  What differs:
//
//   operands   every A operand is a pair of FP16 arrays, hi = fp16(x) and
//              lo = fp16(x - hi); each radix-16 stage accumulates
//                  D = A_hi * B_hi + A_lo * B_hi + A_hi * B_lo
//              in FP32 (six tcgen05.mma per 128-row M-tile, K = 16 each);
//              the dropped A_lo * B_lo term is ~2^-22 relative
//   staging    FP32 complex (8 bytes) out, FP32 or FP16 complex in; the
//              operand pair (hi + lo) has the size of the FP32 staging, so
//              the plain kernel's ping-pong between the A buffer and the
//              staging buffer carries over
//   range      the prologue first reduces the tile's largest component m,
//              then scales the tile by 2^e with m 2^e in [2^13, 2^14): hi
//              stays finite and lo normal for every value within 2^-16 of
//              the tile maximum.  Complex moduli never grow through the
//              stages (radix-R twiddles carry 1/R, stage twiddles 1/16), so
//              every component stays below sqrt(2) 2^14
//   output     the last stage multiplies by L / (16 2^e), an exact power of
//              two: the output is the unnormalised DFT (the FFTW_FORWARD /
//              FFTW_BACKWARD convention of the reference's accuracy harness,
//              benchmark/accuracy_1d.cpp:15)
//   twiddles   FP32 (stage rows carry the 1/16; the DFT-16 matrix is not
//              scaled, so its low part stays in FP16's normal range), applied
//              to the FP32 accumulators with packed FP32x2 products
//
// Prologue work units: with FP16 input a unit is one layout item (4
// sub-vectors); with FP32 input a 16-byte load holds 2 points, so a unit is
// half an item (sub-vectors 2h, 2h+1), and unit u covers item u % ITEMS,
// half u / ITEMS.
#pragma once
#include "fft_pass_split.cuh"
#include "fft_tile.cuh"

namespace mcfft {

template <int L, int R, int C, bool POSTTW, int NCW, bool IN16>
struct TileSplit {
  using S = TileShape<L, R, C, NCW>;
  static constexpr int TP = L * C;       // points per tile
  static constexpr int BUF = TP * 8;     // FP32 staging == operand pair
  static constexpr int HALF = TP * 4;    // offset of the lo part in an operand buffer
  static constexpr int TW_ROWS = stage_tw_rows<L, R>();
  static constexpr bool TW_SMEM = TW_ROWS <= 128;
  static constexpr int TAIL_BYTES = R > 1 ? L * 8 : 0;
  static constexpr int TWS_BYTES = TW_SMEM ? TW_ROWS * 128 : 0;
  static constexpr int OFF_S0 = 0;
  static constexpr int OFF_S1 = BUF;
  static constexpr int OFF_A = 2 * BUF;
  static constexpr int OFF_B = 3 * BUF;  // hi 2 KB, then lo 2 KB
  static constexpr int OFF_TAIL = OFF_B + 4096;
  static constexpr int OFF_TWS = OFF_TAIL + TAIL_BYTES;
  static constexpr int OFF_BAR = OFF_TWS + TWS_BYTES;
  static constexpr int SMEM_BYTES = OFF_BAR + 256 + 1024;  // + alignment slack
  static_assert(SMEM_BYTES <= 232448, "shared memory budget");
};

__device__ __forceinline__ void sts64w(uint32_t a, float x, float y) {
  asm volatile("st.shared.v2.f32 [%0+1024], {%1,%2};" ::"r"(a), "f"(x), "f"(y) : "memory");
}
__device__ __forceinline__ float2 lds64w(uint32_t a) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0,%1}, [%2+1024];" : "=f"(v.x), "=f"(v.y) : "r"(a));
  return v;
}

// hi at window-relative address a, lo HALF bytes further (the low operand
// lies HALF bytes after the high one in every operand buffer): one address
// computation for both stores.
template <int HALF>
__device__ __forceinline__ void sts32_hl(uint32_t a, uint32_t hi, uint32_t lo) {
  asm volatile("st.shared.b32 [%0+1024], %1;" ::"r"(a), "r"(hi) : "memory");
  asm volatile("st.shared.b32 [%0+%2], %1;" ::"r"(a), "r"(lo), "n"(1024 + HALF) : "memory");
}
template <int HALF>
__device__ __forceinline__ void sts128_hl(uint32_t a, uint4 hi, uint4 lo) {
  asm volatile("st.shared.v4.b32 [%0+1024], {%1,%2,%3,%4};" ::"r"(a), "r"(hi.x), "r"(hi.y),
               "r"(hi.z), "r"(hi.w)
               : "memory");
  asm volatile("st.shared.v4.b32 [%0+%5], {%1,%2,%3,%4};" ::"r"(a), "r"(lo.x), "r"(lo.y),
               "r"(lo.z), "r"(lo.w), "n"(1024 + HALF)
               : "memory");
}

// Splits the FP32 pairs (re_0, re_1), (im_0, im_1) of two points into
// packed-FP16 hi and lo words per point.
__device__ __forceinline__ void split_pair(uint64_t yr, uint64_t yi, uint32_t& hi0, uint32_t& hi1,
                                           uint32_t& lo0, uint32_t& lo1) {
  float r0, r1, i0, i1;
  f2u(yr, r0, r1);
  f2u(yi, i0, i1);
  const __half2 h0 = __floats2half2_rn(r0, i0), h1 = __floats2half2_rn(r1, i1);
  const float2 f0 = __half22float2(h0), f1 = __half22float2(h1);
  float lr0, lr1, li0, li1;
  f2u(sub2(yr, f2p(f0.x, f1.x)), lr0, lr1);
  f2u(sub2(yi, f2p(f0.y, f1.y)), li0, li1);
  const __half2 l0 = __floats2half2_rn(lr0, li0), l1 = __floats2half2_rn(lr1, li1);
  hi0 = *reinterpret_cast<const uint32_t*>(&h0);
  hi1 = *reinterpret_cast<const uint32_t*>(&h1);
  lo0 = *reinterpret_cast<const uint32_t*>(&l0);
  lo1 = *reinterpret_cast<const uint32_t*>(&l1);
}

// One complex point of a 16-byte staging load: FP16 input holds 4 points
// (index 0..3), FP32 input 2 points (index 0..1).
template <bool IN16>
__device__ __forceinline__ float2 load_point(const uint4& q, int i) {
  if constexpr (IN16) {
    const uint32_t w = i == 0 ? q.x : i == 1 ? q.y : i == 2 ? q.z : q.w;
    return __half22float2(*reinterpret_cast<const __half2*>(&w));
  } else {
    return i == 0 ? make_float2(__uint_as_float(q.x), __uint_as_float(q.y))
                  : make_float2(__uint_as_float(q.z), __uint_as_float(q.w));
  }
}

// Split-form handles: the plain ones plus the low DFT matrix and the
// per-tile maximum slots.
struct SplitCtx {
  TileCtx t;       // sB = high DFT-16 matrix
  uint32_t sBl;    // low DFT-16 matrix
  uint32_t* red;   // [2] tile maxima (uint bits of a non-negative float)
};

// One tile of one pass, split form (see the file comment), run by the NCW
// consumer warps once the tile's staging buffer b holds its input; k is
// the CTA-local tile index (its parity picks the maximum slot).  `A` is any
// argument block with the pass's tables (TileArgs, or a pass of the batch
// queue).
template <int L, int R, int C, bool POSTTW, int NCW, bool IN16>
struct SplitTile {
  using S = TileShape<L, R, C, NCW>;
  using T = TileSplit<L, R, C, POSTTW, NCW, IN16>;
  static constexpr int NCT = S::NCT;
  static constexpr int NH = IN16 ? 1 : 2;               // loads per point group
  static constexpr int SUBV = 4 / NH;                   // sub-vectors per prologue unit
  static constexpr int UNITS = S::ITEMS * NH;
  static constexpr int NIT_P = (UNITS + NCT - 1) / NCT;  // prologue units per consumer thread
  static constexpr int NLD = R == 1 ? 4 : R;            // 16-byte loads per unit
  static constexpr int NIT_E = S::NMT * 4 / NCW;
  static constexpr int NMT = S::NMT;
  static constexpr int NST = S::NST;
  // Each M-tile accumulates 64 columns: [0, 32) A_hi B_hi + A_lo B_hi,
  // [32, 64) A_hi B_lo (one N = 64 MMA reads A_hi once for both B parts).
  static constexpr int TMEM_COLS = 2 * S::TMEM_COLS;
  static_assert(TMEM_COLS <= 512, "tensor memory");
  static_assert(S::NMT * 4 % NCW == 0, "row blocks per warp");
  static_assert(NMT <= 16, "per-M-tile barriers");
  static_assert(NIT_P * NLD <= 8, "prologue registers");
  static constexpr bool INPLACE_PROLOGUE = (S::NST % 2) == 0;
  static constexpr int LGL = ilog2c(L);

  template <class A>
  static __device__ __forceinline__ void entries(const A& a, int ctid, uint2 (&ient)[NIT_P],
                                                 uint32_t (&eent)[NST][NIT_E]) {
    const int warp = ctid >> 5, lane = ctid & 31, sp = warp & 3;
#pragma unroll
    for (int j = 0; j < NIT_P; ++j) {
      const int u = ctid + j * NCT;
      ient[j] = u < UNITS ? __ldg(a.item_tab + (u % S::ITEMS)) : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int s = 0; s < NST; ++s)
#pragma unroll
      for (int j = 0; j < NIT_E; ++j) {
        const uint32_t m = (warp >> 2) + j * (NCW / 4);
        eent[s][j] = __ldg(a.epi_tab + s * S::NROWS + m * 128 + sp * 32 + lane);
      }
  }

  // Radix-R twiddles (FP32, 1/R) and stage twiddle rows into shared memory;
  // consumer threads only.
  template <class A>
  static __device__ __forceinline__ void tables(const A& a, uint8_t* tail, uint8_t* tws, int ctid) {
    if constexpr (R > 1) {
      for (int i = ctid; i < L; i += NCT)
        *reinterpret_cast<float2*>(tail + tail_entry(i / R, i % R, R, a.tail_pm)) =
            __ldg(a.tail_tw + i);
    }
    if constexpr (T::TW_SMEM && T::TW_ROWS > 0) {
      for (int i = ctid; i < T::TW_ROWS * 8; i += NCT)
        *reinterpret_cast<float4*>(tws + 16 * i) = __ldg(a.tw + i);
    }
  }

  template <class A>
  static __device__ __forceinline__ void run(const A& a, const SplitCtx& x, int ctid, int b,
                                             int64_t cb, int64_t k, uint32_t& mphase,
                                             const uint2 (&ient)[NIT_P],
                                             const uint32_t (&eent)[NST][NIT_E]) {
    const int warp = ctid >> 5, lane = ctid & 31, sp = warp & 3;
    constexpr uint32_t IDESC = sm100::idesc_f16_f32(128, 32);
    constexpr uint32_t IDESC64 = sm100::idesc_f16_f32(128, 64);
    const float tsgn = a.inverse ? 1.f : -1.f;
    const uint32_t sb = b ? x.t.sS1 : x.t.sS0;
    const uint32_t bb = b ? x.t.bS1 : x.t.bS0;
    // A pass with fewer columns than C loads only its own column blocks,
    // the leading part of the staging buffer; zero the rest so that stale
    // data does not enter the tile maximum.
    constexpr uint32_t kInBytes = (uint32_t)T::TP * (IN16 ? 4 : 8);
    if (a.in_tile_bytes < kInBytes) {
      for (uint32_t o = a.in_tile_bytes + 16u * ctid; o < kInBytes; o += 16u * NCT)
        sts128w(bb + o, make_uint4(0u, 0u, 0u, 0u));
      tile::named_bar(1, NCT);
    }
    // ------------------------------------------- tile maximum and scale
    uint4 q[NIT_P][NLD];
    {
      uint32_t amax = 0;
#pragma unroll
      for (int j = 0; j < NIT_P; ++j) {
        const int u = ctid + j * NCT;
        const uint32_t h = (uint32_t)(u / S::ITEMS);
        const uint32_t lb = (ient[j].x & 0xFFFFu) << 2;
#pragma unroll
        for (int n = 0; n < NLD; ++n) {
          q[j][n] = u < UNITS ? lds128w(xo(lb, a.lofs[n * NH + h], bb)) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
          for (int pp = 0; pp < 4 / NH; ++pp) {
            const float2 x = load_point<IN16>(q[j][n], pp);
            amax = max(amax, __float_as_uint(fabsf(x.x)));
            amax = max(amax, __float_as_uint(fabsf(x.y)));
          }
        }
      }
      amax = __reduce_max_sync(0xffffffffu, amax);
      if (lane == 0) atomicMax(&x.red[k & 1], amax);
    }
    tile::named_bar(1, NCT);
    const uint32_t tmax = x.red[k & 1];
    if (ctid == 0) x.red[(k + 1) & 1] = 0u;  // next tile's slot; last read a tile ago
    // 2^sexp puts the tile maximum in [2^13, 2^14)
    const int sexp = tmax == 0 ? 0 : 13 - ((int)((tmax >> 23) & 0xff) - 127);
    const float sc = exp2i(sexp);
    // L / (16 2^sexp): undoes the stage scalings (1/L in total) and the tile scale
    const float fm = exp2i(LGL - 4 - sexp);

    // ---------------------------------------------------------- prologue
    const uint32_t x0 = INPLACE_PROLOGUE ? bb : x.t.bA;  // stage-0 operand (hi; lo at + HALF)
    // The maximum pass already holds every unit's loads in q; staging is
    // rewritten in place only after all consumers are past the barrier
    // above, which they are.
#pragma unroll
    for (int j = 0; j < NIT_P; ++j) {
      const int u = ctid + j * NCT;
      if (UNITS % NCT != 0 && u >= UNITS) break;
      const uint32_t h = (uint32_t)(u / S::ITEMS);
      const uint32_t st = (ient[j].x >> 16) << 2;
      if constexpr (R == 1) {
#pragma unroll
        for (int jj = 0; jj < SUBV; ++jj) {
          const int sv = SUBV * h + jj;  // sub-vector within the item
          uint32_t hi[4], lo[4];
#pragma unroll
          for (int n = 0; n < 4; ++n) {
            const float2 x = load_point<IN16>(q[j][n], jj);
            split2(make_float2(x.x * sc, x.y * sc), hi[n], lo[n]);
          }
          sts128_hl<T::HALF>(xo(st, a.sofs[sv], x0), make_uint4(hi[0], hi[1], hi[2], hi[3]),
                             make_uint4(lo[0], lo[1], lo[2], lo[3]));
        }
      } else {
        const uint32_t trow = ient[j].y & 0x7FFFFFFFu;
        const bool colitem = (ient[j].y >> 31) != 0;
        // Sub-vector jj of the unit: radix-R butterflies, twiddle times
        // the tile scale, split, stores.
        auto subvec = [&](int jj, auto tw_of) {
          const int sv = SUBV * h + jj;
          float2 x[R];
#pragma unroll
          for (int n = 0; n < R; ++n) x[n] = load_point<IN16>(q[j][n], jj);
          small_dft<R>(x, tsgn);
#pragma unroll
          for (int k = 0; k < R; ++k) {
            // entry 0 of the table is W^0 / R = 1 / R: output 0 only takes
            // the (power-of-two) scale sc / R
            uint32_t hi, lo;
            split2(k == 0 ? make_float2(x[0].x * (sc * (1.f / R)), x[0].y * (sc * (1.f / R)))
                          : cmulf(x[k], tw_of(k)),
                   hi, lo);
            sts32_hl<T::HALF>(xo(st, a.sofs[sv * R + k], x0), hi, lo);
          }
        };
        if (colitem) {
          // column items: the sub-vectors share one twiddle row
          float2 wc[R];
          wc[0] = make_float2(sc, 0.f);  // unused (entry 0 is 1 / R)
#pragma unroll
          for (int k = 1; k < R; ++k) {
            const float2 w = lds64f(x.t.sTail + tail_offset(trow, k, R));
            wc[k] = make_float2(w.x * sc, w.y * sc);
          }
#pragma unroll
          for (int jj = 0; jj < SUBV; ++jj) subvec(jj, [&](int k) { return wc[k]; });
        } else {
#pragma unroll
          for (int jj = 0; jj < SUBV; ++jj)
            subvec(jj, [&](int k) {
              const float2 w = lds64f(x.t.sTail + ((trow + SUBV * h + jj) * R + k) * 8);
              return make_float2(w.x * sc, w.y * sc);
            });
        }
      }
    }
    sm100::fence_proxy_async_smem();
    sm100::tc_fence_before();
    tile::named_bar(1, NCT);
    sm100::tc_fence_after();

    // ------------------------------------------------------------ stages
#pragma unroll
    for (int s = 0; s < S::NST; ++s) {
      const uint32_t xs = ((S::NST - s) & 1) ? x.t.sA : sb;   // this stage's operand (hi)
      const uint32_t xn = ((S::NST - s) & 1) ? bb : x.t.bA;   // next stage's operand (window-relative)
      if (sp == ((warp >> 2) & 3) && lane == 0) {  // issuers on all four sub-partitions
#pragma unroll
        for (int j = 0; j < NIT_E; ++j) {
          const uint32_t m = (warp >> 2) + j * (NCW / 4);
          const uint32_t d = x.t.tmem + 64u * m;
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            const uint64_t ah = tile::sdesc_sw64(xs + m * 8192u + ks * 32u);
            const uint64_t al = tile::sdesc_sw64(xs + T::HALF + m * 8192u + ks * 32u);
            // B_hi rows then B_lo rows (contiguous): N = 64 over both
            const uint64_t bhl = tile::sdesc_sw64(x.t.sB + ks * 32u);
            sm100::umma_f16(d, ah, bhl, IDESC64, ks);
            sm100::umma_f16(d, al, bhl, IDESC, 1);
          }
          sm100::umma_commit(&x.t.mmab[m]);
        }
      }
      const bool last = s == S::NST - 1;
      const uint32_t row0 = stage_tw_row0<L, R>(s);
      float2 pt[NIT_E][2];
      if (POSTTW && last) post_twiddles<C, S::NV, false>(a, cb, s, eent, pt);
#pragma unroll
      for (int j = 0; j < NIT_E; ++j) {
        const uint32_t m = (warp >> 2) + j * (NCW / 4);
        const uint32_t e = eent[s][j];
        const uint32_t aux = e >> 16;
        const uint32_t dst = (e & 0xFFFFu) << 2;
        float4 wg[8];
        if (!last && !T::TW_SMEM) {
          const float4* t4 = a.tw + (size_t)(row0 + aux) * 8;
#pragma unroll
          for (int p = 0; p < 8; ++p) wg[p] = __ldg(t4 + (p ^ tw_fold(aux)));
        }
        if (!sm100::mbar_wait_bounded(&x.t.mmab[m], (mphase >> m) & 1u, kWaitLimit)) *x.t.abort_flag = 1;
        sm100::tc_fence_after();
        uint32_t d[32];
        {
          // D = columns [0, 32) + columns [32, 64) of this M-tile
          const uint32_t ta = x.t.tmem + ((uint32_t)(32 * sp) << 16) + 64u * m;
          sm100::tmem_ld32(ta, d);
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            uint32_t e2[16];
            sm100::tmem_ld16(ta + 32u + 16u * hh, e2);
            sm100::tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              float u0, u1;
              f2u(add2(f2p(__uint_as_float(d[16 * hh + 2 * q]), __uint_as_float(d[16 * hh + 2 * q + 1])),
                       f2p(__uint_as_float(e2[2 * q]), __uint_as_float(e2[2 * q + 1]))),
                  u0, u1);
              d[16 * hh + 2 * q] = __float_as_uint(u0);
              d[16 * hh + 2 * q + 1] = __float_as_uint(u1);
            }
          }
        }
        if (!last) {
          const uint32_t trow = x.t.sTws + (row0 + aux) * 128u;
          const uint32_t fold = tw_fold(aux);
          sm100::tmem_wait_ld();
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            float4 w[4];
#pragma unroll
            for (int pp = 0; pp < 4; ++pp)
              w[pp] = T::TW_SMEM ? lds128f(trow + (((4 * hh + pp) ^ fold) << 4)) : wg[4 * hh + pp];
#pragma unroll
            for (int pp = 0; pp < 4; ++pp) {
              const int p = 4 * hh + pp;
              uint64_t yr, yi;
              cmul2(f2p(__uint_as_float(d[4 * p]), __uint_as_float(d[4 * p + 1])),
                    f2p(__uint_as_float(d[4 * p + 2]), __uint_as_float(d[4 * p + 3])),
                    f2p(w[pp].x, w[pp].y), f2p(w[pp].z, w[pp].w), yr, yi);
              uint32_t h0, h1, l0, l1;
              split_pair(yr, yi, h0, h1, l0, l1);
              sts32_hl<T::HALF>(xo(dst, a.kofs[s][2 * p], xn), h0, l0);
              sts32_hl<T::HALF>(xo(dst, a.kofs[s][2 * p + 1], xn), h1, l1);
            }
          }
        } else if (POSTTW) {
          // Four-step twiddle W_N^((v + NV k) g) times L / (16 2^sexp):
          // pairs (w_2p, w_2p+1) advanced by ws^2 (FP32 recurrence, 7
          // steps, ~1e-7 relative).
          float2 w0 = pt[j][0];
          const float2 ws = pt[j][1];
          w0.x *= fm;
          w0.y *= fm;
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
            sts64w(xo(dst, a.kofs[s][2 * p], bb), r0, i0);
            sts64w(xo(dst, a.kofs[s][2 * p + 1], bb), r1, i1);
            if (p < 7) {
              uint64_t nr, ni;
              cmul2(wr, wi, s2r, s2i, nr, ni);
              wr = nr;
              wi = ni;
            }
          }
        } else {
          sm100::tmem_wait_ld();
          const uint64_t fm2 = f2p(fm, fm);
#pragma unroll
          for (int p = 0; p < 8; ++p) {
            float r0, r1, i0, i1;
            f2u(mul2(f2p(__uint_as_float(d[4 * p]), __uint_as_float(d[4 * p + 1])), fm2), r0, r1);
            f2u(mul2(f2p(__uint_as_float(d[4 * p + 2]), __uint_as_float(d[4 * p + 3])), fm2), i0, i1);
            sts64w(xo(dst, a.kofs[s][2 * p], bb), r0, i0);
            sts64w(xo(dst, a.kofs[s][2 * p + 1], bb), r1, i1);
          }
        }
      }
      mphase ^= (1u << NMT) - 1u;
      sm100::fence_proxy_async_smem();
      sm100::tc_fence_before();
      tile::named_bar(1, NCT);
      sm100::tc_fence_after();
      if (*x.t.abort_flag) break;
    }
  }
};

template <int L, int R, int C, bool POSTTW, int NCW, bool IN16>
// 17 warps are granted registers as 20: 65536 / 640 -> 96 per thread.
__global__ void __maxnreg__(96) fft_tile_split(const __grid_constant__ TileArgs a) {
  using S = TileShape<L, R, C, NCW>;
  using T = TileSplit<L, R, C, POSTTW, NCW, IN16>;
  using TL = SplitTile<L, R, C, POSTTW, NCW, IN16>;
  constexpr int NCT = S::NCT;
  constexpr int NMT = S::NMT;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw_u = sm100::smem_u32(smem_raw);
  const uint32_t base_u = (raw_u + 1023u) & ~1023u;
  uint8_t* smem = smem_raw + (base_u - raw_u);
  const uint32_t sS0 = base_u + T::OFF_S0, sS1 = base_u + T::OFF_S1;
  const uint32_t sA = base_u + T::OFF_A;
  const uint32_t sBh = base_u + T::OFF_B, sBl = sBh + 2048;
  const uint32_t sTail = base_u + T::OFF_TAIL;
  const uint32_t sTws = base_u + T::OFF_TWS;
  const uint32_t bS0 = sS0 - kWinBase, bS1 = sS1 - kWinBase, bA = sA - kWinBase;
  if (((bS0 | bS1 | bA) & (uint32_t)(T::BUF - 1)) != 0) {
    if (threadIdx.x == 0 && a.status) atomicExch(a.status, kStatusLayout);
    return;
  }
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + T::OFF_BAR);  // [2]
  uint64_t* outrdy = full + 2;                                      // [2]
  uint64_t* mmab = full + 4;                                        // [NMT]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(full + 4 + 16);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(full + 4 + 17);
  uint32_t* red = reinterpret_cast<uint32_t*>(full + 4 + 18);       // [2] tile maxima
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
      red[0] = 0u;
      red[1] = 0u;
      sm100::fence_mbar_init();
    }
    __syncwarp();
    sm100::tmem_alloc(tmem_slot, TL::TMEM_COLS);
    sm100::tmem_relinquish();
  } else {
    for (int i = tid; i < 128; i += NCT) {
      *reinterpret_cast<uint4*>(smem + T::OFF_B + 16 * i) = __ldg(a.bmat + i);
      *reinterpret_cast<uint4*>(smem + T::OFF_B + 2048 + 16 * i) = __ldg(a.bmat_lo + i);
    }
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
  const SplitCtx x{{sS0, sS1, sA, sBh, sTail, sTws, bS0, bS1, bA, tmem_base, mmab, abort_flag},
                   sBl, red};

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
        pending[b] = false;
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
      for (int b = 0; b < 2; ++b)
        if (pending[b]) sm100::mbar_wait_bounded(&full[b], pend_par[b], kWaitLimit);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ consumers
    uint2 ient[TL::NIT_P];
    uint32_t eent[TL::NST][TL::NIT_E];
    TL::entries(a, tid, ient, eent);
    uint32_t mphase = 0;  // bit m: completions of M-tile barrier m so far, mod 2
    int i = 0;
    for (int64_t t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++i) {
      const int b = i & 1;
      if (!sm100::mbar_wait_bounded(&full[b], (i >> 1) & 1, kWaitLimit)) *abort_flag = 1;
      if (*abort_flag) break;
      TL::run(a, x, tid, b, t % a.col_blocks, i, mphase, ient, eent);
      if (*abort_flag) break;
      if (tid == 0) tile::mbar_arrive(&outrdy[b]);
    }
  }
  __syncthreads();
  if (tid == 0 && *abort_flag && a.status) atomicExch(a.status, kStatusTimeout);
  if (producer) sm100::tmem_dealloc(tmem_base, TL::TMEM_COLS);
}

}  // namespace mcfft
