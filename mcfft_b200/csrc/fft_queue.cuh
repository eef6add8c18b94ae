// fft_queue.cuh -- persistent batch kernel: one launch runs every pass of a
// plan (many transforms of uneven lengths and dimensionality) from a device
// work queue of (pass, tile) items; one instantiation per precision form.
//
// Each CTA takes items blockIdx.x, blockIdx.x + gridDim.x, ... of the queue
// in order.  Per item the producer warp issues the TMA load of the tile's
// input and, once the consumers are done, the TMA store of its output; the
// consumer warps run the same per-tile routine as the per-pass kernels
// (F16Tile::run, SplitTile::run), instantiated for every pass variant (L,
// four-step twiddle, tile size or input type) and selected per item.  Layout tables and tensor maps of all
// passes live in the kernel's parameter block (constant bank).
//
// Dependencies between passes of one transform (the second pass of a
// four-step 1D transform, the column passes of 2D/3D transforms) go through
// counters in global memory: after its output tile is written, a producing
// tile adds 1 to the counter of every key (transform / slab) it covers; the
// producer warp of a consuming tile polls its key's counter until it holds
// the producing pass's tile count before loading.  The host orders the
// queue so that every dependency points to an earlier item, the kernel is
// launched cooperatively (all CTAs resident), and the producer never blocks
// its own stores while it waits for a dependency, so every wait ends.  All
// waits are bounded by kWaitLimit nanoseconds of global time; on timeout
// the kernel records kStatusTimeout, drains its own copies in flight,
// frees its tensor memory and returns.
//
// Memory ordering of a dependency: writer = bulk store, wait for its
// completion (cp.async.bulk.wait_group 0), proxy fence, release add;
// reader = acquire load, proxy fence, bulk tensor load.
#pragma once
#include "fft_tile.cuh"
#include "fft_tile_split.cuh"

namespace mcfft {

constexpr int kQueueMaxPasses = 33;

// One pass of the queue.  Field names match TileArgs where F16Tile reads
// them.
struct alignas(64) QPass {
  CUtensorMap tmap_in;
  CUtensorMap tmap_out;
  const uint2* item_tab;
  const uint32_t* epi_tab;
  uint32_t lofs[16];
  uint32_t sofs[32];
  uint32_t kofs[kMaxStages][16];
  const float4* tw;
  const float2* tail_tw;
  const float2* post_a;
  const float2* post_b;
  uint64_t post_mask;
  uint32_t post_shift;
  float post_scale;
  int inverse;
  int32_t in_cmul[5], in_omul[5], out_cmul[5], out_omul[5];
  int32_t in_ndims, out_ndims;
  int64_t col_blocks;
  uint32_t in_tile_bytes;
  int32_t variant;      // which compiled tile routine runs this pass
  int32_t wait_base;    // counters[wait_base + outer] >= wait_count before loading; -1: none
  int32_t wait_count;
  int32_t sig_base;     // after the store of tile t: +1 on counters[sig_base + k] for every
                        //   k in [t sig_mul / sig_div, ((t + 1) sig_mul - 1) / sig_div],
  int32_t tail_pm;      // radix-R table layout (tail_layout.h)
  int64_t sig_mul, sig_div, sig_kmax;  // k <= sig_kmax; sig_base -1: none
  // L2 eviction priority of the pass's tile loads and stores (kL2Normal,
  // kL2EvictFirst, kL2EvictLast).
  int32_t l2_in, l2_out;
  const struct QPassAux* aux;  // device; null: none of its features
};

// Per-pass features kept out of the parameter block (plan-owned device
// memory, fixed for the plan's life).
struct QPassAux {
  // Input read for the last time (an intermediate between passes): once a
  // tile is in shared memory its source lines are dropped from L2 without
  // write-back.  Row-input passes only: tile (cb, outer) covers rows
  // cb * C + r (r < C) of disc_row_bytes at disc_base + outer * disc_so +
  // row * disc_sc.  disc_base null: none.
  const char* disc_base;
  int64_t disc_sc, disc_so;
  uint32_t disc_row_bytes;
  int32_t disc_C;
  // Transforms at unrelated offsets of the user's buffers (descriptors of
  // one shape that do not follow each other):
  //  - in_otab / out_otab: the outer (transform) coordinate of tile outer
  //    index o is otab[o] instead of o (the map's outer stride is the
  //    offsets' common unit);
  //  - in_gtab / out_gtab (one-pass 1D groups, whose tiles span several
  //    transforms): the tile's staging is filled / drained by row gathers /
  //    scatters of a map whose rows hold one staging row (g_row_bytes),
  //    column c's rows at gtab[c] + j, j < gin_rows / gout_rows; four
  //    columns per instruction.
  const int32_t* in_otab;
  const int32_t* out_otab;
  const int32_t* in_gtab;
  const int32_t* out_gtab;
  int32_t gin_rows, gout_rows, g_C, g_row_bytes;
};

constexpr int32_t kL2Normal = 0, kL2EvictFirst = 1, kL2EvictLast = 2;

struct QItem {
  uint32_t pass;
  uint32_t tile;
};

struct alignas(64) QArgs {
  const QItem* items;
  int64_t nitems;
  int* counters;
  int* status;
  const uint4* bmat;     // DFT-16 embedding, 64B-swizzled K-major, 2 KB (plain: scaled by 1/16)
  const uint4* bmat_lo;  // split form: its low part
  int npass;
  QPass pass[kQueueMaxPasses];
};
static_assert(sizeof(QArgs) <= 32764, "kernel parameter block");

// Queue-kernel shared memory: three 64 KB tile buffers (16K FP16 or 8K
// FP32 points), the DFT-16 matrices, then the largest radix-R and stage-row
// tables any variant keeps in shared memory.
struct QueueSmem {
  static constexpr int STAGE_BYTES = 65536;
  static constexpr int OFF_S0 = 0;
  static constexpr int OFF_S1 = STAGE_BYTES;
  static constexpr int OFF_A = 2 * STAGE_BYTES;
  static constexpr int OFF_B = 3 * STAGE_BYTES;        // high, then low (split) matrix
  static constexpr int OFF_TAIL = OFF_B + 4096;
  static constexpr int OFF_TWS = OFF_TAIL + 2048 * 8;  // radix-R table of L <= 2048
  static constexpr int TWS_BYTES = 32 * 128;           // up to 32 stage rows
  static constexpr int OFF_BAR = OFF_TWS + TWS_BYTES;
  static constexpr int SMEM_BYTES = OFF_BAR + 256;     // the window base must be 1 KB aligned
  static_assert(SMEM_BYTES <= 232448, "shared memory budget");
};

namespace queue {

// Variant index of a pass: L = 32 .. 4096, with and without the four-step
// twiddle; plain form: 16K- or 8K-point tiles (4096 only 16K), variant =
// 16 * (8K tile) + 2 * index(L) + posttw; split form (8K tiles, L <= 2048):
// variant = 16 * (FP16 input) + 2 * index(L) + posttw.
__host__ __device__ constexpr int variant_of(int L, bool posttw, bool alt) {
  int i = 0;
  for (int l = 32; l < L; l <<= 1) ++i;
  return 16 * (alt ? 1 : 0) + 2 * i + (posttw ? 1 : 0);
}

}  // namespace queue

// The kernel itself is compiled in one translation unit (queue.cu).
#ifdef MCFFT_QUEUE_KERNEL
namespace queue {

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(sm100::smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add(int* p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

template <int V>
struct Variant {
  static constexpr int LI = (V >> 1) & 7;  // L = 32 << LI
  static constexpr int L = 32 << LI;
  static constexpr int R = 1 << ((5 + LI) % 4);
  static constexpr bool PT = (V & 1) != 0;
  static constexpr bool ALT = V >= 16;     // plain: 8K tiles; split: FP16 input
};

// Runs this CTA's consecutive items k, k+1, ... that belong to pass `pi`
// with tile routine TL; returns the local index of the first item of
// another pass.  The pass's tables go to shared memory and its layout
// entries to registers once per run.
// The (pass, tile) of the item in staging buffer b, written by the producer
// before it arms that buffer's load barrier (its arrive releases the write;
// the consumers' wait on the barrier acquires it), so that the consumers
// never read the item list in global memory.  Two 8-byte slots after the
// other barrier-area words.
__device__ __forceinline__ volatile QItem* item_ring(uint64_t* full) {
  return reinterpret_cast<volatile QItem*>(full + 4 + 20);
}
__device__ __forceinline__ QItem ring_item(uint64_t* full, int b) {
  volatile QItem* r = item_ring(full);
  return QItem{r[b].pass, r[b].tile};
}

// Drops the source lines of tile t of a pass whose input is read for the
// last time (QPassAux::disc_base); the consumer threads share the lines.
// Runs once the tile's load has completed.
__device__ __forceinline__ void discard_tile(const QPassAux& X, int64_t col_blocks, int64_t t,
                                             int ctid, int nct) {
  const int64_t cb = t % col_blocks, outer = t / col_blocks;
  // rows hold a power of two of 128-byte lines: line i of the tile is line
  // i & (per_row - 1) of row i >> lg
  const uint32_t lg = (uint32_t)(__ffs(X.disc_row_bytes) - 8);
  const uint32_t lines = (uint32_t)X.disc_C << lg;
  const char* base = X.disc_base + outer * X.disc_so + cb * X.disc_C * X.disc_sc;
  for (uint32_t i = (uint32_t)ctid; i < lines; i += (uint32_t)nct)
    tile::discard_l2_line(base + (int64_t)(i >> lg) * X.disc_sc +
                          ((int64_t)(i & ((1u << lg) - 1u)) << 7));
}

// RESIDENT: the pass's tables are already in shared memory (x points at
// them); otherwise they are loaded here, at the start of the run.
template <class TL, bool SPLIT, bool RESIDENT = false, class X>
__device__ __forceinline__ int64_t run_items(const QArgs& a, uint32_t pi, const X& x,
                                             uint8_t* smem, uint64_t* full, uint64_t* outrdy,
                                             int ctid, int64_t k, int64_t nlocal,
                                             uint32_t& mphase) {
  static_assert(RESIDENT || !TL::T::TW_SMEM || TL::T::TW_ROWS * 128 <= QueueSmem::TWS_BYTES,
                "stage rows");
  const QPass& P = a.pass[pi];
  // The layout entries' loads are issued first, so that they are in flight
  // while the tables are copied (one L2 round trip per run instead of two).
  uint2 ient[TL::NIT_P];
  uint32_t eent[TL::NST][TL::NIT_E];
  TL::entries(P, ctid, ient, eent);
  if constexpr (!RESIDENT) {
    // every consumer is past the previous tile's last barrier, so nobody
    // still reads the old tables
    TL::tables(P, smem + QueueSmem::OFF_TAIL, smem + QueueSmem::OFF_TWS, ctid);
    tile::named_bar(1, TL::NCT);
  }
  volatile int* abort_flag;
  if constexpr (SPLIT) abort_flag = x.t.abort_flag;
  else abort_flag = x.abort_flag;
  const bool disc = P.aux && P.aux->disc_base;
  for (;;) {
    const int b = (int)(k & 1);
    const int64_t t = ring_item(full, b).tile;  // the tile in buffer b (loaded: full[b] waited)
    if (disc) discard_tile(*P.aux, P.col_blocks, t, ctid, TL::NCT);
    if constexpr (SPLIT) {
      TL::run(P, x, ctid, b, t % P.col_blocks, k, mphase, ient, eent);
    } else {
      TL::run(P, x, ctid, b, t % P.col_blocks, mphase, ient, eent);
    }
    if (*abort_flag) return nlocal;
    if (ctid == 0) tile::mbar_arrive(&outrdy[b]);
    if (++k >= nlocal) return k;
    // the next item's buffer: once it is loaded, its ring slot tells its pass
    // (a run that ends here returns with that wait done; repeating it is free)
    if (!sm100::mbar_wait_bounded(&full[k & 1], (uint32_t)(k >> 1) & 1u, kWaitLimit)) {
      *abort_flag = 1;
      return nlocal;
    }
    if (*abort_flag) return nlocal;
    if (ring_item(full, (int)(k & 1)).pass != pi) return k;
  }
}

// A gathered tile: staging row (j, c) of g_row_bytes (rows j, columns c
// innermost, no swizzle) is buffer row gtab[c] + j; four columns per
// gather.
__device__ __forceinline__ void gather_tile(const CUtensorMap* map, const QPassAux& X,
                                            const int32_t* gtab, uint32_t dst, uint64_t* bar) {
  for (int c = 0; c < X.g_C; c += 4) {
    const int32_t r0 = gtab[c], r1 = gtab[c + 1], r2 = gtab[c + 2], r3 = gtab[c + 3];
    for (int j = 0; j < X.gin_rows; ++j)
      tile::tma_gather4(map, dst + (uint32_t)((j * X.g_C + c) * X.g_row_bytes), bar, r0 + j,
                        r1 + j, r2 + j, r3 + j);
  }
}
__device__ __forceinline__ void scatter_tile(const CUtensorMap* map, const QPassAux& X,
                                             const int32_t* gtab, uint32_t src) {
  for (int c = 0; c < X.g_C; c += 4) {
    const int32_t r0 = gtab[c], r1 = gtab[c + 1], r2 = gtab[c + 2], r3 = gtab[c + 3];
    for (int j = 0; j < X.gout_rows; ++j)
      tile::tma_scatter4(map, src + (uint32_t)((j * X.g_C + c) * X.g_row_bytes), r0 + j, r1 + j,
                         r2 + j, r3 + j);
  }
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// The producer warp's event loop (one thread): store finished tiles as
// soon as the consumers release them; load the next tile once its buffer is
// free and its dependency is met.  Never blocks on one while the other
// could proceed.
__device__ __forceinline__ void producer_loop(const QArgs& a, uint32_t sS0, uint32_t sS1,
                                              uint64_t* full, uint64_t* outrdy,
                                              volatile int* abort_flag, int64_t nlocal) {
  const int64_t G = gridDim.x;
  const uint64_t pol_first = tile::policy_evict_first(), pol_last = tile::policy_evict_last();
  auto pol = [&](int32_t h) -> uint64_t {
    return h == kL2EvictFirst ? pol_first : h == kL2EvictLast ? pol_last : 0ull;
  };
  int64_t il = 0, is = 0;  // next local item to load / to store
  int64_t sig = -1;        // stored item whose completion is still to be signalled
  QItem sig_it{0u, 0u};    // that item
  bool idle = false;       // no progress since idle_since (global timer, ns)
  uint32_t idle_since = 0;
  // Item il, read one load ahead so that its latency overlaps the wait for
  // the consumers (a stored item is read back from its ring slot).
  QItem nxt = nlocal > 0 ? a.items[blockIdx.x] : QItem{0u, 0u};
  bool nxt_ready = false;  // item il's dependency seen complete (counters only grow)
  // Acquire check of item il's dependency: once seen complete it stays so.
  auto dep_met = [&]() -> bool {
    if (nxt_ready) return true;
    const QPass& P = a.pass[nxt.pass];
    if (P.wait_base >= 0) {
      if (queue::ld_acquire(a.counters + P.wait_base + nxt.tile / P.col_blocks) < P.wait_count)
        return false;
      queue::fence_proxy_async_global();
    }
    nxt_ready = true;
    return true;
  };
  // Completion of a producing tile: its bulk store has finished writing,
  // then a release add on every key it covers.
  auto signal = [&](const QItem& it) {
    const QPass& P = a.pass[it.pass];
    tile::tma_store_wait_all();
    queue::fence_proxy_async_global();
    const int64_t k0 = (int64_t)it.tile * P.sig_mul / P.sig_div;
    int64_t k1 = ((int64_t)it.tile * P.sig_mul + P.sig_mul - 1) / P.sig_div;
    if (k1 > P.sig_kmax) k1 = P.sig_kmax;
    for (int64_t key = k0; key <= k1; ++key)
      queue::red_release_add(a.counters + P.sig_base + key, 1);
  };
  while (is < nlocal) {
    bool moved = false;
    if (is < il && queue::mbar_test(&outrdy[is & 1], (uint32_t)(is >> 1) & 1u)) {
      const QItem it = ring_item(full, (int)(is & 1));  // item is, written when it was loaded
      const QPass& P = a.pass[it.pass];
      const uint32_t src = (is & 1) ? sS1 : sS0;
      const int64_t cb = it.tile % P.col_blocks, outer = it.tile / P.col_blocks;
      const QPassAux* X = P.aux;
      if (X && X->out_gtab) {
        scatter_tile(&P.tmap_out, *X, X->out_gtab + cb * X->g_C, src);
      } else {
        int32_t crd[5];
        tile::tile_coords(P.out_cmul, P.out_omul, cb,
                          X && X->out_otab ? X->out_otab[outer] : outer, crd);
        tile::tma_store_pol(&P.tmap_out, P.out_ndims, crd, src, pol(P.l2_out));
      }
      tile::tma_store_wait_read();
      if (sig >= 0) signal(sig_it);
      sig = P.sig_base >= 0 ? is : -1;
      sig_it = it;
      ++is;
      moved = true;
    }
    if (il < nlocal && il < is + 2 && !*abort_flag) {
      const QItem it = nxt;
      const QPass& P = a.pass[it.pass];
      const int64_t outer = it.tile / P.col_blocks;
      if (dep_met()) {
        const uint32_t dst = (il & 1) ? sS1 : sS0;
        const int64_t cb = it.tile % P.col_blocks;
        volatile QItem* ring = item_ring(full);
        ring[il & 1].pass = it.pass;
        ring[il & 1].tile = it.tile;
        sm100::mbar_arrive_expect_tx(&full[il & 1], P.in_tile_bytes);
        const QPassAux* X = P.aux;
        if (X && X->in_gtab) {
          gather_tile(&P.tmap_in, *X, X->in_gtab + cb * X->g_C, dst, &full[il & 1]);
        } else {
          int32_t crd[5];
          tile::tile_coords(P.in_cmul, P.in_omul, cb,
                            X && X->in_otab ? X->in_otab[outer] : outer, crd);
          tile::tma_load_pol(&P.tmap_in, P.in_ndims, crd, dst, &full[il & 1], pol(P.l2_in));
        }
        tile::prefetch_tmap(&P.tmap_out);  // for this tile's store
        ++il;
        if (il < nlocal) nxt = a.items[blockIdx.x + il * G];
        nxt_ready = false;
        moved = true;
      }
    }
    // Signal after the attempt to issue the next load, so that waiting
    // for the store's completion does not delay it (and never later: the
    // next load may depend on this very tile).
    if (sig >= 0) {
      signal(sig_it);
      sig = -1;
    }
    if (moved) {
      idle = false;
    } else if (is < il && (il == is + 2 || il == nlocal || *abort_flag)) {
      // Only the consumers' release of tile `is` can make progress: check
      // the next load's dependency now (its latency then overlaps the
      // wait), then wait for the release on the barrier (a bounded try-wait
      // suspends the thread instead of spinning, which would take issue
      // slots from the consumers).
      if (il < nlocal && !*abort_flag) {
        tile::prefetch_tmap(&a.pass[nxt.pass].tmap_in);
        dep_met();
      }
      if (!sm100::mbar_wait_bounded(&outrdy[is & 1], (uint32_t)(is >> 1) & 1u, kWaitLimit) ||
          *abort_flag) {
        *abort_flag = 1;
        break;
      }
    } else {
      // Waiting for a dependency (or for both events): poll with a back-off.
      const uint32_t now = sm100::globaltimer_ns();
      if (!idle) {
        idle = true;
        idle_since = now;
      }
      if (*abort_flag || now - idle_since > kWaitLimit) {
        *abort_flag = 1;
        break;
      }
      __nanosleep(128);
    }
  }
  if (sig >= 0) signal(sig_it);
  tile::tma_store_wait_all();
  // Loads issued but not consumed (abort path) must land before the
  // CTA's shared memory is released.
  for (int64_t k = is; k < il; ++k)
    sm100::mbar_wait_bounded(&full[k & 1], (uint32_t)(k >> 1) & 1u, kWaitLimit);
}

template <int V>
__device__ __forceinline__ int64_t run_variant(const QArgs& a, uint32_t pi, const TileCtx& x,
                                               uint8_t* smem, uint64_t* full, uint64_t* outrdy,
                                               int ctid, int64_t k, int64_t nlocal,
                                               uint32_t& mphase) {
  using VV = Variant<V>;
  constexpr int C = (VV::ALT ? 8192 : 16384) / VV::L;
  static_assert(C >= 4, "columns per tile");
  using TL = F16Tile<VV::L, VV::R, C, VV::PT, 16>;
  return run_items<TL, false>(a, pi, x, smem, full, outrdy, ctid, k, nlocal, mphase);
}

template <int V>
__device__ __forceinline__ int64_t run_variant_split(const QArgs& a, uint32_t pi,
                                                     const SplitCtx& x, uint8_t* smem,
                                                     uint64_t* full, uint64_t* outrdy, int ctid,
                                                     int64_t k, int64_t nlocal,
                                                     uint32_t& mphase) {
  using VV = Variant<V>;
  static_assert(VV::L <= 2048, "split tiles hold at least four columns");
  using TL = SplitTile<VV::L, VV::R, 8192 / VV::L, VV::PT, 16, VV::ALT>;
  return run_items<TL, true>(a, pi, x, smem, full, outrdy, ctid, k, nlocal, mphase);
}

}  // namespace queue

// 16 consumer warps + 1 producer warp; 96 registers (17 warps are granted
// registers as 20).  SPLIT selects the precision form.
template <bool SPLIT>
__global__ void __maxnreg__(96) fft_queue(const __grid_constant__ QArgs a) {
  constexpr int NCW = 16, NCT = NCW * 32, NMTMAX = 8;
  constexpr int TMEM_COLS = 256;  // plain: 8 M-tiles x 32; split: 4 M-tiles x 64
  using Q = QueueSmem;
  extern __shared__ uint8_t smem[];
  const uint32_t base_u = sm100::smem_u32(smem);
  const uint32_t sS0 = base_u + Q::OFF_S0, sS1 = base_u + Q::OFF_S1, sA = base_u + Q::OFF_A;
  const uint32_t bS0 = sS0 - kWinBase, bS1 = sS1 - kWinBase, bA = sA - kWinBase;
  if ((base_u & 1023u) != 0 || ((bS0 | bS1 | bA) & (uint32_t)(Q::STAGE_BYTES - 1)) != 0) {
    if (threadIdx.x == 0 && a.status) atomicExch(a.status, kStatusLayout);
    return;
  }
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + Q::OFF_BAR);  // [2]
  uint64_t* outrdy = full + 2;                                      // [2]
  uint64_t* mmab = full + 4;                                        // [up to 16]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(full + 4 + 16);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(full + 4 + 17);
  uint32_t* red = reinterpret_cast<uint32_t*>(full + 4 + 18);       // [2] split: tile maxima
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const bool producer = warp == NCW;
  const int64_t G = gridDim.x;
  const int64_t nlocal = a.nitems > blockIdx.x ? (a.nitems - blockIdx.x + G - 1) / G : 0;

  if (producer) {
    if (lane == 0) {
      sm100::mbar_init(&full[0], 1);
      sm100::mbar_init(&full[1], 1);
      sm100::mbar_init(&outrdy[0], 1);
      sm100::mbar_init(&outrdy[1], 1);
      for (int m = 0; m < NMTMAX; ++m) sm100::mbar_init(&mmab[m], 1);
      *abort_flag = 0;
      red[0] = 0u;
      red[1] = 0u;
      sm100::fence_mbar_init();
    }
    __syncwarp();
    sm100::tmem_alloc(tmem_slot, TMEM_COLS);
    sm100::tmem_relinquish();
  } else {
    for (int i = tid; i < 128; i += NCT) {
      *reinterpret_cast<uint4*>(smem + Q::OFF_B + 16 * i) = __ldg(a.bmat + i);
      if (SPLIT) *reinterpret_cast<uint4*>(smem + Q::OFF_B + 2048 + 16 * i) = __ldg(a.bmat_lo + i);
    }
  }
  sm100::fence_proxy_async_smem();
  sm100::tc_fence_before();
  __syncthreads();
  sm100::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const TileCtx x{sS0, sS1, sA, base_u + Q::OFF_B, base_u + Q::OFF_TAIL, base_u + Q::OFF_TWS,
                  bS0, bS1, bA, tmem_base, mmab, abort_flag};
  const SplitCtx xs{x, base_u + Q::OFF_B + 2048, red};

  if (producer) {
    if (lane == 0) queue::producer_loop(a, sS0, sS1, full, outrdy, abort_flag, nlocal);
    __syncwarp();
  } else {
    // ------------------------------------------------------------ consumers
    uint32_t mphase = 0;  // bit m: phase of mmab[m] (variants use 4 or 8 M-tiles)
    for (int64_t k = 0; k < nlocal;) {
      if (!sm100::mbar_wait_bounded(&full[k & 1], (uint32_t)(k >> 1) & 1u, kWaitLimit)) *abort_flag = 1;
      if (*abort_flag) break;
      const uint32_t pi = queue::ring_item(full, (int)(k & 1)).pass;
      if constexpr (SPLIT) {
        switch (a.pass[pi].variant) {
#define MCFFT_QCASE(V)                                                                          \
  case V:                                                                                       \
    k = queue::run_variant_split<V>(a, pi, xs, smem, full, outrdy, tid, k, nlocal, mphase); \
    break;
          MCFFT_QCASE(0) MCFFT_QCASE(1) MCFFT_QCASE(2) MCFFT_QCASE(3)
          MCFFT_QCASE(4) MCFFT_QCASE(5) MCFFT_QCASE(6) MCFFT_QCASE(7)
          MCFFT_QCASE(8) MCFFT_QCASE(9) MCFFT_QCASE(10) MCFFT_QCASE(11)
          MCFFT_QCASE(12) MCFFT_QCASE(13)
          MCFFT_QCASE(16) MCFFT_QCASE(17) MCFFT_QCASE(18) MCFFT_QCASE(19)
          MCFFT_QCASE(20) MCFFT_QCASE(21) MCFFT_QCASE(22) MCFFT_QCASE(23)
          MCFFT_QCASE(24) MCFFT_QCASE(25) MCFFT_QCASE(26) MCFFT_QCASE(27)
          MCFFT_QCASE(28) MCFFT_QCASE(29)
#undef MCFFT_QCASE
          default: *abort_flag = 1; break;
        }
      } else {
        switch (a.pass[pi].variant) {
#define MCFFT_QCASE(V)                                                                 \
  case V:                                                                              \
    k = queue::run_variant<V>(a, pi, x, smem, full, outrdy, tid, k, nlocal, mphase); \
    break;
          MCFFT_QCASE(0) MCFFT_QCASE(1) MCFFT_QCASE(2) MCFFT_QCASE(3)
          MCFFT_QCASE(4) MCFFT_QCASE(5) MCFFT_QCASE(6) MCFFT_QCASE(7)
          MCFFT_QCASE(8) MCFFT_QCASE(9) MCFFT_QCASE(10) MCFFT_QCASE(11)
          MCFFT_QCASE(12) MCFFT_QCASE(13) MCFFT_QCASE(14) MCFFT_QCASE(15)
          MCFFT_QCASE(16) MCFFT_QCASE(17)
          MCFFT_QCASE(18) MCFFT_QCASE(19) MCFFT_QCASE(20) MCFFT_QCASE(21)
          MCFFT_QCASE(22) MCFFT_QCASE(23) MCFFT_QCASE(24) MCFFT_QCASE(25)
          MCFFT_QCASE(26) MCFFT_QCASE(27) MCFFT_QCASE(28) MCFFT_QCASE(29)
#undef MCFFT_QCASE
          default: *abort_flag = 1; break;
        }
      }
      if (*abort_flag) break;
    }
  }
  __syncthreads();
  if (tid == 0 && *abort_flag && a.status) atomicExch(a.status, kStatusTimeout);
  if (producer) sm100::tmem_dealloc(tmem_base, TMEM_COLS);
}

namespace queue {

// The tile routine of variant V (see variant_of).
template <int V, bool SPLIT>
struct VariantTile;
template <int V>
struct VariantTile<V, false> {
  using VV = Variant<V>;
  using type = F16Tile<VV::L, VV::R, (VV::ALT ? 8192 : 16384) / VV::L, VV::PT, 16>;
};
template <int V>
struct VariantTile<V, true> {
  using VV = Variant<V>;
  using type = SplitTile<VV::L, VV::R, 8192 / VV::L, VV::PT, 16, VV::ALT>;
};

}  // namespace queue

// Shared memory of a fused pair of passes: the batch kernel's three tile
// buffers and DFT-16 matrices, then both passes' tables side by side.
template <bool SPLIT, int V1, int V2>
struct FusedSmem {
  using TL1 = typename queue::VariantTile<V1, SPLIT>::type;
  using TL2 = typename queue::VariantTile<V2, SPLIT>::type;
  static constexpr int OFF_S0 = QueueSmem::OFF_S0;
  static constexpr int OFF_S1 = QueueSmem::OFF_S1;
  static constexpr int OFF_A = QueueSmem::OFF_A;
  static constexpr int OFF_B = QueueSmem::OFF_B;
  static constexpr int OFF_TAIL1 = OFF_B + 4096;
  static constexpr int OFF_TWS1 = OFF_TAIL1 + TL1::T::TAIL_BYTES;
  static constexpr int OFF_TAIL2 = OFF_TWS1 + TL1::T::TWS_BYTES;
  static constexpr int OFF_TWS2 = OFF_TAIL2 + TL2::T::TAIL_BYTES;
  static constexpr int OFF_BAR = OFF_TWS2 + TL2::T::TWS_BYTES;
  static constexpr int SMEM_BYTES = OFF_BAR + 256;
  static_assert(SMEM_BYTES <= 232448, "shared memory budget");
};

// A four-step pair of passes (pass 0 on tile variant V1 with the four-step
// twiddle, pass 1 on V2) in one persistent launch: the batch queue's
// producer, dependency counters and item order, restricted to the two
// variants, with both passes' tables resident in shared memory so that a
// CTA may switch pass every few tiles at no cost.  The host orders the
// items so that a transform's second pass follows its first pass closely
// and the intermediate is still in L2 when it is read (the passes' L2
// policies and scratch discards keep it there and keep it from being
// written back).  Launched cooperatively, like the batch kernel.
template <bool SPLIT, int V1, int V2>
__global__ void __maxnreg__(96) fft_fused(const __grid_constant__ QArgs a) {
  constexpr int NCW = 16, NCT = NCW * 32, NMTMAX = 8;
  constexpr int TMEM_COLS = 256;
  using F = FusedSmem<SPLIT, V1, V2>;
  using TL1 = typename F::TL1;
  using TL2 = typename F::TL2;
  extern __shared__ uint8_t smem[];
  const uint32_t base_u = sm100::smem_u32(smem);
  const uint32_t sS0 = base_u + F::OFF_S0, sS1 = base_u + F::OFF_S1, sA = base_u + F::OFF_A;
  const uint32_t bS0 = sS0 - kWinBase, bS1 = sS1 - kWinBase, bA = sA - kWinBase;
  if ((base_u & 1023u) != 0 || ((bS0 | bS1 | bA) & (uint32_t)(QueueSmem::STAGE_BYTES - 1)) != 0 ||
      a.npass != 2) {
    if (threadIdx.x == 0 && a.status) atomicExch(a.status, kStatusLayout);
    return;
  }
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + F::OFF_BAR);  // [2]
  uint64_t* outrdy = full + 2;                                      // [2]
  uint64_t* mmab = full + 4;                                        // [up to 16]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(full + 4 + 16);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(full + 4 + 17);
  uint32_t* red = reinterpret_cast<uint32_t*>(full + 4 + 18);       // [2] split: tile maxima
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const bool producer = warp == NCW;
  const int64_t G = gridDim.x;
  const int64_t nlocal = a.nitems > blockIdx.x ? (a.nitems - blockIdx.x + G - 1) / G : 0;

  if (producer) {
    if (lane == 0) {
      sm100::mbar_init(&full[0], 1);
      sm100::mbar_init(&full[1], 1);
      sm100::mbar_init(&outrdy[0], 1);
      sm100::mbar_init(&outrdy[1], 1);
      for (int m = 0; m < NMTMAX; ++m) sm100::mbar_init(&mmab[m], 1);
      *abort_flag = 0;
      red[0] = 0u;
      red[1] = 0u;
      sm100::fence_mbar_init();
    }
    __syncwarp();
    sm100::tmem_alloc(tmem_slot, TMEM_COLS);
    sm100::tmem_relinquish();
  } else {
    for (int i = tid; i < 128; i += NCT) {
      *reinterpret_cast<uint4*>(smem + F::OFF_B + 16 * i) = __ldg(a.bmat + i);
      if (SPLIT) *reinterpret_cast<uint4*>(smem + F::OFF_B + 2048 + 16 * i) = __ldg(a.bmat_lo + i);
    }
    TL1::tables(a.pass[0], smem + F::OFF_TAIL1, smem + F::OFF_TWS1, tid);
    TL2::tables(a.pass[1], smem + F::OFF_TAIL2, smem + F::OFF_TWS2, tid);
  }
  sm100::fence_proxy_async_smem();
  sm100::tc_fence_before();
  __syncthreads();
  sm100::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const TileCtx x1{sS0, sS1, sA, base_u + F::OFF_B, base_u + F::OFF_TAIL1, base_u + F::OFF_TWS1,
                   bS0, bS1, bA, tmem_base, mmab, abort_flag};
  const TileCtx x2{sS0, sS1, sA, base_u + F::OFF_B, base_u + F::OFF_TAIL2, base_u + F::OFF_TWS2,
                   bS0, bS1, bA, tmem_base, mmab, abort_flag};

  if (producer) {
    if (lane == 0) queue::producer_loop(a, sS0, sS1, full, outrdy, abort_flag, nlocal);
    __syncwarp();
  } else {
    uint32_t mphase = 0;  // bit m: phase of mmab[m]
    for (int64_t k = 0; k < nlocal;) {
      if (!sm100::mbar_wait_bounded(&full[k & 1], (uint32_t)(k >> 1) & 1u, kWaitLimit)) *abort_flag = 1;
      if (*abort_flag) break;
      const uint32_t pi = queue::ring_item(full, (int)(k & 1)).pass;
      if constexpr (SPLIT) {
        const SplitCtx s1{x1, base_u + F::OFF_B + 2048, red};
        const SplitCtx s2{x2, base_u + F::OFF_B + 2048, red};
        k = pi == 0 ? queue::run_items<TL1, true, true>(a, 0, s1, smem, full, outrdy, tid, k, nlocal, mphase)
                    : queue::run_items<TL2, true, true>(a, 1, s2, smem, full, outrdy, tid, k, nlocal, mphase);
      } else {
        k = pi == 0 ? queue::run_items<TL1, false, true>(a, 0, x1, smem, full, outrdy, tid, k, nlocal, mphase)
                    : queue::run_items<TL2, false, true>(a, 1, x2, smem, full, outrdy, tid, k, nlocal, mphase);
      }
      if (*abort_flag) break;
    }
  }
  __syncthreads();
  if (tid == 0 && *abort_flag && a.status) atomicExch(a.status, kStatusTimeout);
  if (producer) sm100::tmem_dealloc(tmem_base, TMEM_COLS);
}

#endif  // MCFFT_QUEUE_KERNEL

}  // namespace mcfft
