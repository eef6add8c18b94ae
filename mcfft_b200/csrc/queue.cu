// queue.cu -- host side of the persistent batch kernel (fft_queue.cuh):
// parameter-block construction and cooperative launch.
#include <cstring>
#include <mutex>

#define MCFFT_QUEUE_KERNEL
#include "fft_queue.cuh"
#include "queue.h"
#include "tile_pass.h"

namespace mcfft {

int queue_variant(const TileKernel& k) {
  const int L = k.L;
  if (L < 32 || L > 4096 || (L & (L - 1))) return -1;
  if (k.split) {
    if (k.tile_points != 8192 || L > 2048) return -1;
    return queue::variant_of(L, k.posttw, k.in16);
  }
  if (k.tile_points != 16384 && k.tile_points != 8192) return -1;
  if (L * 4 > k.tile_points) return -1;
  return queue::variant_of(L, k.posttw, k.tile_points == 8192);
}

bool fill_qpass(const TilePass& tp, int dir, const void* in, void* out, QPass* q) {
  const TileArgs& a = tp.args;
  std::memset(q, 0, sizeof(*q));
  if (!tile_encode(&q->tmap_in, tp.lay.in, in) || !tile_encode(&q->tmap_out, tp.lay.out, out))
    return false;
  q->item_tab = a.item_tab;
  q->epi_tab = a.epi_tab;
  std::memcpy(q->lofs, a.lofs, sizeof(q->lofs));
  std::memcpy(q->sofs, a.sofs, sizeof(q->sofs));
  std::memcpy(q->kofs, a.kofs, sizeof(q->kofs));
  q->tw = tp.tw[dir];
  q->tail_tw = tp.tail[dir];
  q->post_a = tp.post_a[dir];
  q->post_b = tp.post_b[dir];
  q->post_mask = a.post_mask;
  q->post_shift = a.post_shift;
  q->post_scale = a.post_scale;
  q->inverse = dir;
  q->tail_pm = a.tail_pm;
  std::memcpy(q->in_cmul, a.in_cmul, sizeof(q->in_cmul));
  std::memcpy(q->in_omul, a.in_omul, sizeof(q->in_omul));
  std::memcpy(q->out_cmul, a.out_cmul, sizeof(q->out_cmul));
  std::memcpy(q->out_omul, a.out_omul, sizeof(q->out_omul));
  q->in_ndims = a.in_ndims;
  q->out_ndims = a.out_ndims;
  q->col_blocks = a.col_blocks;
  q->in_tile_bytes = a.in_tile_bytes;
  q->variant = queue_variant(*tp.k);
  q->l2_in = kL2Normal;
  q->l2_out = kL2Normal;
  q->aux = nullptr;
  q->wait_base = -1;
  q->sig_base = -1;
  q->sig_mul = 1;
  q->sig_div = 1;
  return q->variant >= 0;
}

const void* queue_fn_split();  // queue_split.cu

namespace {
const void* queue_fn(bool split) {
  return split ? queue_fn_split() : reinterpret_cast<const void*>(&fft_queue<false>);
}
}  // namespace

cudaError_t launch_queue_fn(const void* fn, int smem_bytes, const QArgs& a, int grid,
                            cudaStream_t st) {
  void* args[] = {const_cast<QArgs*>(&a)};
  // Cooperative: every CTA is resident, so a tile waiting for another
  // CTA's output never waits for a CTA that has not started.
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(17 * 32), args, (size_t)smem_bytes, st);
}

int queue_max_grid_fn(const void* fn, int smem_bytes, int sms) {
  int occ = 0;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 17 * 32, smem_bytes) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return occ * sms;
}

cudaError_t launch_queue(const QArgs& a, int grid, bool split, cudaStream_t st) {
  return launch_queue_fn(queue_fn(split), QueueSmem::SMEM_BYTES, a, grid, st);
}

int queue_max_grid(int sms, bool split) {
  return queue_max_grid_fn(queue_fn(split), QueueSmem::SMEM_BYTES, sms);
}

}  // namespace mcfft
