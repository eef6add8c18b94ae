// noalloc.cu -- mcfftExec1dNoAlloc: the two-pass (four-step) 1D transform
// without any device allocation.
//
// Who needs it: callers that may not call cudaMalloc at the point where the
// transform runs -- code inside a framework whose caching allocator owns all
// device memory, real-time or embedded hosts that forbid allocation after
// start-up, and code that must not risk the device-wide synchronisation
// cudaMalloc/cudaFree can imply.  Plans (mcfftPlanCreate*) allocate their
// tables and, for 1D lengths above 8192, a scratch buffer for the
// intermediate between the two passes; this entry point instead uses
// file-scope __device__ arrays that every GPU loading the library holds
// until the process exits.
//
// Limits: plain FP16 form only; n a power of two in [2^14, 2^22]; n * batch
// <= kNoAllocMaxPoints (4 Mi complex points, the 16 MiB scratch array).
//
// The first call on a device resolves the arrays' device addresses with
// cudaGetSymbolAddress (with that device current) and creates one event and
// one private stream; make that first call before any stream capture.  Every call shares the
// arrays and leaves its contents behind: two calls that overlap on the GPU
// (different streams, different host threads) race on them.  The scratch
// needs no clearing -- pass 1 writes every element pass 2 reads.  The
// twiddle tables and the DFT-16 matrix depend only on (n, direction): a call
// whose (n, direction) equals the previous call's on that device reuses
// them (the same overlap race covers this record).
//
// Device-side waits are bounded; a pass that gives up records a timeout in
// a file-scope status word.  A call returns MCFFT_DEVICE_TIMEOUT, without
// transforming, when it finds the status word of an earlier call on this
// device set: the word is read back (4 bytes, on the private stream) only
// once that earlier call's work has completed (an event query, so the call
// never waits for it), and cleared.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/mcfft.h"
#include "mcfft_internal.h"

namespace mcfft {
namespace {

constexpr int64_t kNoAllocMaxPoints = int64_t(1) << 22;  // 16 MiB of FP16 complex
constexpr int kMaxTwEntries = 2 * 4096 + 2 * 256;         // stage tables of both passes
constexpr int kMaxTail = 2 * 2048;                          // radix-R tables of both passes
constexpr int kMaxPost = 2048;                              // each half of the four-step table

static __device__ __align__(256) uint32_t g_scratch[kNoAllocMaxPoints];  // FP16 complex
static __device__ __align__(256) float2 g_tw[kMaxTwEntries];
static __device__ __align__(256) float2 g_tail[kMaxTail];
static __device__ __align__(256) float2 g_post_lo[kMaxPost];
static __device__ __align__(256) float2 g_post_hi[kMaxPost];
static __device__ __align__(256) uint4 g_bmat[128];
static __device__ __align__(256) int g_status;

struct DevAddrs {
  bool ready = false;
  void* scratch = nullptr;
  float2 *tw = nullptr, *tail = nullptr, *post_lo = nullptr, *post_hi = nullptr;
  uint4* bmat = nullptr;
  int* status = nullptr;
  cudaEvent_t done = nullptr;  // recorded after each call's passes
  cudaStream_t aux = nullptr;  // status read-back, never waits on the caller's work
  bool pending = false;        // a call's status word has not been checked yet
  int64_t tab_n = 0;           // (n, sign) whose tables are resident; 0: none
  int tab_sign = 0;
};
constexpr int kMaxDevices = 64;
DevAddrs g_addr[kMaxDevices];
std::mutex g_mu;

mcfftResult setup_device(int dev, DevAddrs* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  DevAddrs& d = g_addr[dev];
  if (!d.ready) {
    void* p[7];
    const void* syms[7] = {g_scratch, g_tw, g_tail, g_post_lo, g_post_hi, g_bmat, &g_status};
    for (int i = 0; i < 7; ++i) {
      if (cudaGetSymbolAddress(&p[i], syms[i]) != cudaSuccess) {
        cudaGetLastError();
        return MCFFT_CUDA_ERROR;
      }
    }
    d.scratch = p[0];
    d.tw = static_cast<float2*>(p[1]);
    d.tail = static_cast<float2*>(p[2]);
    d.post_lo = static_cast<float2*>(p[3]);
    d.post_hi = static_cast<float2*>(p[4]);
    d.bmat = static_cast<uint4*>(p[5]);
    d.status = static_cast<int*>(p[6]);
    if (!d.done && cudaEventCreateWithFlags(&d.done, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      d.done = nullptr;
      return MCFFT_CUDA_ERROR;
    }
    if (!d.aux && cudaStreamCreateWithFlags(&d.aux, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      d.aux = nullptr;
      return MCFFT_CUDA_ERROR;
    }
    d.ready = true;
  }
  *out = d;
  return MCFFT_SUCCESS;
}

// Status of the earlier call on this device, if its passes have finished:
// MCFFT_DEVICE_TIMEOUT (and the word cleared) when one of them gave up.
// A call still running is checked by a later call.
mcfftResult check_earlier(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  DevAddrs& d = g_addr[dev];
  if (!d.pending) return MCFFT_SUCCESS;
  const cudaError_t q = cudaEventQuery(d.done);
  if (q == cudaErrorNotReady) {
    cudaGetLastError();
    return MCFFT_SUCCESS;
  }
  if (q != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }
  d.pending = false;
  int h = 0;
  // The earlier call's work is complete and the private stream holds no
  // other work, so neither this copy nor the clearing below waits for
  // anything the caller enqueued.
  if (cudaMemcpyFromSymbolAsync(&h, g_status, sizeof(int), 0, cudaMemcpyDeviceToHost, d.aux) !=
          cudaSuccess ||
      cudaStreamSynchronize(d.aux) != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }
  if (h == kStatusOk) return MCFFT_SUCCESS;
  d.tab_n = 0;  // tables may be incomplete after an aborted call
  if (cudaMemsetAsync(d.status, 0, sizeof(int), d.aux) != cudaSuccess ||
      cudaStreamSynchronize(d.aux) != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }
  return h == kStatusTimeout ? MCFFT_DEVICE_TIMEOUT : MCFFT_INTERNAL_ERROR;
}

int ilog2i(int64_t x) {
  int r = 0;
  while ((int64_t(1) << r) < x) ++r;
  return r;
}

// L = 16^a * R with R = 2^(log2(L) mod 4).
int tail_radix(int L) { return 1 << (ilog2i(L) % 4); }

// Stage and radix-R tables of one pass into the given slots.
cudaError_t pass_tables(int L, int R, float2* tw, float2* tail, int sign, cudaStream_t st) {
  int nst = 0;
  for (int64_t t = L / R; t > 1; t >>= 4) ++nst;
  int64_t off = 0, Ls = L / R;
  for (int s = 0; s < nst - 1; ++s) {
    cudaError_t e = gen_twiddle_table(tw + off, Ls, 0, 16, 0, Ls, sign, 1.0 / 16.0, st);
    if (e != cudaSuccess) return e;
    off += Ls;
    Ls >>= 4;
  }
  if (R > 1) return gen_twiddle_table(tail, L, 0, R, 0, L, sign, 1.0 / R, st);
  return cudaSuccess;
}

}  // namespace
}  // namespace mcfft

using namespace mcfft;

extern "C" MCFFT_API mcfftResult mcfftExec1dNoAlloc(const void* in, void* out, int64_t n,
                                                    int64_t batch, int direction, void* stream) {
  if (!in || !out || batch < 1) return MCFFT_INVALID_VALUE;
  if (direction != MCFFT_FORWARD && direction != MCFFT_INVERSE) return MCFFT_INVALID_VALUE;
  if (n < (int64_t(1) << 14) || n > (int64_t(1) << 22) || (n & (n - 1))) return MCFFT_UNSUPPORTED_SIZE;
  // n * batch <= kNoAllocMaxPoints, written so that the product cannot overflow
  if (batch > kNoAllocMaxPoints / n) return MCFFT_INVALID_VALUE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return MCFFT_NO_DEVICE;
  }
  DevAddrs d;
  mcfftResult r = setup_device(dev, &d);
  if (r != MCFFT_SUCCESS) return r;
  r = check_earlier(dev);
  if (r != MCFFT_SUCCESS) return r;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int sign = direction == MCFFT_FORWARD ? -1 : 1;

  // n = n1 * n2: pass 1 = n1-point column transforms with the four-step
  // twiddle into the scratch array, pass 2 = n2-point rows written with
  // stride n1 (the same decomposition the plan uses).
  const int lg = ilog2i(n), lg1 = lg / 2;
  const int n1 = 1 << lg1, n2 = (int)(n >> lg1);
  const int R1 = tail_radix(n1), R2 = tail_radix(n2);
  const PassKernel* k1 = pick_pass_kernel(n1, true, true, false, n2, 16384);
  const PassKernel* k2 = pick_pass_kernel(n2, false, false, false, n1, 16384);
  if (!k1 || !k2 || k1->R != R1 || k2->R != R2) return MCFFT_UNSUPPORTED_SIZE;

  float2* tw2 = d.tw + 4096 + 256;
  float2* tail2 = d.tail + 2048;
  const int sh = lg / 2;
  bool reuse = false;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    reuse = g_addr[dev].tab_n == n && g_addr[dev].tab_sign == sign;
    g_addr[dev].tab_n = 0;  // set again once this call's tables are enqueued
  }
  cudaError_t e = cudaSuccess;
  if (!reuse) {
    e = gen_dft16_embedding(d.bmat, nullptr, sign, st);
    if (e == cudaSuccess) e = pass_tables(n1, R1, d.tw, d.tail, sign, st);
    if (e == cudaSuccess) e = pass_tables(n2, R2, tw2, tail2, sign, st);
    if (e == cudaSuccess)
      e = gen_twiddle_table(d.post_lo, int64_t(1) << sh, 1, 0, 0, n, sign, 1.0, st);
    if (e == cudaSuccess) e = gen_twiddle_table(d.post_hi, n >> sh, 1, 0, sh, n, sign, 1.0, st);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }

  PassArgs a1{};
  a1.in = in;
  a1.out = d.scratch;
  a1.in_sp = n2; a1.in_sc = 1; a1.in_so = n;
  a1.out_sp = n2; a1.out_sc = 1; a1.out_so = n;
  a1.ncols = n2;
  a1.col_blocks = (n2 + k1->C - 1) / k1->C;
  a1.ntiles = a1.col_blocks * batch;
  a1.tw = d.tw;
  a1.tail_tw = d.tail;
  a1.bmat = d.bmat;
  a1.post_lo = d.post_lo;
  a1.post_hi = d.post_hi;
  a1.post_mask = (uint64_t)n - 1;
  a1.post_shift = (uint32_t)sh;
  a1.inverse = direction == MCFFT_INVERSE;
  a1.out_scale = 1.0f / 16.0f;
  a1.status = d.status;

  PassArgs a2 = a1;
  a2.in = d.scratch;
  a2.out = out;
  a2.in_sp = 1; a2.in_sc = n2; a2.in_so = n;
  a2.out_sp = n1; a2.out_sc = 1; a2.out_so = n;
  a2.ncols = n1;
  a2.col_blocks = (n1 + k2->C - 1) / k2->C;
  a2.ntiles = a2.col_blocks * batch;
  a2.tw = tw2;
  a2.tail_tw = tail2;
  a2.post_lo = nullptr;
  a2.post_hi = nullptr;

  const int g1 = (int)(a1.ntiles < 2 * sms ? a1.ntiles : 2 * sms);
  const int g2 = (int)(a2.ntiles < 2 * sms ? a2.ntiles : 2 * sms);
  e = launch_pass(*k1, a1, g1, st);
  if (e == cudaSuccess) e = launch_pass(*k2, a2, g2, st);
  if (e == cudaSuccess) e = cudaEventRecord(d.done, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return MCFFT_CUDA_ERROR;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g_addr[dev].pending = true;
  g_addr[dev].tab_n = n;
  g_addr[dev].tab_sign = sign;
  return MCFFT_SUCCESS;
}
