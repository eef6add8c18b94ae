/*
 * mcfft.h -- C ABI of the B200 (sm_100a) batched complex-to-complex
 * tensor-core FFT.
 *
 * This is the drop-in boundary.  The reference exports only C++-linkage
 * entry points with no status returns and one global plan per process:
 *   mcfftCreate(mcfftHandle*, int n, int n_batch)        include/mcfft_1d_device.h:38
 *   mcfftCreate(mcfftHandle*, int nx, int ny, int n_batch) include/mcfft_2d_device.h:38
 *   mcfftExec(mcfftHandle, MCTYPE* data)                 include/mcfft_1d_device.h:37
 *   setup / doit / finalize / generate_data              include/mcfft_1d_utils.h:8-11
 * Those keep their signatures in include/mcfft_{1d,2d,3d}_utils.h (compat
 * shims over this ABI).  The functions below are the plan-based core every
 * binding (C, C++, ctypes, cgo, JNI) calls: plain pointers and integers,
 * status codes, no CUDA or framework types in the signatures (the stream is
 * a cudaStream_t passed as void*).
 *
 * Data layout: interleaved complex (re, im), batch-major, row-major
 * multi-dimensional arrays with the last dimension contiguous -- the
 * reference's layout (source/mcfft_2d_utils.cpp:49-50).  Input and output
 * are natural order (the reference required digit-reversed input,
 * source/mcfft_1d_utils.cpp:43-59).
 *
 * Precision forms:
 *   MCFFT_PREC_FP16   plain: FP16 in, FP16 out, FP32 accumulation, each
 *                     radix-16 stage scaled by 1/16 (radix-R tail by 1/R),
 *                     so out = DFT(in) * 2^scale_log2 with scale_log2 =
 *                     -log2(number of points of one transform).
 *   MCFFT_PREC_SPLIT  split hi+lo FP16 operands, three products per stage,
 *                     FP32 accumulation: FP32 in (or FP16 in with
 *                     MCFFT_FLAG_INPUT_F16), FP32 out, unnormalised DFT
 *                     (scale_log2 = 0), like FFTW_FORWARD/FFTW_BACKWARD.
 *
 * Sizes: every dimension a power of two >= 16; 1D lengths up to 2^27 (one
 * pass up to 8192, split form 4096; past that a four-step pair of passes,
 * or three passes from 2^24 points (split form 2^23) and for 2^27, the
 * decomposition tuned at plan time); 2D/3D sides up to 8192 (one pass per
 * axis).
 */
#ifndef MCFFT_H_
#define MCFFT_H_

#include <stdint.h>

#if defined(__GNUC__)
#define MCFFT_API __attribute__((visibility("default")))
#else
#define MCFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MCFFT_SUCCESS = 0,
  MCFFT_INVALID_PLAN = 1,
  MCFFT_ALLOC_FAILED = 2,
  MCFFT_INVALID_VALUE = 3,
  MCFFT_UNSUPPORTED_SIZE = 4,
  MCFFT_CUDA_ERROR = 5,
  MCFFT_DEVICE_TIMEOUT = 6,
  MCFFT_INTERNAL_ERROR = 7,
  MCFFT_NO_DEVICE = 8
} mcfftResult;

typedef enum { MCFFT_PREC_FP16 = 0, MCFFT_PREC_SPLIT = 1 } mcfftPrecision;

#define MCFFT_FORWARD (-1)
#define MCFFT_INVERSE (1)

/* Plan flags. */
#define MCFFT_FLAG_NONE 0u
/* Split form only: the input is FP16 complex instead of FP32. */
#define MCFFT_FLAG_INPUT_F16 1u

typedef struct mcfftPlan_st* mcfftPlan;

/* One transform description for mcfftPlanCreateBatch. */
typedef struct {
  int ndim;          /* 1, 2 or 3 */
  int64_t dims[3];   /* dims[0..ndim), last contiguous */
  int64_t batch;     /* transforms of this shape */
  int64_t in_offset; /* element offset of the first one in the input */
  int64_t out_offset;/* element offset of the first one in the output */
} mcfftDesc;

/* Plan information. */
typedef struct {
  int ndim;
  int64_t dims[3];
  int64_t batch;
  int precision;
  int num_passes;          /* HBM passes per exec (kernel launches unless fused) */
  int scale_log2;          /* out = DFT(in) * 2^scale_log2 */
  int64_t elements;        /* complex elements per exec (all transforms) */
  int64_t in_bytes;        /* bytes read from the input per exec */
  int64_t out_bytes;       /* bytes written to the output per exec */
  int64_t workspace_bytes; /* device scratch held by the plan */
  int num_descs;           /* transform groups (mcfftPlanCreateBatch) */
  int launches;            /* this library's kernel launches per exec (1: batch queue) */
  int timed_passes;        /* passes the plan-time tuner timed (0: all from wisdom or untuned) */
  /* Added in 0.2.0 (the struct grew at its end). */
  int64_t fourstep_n1;     /* first group, 1D past one pass: the chosen n1 of n = n1 * n2
                              (three passes, num_passes 3: of n = n1 * n2 * n3); else 0 */
  int tile_points;         /* points per tile of the first pass (0: direct-load kernel) */
  int ctas;                /* CTAs of the first launch */
} mcfftPlanInfo;

MCFFT_API mcfftResult mcfftPlanCreate1d(mcfftPlan* plan, int64_t n, int64_t batch,
                              mcfftPrecision precision, unsigned flags);
MCFFT_API mcfftResult mcfftPlanCreate2d(mcfftPlan* plan, int64_t nx, int64_t ny, int64_t batch,
                              mcfftPrecision precision, unsigned flags);
MCFFT_API mcfftResult mcfftPlanCreate3d(mcfftPlan* plan, int64_t nx, int64_t ny, int64_t nz,
                              int64_t batch, mcfftPrecision precision, unsigned flags);
/* Many transforms of uneven size/dimensionality executed together. */
MCFFT_API mcfftResult mcfftPlanCreateBatch(mcfftPlan* plan, const mcfftDesc* descs, int count,
                                 mcfftPrecision precision, unsigned flags);

/* Stream-ordered; `in` and `out` are device pointers (may be equal for
 * single-pass plans).  direction: MCFFT_FORWARD or MCFFT_INVERSE.  One plan
 * must not run concurrently on two streams (its workspace is shared).
 * The second exec on the same (in, out, direction) captures the plan's
 * launches into a CUDA graph that later execs replay (up to four such
 * graphs per plan; MCFFT_GRAPH=0 in the environment disables this). */
MCFFT_API mcfftResult mcfftExec(mcfftPlan plan, const void* in, void* out, int direction,
                      void* stream);

/* Host-buffer exec: copies `host_in` to the device, transforms it and copies
 * the result to `host_out`, ordered on `stream` (the three steps the
 * reference's harness runs one after another in setup / doit / finalize,
 * source/mcfft_1d_utils.cpp; no single-call counterpart in the reference).
 * A single-shape plan (one descriptor, zero offsets) is cut into chunks of
 * whole transforms (1, 2, 4, .. transforms rising to the largest power of
 * two within 32 MiB of input -- MCFFT_HOST_CHUNK_BYTES in the environment
 * overrides -- and falling again at the end), and the copy in of one chunk,
 * the transforms of earlier ones and their copies out run at the same time;
 * the copies overlap only for page-locked host buffers (cudaHostAlloc /
 * cudaHostRegister).  The first call creates a plan per chunk length and a
 * ring of up to four device buffers per side, held until the plan is
 * destroyed (it synchronises the device: make it before any stream
 * capture).  The host buffers must stay valid until `stream` passes the
 * call and must be disjoint, or identical when input and output elements
 * have the same size.  Layout and scale as mcfftExec. */
MCFFT_API mcfftResult mcfftExecHost(mcfftPlan plan, const void* host_in, void* host_out,
                                    int direction, void* stream);

/* Reads back and clears the plan's device status word (synchronises the
 * plan's last stream).  MCFFT_DEVICE_TIMEOUT if a kernel gave up waiting. */
MCFFT_API mcfftResult mcfftPlanCheckStatus(mcfftPlan plan);

MCFFT_API mcfftResult mcfftPlanGetInfo(mcfftPlan plan, mcfftPlanInfo* info);
MCFFT_API mcfftResult mcfftPlanDestroy(mcfftPlan plan);
MCFFT_API const char* mcfftGetErrorString(mcfftResult result);

/* Two-pass (four-step) 1D transform that allocates nothing.  No counterpart
 * in the reference.  For callers that must not call cudaMalloc where the
 * transform runs (a framework's caching allocator owns device memory, hosts
 * that forbid allocation after start-up, code that cannot afford the
 * synchronisation an allocation may imply): no plan is created and the
 * intermediate between the two passes, the twiddle tables and the DFT-16
 * matrix live in fixed __device__ arrays the library holds on every GPU
 * until exit.  Plain FP16 form (as mcfftExec with MCFFT_PREC_FP16: out =
 * DFT(in) / n), natural order, `in` and `out` distinct device buffers of
 * n * batch FP16 complex values.  Limits: n a power of two in
 * [2^14, 2^22], n * batch <= 2^22 (16 MiB scratch); larger sizes return
 * MCFFT_UNSUPPORTED_SIZE or MCFFT_INVALID_VALUE.  The first call on a device
 * looks up the arrays' device addresses (and creates one event and one
 * stream) and should come before any stream capture.  All calls share the
 * arrays: calls that overlap on the GPU race.  The tables are regenerated
 * only when (n, direction) differs from the previous call's on the device.
 * A device-side wait that ran out in an earlier call is reported by a later
 * call, once the earlier one has completed, as MCFFT_DEVICE_TIMEOUT (that
 * call does not transform; the condition is then cleared). */
MCFFT_API mcfftResult mcfftExec1dNoAlloc(const void* in, void* out, int64_t n, int64_t batch,
                                         int direction, void* stream);

/* Error norms of a result against an FP64 reference, reduced in FP64 on
 * the GPU.  Replaces the host-side error reduction of the reference's
 * accuracy harness (get_error, benchmark/accuracy_1d.cpp:26-56, and
 * benchmark/accuracy_2d.cpp:26-56), which walks the whole result on the
 * CPU.  `y`: device, complex FP16 (y_f16 = 1) or FP32 (y_f16 = 0)
 * interleaved; `ref`: device, complex FP64 interleaved, same element count.
 * The elements are cut into `nseg` segments [seg_off[i], seg_off[i + 1])
 * (host array of nseg + 1 offsets, e.g. one per transform); y of segment i
 * is scaled by 2^seg_scale_log2[i] first (host array, or NULL for no
 * scaling; the plain form's output carries 2^scale_log2, so pass
 * -scale_log2 to compare it with the unscaled DFT).  out (host,
 * 5 * nseg doubles), per segment: sum |y - ref|^2, sum |ref|^2,
 * max |y - ref| and max |ref| (over real and imaginary parts separately),
 * and the reference harness's sum over real and
 * imaginary components of min(1, |(y - ref) / ref|) (divide by the number
 * of complex elements for its get_error value).  Allocates a small device
 * block for its tables and synchronises `stream` before returning. */
MCFFT_API mcfftResult mcfftErrorNorms(const void* y, int y_f16, const void* ref, int nseg,
                                      const int64_t* seg_off, const int* seg_scale_log2,
                                      double* out, void* stream);

/* Autotuning records ("wisdom"; the reference has no tuner and no such
 * file).  Creating a plain-form plan times each pass's two tile shapes once
 * and records the faster per GPU model and pass; a 1D plan past one pass
 * also times its decompositions (four-step splits n1 * n2 and, from 2^21
 * points, three passes) and records the fastest; later plans in the process
 * reuse the record instead of timing.  Export writes this process's records
 * to a text file, Import reads such a file (adding to and replacing records;
 * a malformed file changes nothing and returns MCFFT_INVALID_VALUE), Forget
 * drops every record.  Records of another GPU model are kept but unused. */
MCFFT_API mcfftResult mcfftWisdomExport(const char* path);
MCFFT_API mcfftResult mcfftWisdomImport(const char* path);
MCFFT_API mcfftResult mcfftWisdomForget(void);

/* Library version as 10000*major + 100*minor + patch. */
MCFFT_API int mcfftGetVersion(void);

#ifdef __cplusplus
}
#endif

#endif /* MCFFT_H_ */
