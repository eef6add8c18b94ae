/*
 * oracle/fft64.c -- CPU oracle for the batched complex-to-complex FFT.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (mcfft_b200/, include/)
 * links, loads or calls this file; only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / --impl reference legs use it, as the checker.
 *
 * Two things live here:
 *
 *  1. An FP64 FFT written from the DFT definition (iterative Stockham radix-2
 *     with twiddles from long-double sin/cos).  This is the stand-in for the
 *     FFTW double oracle that the reference's accuracy drivers call
 *     (benchmark/accuracy_1d.cpp:12-24, fftw_plan_dft_1d(..., FFTW_FORWARD,
 *     FFTW_ESTIMATE); benchmark/accuracy_2d.cpp:12-24, fftw_plan_dft_2d).
 *     FFTW is not installed in this image; the FFT is pinned against FFTW's
 *     own printed outputs in the reference's dump 2.txt and against rocFFT's
 *     in 3.txt (tests/golden/).
 *
 *  2. A restatement of the reference's own algorithm: the host digit
 *     reversal (source/mcfft_1d_utils.cpp:8-35), the size->schedule table
 *     (source/mcfft_1d_device.cpp:695-775, source/mcfft_2d_device.cpp:659-691),
 *     the DFT-16 matrix stages of every layer kernel
 *     (source/mcfft_1d_device.cpp:58-593, source/mcfft_2d_device.cpp:335-592)
 *     and the executors (source/mcfft_1d_device.cpp:596-678,
 *     source/mcfft_2d_device.cpp:594-622).  It reproduces the reference's
 *     arithmetic: FP64 data, twiddles from single-precision cosf/sinf
 *     advanced by complex multiplication, the same accumulation order of the
 *     16x16 products.  The rocWMMA fragment plumbing is not restated, only
 *     the matrices it multiplies.
 *
 *  3. The reference's input generator (glibc rand scaled by 1e-4 in float,
 *     source/mcfft_1d_utils.cpp:88-100) and its error metric get_error
 *     (benchmark/accuracy_1d.cpp:26-56).
 *
 * Complex data is interleaved double (re, im), batch-major, as the reference
 * lays it out.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

static inline cplx cmul(cplx a, cplx b) {
  cplx t = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return t;
}

/* ------------------------------------------------------------------------ */
/* 1. FP64 FFT                                                              */
/* ------------------------------------------------------------------------ */

/* exp(sign * 2*pi*i * k / n), computed in long double and rounded once. */
static cplx twid(int64_t k, int64_t n, int sign) {
  long double a = 2.0L * 3.141592653589793238462643383279502884L *
                  (long double)(k % n) / (long double)n;
  cplx t = {(double)cosl(a), (double)(sign * sinl(a))};
  return t;
}

/* Stockham autosort radix-2, n a power of two.  x is the input (destroyed),
 * y is scratch; the result ends up in whichever buffer is returned. */
static cplx *stockham(cplx *x, cplx *y, int64_t n, const cplx *w) {
  /* w[j] = exp(sign 2 pi i j / n), j < n/2 */
  for (int64_t l = n / 2, m = 1; l >= 1; l /= 2, m *= 2) {
    for (int64_t j = 0; j < l; ++j) {
      cplx wj = w[j * m];
      for (int64_t k = 0; k < m; ++k) {
        cplx c0 = x[k + j * m], c1 = x[k + j * m + l * m];
        cplx s = {c0.re + c1.re, c0.im + c1.im};
        cplx d = {c0.re - c1.re, c0.im - c1.im};
        y[k + 2 * j * m] = s;
        y[k + 2 * j * m + m] = cmul(wj, d);
      }
    }
    cplx *t = x; x = y; y = t;
  }
  return x;
}

static int is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }

/* Direct O(n^2) DFT in long double, for small n and for checking. */
static void dft_direct(const cplx *in, cplx *out, int64_t n, int sign) {
  const long double tp = 2.0L * 3.141592653589793238462643383279502884L;
  for (int64_t k = 0; k < n; ++k) {
    long double sr = 0, si = 0;
    for (int64_t j = 0; j < n; ++j) {
      long double a = tp * (long double)((j * k) % n) / (long double)n;
      long double c = cosl(a), s = sign * sinl(a);
      sr += in[j].re * c - in[j].im * s;
      si += in[j].re * s + in[j].im * c;
    }
    out[k].re = (double)sr;
    out[k].im = (double)si;
  }
}

/* One 1D transform of length n along a strided line (in place).  Work
 * buffers a, b hold 2n complex. */
static void line_fft(double *data, int64_t n, int64_t stride, int sign,
                     const cplx *w, cplx *a, cplx *b) {
  cplx *d = (cplx *)data;
  for (int64_t i = 0; i < n; ++i) a[i] = d[i * stride];
  cplx *r;
  if (is_pow2(n)) {
    r = stockham(a, b, n, w);
  } else {
    dft_direct(a, b, n, sign);
    r = b;
  }
  for (int64_t i = 0; i < n; ++i) d[i * stride] = r[i];
}

/* In-place multi-dimensional C2C FFT of `batch` row-major arrays with dims
 * dims[0..ndim) (last dimension contiguous).  sign = -1 forward (FFTW_FORWARD),
 * +1 backward (unnormalised, like FFTW_BACKWARD).  Returns 0 on success. */
int oracle_fftnd(double *data, int ndim, const int64_t *dims, int64_t batch,
                 int sign) {
  int64_t total = 1;
  for (int d = 0; d < ndim; ++d) total *= dims[d];
  for (int ax = ndim - 1; ax >= 0; --ax) {
    int64_t n = dims[ax];
    int64_t inner = 1, outer = batch;
    for (int d = ax + 1; d < ndim; ++d) inner *= dims[d];
    for (int d = 0; d < ax; ++d) outer *= dims[d];
    cplx *w = (cplx *)malloc(sizeof(cplx) * (size_t)(n / 2 + 1));
    if (!w) return -1;
    for (int64_t j = 0; j <= n / 2; ++j) w[j] = twid(j, n, sign);
    int64_t lines = outer * inner;
    int fail = 0;
#pragma omp parallel
    {
      cplx *a = (cplx *)malloc(sizeof(cplx) * (size_t)n);
      cplx *b = (cplx *)malloc(sizeof(cplx) * (size_t)n);
      if (!a || !b) {
#pragma omp atomic write
        fail = 1;
      } else {
#pragma omp for schedule(static)
        for (int64_t li = 0; li < lines; ++li) {
          int64_t o = li / inner, i = li % inner;
          line_fft(data + 2 * (o * n * inner + i), n, inner, sign, w, a, b);
        }
      }
      free(a);
      free(b);
    }
    free(w);
    if (fail) return -1;
  }
  (void)total;
  return 0;
}

int oracle_fft1d(double *data, int64_t n, int64_t batch, int sign) {
  return oracle_fftnd(data, 1, &n, batch, sign);
}

int oracle_dft_direct(const double *in, double *out, int64_t n, int sign) {
  dft_direct((const cplx *)in, (cplx *)out, n, sign);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* 3. The reference's input generator and error metric                     */
/* ------------------------------------------------------------------------ */

/* source/mcfft_1d_utils.cpp:88-100: srand(seed); each value is
 * 0.0001f * rand() / RAND_MAX evaluated in single precision, re then im.
 * (The OpenMP pragma there is inert: the makefile never enables OpenMP.) */
void oracle_generate_data(double *data, int64_t n, int64_t n_batch, int seed) {
  srand((unsigned)seed);
  for (int64_t i = 0; i < n_batch; ++i)
    for (int64_t j = 0; j < n; ++j) {
      float re = 0.0001f * (float)rand() / (float)RAND_MAX;
      float im = 0.0001f * (float)rand() / (float)RAND_MAX;
      data[0 + j * 2 + i * n * 2] = re;
      data[1 + j * 2 + i * n * 2] = im;
    }
}

/* benchmark/accuracy_1d.cpp:26-56: mean over elements of
 * min(1, |rel err|) summed over re and im (range 0..2). */
double oracle_get_error(const double *tested, const double *standard, int64_t n,
                        int64_t n_batch) {
  double error = 0;
  for (int64_t i = 0; i < n_batch; ++i)
    for (int64_t j = 0; j < n; ++j) {
      for (int c = 0; c < 2; ++c) {
        double t = tested[c + j * 2 + i * n * 2];
        double s = standard[c + j * 2 + i * n * 2];
        double e = fabs((t - s) / s);
        error += e < 1.0 ? e : 1.0;
      }
    }
  return error / (double)n / (double)n_batch;
}

/* rel-L2 and max-abs/max|ref| error, reduced in long double. */
void oracle_error_norms(const double *y, const double *ref, int64_t count,
                        double *rel_l2, double *max_rel) {
  long double num = 0, den = 0;
  double mx = 0, mref = 0;
  for (int64_t i = 0; i < 2 * count; ++i) {
    double d = y[i] - ref[i];
    num += (long double)d * d;
    den += (long double)ref[i] * ref[i];
    if (fabs(d) > mx) mx = fabs(d);
    if (fabs(ref[i]) > mref) mref = fabs(ref[i]);
  }
  *rel_l2 = den > 0 ? (double)sqrtl(num / den) : (double)sqrtl(num);
  *max_rel = mref > 0 ? mx / mref : mx;
}

/* ------------------------------------------------------------------------ */
/* 2. Restatement of the reference algorithm                                */
/* ------------------------------------------------------------------------ */

/* source/mcfft_1d_utils.cpp:8-35 (gen_rev): mixed-radix digit reversal.
 * Starting from the identity, for radices taken from last to first, every
 * block of now_N elements is regrouped so that element l*radix + k moves to
 * l + k*(now_N/radix). */
void ref_gen_rev(int N, int *rev, const int *radices, int n_radices) {
  int *t0 = (int *)malloc(sizeof(int) * (size_t)N);
  int *t1 = (int *)malloc(sizeof(int) * (size_t)N);
  int now_N = N;
  for (int i = 0; i < N; ++i) t0[i] = i;
  for (int i = n_radices - 1; i >= 0; --i) {
    int r = radices[i];
    for (int j = 0; j < N; j += now_N)
      for (int k = 0; k < r; ++k)
        for (int l = 0; l < now_N / r; ++l)
          t1[j + l + k * (now_N / r)] = t0[j + l * r + k];
    now_N /= r;
    int *t = t0; t0 = t1; t1 = t;
  }
  memcpy(rev, t0, sizeof(int) * (size_t)N);
  free(t0);
  free(t1);
}

/* source/mcfft_1d_device.cpp:695-775: the fixed size table.  radices[9]
 * default to 16, mergings[3] default to 0 (0 = 256-point, 1 = 512-point,
 * 2 = 1024-point pass).  Returns -1 for sizes the reference leaves
 * uninitialised (its `default: break`). */
int ref_plan_1d(int n, int *radices, int *n_radices, int *mergings,
                int *n_mergings) {
  for (int i = 0; i < 9; ++i) radices[i] = 16;
  for (int i = 0; i < 3; ++i) mergings[i] = 0;
  switch (n) {
    case 256: *n_radices = 2; *n_mergings = 1; break;
    case 512: *n_radices = 3; radices[2] = 2; *n_mergings = 1; mergings[0] = 1; break;
    case 1024: *n_radices = 3; radices[2] = 4; *n_mergings = 1; mergings[0] = 2; break;
    case 131072: *n_radices = 5; radices[2] = 2; *n_mergings = 2; mergings[0] = 1; break;
    case 262144:
      *n_radices = 6; radices[2] = 2; radices[5] = 2; *n_mergings = 2;
      mergings[0] = 1; mergings[1] = 1; break;
    case 524288:
      *n_radices = 6; radices[2] = 4; radices[5] = 2; *n_mergings = 2;
      mergings[0] = 2; mergings[1] = 1; break;
    case 16777216: *n_radices = 6; *n_mergings = 3; break;
    case 33554432: *n_radices = 7; radices[2] = 2; *n_mergings = 3; mergings[0] = 1; break;
    case 67108864:
      *n_radices = 8; radices[2] = 2; radices[5] = 2; *n_mergings = 3;
      mergings[0] = 1; mergings[1] = 1; break;
    case 134217728:
      *n_radices = 9; radices[2] = 2; radices[5] = 2; radices[8] = 2;
      *n_mergings = 3; mergings[0] = 1; mergings[1] = 1; mergings[2] = 1; break;
    default: return -1;
  }
  return 0;
}

/* source/mcfft_2d_device.cpp:659-691: per-axis table for Nx, Ny in
 * {256, 512, 1024}.  Returns -1 otherwise, and -2 for Nx = 1024, whose
 * column pass would launch the never-assigned layer_1[2]
 * (source/mcfft_2d_device.cpp:635-639 assign layer_1[0..1] only). */
int ref_plan_2d(int nx, int ny, int *radices_x, int *n_radices_x, int *radices_y,
                int *n_radices_y, int *mergings) {
  radices_x[0] = radices_x[1] = 16; radices_x[2] = 2;
  radices_y[0] = radices_y[1] = 16; radices_y[2] = 2;
  mergings[0] = mergings[1] = 0;
  switch (nx) {
    case 256: *n_radices_x = 2; break;
    case 512: *n_radices_x = 3; mergings[1] = 1; break;
    case 1024: *n_radices_x = 3; radices_x[2] = 4; mergings[1] = 2; break;
    default: return -1;
  }
  switch (ny) {
    case 256: *n_radices_y = 2; break;
    case 512: *n_radices_y = 3; mergings[0] = 1; break;
    case 1024: *n_radices_y = 3; radices_y[2] = 4; mergings[0] = 2; break;
    default: return -1;
  }
  return mergings[1] == 2 ? -2 : 0;
}

/* source/mcfft_1d_device.cpp:32-36 (W_N_K): {cosf(2*M_PI*K*M/N),
 * -sinf(...)}; the angle is formed in double and rounded to float for the
 * single-precision cosf/sinf. */
static cplx W_N_K(long N, long K, long M) {
  double ang = 2 * M_PI * (double)K * (double)M / (double)N;
  cplx t = {(double)cosf((float)ang), (double)(-sinf((float)ang))};
  return t;
}

/* The 16x16 DFT matrix as the reference builds it
 * (source/mcfft_1d_device.cpp:776-785): F[i][j] = cosf(2*pi*i*j/16),
 * -sinf(...), stored as doubles. */
static void dft16_matrix(double Fr[16][16], double Fi[16][16]) {
  for (int i = 0; i < 16; ++i)
    for (int j = 0; j < 16; ++j) {
      Fr[i][j] = cosf((float)(2 * M_PI * i * j / 16));
      Fi[i][j] = -sinf((float)(2 * M_PI * i * j / 16));
    }
}

/* complex_mul (source/mcfft_1d_device.cpp:10-30): out = F * in for one
 * 16-vector, as four real products with the reference's order:
 * re = Fr*xr - Fi*xi computed as -(Fi*xi) + Fr*xr; im = Fr*xi + Fi*xr. */
static void dft16(const double Fr[16][16], const double Fi[16][16], const cplx *x,
                  cplx *y) {
  for (int k = 0; k < 16; ++k) {
    double a = 0, b = 0;
    for (int n = 0; n < 16; ++n) a += Fi[k][n] * x[n].im;
    a = -a;
    for (int n = 0; n < 16; ++n) a += Fr[k][n] * x[n].re;
    for (int n = 0; n < 16; ++n) b += Fr[k][n] * x[n].im;
    for (int n = 0; n < 16; ++n) b += Fi[k][n] * x[n].re;
    y[k].re = a;
    y[k].im = b;
  }
}

/* Twiddle of thread column `col` at row `row` as the reference forms it:
 * start at W(N, col, 4*(row/4)) and advance by W(N, col, 1) once per row of
 * the thread's 4-row slice (raw_row = threadIdx.x/16*4, loop j < 4). */
static cplx thread_twiddle(long N, long col, int row) {
  cplx t = W_N_K(N, col, (row / 4) * 4);
  cplx f = W_N_K(N, col, 1);
  for (int j = 0; j < row % 4; ++j) t = cmul(t, f);
  return t;
}

/* layer_256_0 (source/mcfft_1d_device.cpp:58-137) on one contiguous
 * 256-block holding digit-reversed input: DFT16 of each column
 * x[16c + r] over r, transpose, multiply by W256^(c*r), DFT16 again,
 * store natural order. */
static void ref_block256(cplx *blk, const double Fr[16][16], const double Fi[16][16]) {
  cplx Y[16][16], col[16], out[16];
  for (int c = 0; c < 16; ++c) dft16(Fr, Fi, blk + 16 * c, Y[c]);
  for (int c = 0; c < 16; ++c) {          /* second product: column c    */
    for (int r = 0; r < 16; ++r)           /* row r of the new B matrix   */
      col[r] = cmul(Y[r][c], thread_twiddle(256, c, r));
    dft16(Fr, Fi, col, out);
    for (int k = 0; k < 16; ++k) blk[k * 16 + c] = out[k];
  }
}

static void ref_layer_256_0(cplx *d, long total, const double Fr[16][16],
                            const double Fi[16][16]) {
  for (long b = 0; b < total; b += 256) ref_block256(d + b, Fr, Fi);
}

/* layer_512_0 (source/mcfft_1d_device.cpp:139-229): two 256-blocks, then
 * a radix-2 epilogue with W512^e (e < 256) from W_N_K directly. */
static void ref_layer_512_0(cplx *d, long total, const double Fr[16][16],
                            const double Fi[16][16]) {
  for (long b = 0; b < total; b += 512) {
    ref_block256(d + b, Fr, Fi);
    ref_block256(d + b + 256, Fr, Fi);
    for (int e = 0; e < 256; ++e) {
      cplx a0 = d[b + e], a1 = cmul(d[b + e + 256], W_N_K(512, e, 1));
      d[b + e].re = a0.re + a1.re; d[b + e].im = a0.im + a1.im;
      d[b + e + 256].re = a0.re - a1.re; d[b + e + 256].im = a0.im - a1.im;
    }
  }
}

/* layer_1024_0 (source/mcfft_1d_device.cpp:231-333): four 256-blocks, then
 * radix-4 with W1024^e, its square and cube (by complex multiplication). */
static void ref_layer_1024_0(cplx *d, long total, const double Fr[16][16],
                             const double Fi[16][16]) {
  for (long b = 0; b < total; b += 1024) {
    for (int q = 0; q < 4; ++q) ref_block256(d + b + 256 * q, Fr, Fi);
    for (int e = 0; e < 256; ++e) {
      cplx t1 = W_N_K(1024, e, 1), t2 = cmul(t1, t1), t3 = cmul(t2, t1);
      cplx a0 = d[b + e], a1 = cmul(d[b + e + 256], t1);
      cplx a2 = cmul(d[b + e + 512], t2), a3 = cmul(d[b + e + 768], t3);
      cplx o0 = {a0.re + a1.re + a2.re + a3.re, a0.im + a1.im + a2.im + a3.im};
      cplx o1 = {a0.re + a1.im - a2.re - a3.im, a0.im - a1.re - a2.im + a3.re};
      cplx o2 = {a0.re - a1.re + a2.re - a3.re, a0.im - a1.im + a2.im - a3.im};
      cplx o3 = {a0.re - a1.im - a2.re + a3.im, a0.im + a1.re - a2.im - a3.re};
      d[b + e] = o0; d[b + e + 256] = o1; d[b + e + 512] = o2; d[b + e + 768] = o3;
    }
  }
}

/* layer_256_1 / layer_512_1 strided passes (source/mcfft_1d_device.cpp:
 * 335-593; 2D variant source/mcfft_2d_device.cpp:335-592).  For every
 * column g (0 <= g < step) of every (radix*step)-block, rows R = 16a + b at
 * stride `step`:
 *   stage 1: Y[16a + k1] = sum_b F[k1][b] * W(16 step, g, b) * Z[16a + b]
 *   stage 2: X[16k2 + k1] = sum_a F[k2][a] * W(256 step, g + step*k1, a)
 *                                           * Y[16a + k1]
 * The 2D file drops the stage-1 twiddle and uses W(256, k1, a) in stage 2.
 * layer_512_1 runs this on rows 0..255 and 256..511, then a radix-2 step
 * (see ref_layer_1 for where the restatement follows the intended math
 * rather than the reference's indexing). */
static void ref_strided256(cplx *d, long base, long step, long g, int twod,
                           const double Fr[16][16], const double Fi[16][16]) {
  cplx v[16], o[16], Y[256];
  for (int a = 0; a < 16; ++a) {
    for (int b = 0; b < 16; ++b) {
      cplx z = d[base + (long)(16 * a + b) * step + g];
      v[b] = twod ? z : cmul(z, thread_twiddle(16 * step, g, b));
    }
    dft16(Fr, Fi, v, o);
    for (int k1 = 0; k1 < 16; ++k1) Y[16 * a + k1] = o[k1];
  }
  for (int k1 = 0; k1 < 16; ++k1) {
    for (int a = 0; a < 16; ++a) {
      cplx tw = twod ? thread_twiddle(256, k1, a)
                     : thread_twiddle(256 * step, g + step * k1, a);
      v[a] = cmul(Y[16 * a + k1], tw);
    }
    dft16(Fr, Fi, v, o);
    for (int k2 = 0; k2 < 16; ++k2) d[base + (long)(16 * k2 + k1) * step + g] = o[k2];
  }
}

static void ref_layer_1(cplx *d, long total, long step, int merging, int twod,
                        const double Fr[16][16], const double Fi[16][16]) {
  long radix = merging == 0 ? 256 : 512;
  for (long blk = 0; blk < total; blk += radix * step) {
    for (long g = 0; g < step; ++g) {
      ref_strided256(d, blk, step, g, twod, Fr, Fi);
      if (radix == 512) ref_strided256(d, blk + 256 * step, step, g, twod, Fr, Fi);
    }
    if (radix == 512) {
      /* Radix-2 epilogue (source/mcfft_1d_device.cpp:575-592): row R < 256
       * pairs with R + 256 under the twiddle W(512 step, g + step*R).
       * Restated as intended, not as written: the reference advances the
       * twiddle by W(512 step, 16 step) per loop trip while its row advances
       * by 64 (:582, :591), and its second sub-stage addresses rows
       * 272..527 for the upper half (:529-530, warp_start includes both
       * i*NUM_WARP*16 and i*256*CONT_SIZE), past its 8192-element LDS tile.
       * The 2D copy (source/mcfft_2d_device.cpp:576-591) keeps the 1D
       * twiddle W(512 step, ...) for a separable column pass; the intended
       * column twiddle is W(512, R). */
      for (long g = 0; g < step; ++g)
        for (long R = 0; R < 256; ++R) {
          cplx tf = twod ? W_N_K(512, R, 1) : W_N_K(512 * step, g + step * R, 1);
          long p0 = blk + R * step + g, p1 = blk + (R + 256) * step + g;
          cplx a0 = d[p0], a1 = cmul(d[p1], tf);
          d[p0].re = a0.re + a1.re; d[p0].im = a0.im + a1.im;
          d[p1].re = a0.re - a1.re; d[p1].im = a0.im - a1.im;
        }
    }
  }
}

/* mcfftExec 1D (source/mcfft_1d_device.cpp:596-678) on digit-reversed
 * input, in place: layer_0[mergings[0]], then layer_1[mergings[i]] with
 * step growing by each pass's radix. */
int ref_exec_1d(double *data, int n, int n_batch) {
  int radices[9], n_radices, mergings[3], n_mergings;
  if (ref_plan_1d(n, radices, &n_radices, mergings, &n_mergings)) return -1;
  double Fr[16][16], Fi[16][16];
  dft16_matrix(Fr, Fi);
  cplx *d = (cplx *)data;
  long total = (long)n * n_batch;
  static const long rad[3] = {256, 512, 1024};
  if (mergings[0] == 0) ref_layer_256_0(d, total, Fr, Fi);
  else if (mergings[0] == 1) ref_layer_512_0(d, total, Fr, Fi);
  else ref_layer_1024_0(d, total, Fr, Fi);
  long step = rad[mergings[0]];
  for (int i = 1; i < n_mergings; ++i) {
    if (mergings[i] == 2) return -3; /* layer_1[2] is never assigned */
    ref_layer_1(d, total, step, mergings[i], 0, Fr, Fi);
    step *= rad[mergings[i]];
  }
  return 0;
}

/* The harness path: setup's permuted scatter (source/mcfft_1d_utils.cpp:
 * 37-66) + exec + finalize's copy.  `in` natural order, `out` natural. */
int ref_transform_1d(const double *in, double *out, int n, int n_batch) {
  int radices[9], n_radices, mergings[3], n_mergings;
  if (ref_plan_1d(n, radices, &n_radices, mergings, &n_mergings)) return -1;
  int *rev = (int *)malloc(sizeof(int) * (size_t)n);
  ref_gen_rev(n, rev, radices, n_radices);
  for (long j = 0; j < n_batch; ++j)
    for (long i = 0; i < n; ++i) {
      out[2 * n * j + 2 * i] = in[2 * n * j + 2 * (long)rev[i]];
      out[2 * n * j + 2 * i + 1] = in[2 * n * j + 2 * (long)rev[i] + 1];
    }
  free(rev);
  return ref_exec_1d(out, n, n_batch);
}

/* 2D (source/mcfft_2d_utils.cpp:33-61 + source/mcfft_2d_device.cpp:594-622):
 * per-axis digit reversal, row pass layer_0[m0] over rows of length Ny, then
 * column pass layer_1[m1] with step = Ny. */
int ref_transform_2d(const double *in, double *out, int nx, int ny, int n_batch) {
  int rx[3], nrx, ry[3], nry, mergings[2];
  int st = ref_plan_2d(nx, ny, rx, &nrx, ry, &nry, mergings);
  if (st) return st;
  int *rev_x = (int *)malloc(sizeof(int) * (size_t)nx);
  int *rev_y = (int *)malloc(sizeof(int) * (size_t)ny);
  ref_gen_rev(nx, rev_x, rx, nrx);
  ref_gen_rev(ny, rev_y, ry, nry);
  for (long i = 0; i < n_batch; ++i)
    for (long j = 0; j < nx; ++j)
      for (long k = 0; k < ny; ++k) {
        long dst = i * nx * ny + j * ny + k;
        long src = i * nx * ny + (long)rev_x[j] * ny + rev_y[k];
        out[2 * dst] = in[2 * src];
        out[2 * dst + 1] = in[2 * src + 1];
      }
  free(rev_x);
  free(rev_y);
  double Fr[16][16], Fi[16][16];
  dft16_matrix(Fr, Fi);
  cplx *d = (cplx *)out;
  long total = (long)nx * ny * n_batch;
  if (mergings[0] == 0) ref_layer_256_0(d, total, Fr, Fi);
  else if (mergings[0] == 1) ref_layer_512_0(d, total, Fr, Fi);
  else ref_layer_1024_0(d, total, Fr, Fi);
  ref_layer_1(d, total, ny, mergings[1], 1, Fr, Fi);
  return 0;
}
