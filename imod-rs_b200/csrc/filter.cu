// filter.cu -- log transform, per-view means and the fused filter stage:
// R-weighting (batched complex FFT of two packed real rows x radial weight x
// inverse FFT), cosine stretch and packing into the staging format that the
// back-projectors copy into shared memory.
//
// Reference semantics: apps/tilt/src/main.rs:333-381 (apply_rweighting),
// 446-488 (apply_cosine_stretch, 411-441 cubic), 608-623 (log, means),
// crates/imod-math/src/stats.rs:844-861 (min_max_mean).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <math.h>

#include <mutex>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "tg_internal.h"
#include "fft.cuh"
#include "f32x2.cuh"

namespace tg {

// ---------------------------------------------------------------------------
// log10 (main.rs:608-613) fused with the per-view f64 sums (main.rs:616-623).
// The uploaded projections are read, never modified: with --log the log'd
// values go to a second buffer, so every reconstruction repeats the whole
// path.  Grid (CH, nviews); every block owns a contiguous chunk of one view
// (16-byte loads and stores between a scalar head and tail) and writes one f64
// partial; a second kernel adds the CH partials in order, so the result does
// not depend on scheduling.  HBM-bound: 4 B read (+ 4 B written with --log)
// per sample.
// ---------------------------------------------------------------------------
constexpr int MEAN_CH = 32;

// f32::max(0.001).log10(): computed in FP64 then rounded once
__device__ __forceinline__ float log_sample(float x) { return (float)log10((double)fmaxf(x, 0.001f)); }

// The same value, (float)log10((double)max(x, 0.001)), mostly without the
// double-precision library call.  With x = 2^e * m, m in [0.75, 1.5), and
// c_j the nearest of 257 table centres (bit patterns 2^15 apart from 0.75, so
// c_128 = 1) with inv_j = 1/c_j rounded to float:
//   ln x = e*ln2 - ln(inv_j) + log1p(r),  r = m*inv_j - 1,
// r exact in double (a product of two floats minus 1) and |r| < 2^-9, log1p(r)
// by its Taylor series through r^5 (truncation below 2^-47 relative; no
// cancellation: the centre c_128 = 1 takes the samples near 1).  The result z is
// within 2^-44 relative of log10 x (a CPU check of this evaluation over 2.5e7
// samples against the FP64 log10 found at most 2^-47.6), so z rounded to float
// is the correctly rounded log unless z lies within 2^-40 |z| of a midpoint
// between floats; those samples (about 2 in 10^5) and infinite x take
// log_sample (x = 1 gives z = 0 exactly, the true value).  The table (shared memory) holds inv_j (a float value) and
// -ln inv_j as doubles, in separate arrays.  The rounding test: z*(1 - 2^-40) and
// z*(1 + 2^-40) round to the same float exactly when no midpoint between floats
// lies between them, and the true value lies strictly inside that interval.
struct LogTable {
  double inv[257];
  double nl[257];
};
// The evaluation without a branch: the rounded value and whether it is decided
// (ok false: take log_sample), so that several samples' FP64 chains interleave.
__device__ __forceinline__ float log_fast_core(float x, const LogTable &lt, bool &ok) {
  x = fmaxf(x, 0.001f);
  const int ix = __float_as_int(x);
  const int e = (ix - 0x3f400000) >> 23;
  const int mb = ix - (e << 23);
  const int j = (mb - 0x3f400000 + 0x4000) >> 15;
  const double r = __fma_rn((double)__int_as_float(mb), lt.inv[j], -1.0);
  double p = __fma_rn(r, 0.2, -0.25);
  p = __fma_rn(r, p, 1.0 / 3.0);
  p = __fma_rn(r, p, -0.5);
  p = __fma_rn(r, p, 1.0);
  const double z = __dmul_rn(__dadd_rn(__fma_rn((double)e, 0.693147180559945309417232121458176568, lt.nl[j]),
                                       __dmul_rn(r, p)),
                             0.434294481903251827651128918916605082);  // ln 2, log10 e
  const float lo = __double2float_rn(__dmul_rn(z, 1.0 - 0x1p-40)), hi = __double2float_rn(__dmul_rn(z, 1.0 + 0x1p-40));
  ok = lo == hi && ix < 0x7f800000;
  return lo;
}
__device__ __forceinline__ float log_sample_fast(float x, const LogTable &lt) {
  bool ok;
  const float f = log_fast_core(x, lt, ok);
  return ok ? f : log_sample(x);
}

// the 257 centres' (inv_j, -ln inv_j) of log_sample_fast
__device__ __forceinline__ void log_table(LogTable &lt) {
  for (int i = threadIdx.x; i < 257; i += blockDim.x) {
    const float inv = __frcp_rn(__int_as_float(0x3f400000 + (i << 15)));
    lt.inv[i] = (double)inv;
    lt.nl[i] = -log((double)inv);
  }
  __syncthreads();
}

// four samples: the four evaluations first (independent FP64 chains), the rare
// undecided ones after
template <bool LOG> __device__ __forceinline__ float4 log4(float4 x, const LogTable &lt) {
  if (!LOG) return x;
  bool k0, k1, k2, k3;
  float4 r = make_float4(log_fast_core(x.x, lt, k0), log_fast_core(x.y, lt, k1), log_fast_core(x.z, lt, k2),
                         log_fast_core(x.w, lt, k3));
  if (!(k0 && k1 && k2 && k3)) {
    if (!k0) r.x = log_sample(x.x);
    if (!k1) r.y = log_sample(x.y);
    if (!k2) r.z = log_sample(x.z);
    if (!k3) r.w = log_sample(x.w);
  }
  return r;
}

template <bool LOG>
__global__ void __launch_bounds__(256) log_sum_kernel(const float *__restrict__ raw, float *__restrict__ logd,
                                                      long npix, double *partials) {
  const int v = blockIdx.y, c = blockIdx.x;
  __shared__ LogTable lt;
  if (LOG) log_table(lt);
  const size_t base = (size_t)v * npix;
  const long c0 = npix * c / MEAN_CH, c1 = npix * (c + 1) / MEAN_CH;
  // [c0, a0): scalar head up to a 16-byte boundary; [a0, a1): float4; [a1, c1): tail
  long a0 = c0 + (long)((4 - ((base + c0) & 3)) & 3);
  if (a0 > c1) a0 = c1;
  const long a1 = a0 + ((c1 - a0) & ~3L);
  double s = 0.0;
  for (long i = c0 + threadIdx.x; i < a0; i += blockDim.x) {
    float x = raw[base + i];
    if (LOG) logd[base + i] = x = log_sample_fast(x, lt);
    s += (double)x;
  }
  const float4 *r4 = reinterpret_cast<const float4 *>(raw + base + a0);
  float4 *l4 = LOG ? reinterpret_cast<float4 *>(logd + base + a0) : nullptr;
  const long n4 = (a1 - a0) / 4;
  long i = threadIdx.x;
  // two 16-byte loads in flight per thread (the loop is latency-bound on HBM otherwise)
  for (; i + (long)blockDim.x < n4; i += 2L * blockDim.x) {
    const float4 u = __ldcs(r4 + i), w = __ldcs(r4 + i + blockDim.x);
    const float4 x = log4<LOG>(u, lt), y = log4<LOG>(w, lt);
    if (LOG) {
      l4[i] = x;
      l4[i + blockDim.x] = y;
    }
    s += ((double)x.x + (double)x.y) + ((double)x.z + (double)x.w);
    s += ((double)y.x + (double)y.y) + ((double)y.z + (double)y.w);
  }
  if (i < n4) {
    const float4 x = log4<LOG>(__ldcs(r4 + i), lt);
    if (LOG) l4[i] = x;
    s += ((double)x.x + (double)x.y) + ((double)x.z + (double)x.w);
  }
  for (long k = a1 + threadIdx.x; k < c1; k += blockDim.x) {
    float x = raw[base + k];
    if (LOG) logd[base + k] = x = log_sample_fast(x, lt);
    s += (double)x;
  }
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    partials[(size_t)v * MEAN_CH + c] = t;
  }
}

__global__ void means_final_kernel(const double *partials, long npix, int nviews, float *means) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nviews) return;
  double t = 0.0;
  for (int c = 0; c < MEAN_CH; ++c) t += partials[(size_t)v * MEAN_CH + c];
  means[v] = (float)(t / (double)npix);
}

__global__ void view_sums_kernel(const double *partials, int nviews, double *sums) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nviews) return;
  double t = 0.0;
  for (int c = 0; c < MEAN_CH; ++c) t += partials[(size_t)v * MEAN_CH + c];
  sums[v] = t;
}

void launch_log_means(const float *raw, float *logd, int npix, int nviews, double *partials,
                      float *means, cudaStream_t st) {
  if (logd) log_sum_kernel<true><<<dim3(MEAN_CH, nviews), 256, 0, st>>>(raw, logd, npix, partials);
  else log_sum_kernel<false><<<dim3(MEAN_CH, nviews), 256, 0, st>>>(raw, nullptr, npix, partials);
  if (means) means_final_kernel<<<(nviews + 127) / 128, 128, 0, st>>>(partials, npix, nviews, means);
}

void launch_view_sums(const double *partials, int nviews, double *sums, cudaStream_t st) {
  view_sums_kernel<<<(nviews + 127) / 128, 128, 0, st>>>(partials, nviews, sums);
}

// ---------------------------------------------------------------------------
// FFT plan: radices 4, 2, 3, 5, 7 (Stockham, auto-sorting).
// ---------------------------------------------------------------------------
bool fft_plan(int n, FftPlanDev *p) {
  p->n = n;
  p->nfac = 0;
  int m = n;
  while (m % 4 == 0) { p->fac[p->nfac++] = 4; m /= 4; }
  while (m % 2 == 0) { p->fac[p->nfac++] = 2; m /= 2; }
  for (int r : {3, 5, 7})
    while (m % r == 0) { p->fac[p->nfac++] = r; m /= r; }
  return m == 1 && p->nfac <= 24;
}

// apps/tilt/src/main.rs:411-420 (Catmull-Rom), f32 operation order kept
__device__ __forceinline__ float cubic1d(float p0, float p1, float p2, float p3, float t) {
  float t2 = __fmul_rn(t, t);
  float t3 = __fmul_rn(t2, t);
  float a = __fadd_rn(__fsub_rn(__fadd_rn(__fmul_rn(-0.5f, p0), __fmul_rn(1.5f, p1)), __fmul_rn(1.5f, p2)), __fmul_rn(0.5f, p3));
  float b = __fsub_rn(__fadd_rn(__fsub_rn(p0, __fmul_rn(2.5f, p1)), __fmul_rn(2.0f, p2)), __fmul_rn(0.5f, p3));
  float c = __fadd_rn(__fmul_rn(-0.5f, p0), __fmul_rn(0.5f, p2));
  return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(a, t3), __fmul_rn(b, t2)), __fmul_rn(c, t)), p1);
}

// Stretched sample at output column ox (main.rs:469-484, 425-441), zero outside.
__device__ __forceinline__ float stretch_sample(const float *row, int nx, int ox, float stretch,
                                                float center, int cubic) {
  float dx = __fsub_rn((float)ox, center);
  float src_x = __fadd_rn(__fmul_rn(dx, stretch), center);
  float fl = floorf(src_x);
  int sx0 = (int)fl;
  if (fl < -1.0e9f) sx0 = -1000000000;  // far out of range: keep the int conversion safe
  float frac = __fsub_rn(src_x, fl);
  if (cubic && sx0 >= 1 && sx0 + 2 < nx) {
    return cubic1d(row[sx0 - 1], row[sx0], row[sx0 + 1], row[sx0 + 2], frac);
  }
  if (sx0 >= 0 && sx0 + 1 < nx)
    return __fadd_rn(__fmul_rn(row[sx0], __fsub_rn(1.0f, frac)), __fmul_rn(row[sx0 + 1], frac));
  if (sx0 >= 0 && sx0 < nx) return row[sx0];
  return 0.0f;
}

template <int STORE> struct Pack;
template <> struct Pack<TG_STORE_FP16> {
  static __device__ __forceinline__ uint32_t h2(float lo, float hi) {
    __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
  }
};
template <> struct Pack<TG_STORE_BF16> {
  static __device__ __forceinline__ uint32_t h2(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
  }
};

// FP16 staging holds |v| < 65520 (larger values round to infinity).  Every packed
// value's magnitude is tracked; a row that does not fit sets bit 2 of the
// session's error word, which the host reports as TG_ERR_RANGE (a diverging SIRT
// run whose residuals outgrow FP16; FP32 and BF16 staging have the f32 range).
constexpr float FP16_LIMIT = 65520.0f;
template <int STORE> __device__ __forceinline__ void range_track(float &mx, float v0, float v1) {
  if (STORE == TG_STORE_FP16) mx = fmaxf(mx, fmaxf(fabsf(v0), fabsf(v1)));
}
template <int STORE> __device__ __forceinline__ void range_report(const FilterArgs &a, float mx) {
  if (STORE == TG_STORE_FP16 && mx >= FP16_LIMIT && a.err) atomicOr(a.err, 4);
}

// Value pair (a, b) of element k of a final row, with the reference's fill
// rule for samples whose left index is out of [0, nx-2] (main.rs:386-406).
__device__ __forceinline__ void elem_ab(const float *row, int nx, int k, int fill_mode,
                                        float fillv, float &a, float &b) {
  if (k >= 0 && k + 1 < nx) {
    a = row[k];
    b = row[k + 1];
  } else {
    float f = fill_mode == TG_FILL_ZERO ? 0.0f
              : fill_mode == TG_FILL_EDGE ? (k < 0 ? row[0] : row[nx - 1])
                                          : fillv;
    a = f;
    b = f;
  }
}

// One CTA per (row pair, view).  Rows 2j and 2j+1 are packed as the real and
// imaginary part of one complex FFT: with a real, even weight the inverse
// returns both filtered rows at once.
template <int FMT, int STORE>
__global__ void __launch_bounds__(256) filter_kernel(FilterArgs a) {
  extern __shared__ __align__(16) unsigned char fsm[];
  const int n = a.nx;
  float2 *A = reinterpret_cast<float2 *>(fsm);
  float2 *B = A + n;
  const int jp = blockIdx.x, v = blockIdx.y;
  const int r0 = 2 * jp, r1 = 2 * jp + 1;
  const bool has1 = r1 < a.ny;
  const float *in0 = a.in + ((size_t)v * a.ny + r0) * n;
  const float *in1 = in0 + n;
  const float *sb0 = a.sub ? a.sub + ((size_t)v * a.ny + r0) * n : nullptr;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    float x0 = in0[k], x1 = has1 ? in1[k] : 0.0f;
    if (sb0) {  // SIRT residual: orig - reprojection (main.rs:933-935)
      x0 = __fsub_rn(x0, sb0[k]);
      if (has1) x1 = __fsub_rn(x1, sb0[n + k]);
    }
    A[k] = make_float2(x0, x1);
  }
  __syncthreads();
  float2 *R = A;
  if (a.weights) {
    if (a.conv_h == nullptr) {
      R = stockham<false>(A, B, a.plan, a.tw);
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        float w = __ldg(&a.weights[k]);
        float2 z = R[k];
        R[k] = make_float2(__fmul_rn(z.x, w), __fmul_rn(z.y, w));
      }
      __syncthreads();
      R = stockham<true>(R, R == A ? B : A, a.plan, a.tw);
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        float2 z = R[k];
        R[k] = make_float2(__fmul_rn(z.x, a.inv_n), __fmul_rn(z.y, a.inv_n));
      }
    } else {
      // n without a radix-2/3/5/7 plan: circulant convolution with the
      // inverse transform of the weights (h already includes 1/n).
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        float s0 = 0.f, s1 = 0.f;
        for (int m = 0; m < n; ++m) {
          int d = k - m;
          d += d < 0 ? n : 0;
          float h = __ldg(&a.conv_h[d]);
          float2 z = A[m];
          s0 = fmaf(h, z.x, s0);
          s1 = fmaf(h, z.y, s1);
        }
        B[k] = make_float2(s0, s1);
      }
      R = B;
    }
    __syncthreads();
  }
  // R holds the two filtered rows; un-interleave into float rows in the other buffer
  float *row0 = reinterpret_cast<float *>(R == A ? B : A);
  float *row1 = row0 + n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    float2 z = R[k];
    row0[k] = z.x;
    row1[k] = z.y;
  }
  __syncthreads();
  const float stretch = a.stretch ? a.stretch[v] : 0.0f;
  if (stretch != 0.0f) {
    float *s0 = reinterpret_cast<float *>(R);  // R is free now
    float *s1 = s0 + n;
    const float center = __fdiv_rn((float)n, 2.0f);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      s0[k] = stretch_sample(row0, n, k, stretch, center, a.cubic);
      s1[k] = stretch_sample(row1, n, k, stretch, center, a.cubic);
    }
    __syncthreads();
    row0 = s0;
    row1 = s1;
  }
  const float fillv = a.fill ? a.fill[v] : 0.0f;
  float hmax = 0.0f;  // largest |value| packed into FP16 by this thread
  if (FMT == FMT_ROWS) {  // plain filtered rows written back over the input rows
    float *o0 = reinterpret_cast<float *>(a.out) + ((size_t)v * a.ny + r0) * n;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      o0[k] = row0[k];
      if (has1) o0[n + k] = row1[k];
    }
    return;
  }
  if (FMT == FMT_ROWPAIR) {
    uint8_t *out = reinterpret_cast<uint8_t *>(a.out) +
                   ((size_t)v * a.rows_alloc + jp) * (size_t)a.PW * (STORE == TG_STORE_FP32 ? 16 : 8);
    for (int e = threadIdx.x; e < a.PW; e += blockDim.x) {
      int k = e - a.padL;
      float a0, b0, a1, b1;
      elem_ab(row0, n, k, a.fill_mode, fillv, a0, b0);
      if (has1) elem_ab(row1, n, k, a.fill_mode, fillv, a1, b1);
      else a1 = b1 = 0.0f;
      if (STORE == TG_STORE_FP32) {
        reinterpret_cast<float4 *>(out)[e] = make_float4(a0, a1, b0, b1);
      } else {
        uint2 w;
        const float d0 = __fsub_rn(b0, a0), d1 = __fsub_rn(b1, a1);
        range_track<STORE>(hmax, a0, a1);
        range_track<STORE>(hmax, d0, d1);
        w.x = Pack<STORE == TG_STORE_FP32 ? TG_STORE_FP16 : STORE>::h2(a0, a1);
        w.y = Pack<STORE == TG_STORE_FP32 ? TG_STORE_FP16 : STORE>::h2(d0, d1);
        reinterpret_cast<uint2 *>(out)[e] = w;
      }
    }
  } else {
    const int eb = STORE == TG_STORE_FP32 ? 8 : 4;
    uint8_t *o0 = reinterpret_cast<uint8_t *>(a.out) + ((size_t)v * a.rows_alloc + r0) * (size_t)a.PW * eb;
    uint8_t *o1 = o0 + (size_t)a.PW * eb;
    for (int e = threadIdx.x; e < a.PW; e += blockDim.x) {
      int k = e - a.padL;
      float a0, b0;
      elem_ab(row0, n, k, a.fill_mode, fillv, a0, b0);
      float a1 = 0.f, b1 = 0.f;
      if (has1) elem_ab(row1, n, k, a.fill_mode, fillv, a1, b1);
      if (STORE == TG_STORE_FP32) {
        reinterpret_cast<float2 *>(o0)[e] = make_float2(a0, b0);
        if (has1) reinterpret_cast<float2 *>(o1)[e] = make_float2(a1, b1);
      } else {
        const float d0 = __fsub_rn(b0, a0), d1 = __fsub_rn(b1, a1);
        range_track<STORE>(hmax, a0, d0);
        if (has1) range_track<STORE>(hmax, a1, d1);
        reinterpret_cast<uint32_t *>(o0)[e] = Pack<STORE == TG_STORE_FP32 ? TG_STORE_FP16 : STORE>::h2(a0, d0);
        if (has1)
          reinterpret_cast<uint32_t *>(o1)[e] = Pack<STORE == TG_STORE_FP32 ? TG_STORE_FP16 : STORE>::h2(a1, d1);
      }
    }
  }
  range_report<STORE>(a, hmax);
}

// ---------------------------------------------------------------------------
// Rows of 2^k (256..4096) or 3*2^k (384..3072) samples: register-resident
// Stockham FFT.  N/V threads per row pair, each holding V complex values (16 for
// 1024..4096: radix-16 passes and a last radix 4, 8 or 16; 8 for 256 and 512:
// radix-8 passes; 12 or 24 for 3*2^k: radix 8/4/2 passes and a final radix-3
// pass), one shared-memory exchange per pass (the generic kernel above takes one
// pass per factor 4).  The first forward pass reads the rows from global memory,
// the spectrum stays in registers between the transforms, and the epilogue works
// on the complex pairs (row 2j in .x, row 2j+1 in .y) without splitting them.
// ---------------------------------------------------------------------------
// Radix-4 butterfly with the plain complex sums and differences on the packed
// f32x2 pipe (one instruction per complex add); the ones that meet a rotation by
// -+i stay scalar, where the swap and sign fold into the adds.  ROT2: v[2]
// arrives still to be rotated by -+i (the radix-8 butterfly's third odd term).
template <bool INV, bool ROT2> __device__ __forceinline__ void bfly4_p(float2 *v) {
  float2 a0, a1;
  if constexpr (ROT2) {
    const float2 r = rot<INV>(v[2]);
    a0 = cadd(v[0], r);
    a1 = csub(v[0], r);
  } else {
    a0 = cadd_p(v[0], v[2]);
    a1 = csub_p(v[0], v[2]);
  }
  const float2 b0 = cadd_p(v[1], v[3]), b1 = rot<INV>(csub_p(v[1], v[3]));
  v[0] = cadd_p(a0, b0);
  v[1] = cadd(a1, b1);
  v[2] = csub_p(a0, b0);
  v[3] = csub(a1, b1);
}

template <bool INV> __device__ __forceinline__ void dft8(float2 *v) {
  const float h = 0.707106781186547524400844362104849039f;  // 1/sqrt(2)
  float2 t[4], u[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    t[j] = cadd_p(v[j], v[j + 4]);
    u[j] = csub_p(v[j], v[j + 4]);
  }
  // u_j *= exp(-+2 pi i j / 8) (u_2's factor -+i is folded into its butterfly)
  {
    const float2 d = u[1];
    u[1] = INV ? make_float2(h * (d.x - d.y), h * (d.x + d.y)) : make_float2(h * (d.x + d.y), h * (d.y - d.x));
  }
  {
    const float2 d = u[3];
    u[3] = INV ? make_float2(-h * (d.x + d.y), h * (d.x - d.y)) : make_float2(h * (d.y - d.x), -h * (d.x + d.y));
  }
  bfly4_p<INV, false>(t);
  bfly4_p<INV, true>(u);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    v[2 * m] = t[m];
    v[2 * m + 1] = u[m];
  }
}

// 16-point DFT as 4 x 4: radix-4 butterflies over v[j + 4m] (m), the twiddles
// exp(-+2 pi i j k1 / 16), radix-4 butterflies over j; output in natural order.
template <bool INV> __device__ __forceinline__ void dft16(float2 *v) {
  // cos and sin of 2 pi m / 16 for the twiddle exponents m = j*k1 that occur
  constexpr float c1 = 0.923879532511286756128183189396788933f;  // cos(pi/8)
  constexpr float s1 = 0.382683432365089771728459984030398867f;  // sin(pi/8)
  constexpr float h = 0.707106781186547524400844362104849039f;   // cos(pi/4)
  float2 y[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    float2 q[4] = {v[j], v[j + 4], v[j + 8], v[j + 12]};
    bfly4_p<INV, false>(q);
#pragma unroll
    for (int k = 0; k < 4; ++k) y[j][k] = q[k];
  }
  auto tw = [](float2 z, float c, float sn) {  // z * (c - +i sn): the forward root exp(-i a)
    const float2 w = make_float2(c, INV ? sn : -sn);
    return cmul(z, w);
  };
  y[1][1] = tw(y[1][1], c1, s1);   // m = 1
  y[1][2] = tw(y[1][2], h, h);     // m = 2
  y[1][3] = tw(y[1][3], s1, c1);   // m = 3
  y[2][1] = tw(y[2][1], h, h);     // m = 2
  y[2][2] = rot<INV>(y[2][2]);     // m = 4: -+i
  y[2][3] = tw(y[2][3], -h, h);    // m = 6
  y[3][1] = tw(y[3][1], s1, c1);   // m = 3
  y[3][2] = tw(y[3][2], -h, h);    // m = 6
  y[3][3] = tw(y[3][3], -c1, -s1); // m = 9
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    float2 q[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
    bfly4_p<INV, false>(q);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = q[k2];
  }
}

template <int R, bool INV> __device__ __forceinline__ void dft_r(float2 *v) {
  if constexpr (R == 16) dft16<INV>(v);
  else if constexpr (R == 8) dft8<INV>(v);
  else if constexpr (R == 4) bfly4_p<INV, false>(v);
  else if constexpr (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd_p(a, b);
    v[1] = csub_p(a, b);
  } else bfly<R, INV>(v, nullptr, R);
}

// Shared-memory position of row element e: one padding slot after every 16
// complex values (128 bytes, one pass over the 32 banks).  Unpadded, a span-1
// pass stores with a stride of R values (8 or 16), which puts the lanes of a
// half-warp on a few bank pairs; padded, the half-warp's 16 stores land on 16
// distinct bank pairs in the span-1 passes and at spans of 16 or more, and reads
// of consecutive elements stay conflict-free (the radix-8 pass at span 8 writes
// the LAY_XOR8 layout below instead).  A pass's R outputs sit at e + r*NS with the low four bits of e
// and r*NS never carrying into bit 4, so their padded positions are one base plus
// compile-time offsets (no per-element address arithmetic).
__device__ __forceinline__ int swz(int e) { return e + (e >> 4); }
// swz(e + off) for an offset whose low four bits never carry with e's: both the
// pass outputs e = base + r*NS (base's low bits stay below 16 - (r*NS mod 16):
// base - k is a multiple of NS*R and k < NS) and the reads t + j*T (T a multiple
// of 16) -- so the offset is a compile-time constant.
__device__ __forceinline__ int swz_add(int swz_e, int off) { return swz_e + off + (off >> 4); }
template <int N> __host__ __device__ constexpr int padded_len() { return N + N / 16; }

// Radix of pass i of the forward transform, for V values per thread: 16, 8, 4 or 2
// while the remaining length allows it (and V is a multiple), the factor 3 of
// 3*2^k lengths last.
__host__ __device__ constexpr int p2_radix(int N, int V, int i) {
  int NS = 1, R = 1;
  for (int p = 0; p <= i; ++p) {
    const int Q = N / NS;
    R = (Q % 16 == 0 && V % 16 == 0) ? 16 : (Q % 8 == 0 && V % 8 == 0) ? 8 : (Q % 4 == 0 && V % 4 == 0) ? 4
        : (Q % 2 == 0 && V % 2 == 0) ? 2 : 3;
    NS *= R;
  }
  return R;
}
__host__ __device__ constexpr int p2_npass(int N, int V) {
  int NS = 1, p = 0;
  while (NS < N) NS *= p2_radix(N, V, p++);
  return p;
}
// span (product of the earlier passes' radices) of pass i
__host__ __device__ constexpr int p2_span(int N, int V, int i) {
  int NS = 1;
  for (int p = 0; p < i; ++p) NS *= p2_radix(N, V, p);
  return NS;
}
// offset of forward pass i's twiddles in the per-pass table: (R-1)*NS entries
// per earlier pass with twiddles (NS > 1; n - R0 entries in all, R0 the first radix)
__host__ __device__ constexpr int p2_twoff(int N, int V, int i) {
  int off = 0;
  for (int p = 1; p < i; ++p) off += (p2_radix(N, V, p) - 1) * p2_span(N, V, p);
  return off;
}
// Shared-memory layout of the buffer a pass writes.  LAY_PAD (swz): one slot of
// padding per 16 values; LAY_XOR8: no padding, bit 3 of the slot flipped in odd
// 64-value blocks -- for the output of a radix-8 pass at span 8, whose strided
// stores put two groups of 8 lanes 64 values apart, 4 slots apart (two-way bank
// conflicts) in the padded layout and 8 apart here; LAY_LIN: plain, for the
// inverse's result, which the staging epilogue reads at consecutive positions.
// Each layout keeps 16 consecutive values of an aligned block in 16 distinct
// bank pairs, so the lane-contiguous accesses stay conflict-free.
enum { LAY_PAD = 0, LAY_XOR8 = 1, LAY_LIN = 2 };
__host__ __device__ constexpr int p2_layout(int N, int V, int p) {
  return (p2_radix(N, V, p) == 8 && p2_span(N, V, p) == 8) ? LAY_XOR8 : LAY_PAD;
}
// slot of element t + j*T (lane-contiguous accesses)
template <int LAY, int T> __device__ __forceinline__ int p2_cslot(int t, int j) {
  if constexpr (LAY == LAY_PAD) {
    return swz_add(swz(t), j * T);
  } else if constexpr (LAY == LAY_LIN) {
    return t + j * T;
  } else if constexpr (T % 128 == 0) {
    return (t ^ (((t >> 6) & 1) << 3)) + j * T;  // bit 6 of t + j*T is bit 6 of t
  } else {
    const int e = t + j * T;
    return e ^ (((e >> 6) & 1) << 3);
  }
}
// slots of base + r*NS, r = 0..R-1 (a pass's strided accesses), as a base per
// parity of r plus compile-time offsets: even r at sb[0] + r*NS, odd at sb[1] + r*NS
// (LAY_PAD: offsets folded as in swz_add; LAY_XOR8, radix 8 at span 8: base + 8r
// stays in base's 64-value block, so the flip is a +-8 on the parity of r)
template <int LAY, int R, int NS> __device__ __forceinline__ void p2_sslot(int base, int (&sb)[2]) {
  if constexpr (LAY == LAY_PAD) {
    sb[0] = sb[1] = swz(base);
  } else {
    static_assert(R == 8 && NS == 8, "the flipped layout serves the radix-8 pass at span 8");
    const int q8 = ((base >> 6) & 1) << 3;
    sb[0] = base + q8;
    sb[1] = base - q8;
  }
}
template <int LAY> __device__ __forceinline__ int p2_soff(int off) {
  return LAY == LAY_PAD ? off + (off >> 4) : off;
}

// values per thread of the register-resident kernel for rows of n samples (0: none)
static int p2_values(int n) {
  switch (n) {
    case 256: case 512: return 8;
    case 1024: case 2048: case 4096: return 16;
    case 384: return 12;
    case 768: case 1536: case 3072: return 24;
    default: return 0;
  }
}

bool p2_twiddle_table(int n, std::vector<float2> &out) {
  out.clear();
  const int V = p2_values(n);
  if (!V) return false;
  out.resize((size_t)n - p2_radix(n, V, 0));
  for (int p = 0; p < p2_npass(n, V); ++p) {
    const int R = p2_radix(n, V, p), NS = p2_span(n, V, p), off = p2_twoff(n, V, p);
    if (NS == 1) continue;
    for (int r = 1; r < R; ++r)
      for (int k = 0; k < NS; ++k) {
        const double a = -2.0 * M_PI * (double)(r * k) / (double)(NS * R);
        out[(size_t)off + (size_t)(r - 1) * NS + k] = make_float2((float)cos(a), (float)sin(a));
      }
  }
  return true;
}

// Pass I of the forward transform over the values x[j] = X[t + j*N/V] held by
// thread t (V per thread, so a pass of radix R is V/R butterflies per thread):
// twiddles, radix-R DFT, results written to Y at base + r*NS -- or, for the last
// pass (TOREG), back into x: that pass's butterfly m reads and writes the
// positions t + (m + M*r)*T, which are x's own.
template <int N, int V, int I, bool TOREG>
__device__ __forceinline__ void p2_pass(float2 (&x)[V], int t, const float2 *__restrict__ tw, float2 *Y) {
  constexpr int T = N / V;
  constexpr int R = p2_radix(N, V, I);
  constexpr int NS = p2_span(N, V, I);
  constexpr int M = V / R;  // butterflies per thread
  static_assert(V % R == 0, "values per thread must be a multiple of the radix");
  static_assert(!TOREG || NS * R == N, "only the last pass keeps its results in registers");
  static_assert(TOREG || ((NS & (NS - 1)) == 0 && R != 3), "folded offsets need power-of-two spans and radices");
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int b = t + m * T;
    const int k = b % NS;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = x[m + M * r];  // X[b + r*N/R]
    if constexpr (NS > 1) {
      const float2 *tp = tw + p2_twoff(N, V, I) + k;
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(tp + (r - 1) * NS));
    }
    dft_r<R, false>(v);
    if constexpr (TOREG) {
#pragma unroll
      for (int r = 0; r < R; ++r) x[m + M * r] = v[r];
    } else {
      constexpr int LAY = p2_layout(N, V, I);
      int sb[2];
      p2_sslot<LAY, R, NS>((b - k) * R + k, sb);
#pragma unroll
      for (int r = 0; r < R; ++r) Y[sb[r & 1] + p2_soff<LAY>(r * NS)] = v[r];
    }
  }
}

// Forward transform from pass I on: x holds pass I's inputs; on return x holds
// the spectrum values X[t + j*N/V].  Passes alternate between A and B, the
// first one (I = 0) writing A.
template <int N, int V, int I>
__device__ __forceinline__ void p2_forward(float2 (&x)[V], int t, const float2 *__restrict__ tw, float2 *A,
                                           float2 *B) {
  constexpr int T = N / V;
  if constexpr (I == p2_npass(N, V) - 1) {
    p2_pass<N, V, I, true>(x, t, tw, nullptr);
  } else {
    p2_pass<N, V, I, false>(x, t, tw, A);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < V; ++j) x[j] = A[p2_cslot<p2_layout(N, V, I), T>(t, j)];
    p2_forward<N, V, I + 1>(x, t, tw, B, A);
  }
}

// Pass I of the inverse transform: the transpose of forward pass PF = P-1-I
// (the forward matrix is symmetric, so the conjugate of the reversed product of
// its transposed passes is the unnormalised inverse).  It reads where pass PF
// wrote (base + r*NS; for I = 0 the forward's last pass, whose values are still
// in x), applies the inverse radix-R DFT and then the conjugate twiddles, and
// leaves in x[m + M*r] the positions t + (m + M*r)*T that pass PF read.  So
// every shared-memory access is one the forward already makes: lane-contiguous
// stores, and loads in the forward's store pattern (bank-conflict-free in the
// padded layout).
template <int N, int V, int I>
__device__ __forceinline__ void p2_ipass(float2 (&x)[V], int t, const float2 *__restrict__ tw, const float2 *Y) {
  constexpr int T = N / V;
  constexpr int PF = p2_npass(N, V) - 1 - I;
  constexpr int R = p2_radix(N, V, PF);
  constexpr int NS = p2_span(N, V, PF);
  constexpr int M = V / R;
  static_assert(I == 0 || ((NS & (NS - 1)) == 0 && R != 3), "folded offsets need power-of-two spans and radices");
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int b = t + m * T;
    const int k = b % NS;
    float2 v[R];
    if constexpr (I == 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = x[m + M * r];
    } else {
      constexpr int LAY = p2_layout(N, V, PF);
      int sb[2];
      p2_sslot<LAY, R, NS>((b - k) * R + k, sb);
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = Y[sb[r & 1] + p2_soff<LAY>(r * NS)];
    }
    dft_r<R, true>(v);
    if constexpr (NS > 1) {
      const float2 *tp = tw + p2_twoff(N, V, PF) + k;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = __ldg(tp + (r - 1) * NS);
        w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) x[m + M * r] = v[r];
  }
}

// Inverse transform from pass I on (I = 0: x holds the weighted spectrum as the
// forward left it).  Pass I reads B (I > 0) and stores its results, in natural
// positions, to A; returns the buffer holding the result (after a barrier).
template <int N, int V, int I>
__device__ __forceinline__ float2 *p2_inverse(float2 (&x)[V], int t, const float2 *__restrict__ tw, float2 *A,
                                              float2 *B) {
  constexpr int T = N / V;
  p2_ipass<N, V, I>(x, t, tw, B);
  // the next pass reads in the strided pattern of forward pass P-2-I: that pass's
  // layout; the last pass's result is plain
  constexpr int P = p2_npass(N, V);
  constexpr int LAY = I == P - 1 ? LAY_LIN : p2_layout(N, V, P - 2 - I);
#pragma unroll
  for (int j = 0; j < V; ++j) A[p2_cslot<LAY, T>(t, j)] = x[j];
  __syncthreads();
  if constexpr (I == p2_npass(N, V) - 1) return A;
  else return p2_inverse<N, V, I + 1>(x, t, tw, B, A);
}

template <int N, int V, int FMT, int STORE>
__device__ __forceinline__ void filter_p2_body(const FilterArgs &a, const int jp, const int v) {
  extern __shared__ __align__(16) unsigned char fsm[];
  constexpr int T = N / V;
  float2 *A = reinterpret_cast<float2 *>(fsm);
  float2 *B = A + padded_len<N>();
  const int t = threadIdx.x;
  const int r0 = 2 * jp;
  const bool has1 = r0 + 1 < a.ny;
  const float *in0 = a.in + ((size_t)v * a.ny + r0) * N;
  const float *sb0 = a.sub ? a.sub + ((size_t)v * a.ny + r0) * N : nullptr;
  float2 x[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const int k = t + j * T;
    float x0 = __ldg(in0 + k), x1 = has1 ? __ldg(in0 + N + k) : 0.0f;
    if (sb0) {  // SIRT residual: orig - reprojection (main.rs:933-935)
      x0 = __fsub_rn(x0, __ldg(sb0 + k));
      if (has1) x1 = __fsub_rn(x1, __ldg(sb0 + N + k));
    }
    x[j] = make_float2(x0, x1);
  }
  p2_forward<N, V, 0>(x, t, a.tw2, A, B);
  // x[j] = spectrum value t + j*T: x the radial weight, and for 2^k lengths the
  // 1/n of the inverse too (a power of two: exact, and exact through the
  // inverse's linear arithmetic, so the result is the one of scaling afterwards)
  constexpr bool POW2 = (N & (N - 1)) == 0;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    float w = __ldg(&a.weights[t + j * T]);
    if (POW2) w = __fmul_rn(w, a.inv_n);
    x[j] = make_float2(__fmul_rn(x[j].x, w), __fmul_rn(x[j].y, w));
  }
  // the forward's last exchange read buffer A (odd pass count) or B; the
  // inverse's first pass writes the other one
  constexpr int P = p2_npass(N, V);
  const float2 *Rr = P % 2 == 0 ? p2_inverse<N, V, 0>(x, t, a.tw2, B, A) : p2_inverse<N, V, 0>(x, t, a.tw2, A, B);
  const float inv_n = a.inv_n;
  auto sc = [&](int k) {
    const float2 z = Rr[k];  // plain layout
    return POW2 ? z : up2(mul2(pk2(z.x, z.y), pk2(inv_n, inv_n)));
  };
  // final value of both rows at column k (0 <= k < N): the cosine stretch
  // (main.rs:446-488) of the scaled inverse, or the scaled inverse itself
  const float stretch = a.stretch ? a.stretch[v] : 0.0f;
  const float center = __fdiv_rn((float)N, 2.0f);
  auto fin = [&](int k) -> float2 {
    if (stretch == 0.0f) return sc(k);
    const float dx = __fsub_rn((float)k, center);
    const float src_x = __fadd_rn(__fmul_rn(dx, stretch), center);
    const float fl = floorf(src_x);
    const int sx0 = fl < -1.0e9f ? -1000000000 : (int)fl;
    const float frac = __fsub_rn(src_x, fl);
    if (a.cubic && sx0 >= 1 && sx0 + 2 < N) {
      const float2 p0 = sc(sx0 - 1), p1 = sc(sx0), p2 = sc(sx0 + 1), p3 = sc(sx0 + 2);
      return make_float2(cubic1d(p0.x, p1.x, p2.x, p3.x, frac), cubic1d(p0.y, p1.y, p2.y, p3.y, frac));
    }
    if (sx0 >= 0 && sx0 + 1 < N) {
      const float2 p0 = sc(sx0), p1 = sc(sx0 + 1);
      const float omf = __fsub_rn(1.0f, frac);
      // RN(RN(p0*(1-f)) + RN(p1*f)) for both rows on the packed pipe (each lane is
      // the scalar operation: no product contracted into the sum)
      return up2(add2(mul2(pk2(p0.x, p0.y), pk2(omf, omf)), mul2(pk2(p1.x, p1.y), pk2(frac, frac))));
    }
    if (sx0 >= 0 && sx0 < N) return sc(sx0);
    return make_float2(0.0f, 0.0f);
  };
  // pack into the staging format with the reference's fill rule (main.rs:386-406).
  // A warp takes 31 consecutive elements e at a time: lane l computes the final
  // value at k = e - padL straight from the inverse (no second exchange) and
  // takes the value at k + 1 from lane l + 1; lane 31 only supplies its value.
  const float fillv = a.fill ? a.fill[v] : 0.0f;
  auto fill = [&](int k) -> float2 {
    if (a.fill_mode == TG_FILL_ZERO) return make_float2(0.0f, 0.0f);
    if (a.fill_mode == TG_FILL_EDGE) return fin(k < 0 ? 0 : N - 1);
    return make_float2(fillv, fillv);
  };
  float hmax = 0.0f;  // largest |value| packed into FP16 by this thread
  const size_t row0 = (size_t)v * a.rows_alloc;
  const int lane = t & 31;
  static_assert(T % 32 == 0, "whole warps per row pair");
  for (int e0 = (t >> 5) * 31; e0 < a.PW; e0 += (T / 32) * 31) {  // warp-uniform bounds
    const int e = e0 + lane;
    const int k = e - a.padL;
    float2 lo = make_float2(0.0f, 0.0f);
    if (k >= 0 && k < N) lo = fin(k);
    float2 hi = make_float2(__shfl_down_sync(0xffffffffu, lo.x, 1), __shfl_down_sync(0xffffffffu, lo.y, 1));
    if (lane == 31 || e >= a.PW) continue;
    if (!(k >= 0 && k + 1 < N)) lo = hi = fill(k);
    if (!has1) lo.y = hi.y = 0.0f;
    if (FMT == FMT_ROWPAIR) {
      uint8_t *out = reinterpret_cast<uint8_t *>(a.out) +
                     (row0 + jp) * (size_t)a.PW * (STORE == TG_STORE_FP32 ? 16 : 8);
      if (STORE == TG_STORE_FP32) {
        reinterpret_cast<float4 *>(out)[e] = make_float4(lo.x, lo.y, hi.x, hi.y);
      } else {
        using PK = Pack<STORE == TG_STORE_FP32 ? TG_STORE_FP16 : STORE>;
        const float2 d = csub_p(hi, lo);
        const float d0 = d.x, d1 = d.y;
        range_track<STORE>(hmax, lo.x, lo.y);
        range_track<STORE>(hmax, d0, d1);
        reinterpret_cast<uint2 *>(out)[e] = make_uint2(PK::h2(lo.x, lo.y), PK::h2(d0, d1));
      }
    } else {
      const int eb = STORE == TG_STORE_FP32 ? 8 : 4;
      uint8_t *o0 = reinterpret_cast<uint8_t *>(a.out) + (row0 + r0) * (size_t)a.PW * eb;
      uint8_t *o1 = o0 + (size_t)a.PW * eb;
      if (STORE == TG_STORE_FP32) {
        reinterpret_cast<float2 *>(o0)[e] = make_float2(lo.x, hi.x);
        if (has1) reinterpret_cast<float2 *>(o1)[e] = make_float2(lo.y, hi.y);
      } else {
        using PK = Pack<STORE == TG_STORE_FP32 ? TG_STORE_FP16 : STORE>;
        const float d0 = __fsub_rn(hi.x, lo.x), d1 = __fsub_rn(hi.y, lo.y);
        range_track<STORE>(hmax, lo.x, d0);
        if (has1) range_track<STORE>(hmax, lo.y, d1);
        reinterpret_cast<uint32_t *>(o0)[e] = PK::h2(lo.x, d0);
        if (has1) reinterpret_cast<uint32_t *>(o1)[e] = PK::h2(lo.y, d1);
      }
    }
  }
  range_report<STORE>(a, hmax);
}

// resident CTAs per SM the register allocation aims at (the kernel is latency-bound):
// 4 of 256 threads for the radix-8 kernels; 5 of the radix-16 kernels' 64 or 128
// threads (96 registers, no spills at 2048), 2 of 256
__host__ __device__ constexpr int p2_min_blocks(int N, int V) {
  return V == 8 && N / V == 256 ? 4 : V == 16 ? (N / V == 256 ? 2 : 5) : 1;
}
template <int N, int V, int FMT, int STORE>
__global__ void __launch_bounds__(N / V, p2_min_blocks(N, V)) filter_p2_kernel(FilterArgs a) {
  filter_p2_body<N, V, FMT, STORE>(a, blockIdx.x, blockIdx.y);
}

// The same filter over the row pairs of many series of one width: block b
// belongs to series j with blk0[j] <= b < blk0[j+1] ((ny+1)/2 row pairs x views
// each); every series' rows come out as in its own launch.
template <int N, int V, int FMT, int STORE>
__global__ void __launch_bounds__(N / V, p2_min_blocks(N, V)) filter_p2_batch_kernel(FilterBatchDev fb) {
  __shared__ __align__(16) FilterArgs s_a;
  __shared__ int s_j;
  if (threadIdx.x == 0) {
    int lo = 0, hi = fb.njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(&fb.blk0[mid]) <= (int)blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    s_j = lo;
  }
  __syncthreads();
  const int j = s_j;
  const uint32_t *src = reinterpret_cast<const uint32_t *>(&fb.jobs[j]);
  uint32_t *dst = reinterpret_cast<uint32_t *>(&s_a);
  for (int i = threadIdx.x; i < (int)(sizeof(FilterArgs) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  const int t = (int)blockIdx.x - __ldg(&fb.blk0[j]), nrp = (s_a.ny + 1) / 2;
  filter_p2_body<N, V, FMT, STORE>(s_a, t % nrp, t / nrp);
}

template <int N, int V, int FMT, int STORE> static void launch_p2(const FilterArgs &a, cudaStream_t st) {
  const size_t smem = (size_t)padded_len<N>() * 16;
  auto k = filter_p2_kernel<N, V, FMT, STORE>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k<<<dim3((a.ny + 1) / 2, a.nviews), N / V, smem, st>>>(a);
}

template <int FMT, int STORE> static bool try_p2(const FilterArgs &a, cudaStream_t st) {
  if (!a.weights || a.conv_h || !a.tw2 || getenv("TG_FILTER_GENERIC")) return false;
  switch (a.nx) {
    case 256: launch_p2<256, 8, FMT, STORE>(a, st); return true;
    case 512: launch_p2<512, 8, FMT, STORE>(a, st); return true;
    case 1024: launch_p2<1024, 16, FMT, STORE>(a, st); return true;
    case 2048: launch_p2<2048, 16, FMT, STORE>(a, st); return true;
    case 4096: launch_p2<4096, 16, FMT, STORE>(a, st); return true;
    case 384: launch_p2<384, 12, FMT, STORE>(a, st); return true;  // 3 * 2^k: 12 or 24 values per thread
    case 768: launch_p2<768, 24, FMT, STORE>(a, st); return true;
    case 1536: launch_p2<1536, 24, FMT, STORE>(a, st); return true;
    case 3072: launch_p2<3072, 24, FMT, STORE>(a, st); return true;
    default: return false;
  }
}

template <int FMT, int STORE> static void launch_f(const FilterArgs &a, cudaStream_t st) {
  if (try_p2<FMT, STORE>(a, st)) return;
  size_t smem = (size_t)a.nx * 16;  // two complex ping-pong buffers
  auto k = filter_kernel<FMT, STORE>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k<<<dim3((a.ny + 1) / 2, a.nviews), 256, smem, st>>>(a);
}

int filter_batch_width(const FilterArgs &a) {
  if (!a.weights || a.conv_h || !a.tw2 || getenv("TG_FILTER_GENERIC")) return 0;
  switch (a.nx) {
    case 256: case 512: case 1024: case 2048: case 4096: case 384: case 768: case 1536: case 3072: return a.nx;
    default: return 0;
  }
}

template <int N, int V, int FMT, int STORE>
static void launch_p2_batch(const FilterBatchDev &fb, int nblocks, cudaStream_t st) {
  const size_t smem = (size_t)padded_len<N>() * 16;
  auto k = filter_p2_batch_kernel<N, V, FMT, STORE>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k<<<nblocks, N / V, smem, st>>>(fb);
}

template <int FMT, int STORE> static void launch_batch_n(int n, const FilterBatchDev &fb, int nb, cudaStream_t st) {
  switch (n) {
    case 256: launch_p2_batch<256, 8, FMT, STORE>(fb, nb, st); break;
    case 512: launch_p2_batch<512, 8, FMT, STORE>(fb, nb, st); break;
    case 1024: launch_p2_batch<1024, 16, FMT, STORE>(fb, nb, st); break;
    case 2048: launch_p2_batch<2048, 16, FMT, STORE>(fb, nb, st); break;
    case 4096: launch_p2_batch<4096, 16, FMT, STORE>(fb, nb, st); break;
    case 384: launch_p2_batch<384, 12, FMT, STORE>(fb, nb, st); break;
    case 768: launch_p2_batch<768, 24, FMT, STORE>(fb, nb, st); break;
    case 1536: launch_p2_batch<1536, 24, FMT, STORE>(fb, nb, st); break;
    default: launch_p2_batch<3072, 24, FMT, STORE>(fb, nb, st); break;
  }
}

void launch_filter_batch(int n, int fmt, int store, const FilterBatchDev &fb, int nblocks, cudaStream_t st) {
  if (fmt == FMT_ROWPAIR) {
    if (store == TG_STORE_FP32) launch_batch_n<FMT_ROWPAIR, TG_STORE_FP32>(n, fb, nblocks, st);
    else if (store == TG_STORE_FP16) launch_batch_n<FMT_ROWPAIR, TG_STORE_FP16>(n, fb, nblocks, st);
    else launch_batch_n<FMT_ROWPAIR, TG_STORE_BF16>(n, fb, nblocks, st);
  } else {
    if (store == TG_STORE_FP32) launch_batch_n<FMT_SINGLE, TG_STORE_FP32>(n, fb, nblocks, st);
    else if (store == TG_STORE_FP16) launch_batch_n<FMT_SINGLE, TG_STORE_FP16>(n, fb, nblocks, st);
    else launch_batch_n<FMT_SINGLE, TG_STORE_BF16>(n, fb, nblocks, st);
  }
}

void launch_filter(const FilterArgs &a, cudaStream_t st) {
  if (a.fmt == FMT_ROWPAIR) {
    if (a.store == TG_STORE_FP32) launch_f<FMT_ROWPAIR, TG_STORE_FP32>(a, st);
    else if (a.store == TG_STORE_FP16) launch_f<FMT_ROWPAIR, TG_STORE_FP16>(a, st);
    else launch_f<FMT_ROWPAIR, TG_STORE_BF16>(a, st);
  } else {
    if (a.store == TG_STORE_FP32) launch_f<FMT_SINGLE, TG_STORE_FP32>(a, st);
    else if (a.store == TG_STORE_FP16) launch_f<FMT_SINGLE, TG_STORE_FP16>(a, st);
    else launch_f<FMT_SINGLE, TG_STORE_BF16>(a, st);
  }
}


// ---------------------------------------------------------------------------
// Allocation-free R-weighting (tg_apply_rweighting_device_noalloc).
//
// Some callers cannot call cudaMalloc: hosts that hand every byte of device
// memory out of their own pool or arena (a Rust or C++ host with its own
// allocator, a framework's caching allocator), and services that must not
// trigger cudaMalloc's implicit device-wide synchronisation or fragment device
// memory while other streams are running.  For them this entry point filters a
// caller-owned device stack in place and keeps its only scratch -- the
// per-call weight, twiddle and fallback-convolution tables -- in the
// file-scope array below, sized for rows of up to NOALLOC_MAX_NX samples.
// Every GPU that loads this library holds the array (128 KB) until the
// process exits.  All calls on a device share it, so calls whose GPU work
// overlaps (on different streams, or from different host threads without
// ordering) race on the tables; order them on one stream.
// ---------------------------------------------------------------------------
constexpr int NOALLOC_MAX_NX = 8192;
// layout: weights [n] | circulant kernel [n] | twiddles [2n]
static __device__ __align__(256) float g_rw_scratch[4 * NOALLOC_MAX_NX];

// The tables are computed on the host and travel to the array inside kernel
// parameters (copied by value when each launch is issued), so no host buffer
// has to outlive the call.  7680 floats = 30 KB per launch, under the 32 KB
// kernel-parameter limit.
constexpr int NOALLOC_CHUNK = 7680;
struct NoallocChunk { float v[NOALLOC_CHUNK]; };
__global__ void __launch_bounds__(256) noalloc_table_kernel(float *dst, int n, NoallocChunk c) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = c.v[i];
}

static std::mutex g_rw_mu;
// device address of g_rw_scratch, per device ordinal, valid for the CUDA context
// whose unique id is stored beside it (a reset device gets a new context)
static float *g_rw_dev[128];
static unsigned long long g_rw_ctx[128];
static float g_rw_host[4 * NOALLOC_MAX_NX];   // host tables of the current call (under g_rw_mu)

// Unique id of the calling thread's current CUDA context (0 if unavailable),
// through the runtime's driver entry points (the library does not link libcuda).
static unsigned long long current_context_id() {
  typedef int (*CtxGetCurrent)(void **);
  typedef int (*CtxGetId)(void *, unsigned long long *);
  static CtxGetCurrent get_current = nullptr;
  static CtxGetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, nullptr) == cudaSuccess)
      get_current = reinterpret_cast<CtxGetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, nullptr) == cudaSuccess)
      get_id = reinterpret_cast<CtxGetId>(f);
  });
  void *ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

}  // namespace tg

extern "C" int tg_apply_rweighting_device_noalloc(float *dev_proj, size_t in_nx, size_t in_ny,
                                                  size_t nz, float cutoff, float falloff,
                                                  int32_t exact_filter_size, int32_t use_hamming,
                                                  int32_t device, void *cuda_stream) {
  using namespace tg;
  if (!dev_proj || in_nx < 2 || in_ny == 0 || nz == 0) {
    set_error("tg_apply_rweighting_device_noalloc: null pointer or empty stack");
    return TG_ERR_INVALID_ARG;
  }
  if (in_nx > (size_t)NOALLOC_MAX_NX) {
    set_error("tg_apply_rweighting_device_noalloc: rows of " + std::to_string(in_nx) +
              " samples exceed the static scratch limit of " + std::to_string(NOALLOC_MAX_NX));
    return TG_ERR_INVALID_ARG;
  }
  if ((in_ny + 1) / 2 > 65535 || nz > 65535) {
    set_error("tg_apply_rweighting_device_noalloc: too many rows or sections for one launch");
    return TG_ERR_INVALID_ARG;
  }
  if (device < 0 || device >= 128) { set_error("bad device ordinal"); return TG_ERR_INVALID_ARG; }
  std::lock_guard<std::mutex> lk(g_rw_mu);
  int prev = -1;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  auto restore = [&]() { if (prev >= 0 && prev != device) cudaSetDevice(prev); };
  const unsigned long long ctx = current_context_id();
  if (!g_rw_dev[device] || ctx == 0 || ctx != g_rw_ctx[device]) {
    // first call in this device's context: the array's device address (the host
    // symbol is only a stand-in and must never be passed to a kernel)
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_rw_scratch);
    if (e != cudaSuccess) { restore(); return cuda_fail(e, "cudaGetSymbolAddress(g_rw_scratch)"); }
    g_rw_dev[device] = static_cast<float *>(ptr);
    g_rw_ctx[device] = ctx;
  }
  const int n = (int)in_nx;
  float *hw = g_rw_host, *hconv = g_rw_host + NOALLOC_MAX_NX, *htw = g_rw_host + 2 * NOALLOC_MAX_NX;
  weight_table(n, cutoff, falloff, exact_filter_size, use_hamming, hw);
  FilterArgs f{};
  const bool radix = fft_plan(n, &f.plan);
  for (int k = 0; k < n; ++k) {
    double ang = -2.0 * M_PI * (double)k / (double)n;
    htw[2 * k] = (float)cos(ang);
    htw[2 * k + 1] = (float)sin(ang);
  }
  if (!radix)  // h[m] = (1/n) sum_k w[k] cos(2 pi k m / n)
    for (int m = 0; m < n; ++m) {
      double acc = 0.0;
      for (int k = 0; k < n; ++k) acc += (double)hw[k] * cos(2.0 * M_PI * (double)k * m / n);
      hconv[m] = (float)(acc / n);
    }
  float *dev = g_rw_dev[device];
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  // tables -> the static array, in kernel-parameter chunks on the caller's stream
  auto upload = [&](float *dst, const float *src, int count) -> cudaError_t {
    static NoallocChunk chunk;  // under g_rw_mu; copied into each launch's parameters
    for (int o = 0; o < count; o += NOALLOC_CHUNK) {
      const int c = std::min(NOALLOC_CHUNK, count - o);
      memcpy(chunk.v, src + o, (size_t)c * sizeof(float));
      noalloc_table_kernel<<<1, 256, 0, st>>>(dst + o, c, chunk);
      cudaError_t le = cudaGetLastError();
      if (le != cudaSuccess) return le;
    }
    return cudaSuccess;
  };
  if ((e = upload(dev, hw, n)) != cudaSuccess || (!radix && (e = upload(dev + NOALLOC_MAX_NX, hconv, n)) != cudaSuccess) ||
      (e = upload(dev + 2 * NOALLOC_MAX_NX, htw, 2 * n)) != cudaSuccess) {
    restore();
    return cuda_fail(e, "noalloc table upload");
  }
  f.in = dev_proj;
  f.out = dev_proj;
  f.weights = dev;
  f.conv_h = radix ? nullptr : dev + NOALLOC_MAX_NX;
  f.tw = reinterpret_cast<const float2 *>(dev + 2 * NOALLOC_MAX_NX);
  f.nx = n;
  f.ny = (int)in_ny;
  f.nviews = (int)nz;
  f.fill_mode = TG_FILL_ZERO;
  f.fmt = FMT_ROWS;
  f.store = TG_STORE_FP32;
  f.inv_n = 1.0f / (float)n;
  size_t smem = (size_t)n * 16;
  auto k = filter_kernel<FMT_ROWS, TG_STORE_FP32>;
  if (smem > 48 * 1024 &&
      (e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) {
    restore();
    return cuda_fail(e, "cudaFuncSetAttribute(filter)");
  }
  k<<<dim3((unsigned)((in_ny + 1) / 2), (unsigned)nz), 256, smem, st>>>(f);
  e = cudaGetLastError();
  restore();
  if (e != cudaSuccess) return cuda_fail(e, "filter launch (noalloc)");
  return TG_OK;
}
