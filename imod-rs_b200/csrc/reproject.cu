// reproject.cu -- SIRT forward projection as a ray-driven gather.
//
// Semantics: forward_project, apps/tilt/src/main.rs:831-896 (voxel-driven
// splat: each voxel adds val*(1-frac) to bin floor(x) and val*frac to the next
// bin of row floor(y), with the two-row split when x-tilt or local alignment
// moves y).  Here one thread owns one bin (view, row, p) and gathers, for each
// depth oz, the few columns whose exact f32 position lands in [p-1, p+1).  No
// atomics; each bin's sum is formed by one thread in a fixed order.  Without
// x-tilt/local alignment the order (oz ascending, ox ascending) is the
// reference's own order, so the result is bit-identical to the serial splat.
#include <cuda_fp16.h>

#include "tg_internal.h"
#include "f32x2.cuh"
#include "local_dev.cuh"

namespace tg {

constexpr float FMAGIC = 12582912.0f;
constexpr uint32_t FMAGIC_BITS = 0x4B400000u;

__global__ void __launch_bounds__(128) fp_kernel(FpArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y, v = blockIdx.z;
  if (p >= a.nx) return;
  float *out = a.sino + ((size_t)v * a.ny + r) * a.nx + p;
  if (v >= a.nviews) {  // views without a tilt angle contribute nothing (main.rs:683-686)
    *out = 0.0f;
    return;
  }
  const float4 g = __ldg(&a.vg[v]);
  const float4 g2 = __ldg(&a.vg2[v]);
  const float cos_t = g.x, sin_t = g.y, zf = g.z, cos_xt = g.w, sin_xt = g2.x;
  const float lxmax = g2.y, lymax = g2.z;  // bounds of |local dx|, |local dy| for this view
  const bool simple = sin_xt == 0.0f && !a.has_local;
  const float aeff = cos_t * cos_xt;
  const float inv_a = fabsf(aeff) > 1e-3f ? 1.0f / aeff : 0.0f;
  const float pf = (float)p;
  float acc = 0.0f;
  const float *vol_r = a.vol + (size_t)r * a.onz * a.onx;
  for (int oz = 0; oz < a.onz; ++oz) {
    const float dz = __fsub_rn((float)oz, a.cz);
    const float t2 = __fmul_rn(__fmul_rn(dz, sin_t), zf);
    int lo, hi;
    if (inv_a != 0.0f) {
      const float base = a.cx + t2;
      float d1 = (pf - 1.0f - lxmax - base) * inv_a, d2 = (pf + 1.0f + lxmax - base) * inv_a;
      float dmin = fminf(d1, d2) + a.ocx, dmax = fmaxf(d1, d2) + a.ocx;
      dmin = fmaxf(dmin, -1.0f);
      dmax = fminf(dmax, (float)a.onx);
      lo = max((int)floorf(dmin) - 1, 0);
      hi = min((int)ceilf(dmax) + 1, a.onx - 1);
    } else {
      lo = 0;
      hi = a.onx - 1;
    }
    for (int ox = lo; ox <= hi; ++ox) {
      const float dx = __fsub_rn((float)ox, a.ocx);
      const float t1 = __fmul_rn(__fmul_rn(dx, cos_t), cos_xt);
      const float xb = __fadd_rn(__fadd_rn(t1, t2), a.cx);
      if (simple) {
        const float tt = __fadd_rd(xb, FMAGIC);
        const int x0 = (int)(__float_as_uint(tt) - FMAGIC_BITS);
        if ((unsigned)x0 > (unsigned)(a.nx - 2)) continue;
        if (x0 != p && x0 != p - 1) continue;
        const float frac = __fsub_rn(xb, __fsub_rn(tt, FMAGIC));
        const float val = vol_r[(size_t)oz * a.onx + ox];
        acc = __fadd_rn(acc, x0 == p ? __fmul_rn(val, __fsub_rn(1.0f, frac)) : __fmul_rn(val, frac));
      } else {
        const float yoff = __fmul_rn(dx, sin_xt);
        const int c = r - (int)floorf(yoff);
        const int L = (int)ceilf(lymax);
        const int iy_lo = max(c - 2 - L, 0), iy_hi = min(c + 1 + L, a.ny - 1);
        for (int iy = iy_lo; iy <= iy_hi; ++iy) {
          float ldx = 0.0f, ldy = 0.0f;
          bool use_l = false;
          if (a.has_local) use_l = local_corr(a.loc, v, ox, iy, a.ny, ldx, ldy);
          const float x = use_l ? __fadd_rn(xb, ldx) : xb;
          const float fx = floorf(x);
          if (!(fx >= 0.0f && fx + 1.0f < (float)a.nx)) continue;
          const int x0 = (int)fx;
          if (x0 != p && x0 != p - 1) continue;
          const float frac = __fsub_rn(x, fx);
          float sy = __fadd_rn((float)iy, yoff);
          if (use_l) sy = __fadd_rn(sy, ldy);
          const float fsy = floorf(sy);
          if (!(fsy >= 0.0f && fsy < (float)a.ny)) continue;
          const int sy0 = (int)fsy;
          const float syf = __fsub_rn(sy, fsy);
          const bool two = sy0 + 1 < a.ny && (fabsf(yoff) > 1e-6f || a.has_local);
          const float val = a.vol[((size_t)iy * a.onz + oz) * a.onx + ox];
          const float cterm = x0 == p ? __fmul_rn(val, __fsub_rn(1.0f, frac)) : __fmul_rn(val, frac);
          if (two) {
            if (sy0 == r) acc = __fadd_rn(acc, __fmul_rn(cterm, __fsub_rn(1.0f, syf)));
            else if (sy0 + 1 == r) acc = __fadd_rn(acc, __fmul_rn(cterm, syf));
          } else if (sy0 == r) {
            acc = __fadd_rn(acc, cterm);
          }
        }
      }
    }
  }
  *out = acc;
}

// Fast reprojection (no local alignment, every view with cos(tilt)*cos(x-tilt)
// > 0.05).  A voxel's position x does not depend on its slice, so one thread
// owns bin p of S consecutive sinogram rows and shares the candidate search
// among them.  For each depth the columns whose exact position lies in
// [p-1, p+1) are found by an estimate from 1/cos corrected with exact
// evaluations (x is non-decreasing in the column), then visited in increasing
// column order.
//
// XT = false (no x-tilt): slice iy feeds only row iy, and the per-bin order
// (z ascending, x ascending) is the reference's serial order, so every bin is
// bit-identical to main.rs:831-896.
//
// XT = true: column ox moves the sample row by yoff = dx*sin(x-tilt), so slice
// iy feeds rows floor(iy+yoff) and floor(iy+yoff)+1 with weights 1-f and f.
// With n = floor(yoff), the thread's rows r0-1+i (i = 0..S) are the nominal
// lower rows of slices iy_i = r0-1+i-n; f32 rounding of iy+yoff can only move
// the floor one row up (then f = 0 and the slice feeds that row with weight 1).
// The edge rules of the reference follow: a slice whose floor row is the last
// row feeds it alone with weight 1 (the one-row branch), a floor row of -1
// feeds nothing.  Weights and products are the reference's f32 expressions;
// only the summation order differs (z, x, slice instead of slice, z, x).
//
// Grid: (views, bin blocks, row groups) -- the views of one row group run
// together, so their reads of that slab of the volume hit L2.
template <int S, bool XT, bool IL>
__device__ __forceinline__ void fp_fast_body(const FpArgs &a, const int bx, const int by, const int bz) {
  const int v = bx;
  const int p = by * blockDim.x + threadIdx.x;
  const int r0 = bz * S;
  if (p >= a.nx) return;
  const int nrows = min(S, a.ny - r0);
  if (v >= a.nviews) {  // views without a tilt angle contribute nothing (main.rs:683-686)
    for (int s = 0; s < nrows; ++s) a.sino[((size_t)v * a.ny + r0 + s) * a.nx + p] = 0.0f;
    return;
  }
  const float4 g = __ldg(&a.vg[v]);
  const float cos_t = g.x, sin_t = g.y, zf = g.z, cos_xt = XT ? g.w : 1.0f;
  const float sin_xt = XT ? __ldg(&a.vg2[v]).x : 0.0f;
  const float inv_a = 1.0f / (cos_t * cos_xt);
  const float lo_t = (float)(p - 1), hi_t = (float)(p + 1);
  const size_t sstride = (size_t)a.onz * a.onx;
  float acc[S];
#pragma unroll
  for (int s = 0; s < S; ++s) acc[s] = 0.0f;
  // blended copy (one x-tilt for all views): its rows are blends, so this path is
  // within a tolerance of the reference, not bit-exact, and the products are fused
  // into packed accumulator pairs (one fma.f32x2 per two rows of a column visit)
  constexpr bool FUSED = XT && IL;
  uint64_t acc2[FUSED ? S / 2 : 1];
#pragma unroll
  for (int s = 0; s < (FUSED ? S / 2 : 1); ++s) acc2[s] = 0;
  // ((dx*cos)*cos_xt + t2) + cx, exactly as main.rs:842; fo is the column as a float
  // (carried along with the integer column: integers are exact in f32)
  auto X = [&](float fo, float t2) {
    const float dx = __fsub_rn(fo, a.ocx);
    const float t1 = XT ? __fmul_rn(__fmul_rn(dx, cos_t), cos_xt) : __fmul_rn(dx, cos_t);
    return __fadd_rn(__fadd_rn(t1, t2), a.cx);
  };
  // XT: row r0+s is the last row of the series (one-row branch) when s == last_s
  const int last_s = a.ny - 1 - r0;
  float foz = 0.0f;
  for (int oz = 0; oz < a.onz; ++oz, foz += 1.0f) {
    const float dz = __fsub_rn(foz, a.cz);
    const float t2 = __fmul_rn(__fmul_rn(dz, sin_t), zf);
    // first column whose position is >= p-1
    int lo = (int)floorf((lo_t - a.cx - t2) * inv_a + a.ocx) - 1;
    lo = min(max(lo, 0), a.onx);
    float flo = (float)lo;
    while (lo > 0 && X(flo - 1.0f, t2) >= lo_t) { --lo; flo -= 1.0f; }
    float x = X(flo, t2);  // carried into the visit loop: each position is evaluated once
    while (lo < a.onx && x < lo_t) { ++lo; flo += 1.0f; x = X(flo, t2); }
    const float *vz = a.vol + (size_t)oz * a.onx;
    float fo = flo;
#pragma unroll 2
    for (int ox = lo; ox < a.onx; ++ox, fo += 1.0f, x = X(fo, t2)) {
      if (!(x < hi_t)) break;
      const float tt = __fadd_rd(x, FMAGIC);
      const int x0 = (int)(__float_as_uint(tt) - FMAGIC_BITS);
      if ((unsigned)x0 > (unsigned)(a.nx - 2)) continue;  // px0 >= 0 && px0 + 1 < nx
      const float frac = __fsub_rn(x, __fsub_rn(tt, FMAGIC));
      const float w = x0 == p ? __fsub_rn(1.0f, frac) : frac;
      if (IL) {
        // interleaved copy: the S rows of this row group at (oz, ox) are S/4 float4s, one
        // per 4-row plane (neighbouring threads' columns are neighbouring float4s); with
        // x-tilt each holds the row's blend of its two source slices (blend_interleave_kernel)
        const float4 *q = reinterpret_cast<const float4 *>(a.volg) +
                          ((size_t)bz * a.onz + oz) * a.onx * (S / 4) + ox;
        // products on the f32x2 pipe; the sums stay scalar so that no product is
        // contracted into them (each stays RN(acc + RN(v*w)), the reference's operations)
        const uint64_t w2 = pk2(w, w);
#pragma unroll
        for (int k = 0; k < S / 4; ++k) {
          const float4 q4 = __ldg(q + (size_t)k * a.onx);
          if constexpr (FUSED) {
            acc2[2 * k] = fma2(pk2(q4.x, q4.y), w2, acc2[2 * k]);
            acc2[2 * k + 1] = fma2(pk2(q4.z, q4.w), w2, acc2[2 * k + 1]);
          } else {
            const float2 pa = up2(mul2(pk2(q4.x, q4.y), w2)), pb = up2(mul2(pk2(q4.z, q4.w), w2));
            acc[4 * k + 0] = __fadd_rn(acc[4 * k + 0], pa.x);
            acc[4 * k + 1] = __fadd_rn(acc[4 * k + 1], pa.y);
            acc[4 * k + 2] = __fadd_rn(acc[4 * k + 2], pb.x);
            acc[4 * k + 3] = __fadd_rn(acc[4 * k + 3], pb.y);
          }
        }
      } else if (!XT) {
        const float *vrow = vz + (size_t)r0 * sstride + ox;
#pragma unroll
        for (int s = 0; s < S; ++s)
          if (s < nrows) acc[s] = __fadd_rn(acc[s], __fmul_rn(__ldg(vrow + (size_t)s * sstride), w));
      } else {
        const float yoff = __fmul_rn(__fsub_rn(fo, a.ocx), sin_xt);
        const float fn = floorf(yoff);
        const int iy0 = r0 - 1 - (int)fn;  // slice of i = 0
        const float *vcol = vz + ox;
        auto slice_val = [&](int i, int iy) { return __ldg(vcol + (size_t)iy * sstride); };
        // When iy0 + yoff and iy0 + S + yoff are positive and share a binade (so
        // r0 >= 8), f32 rounds every iy + yoff of the group to iy + (the same
        // multiple of the binade's ulp) -- integers are even multiples of it there,
        // so ties go the same way -- and all slices share one fraction and one
        // nominal or raised floor.
        const float s0 = __fadd_rn((float)iy0, yoff), s1 = __fadd_rn((float)(iy0 + S), yoff);
        if (s0 > 0.0f && (__float_as_uint(s0) >> 23) == (__float_as_uint(s1) >> 23)) {
          const float fs0 = floorf(s0);
          const bool nominal = fs0 == (float)(r0 - 1);
          const float syf = __fsub_rn(s0, fs0);
          const float wa = __fsub_rn(1.0f, syf), wb = nominal ? syf : 1.0f;
#pragma unroll
          for (int i = 0; i <= S; ++i) {
            const int iy = iy0 + i;
            if (i > nrows || (unsigned)iy >= (unsigned)a.ny) continue;
            const float c = __fmul_rn(slice_val(i, iy), w);
            if (i >= 1 && nominal)
              acc[i - 1] = __fadd_rn(acc[i - 1], __fmul_rn(c, (i - 1 == last_s) ? 1.0f : wa));
            if (i < nrows && !(nominal && i - 1 == last_s)) acc[i] = __fadd_rn(acc[i], __fmul_rn(c, wb));
          }
          continue;
        }
#pragma unroll
        for (int i = 0; i <= S; ++i) {
          const int iy = iy0 + i;
          if (i > nrows || (unsigned)iy >= (unsigned)a.ny) continue;
          const float A = (float)(r0 - 1 + i);  // nominal lower row
          const float sy = __fadd_rn((float)iy, yoff);
          const float fs = floorf(sy);
          const bool nominal = fs == A;
          const float syf = __fsub_rn(sy, fs);
          const float c = __fmul_rn(slice_val(i, iy), w);
          // lower row A = r0-1+i -> acc[i-1]; upper row A+1 -> acc[i]
          if (i >= 1 && nominal) {
            const float wa = (i - 1 == last_s) ? 1.0f : __fsub_rn(1.0f, syf);
            acc[i - 1] = __fadd_rn(acc[i - 1], __fmul_rn(c, wa));
          }
          if (i < nrows && !(r0 + i - 1 == -1 && nominal) && !(nominal && i - 1 == last_s)) {
            const float wb = nominal ? syf : 1.0f;
            acc[i] = __fadd_rn(acc[i], __fmul_rn(c, wb));
          }
        }
      }
    }
  }
  if constexpr (FUSED) {
#pragma unroll
    for (int k = 0; k < S / 2; ++k) {
      const float2 u = up2(acc2[k]);
      acc[2 * k] = u.x;
      acc[2 * k + 1] = u.y;
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s)
    if (s < nrows) a.sino[((size_t)v * a.ny + r0 + s) * a.nx + p] = acc[s];
}

// volg[g][oz][j/4][ox][j%4] = vol[g*G + j][oz][ox] (zero for rows past ny): per
// (row group, depth) G/4 planes of float4s, each plane a row of columns
template <int G>
__device__ __forceinline__ void interleave_at(size_t i, const float *__restrict__ vol, float *__restrict__ volg, int ny,
                                  int onz, int onx, size_t n) {
  if (i >= n) return;
  const size_t sl = (size_t)onz * onx;
  const size_t g = i / sl, rem = i - g * sl;
  float v[G];
#pragma unroll
  for (int j = 0; j < G; ++j) {
    const size_t iy = g * G + j;
    v[j] = iy < (size_t)ny ? __ldg(vol + iy * sl + rem) : 0.0f;
  }
  const size_t ox = rem % onx;
  float4 *o = reinterpret_cast<float4 *>(volg) + (i - ox) * (G / 4) + ox;
#pragma unroll
  for (int k = 0; k < G / 4; ++k)
    o[(size_t)k * onx] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

template <int G>
__global__ void interleave_kernel(const float *__restrict__ vol, float *__restrict__ volg, int ny, int onz, int onx, size_t n) {
  interleave_at<G>((size_t)blockIdx.x * blockDim.x + threadIdx.x, vol, volg, ny, onz, onx, n);
}

// ---- half-precision reprojection (FP16/BF16 staging forms) ----
// The volume is copied into the row-group-interleaved layout as FP16 scaled by a
// power of two 2^(9-e), where max|v| < 2^e, so every value stays below 2^9 and
// the half partial sums below have headroom; the scale is exact and undone on
// the sums.  A column visit loads S halves in S/8 16-byte loads and adds the
// weighted values to packed half partial sums (fma), which are folded into the
// FP32 accumulators (mixed-precision add) every HALF_FLUSH depths.  Tolerance
// path: each volume value and partial sum carries a relative rounding of
// 2^-11; the accumulation over depths stays FP32.

__device__ __forceinline__ void acc2_f16(float &a0, float &a1, uint32_t h2) {
  asm("{\n .reg .f16 lo, hi;\n mov.b32 {lo, hi}, %2;\n"
      " add.rn.f32.f16 %0, lo, %0;\n add.rn.f32.f16 %1, hi, %1;\n}\n"
      : "+f"(a0), "+f"(a1)
      : "r"(h2));
}

// Power-of-two scale of the FP16 copy: copied values stay below 2^9, so the
// half-precision partial sums of fp_half_kernel (HALF_FLUSH = 4 depths, each
// adding weights that sum to at most 1/0.05 + 1 = 21) stay below 2^9 * 84 < 65504.
// headroom: 1 when the copied values are blends of two slices (|b| < 2 max|v|)
constexpr int HALF_FLUSH = 4;
__device__ __forceinline__ float half_scale(const unsigned *maxbits, bool inverse, int headroom = 0) {
  const float m = __uint_as_float(*maxbits);
  if (!(m > 0.0f) || !(m < 3.0e38f)) return 1.0f;
  int e;
  frexpf(m, &e);  // m < 2^e
  e += headroom;
  return inverse ? ldexpf(1.0f, e - 9) : ldexpf(1.0f, 9 - e);
}

// block blk of nblk blocks folds its share of max|vol| into *maxbits
__device__ __forceinline__ void absmax_at(const float *__restrict__ vol, size_t n, unsigned *maxbits, int blk,
                                          int nblk) {
  float m = 0.0f;
  const size_t n4 = n / 4, stride = (size_t)nblk * blockDim.x;
  const float4 *v4 = reinterpret_cast<const float4 *>(vol);  // cudaMalloc'd: 16-byte aligned
  size_t i = (size_t)blk * blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n4; i += 4 * stride) {  // four independent 16-byte loads in flight
    const float4 a = __ldg(v4 + i), b = __ldg(v4 + i + stride), c = __ldg(v4 + i + 2 * stride),
                 d = __ldg(v4 + i + 3 * stride);
    m = fmaxf(m, fmaxf(fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(a.z), fabsf(a.w))),
                       fmaxf(fmaxf(fabsf(b.x), fabsf(b.y)), fmaxf(fabsf(b.z), fabsf(b.w)))));
    m = fmaxf(m, fmaxf(fmaxf(fmaxf(fabsf(c.x), fabsf(c.y)), fmaxf(fabsf(c.z), fabsf(c.w))),
                       fmaxf(fmaxf(fabsf(d.x), fabsf(d.y)), fmaxf(fabsf(d.z), fabsf(d.w)))));
  }
  for (; i < n4; i += stride) {
    const float4 a = __ldg(v4 + i);
    m = fmaxf(m, fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(a.z), fabsf(a.w))));
  }
  if (blk == 0 && threadIdx.x < n - 4 * n4) m = fmaxf(m, fabsf(__ldg(vol + 4 * n4 + threadIdx.x)));
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(maxbits, __float_as_uint(m));  // |v| orders as its bits
}

__global__ void absmax_kernel(const float *__restrict__ vol, size_t n, unsigned *maxbits) {
  absmax_at(vol, n, maxbits, blockIdx.x, gridDim.x);
}

// volh[g][oz][j/8][ox][j%8] = half(vol[g*G + j][oz][ox] * scale) (zero past ny)
template <int G>
__device__ __forceinline__ void interleave_half_at(size_t i, const float *__restrict__ vol, __half *__restrict__ volh, int ny,
                                       int onz, int onx, size_t n, const unsigned *maxbits) {
  if (i >= n) return;
  const float sc = half_scale(maxbits, false);
  const size_t sl = (size_t)onz * onx;
  const size_t g = i / sl, rem = i - g * sl;
  uint32_t w[G / 2];
#pragma unroll
  for (int j = 0; j < G; j += 2) {
    const size_t iy = g * G + j;
    const float v0 = iy < (size_t)ny ? __ldg(vol + iy * sl + rem) * sc : 0.0f;
    const float v1 = iy + 1 < (size_t)ny ? __ldg(vol + (iy + 1) * sl + rem) * sc : 0.0f;
    const __half2 h = __floats2half2_rn(v0, v1);
    w[j / 2] = *reinterpret_cast<const uint32_t *>(&h);
  }
  const size_t ox = rem % onx;
  uint4 *o = reinterpret_cast<uint4 *>(volh) + (i - ox) * (G / 8) + ox;
#pragma unroll
  for (int k = 0; k < G / 8; ++k)
    o[(size_t)k * onx] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
}

template <int G>
__global__ void interleave_half_kernel(const float *__restrict__ vol, __half *__restrict__ volh, int ny, int onz, int onx, size_t n,
                                       const unsigned *maxbits) {
  interleave_half_at<G>((size_t)blockIdx.x * blockDim.x + threadIdx.x, vol, volh, ny, onz, onx, n, maxbits);
}

template <int S, bool XT>
__device__ __forceinline__ void fp_half_body(const FpArgs &a, const int bx, const int by, const int bz) {
  const int v = bx;
  const int p = by * blockDim.x + threadIdx.x;
  const int r0 = bz * S;
  if (p >= a.nx) return;
  const int nrows = min(S, a.ny - r0);
  if (v >= a.nviews) {  // views without a tilt angle contribute nothing (main.rs:683-686)
    for (int s = 0; s < nrows; ++s) a.sino[((size_t)v * a.ny + r0 + s) * a.nx + p] = 0.0f;
    return;
  }
  const float4 g = __ldg(&a.vg[v]);
  const float cos_t = g.x, sin_t = g.y, zf = g.z, cos_xt = XT ? g.w : 1.0f;
  const float inv_a = 1.0f / (cos_t * cos_xt);
  const float lo_t = (float)(p - 1), hi_t = (float)(p + 1);
  float acc[S];
#pragma unroll
  for (int s = 0; s < S; ++s) acc[s] = 0.0f;
  // FP16 partial sums over HALF_FLUSH depths (packed fma), folded into the FP32
  // accumulators with mixed-precision adds
  __half2 ph[S / 2];
#pragma unroll
  for (int m = 0; m < S / 2; ++m) ph[m] = __float2half2_rn(0.0f);
  // Tolerance path: x(ox) = ox*c + c0 with one FMA (within a few ulp of the reference's
  // ((dx*cos)*cos_xt + t2) + cx, and non-decreasing in ox, which the search needs)
  const float c = XT ? cos_t * cos_xt : cos_t;
  float c0 = 0.0f;
  auto X = [&](float fo) { return fmaf(fo, c, c0); };  // fo: the column as a float
  const uint4 *vg = reinterpret_cast<const uint4 *>(a.volh) + (size_t)bz * a.onz * a.onx * (S / 8);
  float foz = 0.0f;
  for (int oz = 0; oz < a.onz; ++oz, foz += 1.0f) {
    const float dz = __fsub_rn(foz, a.cz);
    const float t2 = __fmul_rn(__fmul_rn(dz, sin_t), zf);
    c0 = fmaf(-a.ocx, c, t2 + a.cx);
    int lo = (int)floorf((lo_t - a.cx - t2) * inv_a + a.ocx) - 1;
    lo = min(max(lo, 0), a.onx);
    float flo = (float)lo;
    while (lo > 0 && X(flo - 1.0f) >= lo_t) { --lo; flo -= 1.0f; }
    float x = X(flo);  // carried into the visit loop
    while (lo < a.onx && x < lo_t) { ++lo; flo += 1.0f; x = X(flo); }
    const uint4 *vz = vg + (size_t)oz * a.onx * (S / 8);
    float fo = flo;
#pragma unroll 2
    for (int ox = lo; ox < a.onx; ++ox, fo += 1.0f, x = X(fo)) {
      if (!(x < hi_t)) break;
      const float tt = __fadd_rd(x, FMAGIC);
      const int x0 = (int)(__float_as_uint(tt) - FMAGIC_BITS);
      if ((unsigned)x0 > (unsigned)(a.nx - 2)) continue;
      const float frac = __fsub_rn(x, __fsub_rn(tt, FMAGIC));
      const __half2 w2 = __float2half2_rn(x0 == p ? __fsub_rn(1.0f, frac) : frac);
      const uint4 *q = vz + ox;  // plane k of this column at q + k*onx
#pragma unroll
      for (int k = 0; k < S / 8; ++k) {
        const uint4 u = __ldg(q + (size_t)k * a.onx);
        const uint32_t uu[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int m = 0; m < 4; ++m)
          ph[4 * k + m] = __hfma2(*reinterpret_cast<const __half2 *>(&uu[m]), w2, ph[4 * k + m]);
      }
    }
    if ((oz + 1) % HALF_FLUSH == 0 || oz + 1 == a.onz) {
#pragma unroll
      for (int m = 0; m < S / 2; ++m) {
        acc2_f16(acc[2 * m], acc[2 * m + 1], *reinterpret_cast<const uint32_t *>(&ph[m]));
        ph[m] = __float2half2_rn(0.0f);
      }
    }
  }
  const float inv = half_scale(a.maxbits, true, XT ? 1 : 0);
#pragma unroll
  for (int s = 0; s < S; ++s)
    if (s < nrows) a.sino[((size_t)v * a.ny + r0 + s) * a.nx + p] = acc[s] * inv;
}

int fp_half_rows(int variant) { return (variant & 4) ? 32 : 16; }


// Blended interleaved copy for one x-tilt shared by all views.  Row r of column ox
// receives, in the reference's forward projection (main.rs:831-896), slice
// s1 = r - floor(yoff) with weight 1-f (1 in the one-row branch: last row or zero
// offset) when its floor row is r, and slice s0 = s1 - 1 with weight f when its
// floor row is r-1 (nothing when that is -1), or with weight 1 when f32 rounding
// of s0 + yoff raised its floor to r.  Those weights depend on (slice, column)
// only, not on the view, so the blend B[r] = v(s1)*w1 + v(s0)*w0 is formed once
// per reprojection and the views then project B like a volume without x-tilt.
// The products are summed in another order than the reference's (tolerance path).
__device__ __forceinline__ float blend_row(const float *__restrict__ vol, int ny, size_t sl, size_t rem, int r,
                                          int nn, float yoff, bool two_ok) {
  float acc = 0.0f;
  if (r >= ny) return acc;
  const int s1 = r - nn, s0 = s1 - 1;
  if (s1 >= 0 && s1 < ny) {
    const float sy = __fadd_rn((float)s1, yoff), fs = floorf(sy);
    if (fs == (float)r) {  // floor row r (not raised)
      const float w1 = (r == ny - 1 || !two_ok) ? 1.0f : __fsub_rn(1.0f, __fsub_rn(sy, fs));
      acc = __fmul_rn(__ldg(vol + (size_t)s1 * sl + rem), w1);
    }
  }
  if (s0 >= 0 && s0 < ny) {
    const float sy = __fadd_rn((float)s0, yoff), fs = floorf(sy);
    const float v0 = __ldg(vol + (size_t)s0 * sl + rem);
    if (fs == (float)r) acc = __fadd_rn(acc, v0);  // raised floor: weight 1
    else if (r >= 1 && two_ok) acc = __fadd_rn(acc, __fmul_rn(v0, __fsub_rn(sy, fs)));
  }
  return acc;
}

template <int G>
__device__ __forceinline__ void blend_interleave_at(size_t i, const float *__restrict__ vol, float *__restrict__ volb, int ny,
                                        int onz, int onx, float ocx, float sin_xt, size_t n) {
  if (i >= n) return;
  const size_t sl = (size_t)onz * onx;
  const size_t g = i / sl, rem = i - g * sl;
  const int ox = (int)(rem % onx);
  const float yoff = __fmul_rn(__fsub_rn((float)ox, ocx), sin_xt);
  const int nn = (int)floorf(yoff);
  const bool two_ok = fabsf(yoff) > 1e-6f;  // the reference's two-row condition
  float b[G];
#pragma unroll
  for (int j = 0; j < G; ++j) b[j] = blend_row(vol, ny, sl, rem, (int)g * G + j, nn, yoff, two_ok);
  float4 *o = reinterpret_cast<float4 *>(volb) + (i - (size_t)ox) * (G / 4) + ox;  // layout of interleave_kernel
#pragma unroll
  for (int k = 0; k < G / 4; ++k)
    o[(size_t)k * onx] = make_float4(b[4 * k], b[4 * k + 1], b[4 * k + 2], b[4 * k + 3]);
}

template <int G>
__global__ void blend_interleave_kernel(const float *__restrict__ vol, float *__restrict__ volb, int ny, int onz, int onx,
                                        float ocx, float sin_xt, size_t n) {
  blend_interleave_at<G>((size_t)blockIdx.x * blockDim.x + threadIdx.x, vol, volb, ny, onz, onx, ocx, sin_xt, n);
}

// The same blend into the scaled FP16 copy of the half-staging forms (a blend of
// two slices is below 2 max|v|: one more bit of headroom).
template <int G>
__device__ __forceinline__ void blend_interleave_half_at(size_t i, const float *__restrict__ vol, __half *__restrict__ volh, int ny,
                                             int onz, int onx, float ocx, float sin_xt, size_t n,
                                             const unsigned *maxbits) {
  if (i >= n) return;
  const float sc = half_scale(maxbits, false, 1);
  const size_t sl = (size_t)onz * onx;
  const size_t g = i / sl, rem = i - g * sl;
  const int ox = (int)(rem % onx);
  const float yoff = __fmul_rn(__fsub_rn((float)ox, ocx), sin_xt);
  const int nn = (int)floorf(yoff);
  const bool two_ok = fabsf(yoff) > 1e-6f;
  uint32_t w[G / 2];
#pragma unroll
  for (int j = 0; j < G; j += 2) {
    const int r = (int)g * G + j;
    const __half2 h = __floats2half2_rn(blend_row(vol, ny, sl, rem, r, nn, yoff, two_ok) * sc,
                                        blend_row(vol, ny, sl, rem, r + 1, nn, yoff, two_ok) * sc);
    w[j / 2] = *reinterpret_cast<const uint32_t *>(&h);
  }
  uint4 *o = reinterpret_cast<uint4 *>(volh) + (i - (size_t)ox) * (G / 8) + ox;  // layout of interleave_half_kernel
#pragma unroll
  for (int k = 0; k < G / 8; ++k)
    o[(size_t)k * onx] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
}

template <int G>
__global__ void blend_interleave_half_kernel(const float *__restrict__ vol, __half *__restrict__ volh, int ny, int onz,
                                             int onx, float ocx, float sin_xt, size_t n, const unsigned *maxbits) {
  blend_interleave_half_at<G>((size_t)blockIdx.x * blockDim.x + threadIdx.x, vol, volh, ny, onz, onx, ocx, sin_xt, n, maxbits);
}

template <int S, bool XT, bool IL>
__global__ void __launch_bounds__(128) fp_fast_kernel(FpArgs a) {
  fp_fast_body<S, XT, IL>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int S, bool XT>
__global__ void __launch_bounds__(128) fp_half_kernel(FpArgs a) {
  fp_half_body<S, XT>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---- batched reprojection: one launch per phase over the blocks of many series ----
// Block b belongs to series j with blk0[j] <= b < blk0[j+1]; its arguments are
// copied to shared memory and the per-series body runs with the block's local
// coordinates, so every series' result is the same as in its own launch.
__device__ __forceinline__ int load_fp_job(const FpBatchDev &b, FpArgs *s_a) {
  __shared__ int s_j;
  if (threadIdx.x == 0) {
    int lo = 0, hi = b.njobs - 1;  // last series whose first block is <= blockIdx.x
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(&b.blk0[mid]) <= (int)blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    s_j = lo;
  }
  __syncthreads();
  const int j = s_j;
  const uint32_t *src = reinterpret_cast<const uint32_t *>(&b.jobs[j]);
  uint32_t *dst = reinterpret_cast<uint32_t *>(s_a);
  for (int i = threadIdx.x; i < (int)(sizeof(FpArgs) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  return (int)blockIdx.x - __ldg(&b.blk0[j]);
}

__global__ void fp_zero_maxbits_kernel(const FpArgs *jobs, int njobs) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < njobs) *jobs[j].maxbits = 0u;
}

__global__ void __launch_bounds__(256) absmax_batch_kernel(FpBatchDev b) {
  __shared__ __align__(16) FpArgs s_a;
  const int t = load_fp_job(b, &s_a);
  const size_t n = (size_t)s_a.ny * s_a.onz * s_a.onx;
  absmax_at(s_a.vol, n, s_a.maxbits, t, fp_absmax_blocks(n));
}

template <int S, bool HALF, bool XT>
__global__ void __launch_bounds__(256) fp_copy_batch_kernel(FpBatchDev b) {
  __shared__ __align__(16) FpArgs s_a;
  const int t = load_fp_job(b, &s_a);
  const FpArgs &a = s_a;
  const size_t n = (size_t)((a.ny + S - 1) / S) * a.onz * a.onx;
  const size_t i = (size_t)t * 256 + threadIdx.x;
  if (HALF) {
    if (XT) blend_interleave_half_at<S>(i, a.vol, (__half *)a.volh, a.ny, a.onz, a.onx, a.ocx, a.sin_xt_common, n, a.maxbits);
    else interleave_half_at<S>(i, a.vol, (__half *)a.volh, a.ny, a.onz, a.onx, n, a.maxbits);
  } else {
    if (XT) blend_interleave_at<S>(i, a.vol, a.volg, a.ny, a.onz, a.onx, a.ocx, a.sin_xt_common, n);
    else interleave_at<S>(i, a.vol, a.volg, a.ny, a.onz, a.onx, n);
  }
}

template <int S, bool XT, bool IL>
__global__ void __launch_bounds__(128) fp_fast_batch_kernel(FpBatchDev b) {
  __shared__ __align__(16) FpArgs s_a;
  const int t = load_fp_job(b, &s_a);
  const int gx = s_a.nviews_all, gy = (s_a.nx + 127) / 128;
  fp_fast_body<S, XT, IL>(s_a, t % gx, (t / gx) % gy, t / (gx * gy));
}

template <int S, bool XT>
__global__ void __launch_bounds__(128) fp_half_batch_kernel(FpBatchDev b) {
  __shared__ __align__(16) FpArgs s_a;
  const int t = load_fp_job(b, &s_a);
  const int gx = s_a.nviews_all, gy = (s_a.nx + 127) / 128;
  fp_half_body<S, XT>(s_a, t % gx, (t / gx) % gy, t / (gx * gy));
}

template <int S>
static int launch_half(const FpArgs &a, cudaStream_t st) {
  const size_t nvol = (size_t)a.ny * a.onz * a.onx;
  cudaMemsetAsync(a.maxbits, 0, sizeof(unsigned), st);
  absmax_kernel<<<8 * 148, 256, 0, st>>>(a.vol, nvol, a.maxbits);
  const size_t n = (size_t)((a.ny + S - 1) / S) * a.onz * a.onx;
  const unsigned nb = (unsigned)((n + 255) / 256);
  dim3 grid(a.nviews_all, (a.nx + 127) / 128, (a.ny + S - 1) / S);
  if (a.fast == 2) {  // one x-tilt for all views: blended rows
    blend_interleave_half_kernel<S><<<nb, 256, 0, st>>>(a.vol, (__half *)a.volh, a.ny, a.onz, a.onx, a.ocx,
                                                        a.sin_xt_common, n, a.maxbits);
    fp_half_kernel<S, true><<<grid, 128, 0, st>>>(a);
  } else {
    interleave_half_kernel<S><<<nb, 256, 0, st>>>(a.vol, (__half *)a.volh, a.ny, a.onz, a.onx, n, a.maxbits);
    fp_half_kernel<S, false><<<grid, 128, 0, st>>>(a);
  }
  return 3;
}

template <int S>
static int launch_fast(const FpArgs &a, cudaStream_t st) {
  dim3 grid(a.nviews_all, (a.nx + 127) / 128, (a.ny + S - 1) / S);
  if (a.fast == 2 && a.volg) {
    const size_t n = (size_t)((a.ny + S - 1) / S) * a.onz * a.onx;
    blend_interleave_kernel<S><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a.vol, a.volg, a.ny, a.onz, a.onx,
                                                                          a.ocx, a.sin_xt_common, n);
    fp_fast_kernel<S, true, true><<<grid, 128, 0, st>>>(a);
    return 2;
  } else if (a.fast == 2) {
    fp_fast_kernel<S, true, false><<<grid, 128, 0, st>>>(a);
    return 1;
  } else if (a.volg) {
    const size_t n = (size_t)((a.ny + S - 1) / S) * a.onz * a.onx;
    interleave_kernel<S><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a.vol, a.volg, a.ny, a.onz, a.onx, n);
    fp_fast_kernel<S, false, true><<<grid, 128, 0, st>>>(a);
    return 2;
  }
  fp_fast_kernel<S, false, false><<<grid, 128, 0, st>>>(a);
  return 1;
}

int fp_group_rows(int variant) { return variant == 1 || variant == 3 ? 16 : 8; }

// key = form * 1000 + rows per thread * 10 + x-tilt * 2 + interleaved copy
// (form 1: scaled FP16 copy, 2: FP32 fast kernel)
int fp_batch_key(const FpArgs &a) {
  if ((a.fast == 1 || a.fast == 2) && a.volh) return 1000 + fp_half_rows(a.variant) * 10 + (a.fast == 2 ? 2 : 0) + 1;
  if (a.fast == 1 || a.fast == 2) return 2000 + fp_group_rows(a.variant) * 10 + (a.fast == 2 ? 2 : 0) + (a.volg ? 1 : 0);
  return -1;
}

void fp_batch_blocks(const FpArgs &a, int key, int *absmax, int *copy, int *fp) {
  const int S = (key % 1000) / 10;
  const bool half = key / 1000 == 1, il = (key & 1) != 0;
  const size_t n = (size_t)((a.ny + S - 1) / S) * a.onz * a.onx;
  *absmax = half ? fp_absmax_blocks((size_t)a.ny * a.onz * a.onx) : 0;
  *copy = (half || il) ? (int)((n + 255) / 256) : 0;
  *fp = a.nviews_all * ((a.nx + 127) / 128) * ((a.ny + S - 1) / S);
}

template <int S, bool HALF, bool XT, bool IL>
static int launch_batch_t(const FpArgs *jobs, int njobs, const int *blk_abs, int nabs, const int *blk_copy,
                          int ncopy, const int *blk_fp, int nfp, cudaStream_t st) {
  int k = 0;
  if constexpr (HALF) {
    fp_zero_maxbits_kernel<<<(njobs + 127) / 128, 128, 0, st>>>(jobs, njobs);
    absmax_batch_kernel<<<nabs, 256, 0, st>>>(FpBatchDev{jobs, blk_abs, njobs});
    k += 2;
  }
  if constexpr (HALF || IL) {
    fp_copy_batch_kernel<S, HALF, XT><<<ncopy, 256, 0, st>>>(FpBatchDev{jobs, blk_copy, njobs});
    ++k;
  }
  if constexpr (HALF) fp_half_batch_kernel<S, XT><<<nfp, 128, 0, st>>>(FpBatchDev{jobs, blk_fp, njobs});
  else fp_fast_batch_kernel<S, XT, IL><<<nfp, 128, 0, st>>>(FpBatchDev{jobs, blk_fp, njobs});
  return k + 1;
}

int launch_reproject_batch(int key, const FpArgs *jobs, int njobs, const int *blk_abs, int nabs,
                           const int *blk_copy, int ncopy, const int *blk_fp, int nfp, cudaStream_t st) {
#define TG_FPB(KEY, S, HALF, XT, IL) \
  case KEY: return launch_batch_t<S, HALF, XT, IL>(jobs, njobs, blk_abs, nabs, blk_copy, ncopy, blk_fp, nfp, st);
  switch (key) {
    TG_FPB(1161, 16, true, false, true)
    TG_FPB(1163, 16, true, true, true)
    TG_FPB(1321, 32, true, false, true)
    TG_FPB(1323, 32, true, true, true)
    TG_FPB(2080, 8, false, false, false)
    TG_FPB(2081, 8, false, false, true)
    TG_FPB(2082, 8, false, true, false)
    TG_FPB(2083, 8, false, true, true)
    TG_FPB(2160, 16, false, false, false)
    TG_FPB(2161, 16, false, false, true)
    TG_FPB(2162, 16, false, true, false)
    TG_FPB(2163, 16, false, true, true)
    default: return 0;
  }
#undef TG_FPB
}

// ---- local alignment ----
// The table of corrections: ViewPatches::interpolate (main.rs:172-228) at every
// integer column of every slice of every view, computed once per session with
// the same f32 expressions as local_interp.
__global__ void local_table_kernel(LocalDev L, int nviews, int ny, int onx, float2 *table) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t n = (size_t)nviews * ny * onx;
  if (i >= n) return;
  const int ox = (int)(i % onx);
  const size_t r = i / onx;
  const int iy = (int)(r % ny), v = (int)(r / ny);
  float dx = 0.0f, dy = 0.0f;
  local_interp(L, v, (float)ox, (float)iy, dx, dy);
  table[i] = make_float2(dx, dy);
}

void launch_local_table(const LocalDev &L, int nviews, int ny, int onx, float2 *table, cudaStream_t st) {
  const size_t n = (size_t)nviews * ny * onx;
  local_table_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(L, nviews, ny, onx, table);
}

// dx range of the corrections per (view, slice tile t, column) over the slices that a
// reprojection block of row group t can read when the x-tilt and dy shifts stay
// within one tile: [LB_TILE*(t-1), LB_TILE*(t+2)) clipped to [0, ny)
__global__ void local_bounds_kernel(const float2 *__restrict__ table, int nviews, int ny, int onx, int ntile,
                                    float2 *bnd) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // (v, t, ox)
  const size_t n = (size_t)nviews * ntile * onx;
  if (i >= n) return;
  const int ox = (int)(i % onx);
  const size_t r = i / onx;
  const int t = (int)(r % ntile), v = (int)(r / ntile);
  const int y0 = max(LB_TILE * (t - 1), 0), y1 = min(LB_TILE * (t + 2), ny);
  float mn = 3.40282347e+38f, mx = -3.40282347e+38f;
  for (int iy = y0; iy < y1; ++iy) {
    const float d = __ldg(&table[((size_t)v * ny + iy) * onx + ox]).x;
    mn = fminf(mn, d);
    mx = fmaxf(mx, d);
  }
  bnd[i] = make_float2(mn, mx);
}

void launch_local_bounds(const float2 *table, int nviews, int ny, int onx, float2 *bnd, cudaStream_t st) {
  const int ntile = (ny + LB_TILE - 1) / LB_TILE;
  const size_t n = (size_t)nviews * ntile * onx;
  if (n == 0) return;
  local_bounds_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(table, nviews, ny, onx, ntile, bnd);
}

// Reprojection with local alignment: one thread owns bin p of S (16) rows of one view
// and gathers, per depth, every (column, slice) whose corrected position lands
// in [p-1, p+1) and whose corrected row reaches one of its rows, with the
// reference's weights (main.rs:831-896: with local alignment every sample splits
// over two rows, the last row takes the one-row branch).  The corrections come
// from the session's table; the thread's S row sums live in shared memory (the
// target row depends on the slice's correction).  Order: z, x, slice.
template <int S>
__global__ void __launch_bounds__(128) fp_local_kernel(FpArgs a) {
  static_assert(S == LB_TILE, "row groups are the slice tiles of FpArgs::lbnd");
  __shared__ float sacc[S][128];
  const int tid = threadIdx.x;
  const int v = blockIdx.x;
  const int p = blockIdx.y * blockDim.x + tid;
  const int r0 = blockIdx.z * S;
  if (p >= a.nx) return;
  const int nrows = min(S, a.ny - r0);
  float *out = a.sino + ((size_t)v * a.ny + r0) * a.nx + p;
  if (v >= a.nviews) {  // views without a tilt angle contribute nothing (main.rs:683-686)
    for (int s = 0; s < nrows; ++s) out[(size_t)s * a.nx] = 0.0f;
    return;
  }
#pragma unroll
  for (int s = 0; s < S; ++s) sacc[s][tid] = 0.0f;
  const float4 g = __ldg(&a.vg[v]);
  const float4 g2 = __ldg(&a.vg2[v]);
  const float cos_t = g.x, sin_t = g.y, zf = g.z, cos_xt = g.w, sin_xt = g2.x;
  const float lxmax = g2.y, lymax = g2.z;  // bounds of |dx|, |dy| of this view's corrections
  const float aeff = cos_t * cos_xt;
  const float inv_a = fabsf(aeff) > 1e-3f ? 1.0f / aeff : 0.0f;
  const float pf = (float)p;
  for (int oz = 0; oz < a.onz; ++oz) {
    const float dz = __fsub_rn((float)oz, a.cz);
    const float t2 = __fmul_rn(__fmul_rn(dz, sin_t), zf);
    int lo = 0, hi = a.onx - 1;
    if (inv_a != 0.0f) {
      // columns whose corrected position xb + dx_local can lie in [p-1, p+1) with
      // |dx_local| <= lxmax; the margin (0.05 px, in columns, plus 1e-3 column) covers
      // the f32 rounding of the positions (a few ulp of values below 2^14) and of 1/a
      const float base = a.cx + t2;
      const float d1 = (pf - 1.0f - lxmax - base) * inv_a, d2 = (pf + 1.0f + lxmax - base) * inv_a;
      const float m = 0.05f * fabsf(inv_a) + 1e-3f;
      const float dmin = fmaxf(fminf(d1, d2) + a.ocx - m, -1.0f), dmax = fminf(fmaxf(d1, d2) + a.ocx + m, (float)a.onx);
      lo = max((int)ceilf(dmin), 0);
      hi = min((int)floorf(dmax), a.onx - 1);
    }
    for (int ox = lo; ox <= hi; ++ox) {
      const float dx = __fsub_rn((float)ox, a.ocx);
      const float xb = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(dx, cos_t), cos_xt), t2), a.cx);
      const float yoff = __fmul_rn(dx, sin_xt);
      // slices whose corrected row iy + yoff + dy_local (|dy_local| <= lymax) lies in
      // [r0 - 1, r0 + nrows): the rows [r0, r0 + nrows) receive from floor rows r0-1 ..
      // r0+nrows-1; margin 0.01 row for rounding
      const int iy_lo = max((int)ceilf((float)r0 - 1.0f - yoff - lymax - 0.01f), 0);
      const int iy_hi = min((int)floorf((float)(r0 + nrows) - yoff + lymax + 0.01f), a.ny - 1);
      // skip the column when no slice of the window can land in [p-1, p+1): f32 addition
      // is monotone, so xb + dx lies in [RN(xb + dx_min), RN(xb + dx_max)] for every slice
      // whose dx the tile bound covers
      if (a.lbnd && iy_lo >= max(r0 - LB_TILE, 0) && iy_hi < min(r0 + 2 * LB_TILE, a.ny)) {
        const float2 b = __ldg(&a.lbnd[((size_t)v * gridDim.z + blockIdx.z) * a.onx + ox]);
        if (__fadd_rn(xb, b.y) < pf - 1.0f || __fadd_rn(xb, b.x) >= pf + 1.0f) continue;
      }
      for (int iy = iy_lo; iy <= iy_hi; ++iy) {
        const float2 l = __ldg(&a.loc.table[((size_t)v * a.ny + iy) * a.loc.table_nx + ox]);
        const float x = __fadd_rn(xb, l.x);
        const float fx = floorf(x);
        if (!(fx >= 0.0f && fx + 1.0f < (float)a.nx)) continue;
        const int x0 = (int)fx;
        if (x0 != p && x0 != p - 1) continue;
        const float sy = __fadd_rn(__fadd_rn((float)iy, yoff), l.y);
        const float fsy = floorf(sy);
        if (!(fsy >= 0.0f && fsy < (float)a.ny)) continue;
        const int s0 = (int)fsy - r0;
        if (s0 < -1 || s0 >= nrows) continue;
        const float frac = __fsub_rn(x, fx);
        const float val = __ldg(a.vol + ((size_t)iy * a.onz + oz) * a.onx + ox);
        const float c = x0 == p ? __fmul_rn(val, __fsub_rn(1.0f, frac)) : __fmul_rn(val, frac);
        if ((int)fsy + 1 < a.ny) {  // two rows (always with local alignment, main.rs:877)
          const float syf = __fsub_rn(sy, fsy);
          if (s0 >= 0) sacc[s0][tid] = __fadd_rn(sacc[s0][tid], __fmul_rn(c, __fsub_rn(1.0f, syf)));
          if (s0 + 1 < nrows) sacc[s0 + 1][tid] = __fadd_rn(sacc[s0 + 1][tid], __fmul_rn(c, syf));
        } else if (s0 >= 0) {
          sacc[s0][tid] = __fadd_rn(sacc[s0][tid], c);
        }
      }
    }
  }
  for (int s = 0; s < nrows; ++s) out[(size_t)s * a.nx] = sacc[s][tid];
}

int launch_reproject(const FpArgs &a, cudaStream_t st) {
  if ((a.fast == 1 || a.fast == 2) && a.volh)
    return fp_half_rows(a.variant) == 32 ? launch_half<32>(a, st) : launch_half<16>(a, st);
  if (a.fast) return fp_group_rows(a.variant) == 16 ? launch_fast<16>(a, st) : launch_fast<8>(a, st);
  if (a.has_local && a.loc.table) {
    constexpr int S = 16;
    dim3 grid(a.nviews_all, (a.nx + 127) / 128, (a.ny + S - 1) / S);
    fp_local_kernel<S><<<grid, 128, 0, st>>>(a);
    return 1;
  }
  dim3 grid((a.nx + 127) / 128, a.ny, a.nviews_all);
  fp_kernel<<<grid, 128, 0, st>>>(a);
  return 1;
}

}  // namespace tg
