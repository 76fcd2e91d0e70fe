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
#include "tg_internal.h"
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
          if (a.has_local) use_l = local_interp(a.loc, v, (float)ox, (float)iy, ldx, ldy);
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

// Fast reprojection (no x-tilt, no local alignment, every view with cos > 0.05):
// slice iy feeds only sinogram row iy, and a voxel's position x does not depend
// on the slice, so one thread owns bin p of S consecutive rows and shares the
// candidate search among them.  For each depth the columns whose exact
// position lies in [p-1, p+1) are found by an estimate from 1/cos corrected
// with exact evaluations (x is non-decreasing in the column), then visited in
// increasing column order: the per-bin order (z ascending, x ascending) of the
// reference's serial splat, so every bin is bit-identical to it.
template <int S>
__global__ void __launch_bounds__(128) fp_fast_kernel(FpArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int r0 = blockIdx.y * S, v = blockIdx.z;
  if (p >= a.nx) return;
  const float4 g = __ldg(&a.vg[v]);
  const float cos_t = g.x, sin_t = g.y, zf = g.z;
  const float inv_a = 1.0f / cos_t;
  const float lo_t = (float)(p - 1), hi_t = (float)(p + 1);
  const size_t sstride = (size_t)a.onz * a.onx;
  const float *vol0 = a.vol + (size_t)r0 * sstride;
  int nrows = min(S, a.ny - r0);
  float acc[S];
#pragma unroll
  for (int s = 0; s < S; ++s) acc[s] = 0.0f;
  auto X = [&](int ox, float t2) {  // ((dx*cos)*1 + t2) + cx, exactly as main.rs:842
    const float dx = __fsub_rn((float)ox, a.ocx);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, cos_t), t2), a.cx);
  };
  for (int oz = 0; oz < a.onz; ++oz) {
    const float dz = __fsub_rn((float)oz, a.cz);
    const float t2 = __fmul_rn(__fmul_rn(dz, sin_t), zf);
    // first column whose position is >= p-1
    int lo = (int)floorf((lo_t - a.cx - t2) * inv_a + a.ocx) - 1;
    lo = min(max(lo, 0), a.onx);
    while (lo > 0 && X(lo - 1, t2) >= lo_t) --lo;
    while (lo < a.onx && X(lo, t2) < lo_t) ++lo;
    const float *vrow = vol0 + (size_t)oz * a.onx;
    for (int ox = lo; ox < a.onx; ++ox) {
      const float x = X(ox, t2);
      if (!(x < hi_t)) break;
      const float tt = __fadd_rd(x, FMAGIC);
      const int x0 = (int)(__float_as_uint(tt) - FMAGIC_BITS);
      if ((unsigned)x0 > (unsigned)(a.nx - 2)) continue;  // px0 >= 0 && px0 + 1 < nx
      const float frac = __fsub_rn(x, __fsub_rn(tt, FMAGIC));
      const float w = x0 == p ? __fsub_rn(1.0f, frac) : frac;
#pragma unroll
      for (int s = 0; s < S; ++s)
        if (s < nrows) acc[s] = __fadd_rn(acc[s], __fmul_rn(__ldg(vrow + (size_t)s * sstride + ox), w));
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s)
    if (s < nrows) a.sino[((size_t)v * a.ny + r0 + s) * a.nx + p] = acc[s];
}

void launch_reproject(const FpArgs &a, cudaStream_t st) {
  if (a.fast) {
    constexpr int S = 8;
    dim3 grid((a.nx + 127) / 128, (a.ny + S - 1) / S, a.nviews);
    fp_fast_kernel<S><<<grid, 128, 0, st>>>(a);
    return;
  }
  dim3 grid((a.nx + 127) / 128, a.ny, a.nviews_all);
  fp_kernel<<<grid, 128, 0, st>>>(a);
}

}  // namespace tg
