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

void launch_reproject(const FpArgs &a, cudaStream_t st) {
  dim3 grid((a.nx + 127) / 128, a.ny, a.nviews_all);
  fp_kernel<<<grid, 128, 0, st>>>(a);
}

}  // namespace tg
