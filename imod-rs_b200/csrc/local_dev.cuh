// local_dev.cuh -- device restatement of the local-alignment interpolation.
#pragma once
#include "tg_internal.h"

namespace tg {

// ---------------------------------------------------------------------------
// Local alignment: ViewPatches::interpolate (apps/tilt/src/main.rs:172-228)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void find_bracket(const float *pos, int n, float val, int &idx,
                                             float &frac) {
  if (n == 1) { idx = 0; frac = 0.0f; return; }
  int lo = 0, hi = n - 1;
  if (val <= pos[lo]) { idx = 0; frac = 0.0f; return; }
  if (val >= pos[hi]) { idx = hi; frac = 0.0f; return; }
  while (hi - lo > 1) {
    int mid = (lo + hi) / 2;
    if (pos[mid] <= val) lo = mid; else hi = mid;
  }
  float span = __fsub_rn(pos[hi], pos[lo]);
  frac = span > 1e-12f ? __fdiv_rn(__fsub_rn(val, pos[lo]), span) : 0.0f;
  idx = lo;
}
__device__ __forceinline__ float lerp_ref(float a, float b, float t) {
  return __fadd_rn(a, __fmul_rn(t, __fsub_rn(b, a)));
}
__device__ __forceinline__ bool local_interp(const LocalDev &L, int v, float x, float y, float &odx, float &ody) {
  const int4 vi = L.vinfo[v];
  if (vi.y == 0 || vi.w == 0) { odx = 0.0f; ody = 0.0f; return false; }
  int ix0, iy0;
  float fx, fy;
  find_bracket(L.xs + vi.x, vi.y, x, ix0, fx);
  find_bracket(L.ys + vi.z, vi.w, y, iy0, fy);
  const int nx = vi.y, ny = vi.w;
  const int ix1 = min(ix0 + 1, nx - 1), iy1 = min(iy0 + 1, ny - 1);
  const float *gx = L.gdx + L.goff[v], *gy = L.gdy + L.goff[v];
  odx = lerp_ref(lerp_ref(gx[iy0 * nx + ix0], gx[iy0 * nx + ix1], fx),
                 lerp_ref(gx[iy1 * nx + ix0], gx[iy1 * nx + ix1], fx), fy);
  ody = lerp_ref(lerp_ref(gy[iy0 * nx + ix0], gy[iy0 * nx + ix1], fx),
                 lerp_ref(gy[iy1 * nx + ix0], gy[iy1 * nx + ix1], fx), fy);
  return true;
}

// The correction at column ox (an integer column, as every caller passes) of
// slice iy: from the per-session table when there is one.
__device__ __forceinline__ bool local_corr(const LocalDev &L, int v, int ox, int iy, int ny, float &odx,
                                           float &ody) {
  if (L.table) {
    const float2 t = __ldg(&L.table[((size_t)v * ny + iy) * L.table_nx + ox]);
    odx = t.x;
    ody = t.y;
    return true;  // (0, 0) for views without patches: adding it changes nothing
  }
  return local_interp(L, v, (float)ox, (float)iy, odx, ody);
}

}  // namespace tg
