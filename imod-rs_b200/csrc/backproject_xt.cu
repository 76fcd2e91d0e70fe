// backproject_xt.cu -- back-projection with x-axis tilt (no local alignment).
//
// Semantics: backproject_all, apps/tilt/src/main.rs:756-828.  With an x-axis
// tilt the sample row of voxel (ox, iy) is sample_y = iy + dx*sin(x-tilt); the
// reference samples rows floor(sample_y) and floor(sample_y)+1 at the same
// position x (sample_row_with_fill, main.rs:386-406) and blends them with the
// fraction of sample_y (two-row branch), or takes one row (the last row, or a
// zero offset).  x = ((dx*cos)*cos_xt + (dz*sin)*zf) + cx does not depend on
// the slice.
//
// Tile: S slices x 32 columns x (4 warps * K) depths; one thread owns one
// column and K depths of all S slices.  Per view the block stages, in shared
// memory, the rows [iy0 + floor(min yoff), ...] that its slices can reach, over
// the window of elements its (x, z) corners span (cp.async, double-buffered
// across views).  For one sample position the thread interpolates the S+2 rows
// its slices can read once each in x and then blends consecutive pairs per
// slice: the row interpolation and the blend are the reference's f32
// expressions, and a row shared by two slices is the same value either way, so
// FP32 staging is bit-identical to the reference (and to bp_general_kernel).
// f32 rounding of iy + yoff can put a slice's floor one row above the nominal
// iy + floor(yoff); its fraction is then 0 and the pair is selected one row up.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "tg_internal.h"

namespace tg {

namespace {

constexpr float XMAGIC = 12582912.0f;  // 1.5 * 2^23: x + XMAGIC rounded down holds floor(x) in its low bits
constexpr uint32_t XMAGIC_BITS = 0x4B400000u;
constexpr int XT_TX = 32, XT_NW = 4, XT_WMAX = 72;

__device__ __forceinline__ uint32_t su32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(src), "n"(BYTES));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// packed FP32x2 multiply: each lane is the IEEE round-to-nearest f32 product
__device__ __forceinline__ float2 mul2f(float a0, float a1, float b0, float b1) {
  uint64_t d, x, y;
  asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "f"(a0), "f"(a1));
  asm("mov.b64 %0, {%1, %2};" : "=l"(y) : "f"(b0), "f"(b1));
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(y));
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(d));
  return r;
}
template <int OFF>
__device__ __forceinline__ float2 lds_f2(uint32_t a) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0,%1}, [%2+%3];" : "=f"(v.x), "=f"(v.y) : "r"(a), "n"(OFF));
  return v;
}
template <int OFF>
__device__ __forceinline__ uint32_t lds_u32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1+%2];" : "=r"(v) : "r"(a), "n"(OFF));
  return v;
}
template <int I, int N, class F>
__device__ __forceinline__ void sfor(F &&f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    sfor<I + 1, N>(f);
  }
}

// the window of one view for this tile: element range [kmin, kmin+W) and rows [rbase, rbase+R)
struct XtWindow {
  int kmin, W, rbase, R;
};

__device__ __forceinline__ float xpos(float dx, float dz, float4 g, float cx) {
  return __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(dx, g.x), g.w), __fmul_rn(__fmul_rn(dz, g.y), g.z)), cx);
}

template <int S>
__device__ __forceinline__ XtWindow xt_window(const BpArgs &a, float4 g, float sin_xt, float dx0, float dx1,
                                              float dz0, float dz1, int iy0) {
  // x is monotone in dx (cos*cos_xt > 0) and in dz: the corners bound the tile
  const float x00 = xpos(dx0, dz0, g, a.cx), x01 = xpos(dx0, dz1, g, a.cx);
  const float x10 = xpos(dx1, dz0, g, a.cx), x11 = xpos(dx1, dz1, g, a.cx);
  const float xmin = fminf(fminf(x00, x01), fminf(x10, x11)), xmax = fmaxf(fmaxf(x00, x01), fmaxf(x10, x11));
  XtWindow w;
  w.kmin = max((int)floorf(xmin), -a.padL);
  const int kmax = min((int)floorf(xmax), a.PW - a.padL - 1);
  w.W = kmax - w.kmin + 1;
  const float y0 = __fmul_rn(dx0, sin_xt), y1 = __fmul_rn(dx1, sin_xt);
  const int nlo = (int)floorf(fminf(y0, y1)), nhi = (int)floorf(fmaxf(y0, y1));
  w.rbase = iy0 + nlo;
  w.R = S + 2 + (nhi - nlo);
  return w;
}

}  // namespace

template <int STORE, int S, int K>
__global__ void __launch_bounds__(XT_TX * XT_NW, 5) bp_xtilt_kernel(BpArgs a) {
  constexpr int TZ = XT_NW * K, RMAX = S + 8;
  constexpr int EB = STORE == TG_STORE_FP32 ? 8 : 4;
  __shared__ __align__(16) unsigned char stage[2][RMAX * XT_WMAX * EB];
  const int tid = threadIdx.x, lane = tid & 31, wz = tid >> 5;
  const int ox = blockIdx.x * XT_TX + lane, oz0 = blockIdx.y * TZ, iy0 = blockIdx.z * S;
  const int oxc = min(ox, a.onx - 1);
  const float dx = __fsub_rn((float)oxc, a.ocx);
  const float dx0 = __fsub_rn((float)(blockIdx.x * XT_TX), a.ocx);
  const float dx1 = __fsub_rn((float)min((int)blockIdx.x * XT_TX + XT_TX - 1, a.onx - 1), a.ocx);
  const float dz0 = __fsub_rn((float)oz0, a.cz);
  const float dz1 = __fsub_rn((float)min(oz0 + TZ - 1, a.onz - 1), a.cz);
  float dz[K];
#pragma unroll
  for (int j = 0; j < K; ++j) dz[j] = __fsub_rn((float)min(oz0 + wz + j * XT_NW, a.onz - 1), a.cz);
  float acc[S][K];
#pragma unroll
  for (int i = 0; i < S; ++i)
#pragma unroll
    for (int j = 0; j < K; ++j) acc[i][j] = 0.0f;
  const uint8_t *pairs = reinterpret_cast<const uint8_t *>(a.pairs);

  auto stage_view = [&](int v, int buf) {
    const XtWindow w = xt_window<S>(a, __ldg(&a.vg[v]), __ldg(&a.vg2[v]).x, dx0, dx1, dz0, dz1, iy0);
    const int W = min(w.W, XT_WMAX), R = min(w.R, RMAX);
    const uint32_t base = su32(stage[buf]);
    for (int r = wz; r < R; r += XT_NW) {  // one warp per row, lanes along the row
      const int row = w.rbase + r;
      if (row < 0 || row >= a.ny) continue;  // never read: such slices take no sample there
      const uint8_t *src = pairs + (((size_t)v * a.rows_alloc + row) * a.PW + (w.kmin + a.padL)) * EB;
      for (int c = lane; c < W; c += 32)
        cp_async<EB>(base + (uint32_t)((r * XT_WMAX + c) * EB), src + (size_t)c * EB);
    }
    cp_commit();
  };

  if (a.nviews > 0) stage_view(0, 0);
  for (int v = 0; v < a.nviews; ++v) {
    const int buf = v & 1;
    if (v + 1 < a.nviews) {
      stage_view(v + 1, buf ^ 1);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
    const float4 g = __ldg(&a.vg[v]);
    const float sin_xt = __ldg(&a.vg2[v]).x;
    const XtWindow w = xt_window<S>(a, g, sin_xt, dx0, dx1, dz0, dz1, iy0);
    if (w.W > XT_WMAX || w.R > RMAX) {  // excluded by the host; flagged, and no shared read past the stage
      if (tid == 0) atomicOr(a.err, 2);
      __syncthreads();
      continue;
    }
    const float t1 = __fmul_rn(__fmul_rn(dx, g.x), g.w);
    const float yoff = __fmul_rn(dx, sin_xt);
    const float fn = floorf(yoff);
    const int rb = iy0 + (int)fn - w.rbase;  // staged row of slice 0's nominal lower row
    const bool yoff_nz = fabsf(yoff) > 1e-6f;
    // per slice: fraction, one-row/two-row branch, and whether f32 rounding moved the floor up
    float fy[S], omfy[S];
    uint32_t two = 0, off = 0, take = 0;
#pragma unroll
    for (int i = 0; i < S; ++i) {
      const int iy = iy0 + i;
      const float sy = __fadd_rn((float)iy, yoff);
      const float fly = floorf(sy);
      fy[i] = __fsub_rn(sy, fly);
      omfy[i] = __fsub_rn(1.0f, fy[i]);
      const bool yin = fly >= 0.0f && fly < (float)a.ny;
      const int sy0 = (int)fly;
      if (yin && iy < a.ny) take |= 1u << i;
      if (yin && sy0 + 1 < a.ny && yoff_nz) two |= 1u << i;
      if (sy0 != iy + (int)fn) off |= 1u << i;
    }
    const uint32_t sb = su32(stage[buf]) + (uint32_t)(rb * XT_WMAX * EB);  // row rb+r at +r*XT_WMAX*EB
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const float t2 = __fmul_rn(__fmul_rn(dz[j], g.y), g.z);
      const float x = __fadd_rn(__fadd_rn(t1, t2), a.cx);
      const float tt = __fadd_rd(x, XMAGIC);
      float f = __fsub_rn(x, __fsub_rn(tt, XMAGIC));
      const int k = (int)(__float_as_uint(tt) - XMAGIC_BITS);
      const uint32_t ca = sb + (uint32_t)(min(max(k - w.kmin, 0), w.W - 1) * EB);  // in the window by construction
      float rv[S + 2];  // the S+2 rows this column's slices can read, interpolated in x
      if constexpr (STORE == TG_STORE_FP32) {
        if ((unsigned)k > (unsigned)(a.nx - 2)) f = 0.0f;  // pads and element nx-1 hold (fill, fill)
        const float omf = __fsub_rn(1.0f, f);
        sfor<0, S + 2>([&](auto rc) {
          constexpr int r = decltype(rc)::value;
          const float2 p = lds_f2<r * XT_WMAX * 8>(ca);
          const float2 q = mul2f(p.x, p.y, omf, f);  // row[k]*(1-f), row[k+1]*f, each rounded
          rv[r] = __fadd_rn(q.x, q.y);
        });
      } else {
        sfor<0, S + 2>([&](auto rc) {
          constexpr int r = decltype(rc)::value;
          const uint32_t e = lds_u32<r * XT_WMAX * 4>(ca);
          float a0, d0;
          if constexpr (STORE == TG_STORE_FP16) {
            a0 = __half2float(__ushort_as_half((uint16_t)(e & 0xffff)));
            d0 = __half2float(__ushort_as_half((uint16_t)(e >> 16)));
          } else {
            a0 = __bfloat162float(__ushort_as_bfloat16((uint16_t)(e & 0xffff)));
            d0 = __bfloat162float(__ushort_as_bfloat16((uint16_t)(e >> 16)));
          }
          rv[r] = fmaf(f, d0, a0);
        });
      }
      if (off == 0) {  // every floor at its nominal row (the usual case)
#pragma unroll
        for (int i = 0; i < S; ++i) {
          const float2 q = mul2f(rv[i], rv[i + 1], omfy[i], fy[i]);
          const float val = ((two >> i) & 1u) ? __fadd_rn(q.x, q.y) : rv[i];
          if ((take >> i) & 1u) acc[i][j] = __fadd_rn(acc[i][j], val);
        }
      } else {
#pragma unroll
        for (int i = 0; i < S; ++i) {
          const bool up = (off >> i) & 1u;
          const float v0 = up ? rv[i + 1] : rv[i];
          const float v1 = up ? rv[i + 2] : rv[i + 1];
          const float2 q = mul2f(v0, v1, omfy[i], fy[i]);
          const float val = ((two >> i) & 1u) ? __fadd_rn(q.x, q.y) : v0;
          if ((take >> i) & 1u) acc[i][j] = __fadd_rn(acc[i][j], val);
        }
      }
    }
    __syncthreads();  // buffer `buf` is restaged for view v+2
  }

  // epilogue: the same transform and statistics as the other back-projectors
  const bool xok = ox < a.onx;
  __shared__ float red_mm[S][XT_NW][2];
  __shared__ double red_s[S][XT_NW];
#pragma unroll
  for (int i = 0; i < S; ++i) {
    const int iy = iy0 + i;
    float mn = 3.40282347e+38f, mx = -3.40282347e+38f;
    double sum = 0.0;
    if (iy < a.ny) {
      // SIRT update: the slice's K old values are loaded before any of its stores
      float old[K];
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const int oz = oz0 + wz + j * XT_NW;
        old[j] = (a.mode == 2 && xok && oz < a.onz) ? a.vol[((size_t)iy * a.onz + oz) * a.onx + ox] : 0.0f;
      }
#pragma unroll
      for (int j = 0; j < K; ++j) {
        const int oz = oz0 + wz + j * XT_NW;
        if (xok && oz < a.onz) {
          const size_t idx = ((size_t)iy * a.onz + oz) * a.onx + ox;
          const float vv = __fmul_rn(acc[i][j], a.inv_n);
          if (a.mode == 0) {
            const float y = __fadd_rn(__fmul_rn(__fmul_rn(vv, a.dw), a.os), a.oa);
            a.vol[idx] = y;
            mn = fminf(mn, y);
            mx = fmaxf(mx, y);
            sum += (double)y;
          } else if (a.mode == 1) {
            a.vol[idx] = vv;
          } else {
            a.vol[idx] = __fadd_rn(old[j], __fmul_rn(a.relax, vv));
          }
        }
      }
    }
    if (a.mode == 0) {
      for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
      }
      if (lane == 0) {
        red_mm[i][wz][0] = mn;
        red_mm[i][wz][1] = mx;
        red_s[i][wz] = sum;
      }
    }
  }
  if (a.mode == 0) {
    __syncthreads();
    if (tid < S && iy0 + tid < a.ny) {
      StatPartial p;
      p.mn = 3.40282347e+38f;
      p.mx = -3.40282347e+38f;
      p.sum = 0.0;
      for (int q = 0; q < XT_NW; ++q) {
        p.mn = fminf(p.mn, red_mm[tid][q][0]);
        p.mx = fmaxf(p.mx, red_mm[tid][q][1]);
        p.sum += red_s[tid][q];
      }
      a.partial[(size_t)(iy0 + tid) * (gridDim.x * gridDim.y) + blockIdx.x + blockIdx.y * gridDim.x] = p;
    }
  }
}

// Row-sum form of the x-tilt back-projection (all views share one x-tilt).
// With a common x-tilt the row pair and fraction of voxel (ox, iy) are the same
// in every view, so the reference's sum over views of v0*(1-f) + v1*f
// (main.rs:802-817, 1045-1063) is B[sy0]*(1-f) + B[sy0+1]*f, B[r] the view sum
// of the row-r samples: the fast kernel's no-x-tilt pass with x =
// ((dx*cos)*cos_xt + (dz*sin)*zf) + cx, which already carries the 1/N.  The row
// choice below is the reference's f32 expression; only the order of the f32
// sums differs.  Block (t, iy): depths [onz*t/XB_TILES, onz*(t+1)/XB_TILES) of
// slice iy, a warp on 32 consecutive columns of one depth row (coalesced);
// slices run in order so the rows that neighbouring slices share stay in L2.
template <int MODE>
__global__ void __launch_bounds__(256) xt_blend_kernel(BpArgs a, const float *__restrict__ rows, float sin_xt) {
  const int t = blockIdx.x, iy = blockIdx.y;
  const int oz0 = (int)((long long)a.onz * t / XB_TILES), oz1 = (int)((long long)a.onz * (t + 1) / XB_TILES);
  const size_t sl = (size_t)a.onz * a.onx;
  float mn = 3.40282347e+38f, mx = -3.40282347e+38f;
  double sum = 0.0;
  const float fiy = (float)iy;
  for (int ox = threadIdx.x; ox < a.onx; ox += blockDim.x) {
    const float yoff = __fmul_rn(__fsub_rn((float)ox, a.ocx), sin_xt);
    const float sy = __fadd_rn(fiy, yoff);
    const float fl = floorf(sy);
    const int sy0 = (int)fl;
    const float fr = __fsub_rn(sy, fl);
    const bool two = sy0 >= 0 && sy0 + 1 < a.ny && fabsf(yoff) > 1e-6f;
    const bool one = !two && sy0 >= 0 && sy0 < a.ny;
    const float w0 = __fsub_rn(1.0f, fr);
    const float *b0 = rows + ((two || one) ? (size_t)sy0 * sl : 0) + ox;
    float *out = a.vol + (size_t)iy * sl + ox;
    auto blend = [&](size_t o) {
      float v = 0.0f;
      if (two) v = __fadd_rn(__fmul_rn(__ldg(b0 + o), w0), __fmul_rn(__ldg(b0 + sl + o), fr));
      else if (one) v = __ldg(b0 + o);
      return v;
    };
    if (MODE == 2) {
      // vol += relax * v, four depths at a time: their old values are loaded
      // before any of their stores (a store through out could alias a later
      // load as far as the compiler knows, so one update at a time would wait
      // for each load's round trip to HBM in turn)
      int oz = oz0;
      for (; oz + 4 <= oz1; oz += 4) {
        float old[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) old[u] = out[(size_t)(oz + u) * a.onx];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const size_t o = (size_t)(oz + u) * a.onx;
          out[o] = __fadd_rn(old[u], __fmul_rn(a.relax, blend(o)));
        }
      }
      for (; oz < oz1; ++oz) {
        const size_t o = (size_t)oz * a.onx;
        out[o] = __fadd_rn(out[o], __fmul_rn(a.relax, blend(o)));
      }
      continue;
    }
#pragma unroll 4
    for (int oz = oz0; oz < oz1; ++oz) {
      const size_t o = (size_t)oz * a.onx;
      const float v = blend(o);
      if (MODE == 0) {
        const float y = __fadd_rn(__fmul_rn(__fmul_rn(v, a.dw), a.os), a.oa);
        out[o] = y;
        mn = fminf(mn, y);
        mx = fmaxf(mx, y);
        sum += (double)y;
      } else {  // MODE 1
        out[o] = v;
      }
    }
  }
  if (MODE == 0) {
    __shared__ float rmn[8], rmx[8];
    __shared__ double rs[8];
    for (int o = 16; o > 0; o >>= 1) {
      mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { rmn[w] = mn; rmx[w] = mx; rs[w] = sum; }
    __syncthreads();
    if (threadIdx.x == 0) {
      StatPartial p;
      p.mn = rmn[0];
      p.mx = rmx[0];
      p.sum = rs[0];
      for (int k = 1; k < 8; ++k) { p.mn = fminf(p.mn, rmn[k]); p.mx = fmaxf(p.mx, rmx[k]); p.sum += rs[k]; }
      a.partial[(size_t)iy * XB_TILES + t] = p;
    }
  }
}

int launch_xt_blend(const BpArgs &a, const float *rows, float sin_xt, cudaStream_t st, int *ntiles) {
  if (ntiles) *ntiles = XB_TILES;
  if (a.ny <= 0 || a.onx <= 0 || a.onz <= 0) return TG_OK;
  if (a.ny > 65535) { set_error("more than 65535 rows"); return TG_ERR_UNSUPPORTED; }
  const dim3 grid(XB_TILES, a.ny);
  if (a.mode == 0) xt_blend_kernel<0><<<grid, 256, 0, st>>>(a, rows, sin_xt);
  else if (a.mode == 1) xt_blend_kernel<1><<<grid, 256, 0, st>>>(a, rows, sin_xt);
  else xt_blend_kernel<2><<<grid, 256, 0, st>>>(a, rows, sin_xt);
  return TG_OK;
}

bool bp_xtilt_supported(int onx, float max_abs_sin_xt, float max_x_extent_per_tile) {
  (void)onx;
  // rows a 32-column tile can reach: S + 2 + (nhi - nlo) <= S + 8, and the element window <= 72
  return max_abs_sin_xt * (XT_TX - 1) <= 5.0f && max_x_extent_per_tile <= (float)(XT_WMAX - 3);
}

int launch_bp_xtilt(const BpArgs &a, int store, cudaStream_t st, int *ntiles) {
  constexpr int S = 8, K = 4, TZ = XT_NW * K;
  dim3 grid((a.onx + XT_TX - 1) / XT_TX, (a.onz + TZ - 1) / TZ, (a.ny + S - 1) / S);
  if (ntiles) *ntiles = grid.x * grid.y;
  if (store == TG_STORE_FP32) bp_xtilt_kernel<TG_STORE_FP32, S, K><<<grid, XT_TX * XT_NW, 0, st>>>(a);
  else if (store == TG_STORE_FP16) bp_xtilt_kernel<TG_STORE_FP16, S, K><<<grid, XT_TX * XT_NW, 0, st>>>(a);
  else bp_xtilt_kernel<TG_STORE_BF16, S, K><<<grid, XT_TX * XT_NW, 0, st>>>(a);
  return TG_OK;
}

}  // namespace tg
