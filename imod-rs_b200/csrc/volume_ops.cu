// volume_ops.cu -- volume passes after back-projection.
//
//   lowpass3d (fake SIRT): apps/tilt/src/main.rs:493-538, separable 3-tap box
//     filter in x, then z, then y, clamped at the edges, (a+b+c)/3 in f32.
//   output transform + statistics: apps/tilt/src/main.rs:1077-1093 with
//     min_max_mean (crates/imod-math/src/stats.rs:844-861): per slice min, max
//     and an f64 sum; the header mean is sum_slices(f32 slice mean as f64 *
//     slice size) / total.  Partial sums are per (slice, tile) and reduced in a
//     fixed order, so the statistics are deterministic.
#include <cuda_fp16.h>

#include <algorithm>

#include "tg_internal.h"

namespace tg {

__global__ void lp_x_kernel(const float *__restrict__ in, float *__restrict__ out, int onx,
                            size_t nrows) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t n = nrows * onx;
  if (i >= n) return;
  int ox = (int)(i % onx);
  size_t r = i - ox;
  int x0 = ox > 0 ? ox - 1 : 0, x2 = ox + 1 < onx ? ox + 1 : onx - 1;
  out[i] = __fdiv_rn(__fadd_rn(__fadd_rn(in[r + x0], in[r + ox]), in[r + x2]), 3.0f);
}
__global__ void lp_z_kernel(const float *__restrict__ in, float *__restrict__ out, int onx, int onz,
                            int ny) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t sl = (size_t)onx * onz;
  if (i >= sl * ny) return;
  size_t iy = i / sl, rem = i - iy * sl;
  int oz = (int)(rem / onx), ox = (int)(rem - (size_t)oz * onx);
  int z0 = oz > 0 ? oz - 1 : 0, z2 = oz + 1 < onz ? oz + 1 : onz - 1;
  const float *b = in + iy * sl;
  out[i] = __fdiv_rn(__fadd_rn(__fadd_rn(b[(size_t)z0 * onx + ox], b[(size_t)oz * onx + ox]),
                               b[(size_t)z2 * onx + ox]),
                     3.0f);
}
__global__ void lp_y_kernel(const float *__restrict__ in, float *__restrict__ out, size_t sl,
                            int ny) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= sl * ny) return;
  size_t iy = i / sl, idx = i - iy * sl;
  size_t y0 = iy > 0 ? iy - 1 : 0, y2 = iy + 1 < (size_t)ny ? iy + 1 : ny - 1;
  out[i] = __fdiv_rn(__fadd_rn(__fadd_rn(in[y0 * sl + idx], in[iy * sl + idx]), in[y2 * sl + idx]), 3.0f);
}

// vol -> tmp (x) -> vol (z) -> tmp (y) -> copy back to vol
void launch_lowpass(float *vol, float *tmp, int onx, int onz, int ny, cudaStream_t st) {
  size_t sl = (size_t)onx * onz, n = sl * ny;
  unsigned blocks = (unsigned)((n + 255) / 256);
  lp_x_kernel<<<blocks, 256, 0, st>>>(vol, tmp, onx, (size_t)onz * ny);
  lp_z_kernel<<<blocks, 256, 0, st>>>(tmp, vol, onx, onz, ny);
  lp_y_kernel<<<blocks, 256, 0, st>>>(vol, tmp, sl, ny);
  cudaMemcpyAsync(vol, tmp, n * sizeof(float), cudaMemcpyDeviceToDevice, st);
}

// grid (tiles, ny): block b of slice iy transforms a contiguous chunk
constexpr int TS_TILES = 64;
__global__ void __launch_bounds__(256) transform_stats_kernel(float *vol, size_t sl, float dw,
                                                              float os, float oa,
                                                              StatPartial *partial) {
  const int t = blockIdx.x, iy = blockIdx.y;
  float *s = vol + (size_t)iy * sl;
  size_t c0 = sl * t / TS_TILES, c1 = sl * (t + 1) / TS_TILES;
  float mn = 3.40282347e+38f, mx = -3.40282347e+38f;
  double sum = 0.0;
  for (size_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
    float y = __fadd_rn(__fmul_rn(__fmul_rn(s[i], dw), os), oa);
    s[i] = y;
    mn = fminf(mn, y);
    mx = fmaxf(mx, y);
    sum += (double)y;
  }
  __shared__ float rmn[8], rmx[8];
  __shared__ double rs[8];
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
  }
  int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { rmn[w] = mn; rmx[w] = mx; rs[w] = sum; }
  __syncthreads();
  if (threadIdx.x == 0) {
    StatPartial p;
    p.mn = rmn[0]; p.mx = rmx[0]; p.sum = rs[0];
    for (int k = 1; k < 8; ++k) { p.mn = fminf(p.mn, rmn[k]); p.mx = fmaxf(p.mx, rmx[k]); p.sum += rs[k]; }
    partial[(size_t)iy * TS_TILES + t] = p;
  }
}

void launch_transform_stats(float *vol, int onx, int onz, int ny, float dw, float os, float oa,
                            StatPartial *partial, int *ntiles_out, cudaStream_t st) {
  transform_stats_kernel<<<dim3(TS_TILES, ny), 256, 0, st>>>(vol, (size_t)onx * onz, dw, os, oa,
                                                             partial);
  if (ntiles_out) *ntiles_out = TS_TILES;
}

// One block per slice: its tiles' partials are combined by a fixed tree (the
// same thread always takes the same tiles), so the statistics are
// deterministic; then one thread folds the slices in Y order exactly as
// main.rs:1080-1092 does.
__global__ void __launch_bounds__(256) slice_stats_kernel(const StatPartial *partial, int ntiles, int count,
                                                          float *slice_stats) {
  const int iy = blockIdx.x;
  float mn = 3.40282347e+38f, mx = -3.40282347e+38f;
  double sum = 0.0;
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) {
    const StatPartial p = partial[(size_t)iy * ntiles + t];
    mn = fminf(mn, p.mn);
    mx = fmaxf(mx, p.mx);
    sum += p.sum;
  }
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
    for (int k = 1; k < 8; ++k) { mn = fminf(mn, rmn[k]); mx = fmaxf(mx, rmx[k]); }
    double t = rs[0];
    for (int k = 1; k < 8; ++k) t += rs[k];
    mn = fminf(rmn[0], mn);
    mx = fmaxf(rmx[0], mx);
    slice_stats[3 * iy + 0] = mn;
    slice_stats[3 * iy + 1] = mx;
    slice_stats[3 * iy + 2] = (float)(t / (double)count);
  }
}

__global__ void fold_slices_kernel(const float *slice_stats, int ny, int count, float *out3) {
  float gmin = 3.40282347e+38f, gmax = -3.40282347e+38f;
  double gsum = 0.0;
  for (int iy = 0; iy < ny; ++iy) {
    const float smin = slice_stats[3 * iy], smax = slice_stats[3 * iy + 1], smean = slice_stats[3 * iy + 2];
    if (smin < gmin) gmin = smin;
    if (smax > gmax) gmax = smax;
    gsum += (double)smean * (double)count;
  }
  out3[0] = gmin;
  out3[1] = gmax;
  out3[2] = (float)(gsum / ((double)count * (double)ny));
}

void launch_stats_reduce(const StatPartial *partial, int ny, int ntiles, int count,
                         float *slice_stats, float *out3, cudaStream_t st) {
  slice_stats_kernel<<<ny, 256, 0, st>>>(partial, ntiles, count, slice_stats);
  fold_slices_kernel<<<1, 1, 0, st>>>(slice_stats, ny, count, out3);
}

// f32 -> IEEE half, round to nearest even, for mode-12 output (n values).  With
// both pointers 16-byte aligned each thread converts 8 values per step; otherwise
// (a slice range whose start is not a multiple of 4 values) one per step.
template <bool VEC>
__global__ void __launch_bounds__(256) to_half_kernel(const float *__restrict__ in, __half *__restrict__ out,
                                                      size_t n) {
  const size_t stride = (size_t)gridDim.x * blockDim.x, t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (!VEC) {
    for (size_t i = t0; i < n; i += stride) out[i] = __float2half_rn(__ldcs(in + i));
    return;
  }
  const size_t n8 = n / 8;
  for (size_t i = t0; i < n8; i += stride) {
    const float4 a = __ldcs(reinterpret_cast<const float4 *>(in) + 2 * i);
    const float4 b = __ldcs(reinterpret_cast<const float4 *>(in) + 2 * i + 1);
    const __half2 h0 = __floats2half2_rn(a.x, a.y), h1 = __floats2half2_rn(a.z, a.w);
    const __half2 h2 = __floats2half2_rn(b.x, b.y), h3 = __floats2half2_rn(b.z, b.w);
    uint4 w;
    w.x = *reinterpret_cast<const uint32_t *>(&h0);
    w.y = *reinterpret_cast<const uint32_t *>(&h1);
    w.z = *reinterpret_cast<const uint32_t *>(&h2);
    w.w = *reinterpret_cast<const uint32_t *>(&h3);
    reinterpret_cast<uint4 *>(out)[i] = w;
  }
  if (t0 < n - 8 * n8) out[8 * n8 + t0] = __float2half_rn(in[8 * n8 + t0]);
}

void launch_to_half(const float *in, void *out, size_t n, cudaStream_t st) {
  if (n == 0) return;
  const bool vec = ((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0);
  const size_t blocks = std::min<size_t>((n / (vec ? 8 : 1) + 255) / 256 + 1, 148 * 8);
  if (vec) to_half_kernel<true><<<(unsigned)blocks, 256, 0, st>>>(in, static_cast<__half *>(out), n);
  else to_half_kernel<false><<<(unsigned)blocks, 256, 0, st>>>(in, static_cast<__half *>(out), n);
}

}  // namespace tg
