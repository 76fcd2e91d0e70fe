// ctf.cu -- CTF phase flip of a tilt series on the GPU.
//
// Semantics: apps/ctfphaseflip/src/main.rs (the default CPU path) and, for the
// per-strip seam, GpuCtfSession::correct_strip with ctf_correct.wgsl
// (apps/ctfphaseflip/src/gpu.rs:107-262).
//
// Each view is cut into strips perpendicular to the tilt axis (main.rs:443-
// 470).  Per strip: the bounding box of its pixels is transformed by a 2D FFT
// (row FFTs, a transpose, row FFTs along the former columns), every frequency
// whose CTF -- computed in f64 as the reference's CPU path does -- is negative
// is negated, the inverse transform runs the same way back, and the strip's
// pixels are added into per-pixel weighted sums with the reference's
// triangular weights; a final pass divides (or keeps the input where no strip
// weighs in).  Strip geometry (centres, bounds, bounding boxes) depends on the
// image size and tilt axis only, so the host works it out once per stack with
// the reference's f64 expressions; the device repeats only the per-pixel
// membership test, in the same f64 operation order (no FMA contraction).
//
// Layout in device memory: the stack [nz][ny][nx] f32 in and out, two complex
// work buffers of the largest strip (sw*sh float2 each), the per-pixel weighted
// sum and weight of one view (ny*nx f32 each), twiddle tables per transform
// length, and the per-(view, tile) partial statistics of volume_ops.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "fft.cuh"
#include "tg_internal.h"

namespace tg {

namespace {

constexpr double PI32_D = (double)3.14159265358979323846f;  // `PI as f64` (f32 constant widened)
constexpr int CTF_MAX_N = 12288;                             // transform length: 2n float2 in shared memory

// One complex row of length n per CTA (grid-stride over rows): Stockham with the
// plan's radices, or a direct DFT for lengths with a prime factor above 7.
template <bool INV>
__global__ void __launch_bounds__(256) ctf_fft_rows_kernel(float2 *data, int n, int nrows, FftPlanDev plan,
                                                           const float2 *__restrict__ tw, int direct) {
  extern __shared__ __align__(16) unsigned char csm[];
  float2 *A = reinterpret_cast<float2 *>(csm);
  float2 *B = A + n;
  for (int row = blockIdx.x; row < nrows; row += gridDim.x) {
    float2 *x = data + (size_t)row * n;
    for (int k = threadIdx.x; k < n; k += blockDim.x) A[k] = x[k];
    __syncthreads();
    if (!direct) {
      const float2 *R = stockham<INV>(A, B, plan, tw);
      for (int k = threadIdx.x; k < n; k += blockDim.x) x[k] = R[k];
    } else {
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        float2 acc = make_float2(0.0f, 0.0f);
        int e = 0;  // (j * k) mod n
        for (int j = 0; j < n; ++j) {
          float2 w = __ldg(&tw[e]);
          if (INV) w.y = -w.y;
          acc = cadd(acc, cmul(A[j], w));
          e += k;
          if (e >= n) e -= n;
        }
        x[k] = acc;
      }
    }
    __syncthreads();  // A and B are reused by the next row
  }
}

// out[c][r] = in[r][c] for an rows x cols complex matrix (32x32 tiles)
__global__ void ctf_transpose_kernel(const float2 *__restrict__ in, float2 *__restrict__ out, int rows, int cols) {
  __shared__ float2 t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[j][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * rows + r] = t[threadIdx.x][j];
  }
}

// A[r][c] = (view[(y0 + r) * nx + x0 + c], 0)
__global__ void ctf_extract_kernel(const float *__restrict__ view, int nx, int x0, int y0, int sw, int sh,
                                   float2 *__restrict__ A) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)sw * sh) return;
  const int r = (int)(i / sw), c = (int)(i % sw);
  A[i] = make_float2(view[(size_t)(y0 + r) * nx + x0 + c], 0.0f);
}

struct FlipArgs {
  int sw, sh;
  double pixel_a, wl, cs_a, amp, w_phase, cuton, base1, base2, astig_rad, plate, tilt_axis_rad, cos_ta, sin_ta;
  int has_astig;
};

// main.rs:553-617 on the transposed strip spectrum B[fx][fy]: negate where the
// CTF (f64) is negative, frequencies below the cut-on untouched.
__global__ void ctf_flip_kernel(float2 *B, FlipArgs f) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)f.sw * f.sh) return;
  const int fx = (int)(i / f.sh), fy = (int)(i % f.sh);
  const double freq_y = fy <= f.sh / 2 ? (double)fy : __dsub_rn((double)fy, (double)f.sh);
  const double freq_x = fx <= f.sw / 2 ? (double)fx : __dsub_rn((double)fx, (double)f.sw);
  double rfx = freq_x, rfy = freq_y;
  if (fabs(f.tilt_axis_rad) > 1e-6) {
    rfx = __dadd_rn(__dmul_rn(freq_x, f.cos_ta), __dmul_rn(freq_y, f.sin_ta));
    rfy = __dadd_rn(__dmul_rn(-freq_x, f.sin_ta), __dmul_rn(freq_y, f.cos_ta));
  }
  const double sx = __ddiv_rn(rfx, __dmul_rn((double)f.sw, f.pixel_a));
  const double sy = __ddiv_rn(rfy, __dmul_rn((double)f.sh, f.pixel_a));
  const double s2 = __dadd_rn(__dmul_rn(sx, sx), __dmul_rn(sy, sy));
  if (sqrt(s2) < f.cuton) return;
  double def = f.base1;
  if (f.has_astig) {  // effective_defocus, main.rs:213-219
    const double da = __dsub_rn(atan2(sy, sx), f.astig_rad);
    const double c = cos(da), s = sin(da);
    def = __dadd_rn(__dmul_rn(f.base1, __dmul_rn(c, c)), __dmul_rn(f.base2, __dmul_rn(s, s)));
  }
  // chi = PI * lambda * s2 * (def - 0.5 * Cs * lambda^2 * s2), left to right
  const double t = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.5, f.cs_a), f.wl), f.wl), s2);
  const double chi = __dmul_rn(__dmul_rn(__dmul_rn(3.14159265358979323846, f.wl), s2), __dsub_rn(def, t));
  const double chi_t = __dadd_rn(chi, f.plate);
  const double ctf = __dadd_rn(__dmul_rn(-sin(chi_t), f.w_phase), __dmul_rn(cos(chi_t), f.amp));
  if (ctf < 0.0) {
    const float2 v = B[i];
    B[i] = make_float2(-v.x, -v.y);
  }
}

struct AccumArgs {
  int nx, x0, y0, sw, sh;
  double cxp, cyp, perp_x, perp_y, lo, hi, center, half_w;
  float scale;
};

// main.rs:654-671: pixels of the strip (d in [lo, hi)) add val*w and w
__global__ void ctf_accumulate_kernel(const float2 *__restrict__ A, AccumArgs a, float *wsum, float *wtot) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)a.sw * a.sh) return;
  const int r = (int)(i / a.sw), c = (int)(i % a.sw);
  const int x = a.x0 + c, y = a.y0 + r;
  const double d = __dadd_rn(__dmul_rn(__dsub_rn((double)x, a.cxp), a.perp_x),
                             __dmul_rn(__dsub_rn((double)y, a.cyp), a.perp_y));
  if (!(d >= a.lo && d < a.hi)) return;
  const float dist = (float)fabs(__ddiv_rn(__dsub_rn(d, a.center), a.half_w));
  const float w = fmaxf(__fsub_rn(1.0f, dist), 0.0f);
  const float val = __fmul_rn(A[i].x, a.scale);
  const size_t p = (size_t)y * a.nx + x;
  wsum[p] = __fadd_rn(wsum[p], __fmul_rn(val, w));
  wtot[p] = __fadd_rn(wtot[p], w);
}

// main.rs:675-680
__global__ void ctf_combine_kernel(const float *__restrict__ in, const float *__restrict__ wsum,
                                   const float *__restrict__ wtot, float *out, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float t = wtot[i];
  out[i] = t > 1e-10f ? __fdiv_rn(wsum[i], t) : in[i];
}

// ctf_correct.wgsl in f32 (the shader's operation order; accurate sin/cos/atan2)
__global__ void ctf_strip_f32_kernel(float *re, float *im, tg_ctf_strip_params p) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)p.sw * p.sh) return;
  const uint32_t fx_idx = (uint32_t)(i % p.sw), fy_idx = (uint32_t)(i / p.sw);
  const float sw = (float)p.sw, sh = (float)p.sh;
  float freq_x = fx_idx <= p.sw / 2u ? (float)fx_idx : __fsub_rn((float)fx_idx, sw);
  float freq_y = fy_idx <= p.sh / 2u ? (float)fy_idx : __fsub_rn((float)fy_idx, sh);
  if (fabsf(p.tilt_axis_rad) > 1e-6f) {
    const float ca = cosf(p.tilt_axis_rad), sa = sinf(p.tilt_axis_rad);
    const float rx = __fadd_rn(__fmul_rn(freq_x, ca), __fmul_rn(freq_y, sa));
    const float ry = __fadd_rn(__fmul_rn(-freq_x, sa), __fmul_rn(freq_y, ca));
    freq_x = rx;
    freq_y = ry;
  }
  const float sx = __fdiv_rn(freq_x, __fmul_rn(sw, p.pixel_a));
  const float sy = __fdiv_rn(freq_y, __fmul_rn(sh, p.pixel_a));
  const float s2 = __fadd_rn(__fmul_rn(sx, sx), __fmul_rn(sy, sy));
  if (__fsqrt_rn(s2) < p.cuton_freq) return;
  float def = p.defocus1;
  if (p.has_astigmatism == 1u) {
    const float da = __fsub_rn(atan2f(sy, sx), p.astig_angle_rad);
    const float c = cosf(da), s = sinf(da);
    def = __fadd_rn(__fmul_rn(p.defocus1, __fmul_rn(c, c)), __fmul_rn(p.defocus2, __fmul_rn(s, s)));
  }
  const float wl = p.wavelength;
  const float t = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(0.5f, p.cs_a), wl), wl), s2);
  const float chi = __fmul_rn(__fmul_rn(__fmul_rn(3.14159265358979323846f, wl), s2), __fsub_rn(def, t));
  const float chi_t = __fadd_rn(chi, p.plate_phase_rad);
  const float w = p.amp_contrast;
  const float w_phase = __fsqrt_rn(__fsub_rn(1.0f, __fmul_rn(w, w)));
  const float ctf = __fadd_rn(__fmul_rn(-sinf(chi_t), w_phase), __fmul_rn(cosf(chi_t), w));
  if (ctf < 0.0f) {
    re[i] = -re[i];
    im[i] = -im[i];
  }
}

double electron_wavelength(float kv) {  // main.rs:706-718
  const double v = (double)kv * 1000.0;
  const double m0 = 9.10938e-31, e = 1.60218e-19, c = 2.99792e8, h = 6.62607e-34;
  const double lam = h / sqrt(2.0 * m0 * e * v * (1.0 + e * v / (2.0 * m0 * c * c)));
  return lam * 1e10;
}

struct StripGeom {
  double center, lo, hi;
  int x0, x1, y0, y1;
};

struct DevBuf {  // device allocations of one call, freed on every return path
  std::vector<void *> ptrs;
  cudaStream_t st = nullptr;
  ~DevBuf() {
    if (st) cudaStreamSynchronize(st);
    for (void *p : ptrs) cudaFree(p);
    if (st) cudaStreamDestroy(st);
  }
  template <class T> cudaError_t alloc(T **p, size_t bytes) {
    cudaError_t e = cudaMalloc((void **)p, std::max<size_t>(bytes, 16));
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

struct Twiddles {
  float2 *d = nullptr;
  FftPlanDev plan{};
  int direct = 0;
};

template <bool INV> void fft_rows(float2 *data, int n, int nrows, const Twiddles &t, cudaStream_t st) {
  const size_t smem = (size_t)n * 16;
  auto k = ctf_fft_rows_kernel<INV>;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int grid = std::min(nrows, 148 * 8);
  k<<<grid, 256, smem, st>>>(data, n, nrows, t.plan, t.d, t.direct);
}

}  // namespace

int ctf_strip_width(const tg_ctf_options *o, int nx, const float *view_def, int nviews) {  // main.rs:284-324
  size_t max_w;
  if (o->max_strip_width > 0) {
    max_w = (size_t)o->max_strip_width;
  } else {
    double max_def = 0.0;
    if (view_def) {
      for (int v = 0; v < nviews; ++v)
        max_def = std::max(max_def, (double)std::max(fabsf(view_def[3 * v]), fabsf(view_def[3 * v + 1])) * 10.0);
    } else {
      max_def = (double)fabsf(o->defocus) * 10.0;
    }
    const double wl = electron_wavelength(o->voltage);
    if (max_def > 1.0 && wl > 0.0) {
      const double safe = std::max((double)o->pixel_size / (wl * (max_def / (double)nx)), 16.0);
      max_w = (size_t)safe;
    } else {
      max_w = (size_t)std::max(o->strip_width, 0);
    }
  }
  return (int)std::min((size_t)std::max(o->strip_width, 0), max_w);
}

}  // namespace tg

using namespace tg;

extern "C" {

void tg_ctf_options_default(tg_ctf_options *o) {
  if (!o) return;
  memset(o, 0, sizeof *o);
  o->defocus = -3000.0f;
  o->voltage = 300.0f;
  o->cs = 2.7f;
  o->pixel_size = 1.0f;
  o->strip_width = 256;
  o->tilt_axis_angle = 0.0f;
  o->max_strip_width = 0;
  o->amplitude_contrast = 0.07f;
  o->cuton_freq = 0.0f;
  o->plate_phase = 0.0f;
  o->device = 0;
}

int tg_ctf_strip_width(const tg_ctf_options *o, int32_t nx, const float *view_defocus, int32_t n_view_defocus,
                       int32_t *out) {
  if (!o || !out || nx < 1) return TG_ERR_INVALID_ARG;
  *out = ctf_strip_width(o, nx, view_defocus, view_defocus ? n_view_defocus : 0);
  return TG_OK;
}

int tg_ctf_phaseflip(const tg_ctf_options *o, const float *host_in, int32_t nx, int32_t ny, int32_t nz,
                     const float *angles, int32_t n_angles, const float *view_defocus, int32_t n_view_defocus,
                     float *host_out, tg_stats *stats) {
  if (!o || !host_in || !host_out || nx < 1 || ny < 1 || nz < 1 || (n_angles > 0 && !angles)) {
    set_error("tg_ctf_phaseflip: null pointer or empty stack");
    return TG_ERR_INVALID_ARG;
  }
  const int strip_width = ctf_strip_width(o, nx, view_defocus, view_defocus ? n_view_defocus : 0);
  if (strip_width < 1) { set_error("strip width must be at least 1"); return TG_ERR_INVALID_ARG; }
  // strip geometry (main.rs:436-509), once for the stack
  const double tilt_axis_rad = (double)o->tilt_axis_angle * PI32_D / 180.0;
  const double perp_x = cos(tilt_axis_rad), perp_y = sin(tilt_axis_rad);
  const double cxp = (double)nx / 2.0, cyp = (double)ny / 2.0;
  double min_perp = 1.79769313486231570e+308, max_perp = -1.79769313486231570e+308;
  const double corners[4][2] = {{0.0, 0.0}, {(double)nx, 0.0}, {0.0, (double)ny}, {(double)nx, (double)ny}};
  for (auto &c : corners) {
    const double d = (c[0] - cxp) * perp_x + (c[1] - cyp) * perp_y;
    min_perp = std::min(min_perp, d);
    max_perp = std::max(max_perp, d);
  }
  const double sw_d = (double)strip_width;
  const size_t n_strips = (size_t)ceil((max_perp - min_perp) / sw_d);
  std::vector<StripGeom> strips;
  size_t work = 1;
  std::map<int, int> lengths;  // transform lengths in use
  for (size_t k = 0; k < n_strips; ++k) {
    StripGeom g;
    g.center = min_perp + ((double)k + 0.5) * sw_d;
    g.lo = g.center - sw_d / 2.0;
    g.hi = g.center + sw_d / 2.0;
    int bx0 = nx, bx1 = 0, by0 = ny, by1 = 0;
    for (int y = 0; y < ny; ++y) {
      const double ty = ((double)y - cyp) * perp_y;
      for (int x = 0; x < nx; ++x) {
        const double d = ((double)x - cxp) * perp_x + ty;
        if (d >= g.lo && d < g.hi) {
          bx0 = std::min(bx0, x);
          bx1 = std::max(bx1, x + 1);
          by0 = std::min(by0, y);
          by1 = std::max(by1, y + 1);
        }
      }
    }
    if (bx1 <= bx0 || by1 <= by0) continue;
    g.x0 = bx0; g.x1 = bx1; g.y0 = by0; g.y1 = by1;
    const int sw = bx1 - bx0, sh = by1 - by0;
    if (sw > CTF_MAX_N || sh > CTF_MAX_N) {
      set_error("strip dimension above " + std::to_string(CTF_MAX_N) + " samples");
      return TG_ERR_UNSUPPORTED;
    }
    work = std::max(work, (size_t)sw * sh);
    lengths[sw] = 0;
    lengths[sh] = 0;
    strips.push_back(g);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("no CUDA device"); return TG_ERR_NO_DEVICE; }
  if (o->device < 0 || o->device >= ndev) { set_error("bad device ordinal"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(o->device));
  DevBuf mem;
  TG_CUDA(cudaStreamCreateWithFlags(&mem.st, cudaStreamNonBlocking));
  cudaStream_t st = mem.st;
  const size_t npix = (size_t)nx * ny, ntot = npix * nz;
  float *d_in, *d_out, *d_wsum, *d_wtot, *d_slice, *d_stats3;
  float2 *d_A, *d_B;
  StatPartial *d_part;
  cudaError_t e;
  if ((e = mem.alloc(&d_in, ntot * 4)) || (e = mem.alloc(&d_out, ntot * 4)) || (e = mem.alloc(&d_wsum, npix * 4)) ||
      (e = mem.alloc(&d_wtot, npix * 4)) || (e = mem.alloc(&d_A, work * 8)) || (e = mem.alloc(&d_B, work * 8)) ||
      (e = mem.alloc(&d_part, (size_t)nz * 64 * sizeof(StatPartial))) || (e = mem.alloc(&d_slice, (size_t)nz * 12)) ||
      (e = mem.alloc(&d_stats3, 16)))
    return cuda_fail(e, "cudaMalloc(ctfphaseflip)");
  std::map<int, Twiddles> tws;
  for (auto &kv : lengths) {
    Twiddles t;
    const int n = kv.first;
    t.direct = fft_plan(n, &t.plan) ? 0 : 1;
    std::vector<float2> h(n);
    for (int k = 0; k < n; ++k) {
      const double a = -2.0 * M_PI * (double)k / (double)n;
      h[k] = make_float2((float)cos(a), (float)sin(a));
    }
    if ((e = mem.alloc(&t.d, (size_t)n * 8))) return cuda_fail(e, "cudaMalloc(twiddles)");
    TG_CUDA(cudaMemcpyAsync(t.d, h.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st));
    TG_CUDA(cudaStreamSynchronize(st));  // h goes out of scope
    tws[n] = t;
  }
  TG_CUDA(cudaMemcpyAsync(d_in, host_in, ntot * 4, cudaMemcpyHostToDevice, st));
  const double wl = electron_wavelength(o->voltage);
  const double amp = (double)o->amplitude_contrast;
  FlipArgs f{};
  f.pixel_a = (double)o->pixel_size;
  f.wl = wl;
  f.cs_a = (double)o->cs * 1e7;
  f.amp = amp;
  f.w_phase = sqrt(1.0 - amp * amp);
  f.cuton = (double)o->cuton_freq;
  f.plate = (double)o->plate_phase * PI32_D / 180.0;
  f.tilt_axis_rad = tilt_axis_rad;
  f.cos_ta = cos(tilt_axis_rad);
  f.sin_ta = sin(tilt_axis_rad);
  {
    NvtxRange nv("tg.ctfphaseflip");
    for (int z = 0; z < nz; ++z) {
      const float tilt_deg = z < n_angles ? angles[z] : 0.0f;
      const double tilt_rad = (double)tilt_deg * PI32_D / 180.0;
      float d1 = o->defocus, d2 = o->defocus, astig = 0.0f;
      if (view_defocus && z < n_view_defocus) {
        d1 = view_defocus[3 * z];
        d2 = view_defocus[3 * z + 1];
        astig = view_defocus[3 * z + 2];
      }
      const double def1_a = (double)d1 * 10.0, def2_a = (double)d2 * 10.0;
      f.astig_rad = (double)astig * PI32_D / 180.0;
      f.has_astig = fabs(def1_a - def2_a) > 0.01 ? 1 : 0;
      const float *view = d_in + (size_t)z * npix;
      TG_CUDA(cudaMemsetAsync(d_wsum, 0, npix * 4, st));
      TG_CUDA(cudaMemsetAsync(d_wtot, 0, npix * 4, st));
      for (const StripGeom &g : strips) {
        const int sw = g.x1 - g.x0, sh = g.y1 - g.y0;
        const size_t n = (size_t)sw * sh;
        const unsigned nb = (unsigned)((n + 255) / 256);
        const double dx_a = g.center * (double)o->pixel_size;
        f.base1 = def1_a + dx_a * sin(tilt_rad);
        f.base2 = def2_a + dx_a * sin(tilt_rad);
        f.sw = sw;
        f.sh = sh;
        ctf_extract_kernel<<<nb, 256, 0, st>>>(view, nx, g.x0, g.y0, sw, sh, d_A);
        fft_rows<false>(d_A, sw, sh, tws[sw], st);
        ctf_transpose_kernel<<<dim3((sw + 31) / 32, (sh + 31) / 32), dim3(32, 8), 0, st>>>(d_A, d_B, sh, sw);
        fft_rows<false>(d_B, sh, sw, tws[sh], st);
        ctf_flip_kernel<<<nb, 256, 0, st>>>(d_B, f);
        fft_rows<true>(d_B, sh, sw, tws[sh], st);
        ctf_transpose_kernel<<<dim3((sh + 31) / 32, (sw + 31) / 32), dim3(32, 8), 0, st>>>(d_B, d_A, sw, sh);
        fft_rows<true>(d_A, sw, sh, tws[sw], st);
        AccumArgs a{};
        a.nx = nx; a.x0 = g.x0; a.y0 = g.y0; a.sw = sw; a.sh = sh;
        a.cxp = cxp; a.cyp = cyp; a.perp_x = perp_x; a.perp_y = perp_y;
        a.lo = g.lo; a.hi = g.hi; a.center = g.center; a.half_w = sw_d / 2.0;
        a.scale = 1.0f / (float)((size_t)sw * sh);
        ctf_accumulate_kernel<<<nb, 256, 0, st>>>(d_A, a, d_wsum, d_wtot);
      }
      ctf_combine_kernel<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>(view, d_wsum, d_wtot,
                                                                          d_out + (size_t)z * npix, npix);
      TG_CUDA(cudaGetLastError());
    }
    // statistics (main.rs:681-693): per-section min, max and f64 sum, folded in order
    int ntiles = 0;
    launch_transform_stats(d_out, nx, ny, nz, 1.0f, 1.0f, 0.0f, d_part, &ntiles, st);
    launch_stats_reduce(d_part, nz, ntiles, (int)npix, d_slice, d_stats3, st);
    TG_CUDA(cudaGetLastError());
  }
  TG_CUDA(cudaMemcpyAsync(host_out, d_out, ntot * 4, cudaMemcpyDeviceToHost, st));
  float s3[3];
  TG_CUDA(cudaMemcpyAsync(s3, d_stats3, 12, cudaMemcpyDeviceToHost, st));
  TG_CUDA(cudaStreamSynchronize(st));
  if (stats) {
    stats->amin = s3[0];
    stats->amax = s3[1];
    stats->amean = s3[2];
  }
  return TG_OK;
}

int tg_ctf_correct_strip(float *strip_re, float *strip_im, const tg_ctf_strip_params *p, int32_t device) {
  if (!strip_re || !strip_im || !p || p->sw == 0 || p->sh == 0) return TG_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("no CUDA device"); return TG_ERR_NO_DEVICE; }
  if (device < 0 || device >= ndev) { set_error("bad device ordinal"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(device));
  const size_t n = (size_t)p->sw * p->sh;
  DevBuf mem;
  TG_CUDA(cudaStreamCreateWithFlags(&mem.st, cudaStreamNonBlocking));
  float *d_re, *d_im;
  cudaError_t e;
  if ((e = mem.alloc(&d_re, n * 4)) || (e = mem.alloc(&d_im, n * 4))) return cuda_fail(e, "cudaMalloc(strip)");
  TG_CUDA(cudaMemcpyAsync(d_re, strip_re, n * 4, cudaMemcpyHostToDevice, mem.st));
  TG_CUDA(cudaMemcpyAsync(d_im, strip_im, n * 4, cudaMemcpyHostToDevice, mem.st));
  ctf_strip_f32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, mem.st>>>(d_re, d_im, *p);
  TG_CUDA(cudaGetLastError());
  TG_CUDA(cudaMemcpyAsync(strip_re, d_re, n * 4, cudaMemcpyDeviceToHost, mem.st));
  TG_CUDA(cudaMemcpyAsync(strip_im, d_im, n * 4, cudaMemcpyDeviceToHost, mem.st));
  TG_CUDA(cudaStreamSynchronize(mem.st));
  return TG_OK;
}

}  // extern "C"
