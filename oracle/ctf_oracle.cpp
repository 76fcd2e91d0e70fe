// ctf_oracle.cpp -- CPU restatement of imod-rs's ctfphaseflip, TEST
// INFRASTRUCTURE ONLY (the tests and the CPU baseline call it; nothing in the
// product path does).
//
// Follows apps/ctfphaseflip/src/main.rs:
//   electron_wavelength            706-718
//   effective_defocus              213-219
//   strip width (auto maximum)     284-324
//   per-view strip loop            385-700: strips perpendicular to the tilt axis,
//     bounding box of the strip's pixels, 2D FFT (rows then columns, f32 like
//     rustfft::<f32>), phase flip where the CTF (computed in f64) is negative
//     (553-617), inverse 2D FFT, 1/(sw*sh), triangular strip weights and the
//     weighted combination (keeping the input where no strip weighs in)
//   statistics                     681-693
// and the GPU seam's shader (apps/ctfphaseflip/src/ctf_correct.wgsl) in f32.
// The FFT is this oracle's mixed-radix restatement of rustfft's published
// method (FftPlan in tilt_oracle.cpp); the reference pins no results at that
// boundary.
#include <math.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "tilt_oracle.h"

// FftPlan<float> of tilt_oracle.cpp
namespace ctf_detail {
void fft32(std::complex<float> *x, int n, bool inverse);
}

namespace {

const double PI32 = (double)3.14159265358979323846f;  // `PI as f64` of std::f32::consts::PI

double wavelength_a(float kv) {  // main.rs:706-718
  const double v = (double)kv * 1000.0;
  const double m0 = 9.10938e-31, e = 1.60218e-19, c = 2.99792e8, h = 6.62607e-34;
  const double lam = h / std::sqrt(2.0 * m0 * e * v * (1.0 + e * v / (2.0 * m0 * c * c)));
  return lam * 1e10;
}

double effective_defocus(double d1, double d2, double ang, double astig) {  // main.rs:213-219
  const double da = ang - astig;
  const double c2 = std::cos(da) * std::cos(da), s2 = std::sin(da) * std::sin(da);
  return d1 * c2 + d2 * s2;
}

}  // namespace

extern "C" {

double or_ctf_wavelength(float kv) { return wavelength_a(kv); }

// main.rs:284-324: strip_width clamped to the given or automatic maximum.
// view_def: 3 floats per view (defocus1 nm, defocus2 nm, astig deg) or NULL.
int or_ctf_strip_width(const or_ctf_params *p, int nx, const float *view_def, int nviews) {
  size_t max_w;
  if (p->max_strip_width > 0) {
    max_w = (size_t)p->max_strip_width;
  } else {
    double max_def = 0.0;
    if (view_def) {
      for (int v = 0; v < nviews; ++v) {
        const double d = (double)std::max(std::fabs(view_def[3 * v]), std::fabs(view_def[3 * v + 1])) * 10.0;
        max_def = std::max(max_def, d);
      }
    } else {
      max_def = (double)std::fabs(p->defocus) * 10.0;
    }
    const double wl = wavelength_a(p->voltage);
    if (max_def > 1.0 && wl > 0.0) {
      const double per_px = max_def / (double)nx;
      double safe = (double)p->pixel_a / (wl * per_px);
      safe = std::max(safe, 16.0);
      max_w = (size_t)safe;
    } else {
      max_w = (size_t)p->strip_width;
    }
  }
  return (int)std::min((size_t)p->strip_width, max_w);
}

// The whole stack: in/out [nz][ny][nx].  Returns 0.
int or_ctfphaseflip32(const or_ctf_params *p, const float *in, int nx, int ny, int nz, const float *angles,
                      int n_angles, const float *view_def, int n_view_def, float *out, or_stats *st) {
  const double wl = wavelength_a(p->voltage);
  const double cs_a = (double)p->cs * 1e7;
  const double amp = (double)p->amplitude_contrast, cuton = (double)p->cuton_freq;
  const double tilt_axis_rad = (double)p->tilt_axis_angle * PI32 / 180.0;
  const double plate = (double)p->plate_phase * PI32 / 180.0;
  const int strip_width = or_ctf_strip_width(p, nx, view_def, n_view_def);
  const double perp_x = std::cos(tilt_axis_rad), perp_y = std::sin(tilt_axis_rad);
  const double cxp = (double)nx / 2.0, cyp = (double)ny / 2.0;
  const float pixel_a = p->pixel_a;
  float gmin = 3.40282347e+38f, gmax = -3.40282347e+38f;
  double gsum = 0.0;
  const size_t npix = (size_t)nx * ny;
  std::vector<float> wsum(npix), wtot(npix);
  std::vector<std::complex<float>> strip, col;
  for (int z = 0; z < nz; ++z) {
    const float *data = in + (size_t)z * npix;
    float *output = out + (size_t)z * npix;
    const float tilt_deg = z < n_angles ? angles[z] : 0.0f;
    const double tilt_rad = (double)tilt_deg * PI32 / 180.0;
    float d1nm = p->defocus, d2nm = p->defocus, astig_deg = 0.0f;
    if (view_def && z < n_view_def) {
      d1nm = view_def[3 * z];
      d2nm = view_def[3 * z + 1];
      astig_deg = view_def[3 * z + 2];
    }
    const double def1_a = (double)d1nm * 10.0, def2_a = (double)d2nm * 10.0;
    const double astig_rad = (double)astig_deg * PI32 / 180.0;
    const bool has_astig = std::fabs(def1_a - def2_a) > 0.01;
    memcpy(output, data, npix * sizeof(float));
    double min_perp = 1.79769313486231570e+308, max_perp = -1.79769313486231570e+308;
    const double corners[4][2] = {{0.0, 0.0}, {(double)nx, 0.0}, {0.0, (double)ny}, {(double)nx, (double)ny}};
    for (auto &c : corners) {
      const double d = (c[0] - cxp) * perp_x + (c[1] - cyp) * perp_y;
      if (d < min_perp) min_perp = d;
      if (d > max_perp) max_perp = d;
    }
    const double sw_d = (double)strip_width;
    const size_t n_strips = (size_t)std::ceil((max_perp - min_perp) / sw_d);
    std::fill(wsum.begin(), wsum.end(), 0.0f);
    std::fill(wtot.begin(), wtot.end(), 0.0f);
    for (size_t k = 0; k < n_strips; ++k) {
      const double center = min_perp + ((double)k + 0.5) * sw_d;
      const double dx_a = center * (double)pixel_a;
      const double base1 = def1_a + dx_a * std::sin(tilt_rad);
      const double base2 = def2_a + dx_a * std::sin(tilt_rad);
      const double lo = center - sw_d / 2.0, hi = center + sw_d / 2.0;
      size_t bx0 = nx, bx1 = 0, by0 = ny, by1 = 0;
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const double d = ((double)x - cxp) * perp_x + ((double)y - cyp) * perp_y;
          if (d >= lo && d < hi) {
            bx0 = std::min(bx0, (size_t)x);
            if ((size_t)x >= bx1) bx1 = x + 1;
            by0 = std::min(by0, (size_t)y);
            if ((size_t)y >= by1) by1 = y + 1;
          }
        }
      if (bx1 <= bx0 || by1 <= by0) continue;
      const int sw = (int)(bx1 - bx0), sh = (int)(by1 - by0);
      strip.assign((size_t)sw * sh, std::complex<float>(0.0f, 0.0f));
      for (int y = 0; y < sh; ++y)
        for (int x = 0; x < sw; ++x) strip[(size_t)y * sw + x] = std::complex<float>(data[(by0 + y) * nx + bx0 + x], 0.0f);
      for (int r = 0; r < sh; ++r) ctf_detail::fft32(&strip[(size_t)r * sw], sw, false);
      col.assign(sh, std::complex<float>(0.0f, 0.0f));
      for (int c = 0; c < sw; ++c) {
        for (int r = 0; r < sh; ++r) col[r] = strip[(size_t)r * sw + c];
        ctf_detail::fft32(col.data(), sh, false);
        for (int r = 0; r < sh; ++r) strip[(size_t)r * sw + c] = col[r];
      }
      const double w_phase = std::sqrt(1.0 - amp * amp);
      for (int fy = 0; fy < sh; ++fy) {
        const double freq_y = fy <= sh / 2 ? (double)fy : (double)fy - (double)sh;
        for (int fx = 0; fx < sw; ++fx) {
          const double freq_x = fx <= sw / 2 ? (double)fx : (double)fx - (double)sw;
          double rfx = freq_x, rfy = freq_y;
          if (std::fabs(tilt_axis_rad) > 1e-6) {
            const double ca = std::cos(tilt_axis_rad), sa = std::sin(tilt_axis_rad);
            rfx = freq_x * ca + freq_y * sa;
            rfy = -freq_x * sa + freq_y * ca;
          }
          const double sx = rfx / ((double)sw * (double)pixel_a), sy = rfy / ((double)sh * (double)pixel_a);
          const double s2 = sx * sx + sy * sy, s = std::sqrt(s2);
          if (s < cuton) continue;
          const double def = has_astig ? effective_defocus(base1, base2, std::atan2(sy, sx), astig_rad) : base1;
          const double chi = 3.14159265358979323846 * wl * s2 * (def - 0.5 * cs_a * wl * wl * s2);
          const double chi_t = chi + plate;
          const double ctf = -std::sin(chi_t) * w_phase + std::cos(chi_t) * amp;
          if (ctf < 0.0) strip[(size_t)fy * sw + fx] = -strip[(size_t)fy * sw + fx];
        }
      }
      for (int c = 0; c < sw; ++c) {
        for (int r = 0; r < sh; ++r) col[r] = strip[(size_t)r * sw + c];
        ctf_detail::fft32(col.data(), sh, true);
        for (int r = 0; r < sh; ++r) strip[(size_t)r * sw + c] = col[r];
      }
      for (int r = 0; r < sh; ++r) ctf_detail::fft32(&strip[(size_t)r * sw], sw, true);
      const float scale = 1.0f / (float)((size_t)sw * sh);
      for (size_t y = by0; y < by1; ++y)
        for (size_t x = bx0; x < bx1; ++x) {
          const double d = ((double)x - cxp) * perp_x + ((double)y - cyp) * perp_y;
          if (d >= lo && d < hi) {
            const float dist = (float)std::fabs((d - center) / (sw_d / 2.0));
            const float w = std::max(1.0f - dist, 0.0f);
            const float val = strip[(y - by0) * sw + (x - bx0)].real() * scale;
            wsum[y * nx + x] += val * w;
            wtot[y * nx + x] += w;
          }
        }
    }
    for (size_t i = 0; i < npix; ++i)
      if (wtot[i] > 1e-10f) output[i] = wsum[i] / wtot[i];
    float smin = 3.40282347e+38f, smax = -3.40282347e+38f;
    double s = 0.0;
    for (size_t i = 0; i < npix; ++i) {
      smin = std::min(smin, output[i]);
      smax = std::max(smax, output[i]);
      s += (double)output[i];
    }
    const float smean = (float)(s / (double)npix);
    gmin = std::min(gmin, smin);
    gmax = std::max(gmax, smax);
    gsum += (double)smean * (double)npix;
  }
  if (st) {
    st->amin = gmin;
    st->amax = gmax;
    st->amean = (float)(gsum / (double)(npix * (size_t)nz));
  }
  return 0;
}

// ctf_correct.wgsl in f32 (the GPU seam, GpuCtfSession::correct_strip): re/im
// of one strip's 2D FFT, sw*sh values each, flipped in place.
void or_ctf_correct_strip32(float *re, float *im, const or_ctf_strip *p) {
  const float PI = 3.14159265358979323846f;
  const float sw = (float)p->sw, sh = (float)p->sh;
  for (uint32_t fy_idx = 0; fy_idx < p->sh; ++fy_idx)
    for (uint32_t fx_idx = 0; fx_idx < p->sw; ++fx_idx) {
      float freq_x = fx_idx <= p->sw / 2u ? (float)fx_idx : (float)fx_idx - sw;
      float freq_y = fy_idx <= p->sh / 2u ? (float)fy_idx : (float)fy_idx - sh;
      if (std::fabs(p->tilt_axis_rad) > 1e-6f) {
        const float ca = cosf(p->tilt_axis_rad), sa = sinf(p->tilt_axis_rad);
        const float rx = freq_x * ca + freq_y * sa;
        const float ry = -freq_x * sa + freq_y * ca;
        freq_x = rx;
        freq_y = ry;
      }
      const float sx = freq_x / (sw * p->pixel_a), sy = freq_y / (sh * p->pixel_a);
      const float s2 = sx * sx + sy * sy, s = sqrtf(s2);
      if (s < p->cuton_freq) continue;
      float def = p->defocus1;
      if (p->has_astigmatism == 1u) {
        const float da = atan2f(sy, sx) - p->astig_angle_rad;
        def = p->defocus1 * (cosf(da) * cosf(da)) + p->defocus2 * (sinf(da) * sinf(da));
      }
      const float wl = p->wavelength;
      const float chi = PI * wl * s2 * (def - 0.5f * p->cs_a * wl * wl * s2);
      const float chi_t = chi + p->plate_phase_rad;
      const float w = p->amp_contrast;
      const float w_phase = sqrtf(1.0f - w * w);
      const float ctf = -sinf(chi_t) * w_phase + cosf(chi_t) * w;
      if (ctf < 0.0f) {
        const size_t idx = (size_t)fy_idx * p->sw + fx_idx;
        re[idx] = -re[idx];
        im[idx] = -im[idx];
      }
    }
}

}  // extern "C"
