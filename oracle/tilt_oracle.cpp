// tilt_oracle.cpp -- CPU restatement of the imod-rs `tilt` path (test infrastructure).
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path and the timed
// CPU baseline.  Every function cites the reference lines it restates
// (paths are relative to the imod-rs project root).  Parity of the arithmetic
// against the Rust reference is UNPINNED (no Rust toolchain; rustfft 6.x not
// vendored); see tilt_oracle.h.
//
// Build: -O3 -ffp-contract=off (no fused multiply-add, as Rust evaluates f32
// expressions), so `T=float` instantiations reproduce the reference's f32
// operation order, and `T=double` instantiations form the FP64 accuracy oracle.
#include "tilt_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

namespace {

// std::f32::consts::PI rounds to 3.14159274f; M_PI in double.
template <typename T> struct K;
template <> struct K<float> {
  static float pi() { return 3.14159265358979323846f; }
  static float cos_(float x) { return cosf(x); }
  static float sin_(float x) { return sinf(x); }
  static float exp_(float x) { return expf(x); }
  static float log10_(float x) { return log10f(x); }
  static float floor_(float x) { return floorf(x); }
  static float fabs_(float x) { return fabsf(x); }
  static float maxv() { return 3.40282347e+38f; }
  static float minv() { return -3.40282347e+38f; }
};
template <> struct K<double> {
  static double pi() { return 3.14159265358979323846; }
  static double cos_(double x) { return std::cos(x); }
  static double sin_(double x) { return std::sin(x); }
  static double exp_(double x) { return std::exp(x); }
  static double log10_(double x) { return std::log10(x); }
  static double floor_(double x) { return std::floor(x); }
  static double fabs_(double x) { return std::fabs(x); }
  static double maxv() { return 1.79769313486231570e+308; }
  static double minv() { return -1.79769313486231570e+308; }
};

template <class F> void parallel_for(int n, int nthreads, F f) {
  if (nthreads <= 1 || n <= 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  int nt = std::min(nthreads, n);
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&] {
      int i;
      while ((i = next.fetch_add(1)) < n) f(i);
    });
  for (auto &x : th) x.join();
}

// ---------------------------------------------------------------------------
// FFT: mixed-radix decimation-in-time Cooley-Tukey, twiddles computed in FP64
// and rounded to T (the published method of rustfft 6's planner for the
// radices it uses).  Unnormalised in both directions, like rustfft.
// Used by apply_rweighting (apps/tilt/src/main.rs:340-346,374).
// ---------------------------------------------------------------------------
template <typename T> struct FftPlan {
  int n;
  std::vector<int> fac;
  std::vector<std::complex<T>> tw;  // exp(-2*pi*i*k/n), k in [0,n)
  explicit FftPlan(int n_) : n(n_) {
    int m = n;
    while (m % 4 == 0) { fac.push_back(4); m /= 4; }
    while (m % 2 == 0) { fac.push_back(2); m /= 2; }
    for (int p = 3; p * p <= m; p += 2)
      while (m % p == 0) { fac.push_back(p); m /= p; }
    if (m > 1) fac.push_back(m);
    tw.resize(n);
    for (int k = 0; k < n; ++k) {
      double a = -2.0 * 3.14159265358979323846 * (double)k / (double)n;
      tw[k] = std::complex<T>((T)std::cos(a), (T)std::sin(a));
    }
  }
  std::complex<T> w(long e, bool inv) const {
    std::complex<T> v = tw[(size_t)(e % n)];
    return inv ? std::conj(v) : v;
  }
  // DFT of size m of in[0], in[s], ..., written to out[0..m); tsc = n/m
  void rec(const std::complex<T> *in, int s, std::complex<T> *out, int m, int fi, int tsc,
           bool inv) const {
    if (m == 1) { out[0] = in[0]; return; }
    int p = fac[fi], q = m / p;
    for (int r = 0; r < p; ++r) rec(in + (size_t)r * s, s * p, out + (size_t)r * q, q, fi + 1, tsc * p, inv);
    std::complex<T> t[64];
    std::vector<std::complex<T>> tb;
    std::complex<T> *tp = t;
    if (p > 64) { tb.resize(p); tp = tb.data(); }
    for (int k = 0; k < q; ++k) {
      for (int r = 0; r < p; ++r) {
        std::complex<T> v = out[(size_t)r * q + k];
        tp[r] = (r == 0 || k == 0) ? v : v * w((long)r * k * tsc, inv);
      }
      if (p == 2) {
        out[k] = tp[0] + tp[1];
        out[k + q] = tp[0] - tp[1];
      } else if (p == 4) {
        std::complex<T> a0 = tp[0] + tp[2], a1 = tp[0] - tp[2];
        std::complex<T> b0 = tp[1] + tp[3], b1 = tp[1] - tp[3];
        // multiply b1 by -i (forward) or +i (inverse)
        std::complex<T> b1r = inv ? std::complex<T>(-b1.imag(), b1.real())
                                  : std::complex<T>(b1.imag(), -b1.real());
        out[k] = a0 + b0;
        out[k + q] = a1 + b1r;
        out[k + 2 * q] = a0 - b0;
        out[k + 3 * q] = a1 - b1r;
      } else {
        for (int j = 0; j < p; ++j) {
          std::complex<T> acc = tp[0];
          for (int r = 1; r < p; ++r) acc += tp[r] * w((long)((r * j) % p) * (n / p), inv);
          out[k + (size_t)j * q] = acc;
        }
      }
    }
  }
  void run(std::complex<T> *x, bool inv, std::vector<std::complex<T>> &scratch) const {
    scratch.assign(x, x + n);
    rec(scratch.data(), 1, x, n, 0, 1, inv);
  }
};

// ---------------------------------------------------------------------------
// Radial weight table: apps/tilt/src/main.rs:348-369
// ---------------------------------------------------------------------------
template <typename T>
void weight_table(int n, T cutoff, T falloff, int efs, int hamming, T *wt) {
  size_t filter_nxc = efs > 0 ? (size_t)efs : (size_t)(n / 2 + 1);
  for (int i = 0; i < n; ++i) {
    int fb = i <= n / 2 ? i : n - i;
    T w = (T)fb / (T)filter_nxc;
    T weight;
    if (hamming) {
      T h;
      if (cutoff > (T)1e-12f && w <= cutoff)
        h = (T)0.54f + (T)0.46f * K<T>::cos_(K<T>::pi() * w / cutoff);
      else if (w > cutoff)
        h = 0;
      else
        h = 1;
      weight = w * h;
    } else if (w <= cutoff) {
      weight = w;
    } else {
      T d = w - cutoff;
      weight = w * K<T>::exp_(-d * d / ((T)2.0 * falloff * falloff));
    }
    wt[i] = weight;
  }
}

// apps/tilt/src/main.rs:333-381 (rows processed in parallel like par_chunks_mut)
template <typename T>
void rweight(T *data, int nx, int nrows, T cutoff, T falloff, int efs, int hamming, int nthreads) {
  std::vector<T> wt(nx);
  weight_table<T>(nx, cutoff, falloff, efs, hamming, wt.data());
  FftPlan<T> plan(nx);
  T inv_n = (T)1.0 / (T)nx;
  int nt = std::max(1, nthreads);
  // contiguous blocks of rows per task keep per-thread buffers reusable
  int nblk = std::min(nrows, nt * 16);
  if (nblk < 1) return;
  parallel_for(nblk, nt, [&](int b) {
    long r0 = (long)nrows * b / nblk, r1 = (long)nrows * (b + 1) / nblk;
    std::vector<std::complex<T>> buf(nx), scratch;
    for (long r = r0; r < r1; ++r) {
      T *row = data + (size_t)r * nx;
      for (int i = 0; i < nx; ++i) buf[i] = std::complex<T>(row[i], (T)0);
      plan.run(buf.data(), false, scratch);
      for (int i = 0; i < nx; ++i) buf[i] = std::complex<T>(buf[i].real() * wt[i], buf[i].imag() * wt[i]);
      plan.run(buf.data(), true, scratch);
      for (int i = 0; i < nx; ++i) row[i] = buf[i].real() * inv_n;
    }
  });
}

// apps/tilt/src/main.rs:411-420
template <typename T> T cubic_interp_1d(T p0, T p1, T p2, T p3, T t) {
  T t2 = t * t;
  T t3 = t2 * t;
  T a = (T)-0.5 * p0 + (T)1.5 * p1 - (T)1.5 * p2 + (T)0.5 * p3;
  T b = p0 - (T)2.5 * p1 + (T)2.0 * p2 - (T)0.5 * p3;
  T c = (T)-0.5 * p0 + (T)0.5 * p2;
  T d = p1;
  return a * t3 + b * t2 + c * t + d;
}

// apps/tilt/src/main.rs:425-441.  G: type of the sampling geometry, T: of the data.
template <typename G, typename T> T sample_row_cubic(const T *row, G src_x, int len) {
  G fl = K<G>::floor_(src_x);
  long sx0 = (long)fl;
  T frac = (T)(src_x - (G)sx0);
  if (sx0 >= 1 && sx0 + 2 < len) {
    long i = sx0;
    return cubic_interp_1d<T>(row[i - 1], row[i], row[i + 1], row[i + 2], frac);
  } else if (sx0 >= 0 && sx0 + 1 < len) {
    T f2 = (T)(src_x - (G)sx0);
    return row[sx0] * ((T)1.0 - f2) + row[sx0 + 1] * f2;
  } else if (sx0 >= 0 && sx0 < len) {
    return row[sx0];
  }
  return (T)0;
}

// apps/tilt/src/main.rs:446-488.  Rows [r0, r1) of every view only.
template <typename G, typename T>
int cosine_stretch(T *data, int nx, int ny, int nz, const float *angles, int n_angles, int cubic,
                   G max_tilt, int r0, int r1) {
  G center = (G)nx / (G)2.0;
  std::vector<T> orig(nx);
  for (int p = 0; p < nz; ++p) {
    if (p >= n_angles) return -10;  // tilt_angles[p] out of bounds: the reference panics
    G ang = (G)angles[p];
    G angle_abs = K<G>::fabs_(ang);
    if (angle_abs > max_tilt) continue;
    G rad = ang * K<G>::pi() / (G)180.0;
    G cos_t = K<G>::cos_(rad);
    if (K<G>::fabs_(cos_t) < (G)1e-6f) continue;
    G stretch = (G)1.0 / cos_t;
    for (int iy = r0; iy < r1; ++iy) {
      T *out = data + ((size_t)p * ny + iy) * nx;
      std::memcpy(orig.data(), out, sizeof(T) * nx);
      for (int ox = 0; ox < nx; ++ox) {
        G dx = (G)ox - center;
        G src_x = dx * stretch + center;
        if (cubic) {
          out[ox] = sample_row_cubic<G, T>(orig.data(), src_x, nx);
        } else {
          long sx0 = (long)K<G>::floor_(src_x);
          if (sx0 >= 0 && sx0 + 1 < nx) {
            T frac = (T)(src_x - (G)sx0);
            out[ox] = orig[sx0] * ((T)1.0 - frac) + orig[sx0 + 1] * frac;
          } else if (sx0 >= 0 && sx0 < nx) {
            out[ox] = orig[sx0];
          } else {
            out[ox] = (T)0;
          }
        }
      }
    }
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Local alignment grid: apps/tilt/src/main.rs:143-307
// ---------------------------------------------------------------------------
template <typename T> struct ViewPatches {
  std::vector<T> xs, ys, dx, dy;
  static void find_bracket(const std::vector<T> &pos, T val, size_t &idx, T &frac) {
    if (pos.size() == 1) { idx = 0; frac = 0; return; }
    size_t lo = 0, hi = pos.size() - 1;
    if (val <= pos[lo]) { idx = 0; frac = 0; return; }
    if (val >= pos[hi]) { idx = hi; frac = 0; return; }
    while (hi - lo > 1) {
      size_t mid = (lo + hi) / 2;
      if (pos[mid] <= val) lo = mid; else hi = mid;
    }
    T span = pos[hi] - pos[lo];
    frac = span > (T)1e-12f ? (val - pos[lo]) / span : (T)0;
    idx = lo;
  }
  void interpolate(T x, T y, T &odx, T &ody) const {
    if (xs.empty() || ys.empty()) { odx = 0; ody = 0; return; }
    size_t nx = xs.size(), ny = ys.size(), ix0, iy0;
    T fx, fy;
    find_bracket(xs, x, ix0, fx);
    find_bracket(ys, y, iy0, fy);
    size_t ix1 = std::min(ix0 + 1, nx - 1), iy1 = std::min(iy0 + 1, ny - 1);
    auto lerp = [](T a, T b, T t) { return a + t * (b - a); };
    odx = lerp(lerp(dx[iy0 * nx + ix0], dx[iy0 * nx + ix1], fx), lerp(dx[iy1 * nx + ix0], dx[iy1 * nx + ix1], fx), fy);
    ody = lerp(lerp(dy[iy0 * nx + ix0], dy[iy0 * nx + ix1], fx), lerp(dy[iy1 * nx + ix0], dy[iy1 * nx + ix1], fx), fy);
  }
};

template <typename T>
std::vector<ViewPatches<T>> load_local(const float *rows, int nrows, int nz) {
  std::vector<ViewPatches<T>> views(nz);
  std::vector<std::vector<int>> by_view(nz);
  for (int i = 0; i < nrows; ++i) {
    long v = (long)rows[i * 5 + 0];
    if (v >= 0 && v < nz) by_view[v].push_back(i);
  }
  auto dedup = [](std::vector<T> &v) {  // Vec::dedup_by(|a,b| |a-b| < 0.01)
    std::vector<T> out;
    for (T e : v)
      if (out.empty() || !(K<T>::fabs_(e - out.back()) < (T)0.01f)) out.push_back(e);
    v.swap(out);
  };
  for (int vi = 0; vi < nz; ++vi) {
    auto &idx = by_view[vi];
    if (idx.empty()) continue;
    ViewPatches<T> vp;
    for (int i : idx) { vp.xs.push_back((T)rows[i * 5 + 1]); vp.ys.push_back((T)rows[i * 5 + 2]); }
    std::stable_sort(vp.xs.begin(), vp.xs.end());
    dedup(vp.xs);
    std::stable_sort(vp.ys.begin(), vp.ys.end());
    dedup(vp.ys);
    size_t nx = vp.xs.size(), ny = vp.ys.size();
    vp.dx.assign(nx * ny, (T)0);
    vp.dy.assign(nx * ny, (T)0);
    for (int i : idx) {
      T px = (T)rows[i * 5 + 1], py = (T)rows[i * 5 + 2];
      size_t ix = 0, iy = 0;
      for (size_t k = 0; k < nx; ++k) if (K<T>::fabs_(vp.xs[k] - px) < (T)0.01f) { ix = k; break; }
      for (size_t k = 0; k < ny; ++k) if (K<T>::fabs_(vp.ys[k] - py) < (T)0.01f) { iy = k; break; }
      vp.dx[iy * nx + ix] = (T)rows[i * 5 + 3];
      vp.dy[iy * nx + ix] = (T)rows[i * 5 + 4];
    }
    views[vi] = std::move(vp);
  }
  return views;
}

// ---------------------------------------------------------------------------
// Per-view geometry: apps/tilt/src/main.rs:683-700 (ProjParams 131-140)
// ---------------------------------------------------------------------------
template <typename T> struct ProjParams { T cos_t, sin_t, cos_xt, sin_xt, zf; };

template <typename T> std::vector<ProjParams<T>> proj_params(const or_params *p) {
  std::vector<ProjParams<T>> out;
  int nv = std::min(p->n_angles, p->nz);  // tilt_angles.iter().take(nz)
  for (int i = 0; i < nv; ++i) {
    T deg = (T)p->angles[i];
    T rad = deg * K<T>::pi() / (T)180.0;
    T xt_deg = (p->xtilt && i < p->n_xtilt) ? (T)p->xtilt[i] : (T)0;
    T xt_rad = xt_deg * K<T>::pi() / (T)180.0;
    T zf = (p->zfac && i < p->n_zfac) ? (T)p->zfac[i] : (T)1;
    out.push_back({K<T>::cos_(rad), K<T>::sin_(rad), K<T>::cos_(xt_rad), K<T>::sin_(xt_rad), zf});
  }
  return out;
}

// apps/tilt/src/main.rs:386-406
template <typename G, typename T>
inline T sample_row_with_fill(const T *row, G proj_x, int row_len, int fill, T mean) {
  long px0 = (long)K<G>::floor_(proj_x);
  if (px0 >= 0 && px0 + 1 < row_len) {
    T frac = (T)(proj_x - (G)px0);
    return row[px0] * ((T)1.0 - frac) + row[px0 + 1] * frac;
  }
  switch (fill) {
    case OR_FILL_ZERO: return (T)0;
    case OR_FILL_EDGE: return px0 < 0 ? row[0] : (row_len > 0 ? row[row_len - 1] : (T)0);
    default: return mean;
  }
}

// WBP of slices [y0,y1): apps/tilt/src/main.rs:756-828 and 1008-1075
template <typename G, typename T>
void backproject(const or_params *p, const T *proj, const T *means, T *vol, int y0, int y1,
                 int nthreads) {
  const int in_nx = p->nx, in_ny = p->ny, nz = p->nz, out_nx = p->out_nx, out_nz = p->out_nz;
  auto pps = proj_params<G>(p);
  std::vector<ViewPatches<G>> la;
  const bool has_la = p->has_local != 0;
  if (has_la) la = load_local<G>(p->local, p->n_local, nz);
  const G center_x = (G)in_nx / (G)2.0, center_z = (G)out_nz / (G)2.0,
          out_center_x = (G)out_nx / (G)2.0;
  const T inv_n = (T)1.0 / (T)nz;
  const int fill = p->fill_mode;
  auto do_row = [&](int iy) {
    T *slice = vol + (size_t)(iy - y0) * out_nz * out_nx;
    std::fill(slice, slice + (size_t)out_nz * out_nx, (T)0);
    for (size_t pi = 0; pi < pps.size(); ++pi) {
      const ProjParams<G> &pp = pps[pi];
      const T pm = means[pi];
      for (int oz = 0; oz < out_nz; ++oz) {
        G dz = (G)oz - center_z;
        G z_contrib = dz * pp.sin_t * pp.zf;
        T *srow = slice + (size_t)oz * out_nx;
        for (int ox = 0; ox < out_nx; ++ox) {
          G dx = (G)ox - out_center_x;
          G proj_x = dx * pp.cos_t * pp.cos_xt + z_contrib + center_x;
          G proj_y_offset = dx * pp.sin_xt;
          G ldx = 0, ldy = 0;
          bool use_l = has_la && !la[pi].xs.empty();
          if (use_l) { la[pi].interpolate((G)ox, (G)iy, ldx, ldy); proj_x += ldx; }
          G sample_y = (G)iy + proj_y_offset;
          if (use_l) sample_y = sample_y + ldy;
          long sy0 = (long)K<G>::floor_(sample_y);
          T sy_frac = (T)(sample_y - (G)sy0);
          if (sy0 >= 0 && sy0 + 1 < in_ny && (K<G>::fabs_(proj_y_offset) > (G)1e-6f || has_la)) {
            const T *row0 = proj + ((size_t)pi * in_ny + sy0) * in_nx;
            const T *row1 = row0 + in_nx;
            T v0 = sample_row_with_fill<G, T>(row0, proj_x, in_nx, fill, pm);
            T v1 = sample_row_with_fill<G, T>(row1, proj_x, in_nx, fill, pm);
            srow[ox] += v0 * ((T)1.0 - sy_frac) + v1 * sy_frac;
          } else if (sy0 >= 0 && sy0 < in_ny) {
            const T *row = proj + ((size_t)pi * in_ny + sy0) * in_nx;
            srow[ox] += sample_row_with_fill<G, T>(row, proj_x, in_nx, fill, pm);
          }
        }
      }
    }
    for (size_t i = 0; i < (size_t)out_nz * out_nx; ++i) slice[i] *= inv_n;
  };
  // rayon-style: chunks of max(32, out_ny/20) rows, rows of a chunk in parallel (main.rs:709,1004-1010)
  int out_ny = in_ny;
  int chunk = std::max(32, out_ny / 20);
  for (int c0 = y0; c0 < y1; c0 += chunk) {
    int c1 = std::min(y1, c0 + chunk);
    parallel_for(c1 - c0, nthreads, [&](int i) { do_row(c0 + i); });
  }
}

// GPU form: apps/tilt/src/backproject.wgsl:26-64 driven by gpu.rs:224-269
template <typename G, typename T>
void backproject_wgsl(const or_params *p, const T *proj, T *vol, int y0, int y1, int nthreads) {
  const int in_nx = p->nx, in_ny = p->ny, nz = p->nz, out_nx = p->out_nx, out_nz = p->out_nz;
  auto pps = proj_params<G>(p);
  const G center_x = (G)in_nx / (G)2.0, center_z = (G)out_nz / (G)2.0,
          out_center_x = (G)out_nx / (G)2.0;
  const T inv_n = (T)1.0 / (T)nz;
  parallel_for(y1 - y0, nthreads, [&](int i) {
    int iy = y0 + i;
    T *slice = vol + (size_t)i * out_nz * out_nx;
    for (int oz = 0; oz < out_nz; ++oz)
      for (int ox = 0; ox < out_nx; ++ox) {
        G dx = (G)ox - out_center_x, dz = (G)oz - center_z;
        T acc = 0;
        for (size_t pi = 0; pi < pps.size(); ++pi) {
          G proj_x = dx * pps[pi].cos_t + dz * pps[pi].sin_t + center_x;
          long px0 = (long)K<G>::floor_(proj_x);
          if (px0 >= 0 && px0 + 1 < in_nx) {
            T frac = (T)(proj_x - (G)px0);
            const T *row = proj + ((size_t)pi * in_ny + iy) * in_nx;
            acc += row[px0] * ((T)1.0 - frac) + row[px0 + 1] * frac;
          }
        }
        slice[(size_t)oz * out_nx + ox] = acc * inv_n;
      }
  });
}

// apps/tilt/src/main.rs:831-896 (serial, as in the reference)
template <typename G, typename T> void forward_project(const or_params *p, const T *vol, T *sino) {
  const int in_nx = p->nx, in_ny = p->ny, nz = p->nz, out_nx = p->out_nx, out_nz = p->out_nz;
  auto pps = proj_params<G>(p);
  std::vector<ViewPatches<G>> la;
  const bool has_la = p->has_local != 0;
  if (has_la) la = load_local<G>(p->local, p->n_local, nz);
  const G center_x = (G)in_nx / (G)2.0, center_z = (G)out_nz / (G)2.0,
          out_center_x = (G)out_nx / (G)2.0;
  std::fill(sino, sino + (size_t)nz * in_nx * in_ny, (T)0);
  for (int iy = 0; iy < in_ny; ++iy) {
    const T *slice = vol + (size_t)iy * out_nz * out_nx;
    for (size_t pi = 0; pi < pps.size(); ++pi) {
      const ProjParams<G> &pp = pps[pi];
      for (int oz = 0; oz < out_nz; ++oz) {
        G dz = (G)oz - center_z;
        G z_contrib = dz * pp.sin_t * pp.zf;
        for (int ox = 0; ox < out_nx; ++ox) {
          G dx = (G)ox - out_center_x;
          G proj_x = dx * pp.cos_t * pp.cos_xt + z_contrib + center_x;
          G proj_y_offset = dx * pp.sin_xt;
          G ldx = 0, ldy = 0;
          bool use_l = has_la && !la[pi].xs.empty();
          if (use_l) { la[pi].interpolate((G)ox, (G)iy, ldx, ldy); proj_x += ldx; }
          G sample_y = (G)iy + proj_y_offset;
          if (use_l) sample_y = sample_y + ldy;
          long px0 = (long)K<G>::floor_(proj_x);
          if (px0 >= 0 && px0 + 1 < in_nx) {
            T frac = (T)(proj_x - (G)px0);
            T val = slice[(size_t)oz * out_nx + ox];
            long sy0 = (long)K<G>::floor_(sample_y);
            T sy_frac = (T)(sample_y - (G)sy0);
            if (sy0 >= 0 && sy0 + 1 < in_ny && (K<G>::fabs_(proj_y_offset) > (G)1e-6f || has_la)) {
              size_t row0 = ((size_t)pi * in_ny + sy0) * in_nx, row1 = row0 + in_nx;
              T w0 = (T)1.0 - sy_frac, w1 = sy_frac;
              sino[row0 + px0] += val * ((T)1.0 - frac) * w0;
              sino[row0 + px0 + 1] += val * frac * w0;
              sino[row1 + px0] += val * ((T)1.0 - frac) * w1;
              sino[row1 + px0 + 1] += val * frac * w1;
            } else if (sy0 >= 0 && sy0 < in_ny) {
              size_t r = ((size_t)pi * in_ny + sy0) * in_nx;
              sino[r + px0] += val * ((T)1.0 - frac);
              sino[r + px0 + 1] += val * frac;
            }
          }
        }
      }
    }
  }
}

// apps/tilt/src/main.rs:493-538
template <typename T> void lowpass3d(T *vol, int out_nx, int out_nz, int out_ny) {
  if (out_ny == 0) return;
  size_t sl = (size_t)out_nx * out_nz;
  std::vector<T> tmp(sl);
  for (int iy = 0; iy < out_ny; ++iy) {
    T *v = vol + iy * sl;
    for (int oz = 0; oz < out_nz; ++oz) {
      size_t r = (size_t)oz * out_nx;
      for (int ox = 0; ox < out_nx; ++ox) {
        int x0 = ox > 0 ? ox - 1 : 0, x2 = ox + 1 < out_nx ? ox + 1 : out_nx - 1;
        tmp[r + ox] = (v[r + x0] + v[r + ox] + v[r + x2]) / (T)3.0;
      }
    }
    std::memcpy(v, tmp.data(), sl * sizeof(T));
  }
  for (int iy = 0; iy < out_ny; ++iy) {
    T *v = vol + iy * sl;
    for (int oz = 0; oz < out_nz; ++oz) {
      int z0 = oz > 0 ? oz - 1 : 0, z2 = oz + 1 < out_nz ? oz + 1 : out_nz - 1;
      for (int ox = 0; ox < out_nx; ++ox)
        tmp[(size_t)oz * out_nx + ox] =
            (v[(size_t)z0 * out_nx + ox] + v[(size_t)oz * out_nx + ox] + v[(size_t)z2 * out_nx + ox]) / (T)3.0;
    }
    std::memcpy(v, tmp.data(), sl * sizeof(T));
  }
  std::vector<T> prev(vol, vol + sl * out_ny);
  for (int iy = 0; iy < out_ny; ++iy) {
    int y0 = iy > 0 ? iy - 1 : 0, y2 = iy + 1 < out_ny ? iy + 1 : out_ny - 1;
    for (size_t i = 0; i < sl; ++i) vol[iy * sl + i] = (prev[y0 * sl + i] + prev[iy * sl + i] + prev[y2 * sl + i]) / (T)3.0;
  }
}

// min_max_mean: crates/imod-math/src/stats.rs:844-861
template <typename T> void min_max_mean(const T *d, size_t n, T &mn, T &mx, T &mean) {
  if (n == 0) { mn = mx = mean = 0; return; }
  mn = K<T>::maxv(); mx = K<T>::minv();
  double sum = 0.0;
  for (size_t i = 0; i < n; ++i) {
    T x = d[i];
    if (x < mn) mn = x;
    if (x > mx) mx = x;
    sum += (double)x;
  }
  mean = (T)(sum / (double)n);
}

// output transform + stats: apps/tilt/src/main.rs:1077-1093 (and 965-975)
template <typename T>
void output_stats(T *vol, int out_nx, int out_nz, int out_ny, T dw, T os, T oa, or_stats *st) {
  T gmin = K<T>::maxv(), gmax = K<T>::minv();
  double gsum = 0.0;
  size_t sl = (size_t)out_nx * out_nz;
  for (int iy = 0; iy < out_ny; ++iy) {
    T *s = vol + iy * sl;
    for (size_t i = 0; i < sl; ++i) s[i] = (s[i] * dw) * os + oa;
    T smin, smax, smean;
    min_max_mean<T>(s, sl, smin, smax, smean);
    if (smin < gmin) gmin = smin;
    if (smax > gmax) gmax = smax;
    gsum += (double)smean * (double)sl;
  }
  if (st) {
    st->amin = (float)gmin;
    st->amax = (float)gmax;
    st->amean = (float)(gsum / (double)(sl * (size_t)out_ny));
  }
}

// The body of main() between reading and writing: apps/tilt/src/main.rs:607-1093.
// G = type of sampling geometry, T = type of data values.
template <typename G, typename T>
int run(const or_params *p, const float *proj_in, T *vol, or_stats *st, int nthreads) {
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  if (nx <= 0 || ny <= 0 || nz <= 0 || p->out_nx <= 0 || p->out_nz <= 0) return -1;
  const size_t n = (size_t)nx * ny * nz;
  std::vector<T> proj(proj_in, proj_in + n);
  if (p->log_transform)
    for (auto &v : proj) v = K<T>::log10_(std::fmax(v, (T)0.001f));  // main.rs:608-613 (f32::max = fmax)
  std::vector<T> means(nz);
  for (int v = 0; v < nz; ++v) {  // main.rs:616-623
    T a, b;
    min_max_mean<T>(proj.data() + (size_t)v * nx * ny, (size_t)nx * ny, a, b, means[v]);
  }
  std::vector<T> orig;
  if (p->sirt_iters > 0) orig = proj;  // main.rs:626-630
  if (!p->no_weight)
    rweight<T>(proj.data(), nx, ny * nz, (T)p->cutoff, (T)p->falloff, p->exact_filter_size,
               p->hamming, nthreads);
  if (!p->no_cosine_stretch) {
    int rc = cosine_stretch<G, T>(proj.data(), nx, ny, nz, p->angles, p->n_angles, p->cosine_cubic,
                                  (G)p->max_cosine_tilt, 0, ny);
    if (rc) return rc;
  }
  const int out_nx = p->out_nx, out_nz = p->out_nz, out_ny = ny;
  const size_t vn = (size_t)out_nx * out_nz * out_ny;
  if (p->gpu_compat) {  // main.rs:898-918 (takes precedence over SIRT)
    backproject_wgsl<G, T>(p, proj.data(), vol, 0, ny, nthreads);
  } else if (p->sirt_iters > 0) {  // main.rs:919-975
    backproject<G, T>(p, proj.data(), means.data(), vol, 0, ny, nthreads);
    std::vector<T> reproj(n), delta(vn);
    for (int it = 0; it < p->sirt_iters; ++it) {
      forward_project<G, T>(p, vol, reproj.data());
      for (size_t i = 0; i < n; ++i) reproj[i] = orig[i] - reproj[i];
      if (!p->no_weight)
        rweight<T>(reproj.data(), nx, ny * nz, (T)p->cutoff, (T)p->falloff, p->exact_filter_size,
                   p->hamming, nthreads);
      backproject<G, T>(p, reproj.data(), means.data(), delta.data(), 0, ny, nthreads);
      T relax = (T)p->sirt_relax;
      for (size_t i = 0; i < vn; ++i) vol[i] += relax * delta[i];
    }
    for (int k = 0; k < p->fake_sirt; ++k) lowpass3d<T>(vol, out_nx, out_nz, out_ny);
  } else {
    backproject<G, T>(p, proj.data(), means.data(), vol, 0, ny, nthreads);
    for (int k = 0; k < p->fake_sirt; ++k) lowpass3d<T>(vol, out_nx, out_nz, out_ny);
  }
  output_stats<T>(vol, out_nx, out_nz, out_ny, (T)p->densweight, (T)p->outscale, (T)p->outadd, st);
  return 0;
}

}  // namespace

extern "C" {

void or_log_transform32(float *d, size_t n) {
  for (size_t i = 0; i < n; ++i) d[i] = log10f(std::fmax(d[i], 0.001f));
}
void or_view_means32(const float *d, int nx, int ny, int nz, float *means) {
  for (int v = 0; v < nz; ++v) {
    float a, b;
    min_max_mean<float>(d + (size_t)v * nx * ny, (size_t)nx * ny, a, b, means[v]);
  }
}
void or_weight_table32(int n, float c, float f, int efs, int h, float *w) { weight_table<float>(n, c, f, efs, h, w); }
void or_weight_table64(int n, double c, double f, int efs, int h, double *w) { weight_table<double>(n, c, f, efs, h, w); }
void or_rweight32(float *d, int nx, int nrows, float c, float f, int efs, int h, int nt) {
  rweight<float>(d, nx, nrows, c, f, efs, h, nt);
}
void or_rweight64(double *d, int nx, int nrows, double c, double f, int efs, int h, int nt) {
  rweight<double>(d, nx, nrows, c, f, efs, h, nt);
}
void or_cosine_stretch32(float *d, int nx, int ny, int nz, const float *a, int na, int cubic, float mt) {
  cosine_stretch<float, float>(d, nx, ny, nz, a, na, cubic, mt, 0, ny);
}
void or_fft32(float *reim, int n, int inverse) {
  FftPlan<float> p(n);
  std::vector<std::complex<float>> s;
  p.run(reinterpret_cast<std::complex<float> *>(reim), inverse != 0, s);
}
void or_fft64(double *reim, int n, int inverse) {
  FftPlan<double> p(n);
  std::vector<std::complex<double>> s;
  p.run(reinterpret_cast<std::complex<double> *>(reim), inverse != 0, s);
}
int or_backproject32(const or_params *p, const float *proj, const float *means, float *vol, int y0, int y1, int nt) {
  if (p->gpu_compat) backproject_wgsl<float, float>(p, proj, vol, y0, y1, nt);
  else backproject<float, float>(p, proj, means, vol, y0, y1, nt);
  return 0;
}
int or_backproject64(const or_params *p, const double *proj, const double *means, double *vol, int y0, int y1, int nt) {
  if (p->gpu_compat) backproject_wgsl<double, double>(p, proj, vol, y0, y1, nt);
  else backproject<double, double>(p, proj, means, vol, y0, y1, nt);
  return 0;
}
int or_forward_project32(const or_params *p, const float *vol, float *sino) { forward_project<float, float>(p, vol, sino); return 0; }
int or_forward_project64(const or_params *p, const double *vol, double *sino) { forward_project<double, double>(p, vol, sino); return 0; }
void or_lowpass32(float *v, int a, int b, int c) { lowpass3d<float>(v, a, b, c); }
void or_lowpass64(double *v, int a, int b, int c) { lowpass3d<double>(v, a, b, c); }
int or_run32(const or_params *p, const float *proj, float *vol, or_stats *st, int nt) { return run<float, float>(p, proj, vol, st, nt); }
int or_run64(const or_params *p, const float *proj, double *vol, or_stats *st, int nt) { return run<double, double>(p, proj, vol, st, nt); }
int or_run64g(const or_params *p, const float *proj, double *vol, or_stats *st, int nt) { return run<float, double>(p, proj, vol, st, nt); }
int or_backproject64g(const or_params *p, const double *proj, const double *means, double *vol, int y0, int y1, int nt) {
  if (p->gpu_compat) backproject_wgsl<float, double>(p, proj, vol, y0, y1, nt);
  else backproject<float, double>(p, proj, means, vol, y0, y1, nt);
  return 0;
}
int or_forward_project64g(const or_params *p, const double *vol, double *sino) { forward_project<float, double>(p, vol, sino); return 0; }
void or_output_stats32(float *vol, int a, int b, int c, float dw, float os, float oa, or_stats *st) {
  output_stats<float>(vol, a, b, c, dw, os, oa, st);
}

}  // extern "C"

namespace {
// The reference's WBP flow (main.rs:607-653, 1002-1090) restricted to slices
// [y0, y1): only the projection rows those slices read are log'd, filtered and
// stretched (all rows when x-tilt or local alignment bends the rays); the
// per-view means still cover the whole view.  G = sampling geometry type,
// T = data type, as in run().
template <typename G, typename T>
int wbp_rows(const or_params *p, const float *proj_in, T *vol_rows, int y0, int y1, int nt) {
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  int halo = 0;
  if (p->xtilt || p->has_local) halo = ny;  // conservative: whole stack
  const int r0 = std::max(0, y0 - halo), r1 = std::min(ny, y1 + halo);
  std::vector<T> proj((size_t)nx * ny * nz, (T)0);
  auto logv = [&](float x) -> T { return p->log_transform ? K<T>::log10_(std::fmax((T)x, (T)0.001f)) : (T)x; };
  for (int v = 0; v < nz; ++v)
    for (size_t i = ((size_t)v * ny + r0) * nx; i < ((size_t)v * ny + r1) * nx; ++i) proj[i] = logv(proj_in[i]);
  std::vector<T> means(nz);
  parallel_for(nz, nt, [&](int v) {  // main.rs:616-623 over the whole view
    double s = 0.0;
    const float *d = proj_in + (size_t)v * nx * ny;
    for (size_t i = 0; i < (size_t)nx * ny; ++i) s += (double)logv(d[i]);
    means[v] = (T)(s / (double)((size_t)nx * ny));
  });
  std::vector<T> rows((size_t)nz * (r1 - r0) * nx);  // the band rows, contiguous for the FFT
  for (int v = 0; v < nz; ++v)
    std::memcpy(&rows[(size_t)v * (r1 - r0) * nx], &proj[((size_t)v * ny + r0) * nx], sizeof(T) * (size_t)(r1 - r0) * nx);
  if (!p->no_weight)
    rweight<T>(rows.data(), nx, nz * (r1 - r0), (T)p->cutoff, (T)p->falloff, p->exact_filter_size, p->hamming, nt);
  for (int v = 0; v < nz; ++v)
    std::memcpy(&proj[((size_t)v * ny + r0) * nx], &rows[(size_t)v * (r1 - r0) * nx], sizeof(T) * (size_t)(r1 - r0) * nx);
  if (!p->no_cosine_stretch) {
    int rc = cosine_stretch<G, T>(proj.data(), nx, ny, nz, p->angles, p->n_angles, p->cosine_cubic,
                                  (G)p->max_cosine_tilt, r0, r1);
    if (rc) return rc;
  }
  backproject<G, T>(p, proj.data(), means.data(), vol_rows, y0, y1, nt);
  return 0;
}
}  // namespace

extern "C" {
// Timed CPU baseline (f32, the reference's arithmetic) and its FP64 form with the
// reference's f32 sampling geometry (ref64g) for error checks on slice subsets.
int or_wbp_rows32(const or_params *p, const float *proj_in, float *vol_rows, int y0, int y1, int nt) {
  return wbp_rows<float, float>(p, proj_in, vol_rows, y0, y1, nt);
}
int or_wbp_rows64g(const or_params *p, const float *proj_in, double *vol_rows, int y0, int y1, int nt) {
  return wbp_rows<float, double>(p, proj_in, vol_rows, y0, y1, nt);
}

// The reconstruction step of imod-studio (apps/imod-studio/src/main.rs:725-776),
// restated on its own: an unweighted back-projection with zero fill, thickness =
// width, x = ((ox - cx) * cos + (oz - cz) * sin) + cx, the two-sample lerp only
// when both samples are inside the row, and the sum scaled by 1/nz (f32, in the
// reference's operation order).  out: [ny][nx (thickness)][nx].
void or_studio_reconstruct32(const float *proj, int nx, int ny, int nz, const float *angles, int n_angles,
                             float *out) {
  const int out_nz = nx;
  const float cx = (float)nx / 2.0f, cz = (float)out_nz / 2.0f;
  const float pi = 3.14159265358979323846f;
  for (int iy = 0; iy < ny; ++iy) {
    float *sl = out + (size_t)iy * out_nz * nx;
    for (size_t i = 0; i < (size_t)out_nz * nx; ++i) sl[i] = 0.0f;
    for (int pi_ = 0; pi_ < n_angles && pi_ < nz; ++pi_) {
      const float r = angles[pi_] * pi / 180.0f;
      const float cos_t = cosf(r), sin_t = sinf(r);
      const float *row = proj + ((size_t)pi_ * ny + iy) * nx;
      for (int oz = 0; oz < out_nz; ++oz) {
        const float bo = ((float)oz - cz) * sin_t;
        for (int ox = 0; ox < nx; ++ox) {
          const float px = ((float)ox - cx) * cos_t + bo + cx;
          const long p0 = (long)floorf(px);
          if (p0 >= 0 && p0 + 1 < nx) {
            const float f = px - (float)p0;
            sl[(size_t)oz * nx + ox] += row[p0] * (1.0f - f) + row[p0 + 1] * f;
          }
        }
      }
    }
    const float inv = 1.0f / (float)nz;
    for (size_t i = 0; i < (size_t)out_nz * nx; ++i) sl[i] *= inv;
  }
}

}  // extern "C"

// f32 transform of any length for the ctfphaseflip restatement (ctf_oracle.cpp),
// plans cached per length and thread
namespace ctf_detail {
void fft32(std::complex<float> *x, int n, bool inverse) {
  thread_local std::vector<std::unique_ptr<FftPlan<float>>> plans;
  thread_local std::vector<std::complex<float>> scratch;
  FftPlan<float> *pl = nullptr;
  for (auto &q : plans)
    if (q->n == n) pl = q.get();
  if (!pl) {
    plans.emplace_back(new FftPlan<float>(n));
    pl = plans.back().get();
  }
  pl->run(x, inverse, scratch);
}
}  // namespace ctf_detail
