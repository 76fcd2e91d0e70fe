// synth.cu -- seeded synthetic tilt series: analytic line integrals through a
// random ellipsoid + bead phantom, in the geometry the back-projector inverts
// (projection x = dx*cos(t)*cos(xi) + dz*sin(t) + nx/2, row = y + dx*sin(xi)),
// plus Gaussian or Poisson noise from a counter-based generator, so every
// pixel is a pure function of (seed, index).  Workload generator only; it has
// no counterpart in the reference.
#include <math.h>

#include <algorithm>
#include <vector>

#include "tg_internal.h"

namespace tg {

struct Ell {  // 16 floats
  float cx, cy, cz, dens;
  float m[9];  // diag(1/axes) * R^T
  float pad[3];
};

static inline uint64_t splitmix64(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline double urand(uint64_t &s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double dev_u01(uint64_t seed, uint64_t idx, uint64_t k) {
  uint64_t z = mix64(seed ^ mix64(idx * 0x9E3779B97F4A7C15ull + k + 1));
  return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

__global__ void project_kernel(const Ell *ells, const int *row_off, const int *row_list,
                               const float *angles, int nx, int ny, float vol_cx, float vol_cz,
                               float xtilt_rad, float *out) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y, v = blockIdx.z;
  if (ix >= nx) return;
  const double th = (double)angles[v] * 3.14159265358979323846 / 180.0;
  const double ct = cos(th), st = sin(th), cxi = cos((double)xtilt_rad), sxi = sin((double)xtilt_rad);
  const double a = ct * cxi, b = st;
  const double den = a * a + b * b;
  const double u = (double)ix - 0.5 * nx;
  // a point on the ray and the ray direction (unit)
  const double dx0 = u * a / den, dz0 = u * b / den, y0 = (double)iy - dx0 * sxi;
  double d0 = b, d1 = -b * sxi, d2 = -a;  // satisfies a*d0 + b*d2 = 0 and d1 + d0*sxi = 0
  const double dn = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  d0 /= dn; d1 /= dn; d2 /= dn;
  double sum = 0.0;
  for (int e = row_off[iy]; e < row_off[iy + 1]; ++e) {
    const Ell E = ells[row_list[e]];
    const double px = dx0 + vol_cx - E.cx, py = y0 - E.cy, pz = dz0 + vol_cz - E.cz;
    const double q0 = E.m[0] * px + E.m[1] * py + E.m[2] * pz;
    const double q1 = E.m[3] * px + E.m[4] * py + E.m[5] * pz;
    const double q2 = E.m[6] * px + E.m[7] * py + E.m[8] * pz;
    const double e0 = E.m[0] * d0 + E.m[1] * d1 + E.m[2] * d2;
    const double e1 = E.m[3] * d0 + E.m[4] * d1 + E.m[5] * d2;
    const double e2 = E.m[6] * d0 + E.m[7] * d1 + E.m[8] * d2;
    const double ee = e0 * e0 + e1 * e1 + e2 * e2, qe = q0 * e0 + q1 * e1 + q2 * e2,
                 qq = q0 * q0 + q1 * q1 + q2 * q2;
    const double disc = qe * qe - ee * (qq - 1.0);
    if (disc > 0.0) sum += (double)E.dens * 2.0 * sqrt(disc) / ee;
  }
  out[((size_t)v * ny + iy) * nx + ix] = (float)sum;
}

__global__ void moments_kernel(const float *x, size_t n, double *part) {
  double s = 0.0, s2 = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double v = x[i];
    s += v;
    s2 += v * v;
  }
  __shared__ double r1[8], r2[8];
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) { r1[threadIdx.x >> 5] = s; r2[threadIdx.x >> 5] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int k = 0; k < 8; ++k) { a += r1[k]; b += r2[k]; }
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

__global__ void noise_kernel(float *x, size_t n, int kind, double sigma, double base, double mu,
                             uint64_t seed) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double u1 = dev_u01(seed, i, 0), u2 = dev_u01(seed, i, 1);
    double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    if (kind == 1) {
      x[i] = (float)((double)x[i] + sigma * z);
    } else {
      double lam = base * exp(-mu * (double)x[i]);
      double c;
      if (lam < 40.0) {  // inversion by multiplication (Knuth)
        double L = exp(-lam), p = 1.0;
        int k = 0;
        for (int t = 0; t < 400; ++t) {
          p *= dev_u01(seed, i, 2 + t);
          if (p <= L) break;
          ++k;
        }
        c = k;
      } else {
        c = floor(lam + sqrt(lam) * z + 0.5);
        if (c < 0) c = 0;
      }
      x[i] = (float)c;
    }
  }
}

int synth_projections(const tg_phantom_spec *sp, const float *angles_host, float *d_out,
                      cudaStream_t st) {
  const int nx = sp->nx, ny = sp->ny, nz = sp->nz;
  if (nx <= 0 || ny <= 0 || nz <= 0 || sp->vol_nx <= 0 || sp->vol_nz <= 0) return TG_ERR_INVALID_ARG;
  uint64_t s = sp->seed * 0x2545F4914F6CDD1Dull + 12345;
  std::vector<Ell> ells;
  std::vector<float> ylo, yhi;
  auto add = [&](double cx, double cy, double cz, double a, double b, double c, double q0, double q1,
                 double q2, double q3, double dens) {
    // rotation matrix from the unit quaternion
    double R[9] = {1 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2),
                   2 * (q1 * q2 + q0 * q3), 1 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1),
                   2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1 - 2 * (q1 * q1 + q2 * q2)};
    double ax[3] = {a, b, c};
    Ell E{};
    E.cx = (float)cx; E.cy = (float)cy; E.cz = (float)cz; E.dens = (float)dens;
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) E.m[r * 3 + k] = (float)(R[k * 3 + r] / ax[r]);  // (R^T)[r][k]/ax[r]
    ells.push_back(E);
    double rm = std::max(a, std::max(b, c));
    ylo.push_back((float)(cy - rm));
    yhi.push_back((float)(cy + rm));
  };
  auto pick = [&](double lo, double hi) { return hi > lo ? lo + (hi - lo) * urand(s) : 0.5 * (lo + hi); };
  for (int i = 0; i < sp->n_ell; ++i) {
    double a = pick(sp->rmin, sp->rmax), b = pick(sp->rmin, sp->rmax), c = pick(sp->rmin, sp->rmax);
    double m = sp->rmax;
    double cx = pick(m, sp->vol_nx - m), cy = pick(m, ny - m), cz = pick(m, sp->vol_nz - m);
    // uniform random rotation (Shoemake)
    double u1 = urand(s), u2 = urand(s), u3 = urand(s);
    double q0 = sqrt(1 - u1) * sin(2 * M_PI * u2), q1 = sqrt(1 - u1) * cos(2 * M_PI * u2);
    double q2 = sqrt(u1) * sin(2 * M_PI * u3), q3 = sqrt(u1) * cos(2 * M_PI * u3);
    add(cx, cy, cz, a, b, c, q0, q1, q2, q3, pick(sp->dmin, sp->dmax));
  }
  for (int i = 0; i < sp->n_beads; ++i) {
    double m = sp->bead_r;
    double cx = pick(m, sp->vol_nx - m), cy = pick(m, ny - m), cz = pick(m, sp->vol_nz - m);
    add(cx, cy, cz, sp->bead_r, sp->bead_r, sp->bead_r, 1, 0, 0, 0, sp->bead_d);
  }
  // rows each ellipsoid can reach (x-tilt bends rows by up to vol_nx/2*|sin(xi)|)
  const double xi = (double)sp->xtilt_deg * M_PI / 180.0;
  const double margin = 0.5 * sp->vol_nx * fabs(sin(xi)) + 2.0;
  std::vector<int> off(ny + 1, 0), list;
  std::vector<std::vector<int>> rows(ny);
  for (size_t e = 0; e < ells.size(); ++e) {
    int a = std::max(0, (int)floor(ylo[e] - margin)), b = std::min(ny - 1, (int)ceil(yhi[e] + margin));
    for (int y = a; y <= b; ++y) rows[y].push_back((int)e);
  }
  for (int y = 0; y < ny; ++y) {
    off[y + 1] = off[y] + (int)rows[y].size();
    list.insert(list.end(), rows[y].begin(), rows[y].end());
  }
  Ell *d_ell = nullptr;
  int *d_off = nullptr, *d_list = nullptr;
  float *d_ang = nullptr;
  double *d_part = nullptr;
  const int NB = 1184;
  TG_CUDA(cudaMalloc(&d_ell, std::max<size_t>(1, ells.size()) * sizeof(Ell)));
  TG_CUDA(cudaMalloc(&d_off, off.size() * sizeof(int)));
  TG_CUDA(cudaMalloc(&d_list, std::max<size_t>(1, list.size()) * sizeof(int)));
  TG_CUDA(cudaMalloc(&d_ang, nz * sizeof(float)));
  TG_CUDA(cudaMalloc(&d_part, 2 * NB * sizeof(double)));
  if (!ells.empty()) TG_CUDA(cudaMemcpyAsync(d_ell, ells.data(), ells.size() * sizeof(Ell), cudaMemcpyHostToDevice, st));
  TG_CUDA(cudaMemcpyAsync(d_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  if (!list.empty()) TG_CUDA(cudaMemcpyAsync(d_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  TG_CUDA(cudaMemcpyAsync(d_ang, angles_host, nz * sizeof(float), cudaMemcpyHostToDevice, st));
  project_kernel<<<dim3((nx + 127) / 128, ny, nz), 128, 0, st>>>(
      d_ell, d_off, d_list, d_ang, nx, ny, 0.5f * sp->vol_nx, 0.5f * sp->vol_nz, (float)xi, d_out);
  TG_CUDA(cudaGetLastError());
  const size_t n = (size_t)nx * ny * nz;
  if (sp->noise_kind == 1) {
    moments_kernel<<<NB, 256, 0, st>>>(d_out, n, d_part);
    std::vector<double> part(2 * NB);
    TG_CUDA(cudaMemcpyAsync(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    TG_CUDA(cudaStreamSynchronize(st));
    double s1 = 0, s2 = 0;
    for (int i = 0; i < NB; ++i) { s1 += part[2 * i]; s2 += part[2 * i + 1]; }
    double mean = s1 / n, var = std::max(0.0, s2 / n - mean * mean);
    noise_kernel<<<NB, 256, 0, st>>>(d_out, n, 1, sp->noise * sqrt(var), 0.0, 0.0, sp->seed);
  } else if (sp->noise_kind == 2) {
    noise_kernel<<<NB, 256, 0, st>>>(d_out, n, 2, 0.0, sp->noise, 1.0 / sp->vol_nz, sp->seed);
  }
  TG_CUDA(cudaGetLastError());
  TG_CUDA(cudaStreamSynchronize(st));
  cudaFree(d_ell);
  cudaFree(d_off);
  cudaFree(d_list);
  cudaFree(d_ang);
  cudaFree(d_part);
  return TG_OK;
}

}  // namespace tg
