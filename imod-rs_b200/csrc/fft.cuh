// fft.cuh -- shared-memory Stockham FFT of one complex row per CTA (radices 4,
// 2, 3, 5, 7; plan from fft_plan()), used by the R-weighting filter and the CTF
// phase flip.  Unnormalised in both directions.
#pragma once
#include "tg_internal.h"

namespace tg {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV> __device__ __forceinline__ float2 rot(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R, bool INV> __device__ __forceinline__ void bfly(float2 *v, const float2 *tw, int n) {
  if constexpr (R == 2) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 4) {
    float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    float2 b0 = cadd(v[1], v[3]), b1 = rot<INV>(csub(v[1], v[3]));
    v[0] = cadd(a0, b0);
    v[1] = cadd(a1, b1);
    v[2] = csub(a0, b0);
    v[3] = csub(a1, b1);
  } else if constexpr (R == 3) {
    const float s = 0.866025403784438646763723170752936183f;  // sin(2pi/3)
    float2 t1 = cadd(v[1], v[2]);
    float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    float2 d = csub(v[1], v[2]);
    float2 t3 = rot<INV>(make_float2(s * d.x, s * d.y));
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  } else if constexpr (R == 5) {
    const float c1 = 0.309016994374947424102293417182819059f;   // cos(2pi/5)
    const float c2 = -0.809016994374947424102293417182819059f;  // cos(4pi/5)
    const float s1 = 0.951056516295153572116439333379382143f;   // sin(2pi/5)
    const float s2 = 0.587785252292473129168705954639072769f;   // sin(4pi/5)
    float2 a1 = cadd(v[1], v[4]), a2 = cadd(v[2], v[3]);
    float2 b1 = csub(v[1], v[4]), b2 = csub(v[2], v[3]);
    float2 x0 = v[0];
    float2 p1 = make_float2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
    float2 p2 = make_float2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
    float2 q1 = rot<INV>(make_float2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    float2 q2 = rot<INV>(make_float2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    v[0] = cadd(x0, cadd(a1, a2));
    v[1] = cadd(p1, q1);
    v[4] = csub(p1, q1);
    v[2] = cadd(p2, q2);
    v[3] = csub(p2, q2);
  } else {  // generic (R = 7): direct DFT with table twiddles
    float2 out[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      float2 acc = v[0];
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = __ldg(&tw[((r * j) % R) * (n / R)]);
        if (INV) w.y = -w.y;
        acc = cadd(acc, cmul(v[r], w));
      }
      out[j] = acc;
    }
#pragma unroll
    for (int j = 0; j < R; ++j) v[j] = out[j];
  }
}

// One Stockham pass of radix R: X -> Y, Ns = product of the radices done so far.
template <int R, bool INV>
__device__ __forceinline__ void stockham_pass(const float2 *X, float2 *Y, int n, int Ns,
                                              const float2 *tw) {
  const int nb = n / R;
  const int tstride = n / (Ns * R);
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
    int k = j % Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = X[j + r * nb];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = __ldg(&tw[r * k * tstride]);
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    bfly<R, INV>(v, tw, n);
    int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) Y[base + r * Ns] = v[r];
  }
}

// Full transform; returns the buffer holding the result.
template <bool INV>
__device__ float2 *stockham(float2 *A, float2 *B, const FftPlanDev &pl, const float2 *tw) {
  int Ns = 1;
  for (int i = 0; i < pl.nfac; ++i) {
    int R = pl.fac[i];
    switch (R) {
      case 4: stockham_pass<4, INV>(A, B, pl.n, Ns, tw); break;
      case 2: stockham_pass<2, INV>(A, B, pl.n, Ns, tw); break;
      case 3: stockham_pass<3, INV>(A, B, pl.n, Ns, tw); break;
      case 5: stockham_pass<5, INV>(A, B, pl.n, Ns, tw); break;
      default: stockham_pass<7, INV>(A, B, pl.n, Ns, tw); break;
    }
    __syncthreads();
    float2 *t = A; A = B; B = t;
    Ns *= R;
  }
  return A;
}

}  // namespace tg
