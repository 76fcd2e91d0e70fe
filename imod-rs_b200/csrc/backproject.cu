// backproject.cu -- weighted back-projection kernels for sm_100a.
//
// Semantics: apps/tilt/src/main.rs:1002-1090 (CPU WBP core, also
// backproject_all 756-828) and sample_row_with_fill 386-406.  The sample
// position of every voxel is computed in the reference's f32 operation order
//     proj_x = ((dx*cos_t)*cos_xt + (dz*sin_t)*zf) + center_x
// with explicitly rounded intrinsics (no FMA contraction), so every floor and
// bounds decision matches the reference; with FP32 storage the interpolation
// row[k]*(1-f) + row[k+1]*f and the per-view accumulation order match too.
//
// bp_fast_kernel (no x-tilt, no local alignment; every output slice iy reads
// projection row iy only):
//   * CTA tile = S slices x TX columns x TZ depth; each thread keeps S x K
//     accumulators (one column, K depths, S slices) in registers.  The sample
//     position depends on (view, x, z) but not on the slice, so one floor and
//     one fraction serve S slices.
//   * Per view the CTA needs only the window of each row that its tile
//     projects onto (<= TX + TZ*|sin*zf| + 2 elements).  Windows of VPS views
//     are copied from HBM to shared memory with cp.async.bulk (the TMA bulk
//     engine) completing on an mbarrier, double buffered against compute.
//   * floor(x) comes from one round-down add of 1.5*2^23 (exact for
//     |x| < 2^22); the float's bit pattern then gives the shared-memory address
//     with one integer multiply-add.
//   * FP16/BF16 storage: one packed fma (f*(b-a) + a) interpolates two slices,
//     and a mixed-precision add (add.rn.f32.f16/bf16) accumulates in FP32.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tg_internal.h"
#include "local_dev.cuh"

namespace tg {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ float4 lds128(uint32_t a) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(a));
  return v;
}
__device__ __forceinline__ uint2 lds64(uint32_t a) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0,%1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(a));
  return v;
}
// d = (f32)h + acc in one instruction (PTX 8.6 mixed precision, sm_100+)
__device__ __forceinline__ float add_f32_f16(float acc, uint16_t h) {
  float d;
  asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(h), "f"(acc));
  return d;
}
__device__ __forceinline__ float add_f32_bf16(float acc, uint16_t h) {
  float d;
  asm("add.rn.f32.bf16 %0, %1, %2;" : "=f"(d) : "h"(h), "f"(acc));
  return d;
}

constexpr float MAGIC = 12582912.0f;      // 1.5 * 2^23
constexpr uint32_t MAGIC_BITS = 0x4B400000u;
constexpr long WAIT_LIMIT = 1L << 26;     // bounded spin on an mbarrier phase

// exact reference position for (dx, dz): ((dx*c)*cxt + (dz*s)*zf) + cx
template <bool ZF>
__device__ __forceinline__ float ref_x(float t1, float dz, float s, float zf, float cx) {
  float t2 = __fmul_rn(dz, s);
  if (ZF) t2 = __fmul_rn(t2, zf);
  return __fadd_rn(__fadd_rn(t1, t2), cx);
}

template <int STORE, int S, int K, int TX, int NT, int VPS, bool ZF>
struct FastCfg {
  static constexpr int SP = S / 2;
  static constexpr int OZG = NT / TX;
  static constexpr int TZ = OZG * K;
  static constexpr int EB = STORE == TG_STORE_FP32 ? 16 : 8;
  static constexpr int WMAX = ((TX + TZ * (ZF ? 2 : 1) + 8) + 1) & ~1;  // elements, even
  static constexpr int SLOT = SP * WMAX * EB;                             // bytes per view
  static constexpr int BUF = 2 * VPS * SLOT;
  static size_t smem(int nviews) { return BUF + 8 * (size_t)nviews + 16 + 16 * (NT / 32) * S + 64; }
};

template <int STORE, int S, int K, int TX, int NT, int VPS, bool ZF>
__global__ void __launch_bounds__(NT) bp_fast_kernel(BpArgs a) {
  using C = FastCfg<STORE, S, K, TX, NT, VPS, ZF>;
  constexpr int SP = C::SP, OZG = C::OZG, TZ = C::TZ, EB = C::EB, WMAX = C::WMAX, SLOT = C::SLOT;
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char *bufs = sm;
  int *win_k0 = reinterpret_cast<int *>(sm + C::BUF);
  int *win_n = win_k0 + a.nviews;
  uint64_t *bars = reinterpret_cast<uint64_t *>(
      (reinterpret_cast<uintptr_t>(win_n + a.nviews) + 15) & ~(uintptr_t)15);
  __shared__ int s_abort;

  const int tid = threadIdx.x;
  const int tx = tid % TX, tzg = tid / TX;
  const int ox0 = blockIdx.x * TX, oz0 = blockIdx.y * TZ, iy0 = blockIdx.z * S;
  const int ox = min(ox0 + tx, a.onx - 1);
  const int oxlo = ox0, oxhi = min(ox0 + TX, a.onx) - 1;
  const int ozlo = oz0, ozhi = min(oz0 + TZ, a.onz) - 1;

  // ---- per-view windows of this tile (corners bound x: it is monotone in dx and dz)
  for (int v = tid; v < a.nviews; v += NT) {
    float4 g = __ldg(&a.vg[v]);
    float t1l = __fmul_rn(__fsub_rn((float)oxlo, a.ocx), g.x);
    float t1h = __fmul_rn(__fsub_rn((float)oxhi, a.ocx), g.x);
    float dzl = __fsub_rn((float)ozlo, a.cz), dzh = __fsub_rn((float)ozhi, a.cz);
    float x0 = ref_x<ZF>(t1l, dzl, g.y, g.z, a.cx), x1 = ref_x<ZF>(t1l, dzh, g.y, g.z, a.cx);
    float x2 = ref_x<ZF>(t1h, dzl, g.y, g.z, a.cx), x3 = ref_x<ZF>(t1h, dzh, g.y, g.z, a.cx);
    float xmn = fminf(fminf(x0, x1), fminf(x2, x3)), xmx = fmaxf(fmaxf(x0, x1), fmaxf(x2, x3));
    int kmin = (int)floorf(xmn), kmax = (int)floorf(xmx);
    if (EB == 8) kmin &= ~1;  // 16-byte aligned bulk copies
    int cnt = kmax - kmin + 1;
    if (EB == 8) cnt = (cnt + 1) & ~1;
    // in-bounds guards (the host sizes WMAX and the row padding so these never fire)
    if (cnt > WMAX || kmin + a.padL < 0 || kmin + a.padL + cnt > a.PW) {
      atomicOr(a.err, 2);
      cnt = min(cnt, WMAX);
      kmin = max(kmin, -a.padL);
      if (kmin + a.padL + cnt > a.PW) kmin = a.PW - a.padL - cnt;
      if (EB == 8) kmin &= ~1;
    }
    win_k0[v] = kmin;
    win_n[v] = cnt;
  }
  if (tid == 0) {
    mbar_init(smem_u32(&bars[0]), 1);
    mbar_init(smem_u32(&bars[1]), 1);
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();

  const int nst = (a.nviews + VPS - 1) / VPS;
  const uint8_t *pairs = reinterpret_cast<const uint8_t *>(a.pairs);
  const int jp0 = iy0 / 2;
  auto issue = [&](int st) {
    const int v0 = st * VPS, nv = min(VPS, a.nviews - v0);
    const uint32_t bar = smem_u32(&bars[st & 1]);
    uint32_t bytes = 0;
    for (int vi = 0; vi < nv; ++vi) bytes += (uint32_t)(SP * win_n[v0 + vi] * EB);
    fence_proxy_async();
    mbar_expect_tx(bar, bytes);
    for (int vi = 0; vi < nv; ++vi) {
      const int v = v0 + vi, k0 = win_k0[v], n = win_n[v];
      const uint32_t dst = smem_u32(bufs) + ((st & 1) * VPS + vi) * SLOT;
      for (int sp = 0; sp < SP; ++sp) {
        const uint8_t *src =
            pairs + (((size_t)v * a.rows_alloc + jp0 + sp) * a.PW + (size_t)(k0 + a.padL)) * EB;
        bulk_g2s(dst + sp * WMAX * EB, src, (uint32_t)(n * EB), bar);
      }
    }
  };

  float acc[S][K];
#pragma unroll
  for (int s = 0; s < S; ++s)
#pragma unroll
    for (int j = 0; j < K; ++j) acc[s][j] = 0.0f;
  const float dx = __fsub_rn((float)ox, a.ocx);
  float dz[K];
#pragma unroll
  for (int j = 0; j < K; ++j) dz[j] = __fsub_rn((float)min(oz0 + tzg + j * OZG, a.onz - 1), a.cz);

  if (tid == 0 && nst > 0) issue(0);
  for (int st = 0; st < nst; ++st) {
    if (tid == 0 && st + 1 < nst) issue(st + 1);
    {
      const uint32_t bar = smem_u32(&bars[st & 1]);
      const uint32_t par = (st >> 1) & 1;
      long spins = 0;
      while (!mbar_try_wait(bar, par)) {
        if (++spins > WAIT_LIMIT) {
          s_abort = 1;
          break;
        }
      }
    }
    if (!s_abort) {
      const int v0 = st * VPS, nv = min(VPS, a.nviews - v0);
      for (int vi = 0; vi < nv; ++vi) {
        const int v = v0 + vi;
        const float4 g = __ldg(&a.vg[v]);
        const float t1 = __fmul_rn(dx, g.x);  // (dx*cos_t)*cos_xt, cos_xt == 1 exactly here
        const int k0 = win_k0[v];
        const uint32_t slot = smem_u32(bufs) + ((st & 1) * VPS + vi) * SLOT;
        const uint32_t adj = slot - (MAGIC_BITS + (uint32_t)k0) * (uint32_t)EB;
#pragma unroll
        for (int j = 0; j < K; ++j) {
          const float x = ref_x<ZF>(t1, dz[j], g.y, g.z, a.cx);
          const float tt = __fadd_rd(x, MAGIC);  // MAGIC + floor(x), exactly
          const float f0 = __fsub_rn(x, __fsub_rn(tt, MAGIC));
          const uint32_t bits = __float_as_uint(tt);
          const uint32_t addr = bits * (uint32_t)EB + adj;
          if constexpr (STORE == TG_STORE_FP32) {
            const bool in = (bits - MAGIC_BITS) <= (uint32_t)(a.nx - 2);
            const float f = in ? f0 : 0.0f;
            const float omf = __fsub_rn(1.0f, f);
#pragma unroll
            for (int sp = 0; sp < SP; ++sp) {
              const float4 e = lds128(addr + sp * WMAX * 16);
              acc[2 * sp][j] = __fadd_rn(acc[2 * sp][j], __fadd_rn(__fmul_rn(e.x, omf), __fmul_rn(e.z, f)));
              acc[2 * sp + 1][j] =
                  __fadd_rn(acc[2 * sp + 1][j], __fadd_rn(__fmul_rn(e.y, omf), __fmul_rn(e.w, f)));
            }
          } else if constexpr (STORE == TG_STORE_FP16) {
            const __half2 f2 = __float2half2_rn(f0);
#pragma unroll
            for (int sp = 0; sp < SP; ++sp) {
              const uint2 e = lds64(addr + sp * WMAX * 8);
              const __half2 r = __hfma2(f2, *reinterpret_cast<const __half2 *>(&e.y),
                                        *reinterpret_cast<const __half2 *>(&e.x));
              const uint32_t rb = *reinterpret_cast<const uint32_t *>(&r);
              acc[2 * sp][j] = add_f32_f16(acc[2 * sp][j], (uint16_t)(rb & 0xffffu));
              acc[2 * sp + 1][j] = add_f32_f16(acc[2 * sp + 1][j], (uint16_t)(rb >> 16));
            }
          } else {
            const __nv_bfloat162 f2 = __float2bfloat162_rn(f0);
#pragma unroll
            for (int sp = 0; sp < SP; ++sp) {
              const uint2 e = lds64(addr + sp * WMAX * 8);
              const __nv_bfloat162 r = __hfma2(f2, *reinterpret_cast<const __nv_bfloat162 *>(&e.y),
                                               *reinterpret_cast<const __nv_bfloat162 *>(&e.x));
              const uint32_t rb = *reinterpret_cast<const uint32_t *>(&r);
              acc[2 * sp][j] = add_f32_bf16(acc[2 * sp][j], (uint16_t)(rb & 0xffffu));
              acc[2 * sp + 1][j] = add_f32_bf16(acc[2 * sp + 1][j], (uint16_t)(rb >> 16));
            }
          }
        }
      }
    }
    __syncthreads();
    if (s_abort) break;
  }
  if (s_abort) {
    if (tid == 0) {
      atomicOr(a.err, 1);
      // bounded drain of copies still in flight on either barrier before the CTA exits
      for (int b = 0; b < 2; ++b) {
        long spins = 0;
        while (!mbar_try_wait(smem_u32(&bars[b]), 0) && !mbar_try_wait(smem_u32(&bars[b]), 1) &&
               ++spins < WAIT_LIMIT) {
        }
      }
    }
    return;
  }

  // ---- epilogue: 1/N, output transform or SIRT update, per-slice partial stats
  const int oxr = ox0 + tx;
  const bool xok = oxr < a.onx;
  float *red = reinterpret_cast<float *>(sm);  // staging buffers are free now
  const int tile = blockIdx.x + blockIdx.y * gridDim.x;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int iy = iy0 + s;
    float mn = 3.40282347e+38f, mx = -3.40282347e+38f;
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const int oz = oz0 + tzg + j * OZG;
      if (xok && oz < a.onz && iy < a.ny) {
        const size_t idx = ((size_t)iy * a.onz + oz) * a.onx + oxr;
        const float v = __fmul_rn(acc[s][j], a.inv_n);
        if (a.mode == 0) {
          const float y = __fadd_rn(__fmul_rn(__fmul_rn(v, a.dw), a.os), a.oa);
          a.vol[idx] = y;
          mn = fminf(mn, y);
          mx = fmaxf(mx, y);
          sum += (double)y;
        } else if (a.mode == 1) {
          a.vol[idx] = v;
        } else {
          a.vol[idx] = __fadd_rn(a.vol[idx], __fmul_rn(a.relax, v));
        }
      }
    }
    if (a.mode == 0) {
      for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
      }
      if ((tid & 31) == 0) {
        float *r = red + ((tid >> 5) * S + s) * 4;
        r[0] = mn;
        r[1] = mx;
        *reinterpret_cast<double *>(r + 2) = sum;
      }
    }
  }
  if (a.mode == 0) {
    __syncthreads();
    if (tid < S && iy0 + tid < a.ny) {
      float mn = 3.40282347e+38f, mx = -3.40282347e+38f;
      double sum = 0.0;
      for (int w = 0; w < NT / 32; ++w) {
        const float *r = red + (w * S + tid) * 4;
        mn = fminf(mn, r[0]);
        mx = fmaxf(mx, r[1]);
        sum += *reinterpret_cast<const double *>(r + 2);
      }
      StatPartial p;
      p.mn = mn;
      p.mx = mx;
      p.sum = sum;
      a.partial[(size_t)(iy0 + tid) * (gridDim.x * gridDim.y) + tile] = p;
    }
  }
}

// ---- variant table (tile shapes the autotuner chooses from) ----
struct FastVariant { int S, K, TX, NT, VPS; const char *name; };
static const FastVariant kFast[] = {
    {8, 4, 64, 256, 4, "S8K4TX64NT256"},
    {8, 8, 64, 256, 2, "S8K8TX64NT256"},
    {8, 4, 32, 128, 4, "S8K4TX32NT128"},
    {4, 8, 64, 256, 4, "S4K8TX64NT256"},
    {8, 2, 128, 256, 4, "S8K2TX128NT256"},
};
int bp_fast_variants() { return (int)(sizeof(kFast) / sizeof(kFast[0])); }
const char *bp_fast_variant_name(int v) { return kFast[v].name; }

template <int STORE, int S, int K, int TX, int NT, int VPS, bool ZF>
static int launch_fast_t(const BpArgs &a, cudaStream_t st, int *ntiles) {
  using C = FastCfg<STORE, S, K, TX, NT, VPS, ZF>;
  auto kern = bp_fast_kernel<STORE, S, K, TX, NT, VPS, ZF>;
  size_t smem = C::smem(a.nviews);
  if (smem > 200 * 1024) return TG_ERR_UNSUPPORTED;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(bp_fast)");
  dim3 grid((a.onx + TX - 1) / TX, (a.onz + C::TZ - 1) / C::TZ, (a.ny + S - 1) / S);
  if (ntiles) *ntiles = grid.x * grid.y;
  kern<<<grid, NT, smem, st>>>(a);
  return TG_OK;
}

template <int STORE, bool ZF>
static int launch_fast_v(const BpArgs &a, int variant, cudaStream_t st, int *ntiles) {
  switch (variant) {
    case 0: return launch_fast_t<STORE, 8, 4, 64, 256, 4, ZF>(a, st, ntiles);
    case 1: return launch_fast_t<STORE, 8, 8, 64, 256, 2, ZF>(a, st, ntiles);
    case 2: return launch_fast_t<STORE, 8, 4, 32, 128, 4, ZF>(a, st, ntiles);
    case 3: return launch_fast_t<STORE, 4, 8, 64, 256, 4, ZF>(a, st, ntiles);
    default: return launch_fast_t<STORE, 8, 2, 128, 256, 4, ZF>(a, st, ntiles);
  }
}

int bp_fast_ntiles(const BpArgs &a, int variant) {
  const FastVariant &f = kFast[variant];
  int tz = (f.NT / f.TX) * f.K;
  return ((a.onx + f.TX - 1) / f.TX) * ((a.onz + tz - 1) / tz);
}

int launch_bp_fast(const BpArgs &a, int store, bool zf, int variant, cudaStream_t st, int *ntiles) {
  if (variant < 0 || variant >= bp_fast_variants()) variant = 0;
  if (store == TG_STORE_FP32)
    return zf ? launch_fast_v<TG_STORE_FP32, true>(a, variant, st, ntiles)
              : launch_fast_v<TG_STORE_FP32, false>(a, variant, st, ntiles);
  if (store == TG_STORE_FP16)
    return zf ? launch_fast_v<TG_STORE_FP16, true>(a, variant, st, ntiles)
              : launch_fast_v<TG_STORE_FP16, false>(a, variant, st, ntiles);
  return zf ? launch_fast_v<TG_STORE_BF16, true>(a, variant, st, ntiles)
            : launch_fast_v<TG_STORE_BF16, false>(a, variant, st, ntiles);
}

// ---------------------------------------------------------------------------
// General kernel: x-tilt (bilinear in y), z-factor, local alignment; SINGLE
// format read through L1 (rows differ per column when x-tilt bends the rays).
// One thread = one column of one slice, K depths.
// ---------------------------------------------------------------------------
template <int STORE, int K, int NT>
__global__ void __launch_bounds__(NT) bp_general_kernel(BpArgs a) {
  constexpr int TX = 32, OZG = NT / TX, TZ = OZG * K;
  constexpr int EB = STORE == TG_STORE_FP32 ? 8 : 4;
  const int tid = threadIdx.x, lane = tid & 31, tzg = tid / TX;
  const int ox = blockIdx.x * TX + lane, oz0 = blockIdx.y * TZ, iy = blockIdx.z;
  const int oxc = min(ox, a.onx - 1);
  const float dx = __fsub_rn((float)oxc, a.ocx);
  float dz[K];
#pragma unroll
  for (int j = 0; j < K; ++j) dz[j] = __fsub_rn((float)min(oz0 + tzg + j * OZG, a.onz - 1), a.cz);
  float acc[K];
#pragma unroll
  for (int j = 0; j < K; ++j) acc[j] = 0.0f;
  const uint8_t *pairs = reinterpret_cast<const uint8_t *>(a.pairs);
  const int kmin = -a.padL, kmax = a.PW - a.padL - 1;
  for (int v = 0; v < a.nviews; ++v) {
    const float4 g = __ldg(&a.vg[v]);
    const float sin_xt = __ldg(&a.vg2[v].x);
    const float t1 = __fmul_rn(__fmul_rn(dx, g.x), g.w);
    const float yoff = __fmul_rn(dx, sin_xt);
    float ldx = 0.0f, ldy = 0.0f;
    bool use_l = false;
    if (a.has_local) use_l = local_interp(a.loc, v, (float)oxc, (float)iy, ldx, ldy);
    float sample_y = __fadd_rn((float)iy, yoff);
    if (use_l) sample_y = __fadd_rn(sample_y, ldy);
    const float fly = floorf(sample_y);
    const float fy = __fsub_rn(sample_y, fly);
    const bool yin = fly >= 0.0f && fly < (float)a.ny;
    const int sy0 = yin ? (int)fly : 0;
    const bool two = yin && sy0 + 1 < a.ny && (fabsf(yoff) > 1e-6f || a.has_local);
    if (!yin) continue;
    const uint8_t *row0 = pairs + ((size_t)v * a.rows_alloc + sy0) * (size_t)a.PW * EB;
    const uint8_t *row1 = two ? row0 + (size_t)a.PW * EB : row0;
    const float omfy = __fsub_rn(1.0f, fy);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      float t2 = __fmul_rn(__fmul_rn(dz[j], g.y), g.z);
      float x = __fadd_rn(__fadd_rn(t1, t2), a.cx);
      if (use_l) x = __fadd_rn(x, ldx);
      const float tt = __fadd_rd(x, MAGIC);
      float f = __fsub_rn(x, __fsub_rn(tt, MAGIC));
      int k = (int)(__float_as_uint(tt) - MAGIC_BITS);
      const bool in = (unsigned)k <= (unsigned)(a.nx - 2);
      if (fabsf(x) > 4.0e6f) { k = x < 0.0f ? kmin : kmax; f = 0.0f; }  // beyond the magic range
      k = min(max(k, kmin), kmax);
      const size_t e = (size_t)(k + a.padL);
      float v0, v1 = 0.0f;
      if constexpr (STORE == TG_STORE_FP32) {
        if (!in) f = 0.0f;
        const float omf = __fsub_rn(1.0f, f);
        const float2 p0 = __ldg(reinterpret_cast<const float2 *>(row0) + e);
        v0 = __fadd_rn(__fmul_rn(p0.x, omf), __fmul_rn(p0.y, f));
        if (two) {
          const float2 p1 = __ldg(reinterpret_cast<const float2 *>(row1) + e);
          v1 = __fadd_rn(__fmul_rn(p1.x, omf), __fmul_rn(p1.y, f));
        }
      } else {
        const uint32_t w0 = __ldg(reinterpret_cast<const uint32_t *>(row0) + e);
        float a0, d0;
        if (STORE == TG_STORE_FP16) {
          a0 = __half2float(__ushort_as_half((uint16_t)(w0 & 0xffff)));
          d0 = __half2float(__ushort_as_half((uint16_t)(w0 >> 16)));
        } else {
          a0 = __bfloat162float(__ushort_as_bfloat16((uint16_t)(w0 & 0xffff)));
          d0 = __bfloat162float(__ushort_as_bfloat16((uint16_t)(w0 >> 16)));
        }
        v0 = fmaf(f, d0, a0);
        if (two) {
          const uint32_t w1 = __ldg(reinterpret_cast<const uint32_t *>(row1) + e);
          float a1, d1;
          if (STORE == TG_STORE_FP16) {
            a1 = __half2float(__ushort_as_half((uint16_t)(w1 & 0xffff)));
            d1 = __half2float(__ushort_as_half((uint16_t)(w1 >> 16)));
          } else {
            a1 = __bfloat162float(__ushort_as_bfloat16((uint16_t)(w1 & 0xffff)));
            d1 = __bfloat162float(__ushort_as_bfloat16((uint16_t)(w1 >> 16)));
          }
          v1 = fmaf(f, d1, a1);
        }
      }
      const float val = two ? __fadd_rn(__fmul_rn(v0, omfy), __fmul_rn(v1, fy)) : v0;
      acc[j] = __fadd_rn(acc[j], val);
    }
  }
  // epilogue (same as the fast kernel)
  const bool xok = ox < a.onx;
  float mn = 3.40282347e+38f, mx = -3.40282347e+38f;
  double sum = 0.0;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const int oz = oz0 + tzg + j * OZG;
    if (xok && oz < a.onz) {
      const size_t idx = ((size_t)iy * a.onz + oz) * a.onx + ox;
      const float v = __fmul_rn(acc[j], a.inv_n);
      if (a.mode == 0) {
        const float y = __fadd_rn(__fmul_rn(__fmul_rn(v, a.dw), a.os), a.oa);
        a.vol[idx] = y;
        mn = fminf(mn, y);
        mx = fmaxf(mx, y);
        sum += (double)y;
      } else if (a.mode == 1) {
        a.vol[idx] = v;
      } else {
        a.vol[idx] = __fadd_rn(a.vol[idx], __fmul_rn(a.relax, v));
      }
    }
  }
  if (a.mode == 0) {
    __shared__ float red[NT / 32][4];
    for (int o = 16; o > 0; o >>= 1) {
      mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    if (lane == 0) {
      red[tid >> 5][0] = mn;
      red[tid >> 5][1] = mx;
      *reinterpret_cast<double *>(&red[tid >> 5][2]) = sum;
    }
    __syncthreads();
    if (tid == 0) {
      StatPartial p;
      p.mn = 3.40282347e+38f;
      p.mx = -3.40282347e+38f;
      p.sum = 0.0;
      for (int w = 0; w < NT / 32; ++w) {
        p.mn = fminf(p.mn, red[w][0]);
        p.mx = fmaxf(p.mx, red[w][1]);
        p.sum += *reinterpret_cast<const double *>(&red[w][2]);
      }
      a.partial[(size_t)iy * (gridDim.x * gridDim.y) + blockIdx.x + blockIdx.y * gridDim.x] = p;
    }
  }
}

int launch_bp_general(const BpArgs &a, int store, cudaStream_t st, int *ntiles) {
  constexpr int K = 4, NT = 128, TZ = (NT / 32) * K;
  dim3 grid((a.onx + 31) / 32, (a.onz + TZ - 1) / TZ, a.ny);
  if (ntiles) *ntiles = grid.x * grid.y;
  if (store == TG_STORE_FP32) bp_general_kernel<TG_STORE_FP32, K, NT><<<grid, NT, 0, st>>>(a);
  else if (store == TG_STORE_FP16) bp_general_kernel<TG_STORE_FP16, K, NT><<<grid, NT, 0, st>>>(a);
  else bp_general_kernel<TG_STORE_BF16, K, NT><<<grid, NT, 0, st>>>(a);
  return TG_OK;
}

}  // namespace tg
