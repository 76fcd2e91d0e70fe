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

#include <algorithm>
#include <type_traits>

#include "tg_internal.h"
#include "f32x2.cuh"
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
// acc0 += (f32)lo(h2), acc1 += (f32)hi(h2): the halves are taken straight from
// the 32-bit register (mov.b32 unpack) instead of being shifted out
__device__ __forceinline__ void add2_f32_f16(float &acc0, float &acc1, uint32_t h2) {
  asm("{\n .reg .f16 lo, hi;\n mov.b32 {lo, hi}, %2;\n"
      " add.rn.f32.f16 %0, lo, %0;\n add.rn.f32.f16 %1, hi, %1;\n}\n"
      : "+f"(acc0), "+f"(acc1)
      : "r"(h2));
}
__device__ __forceinline__ void add2_f32_bf16(float &acc0, float &acc1, uint32_t h2) {
  asm("{\n .reg .b16 lo, hi;\n mov.b32 {lo, hi}, %2;\n"
      " add.rn.f32.bf16 %0, lo, %0;\n add.rn.f32.bf16 %1, hi, %1;\n}\n"
      : "+f"(acc0), "+f"(acc1)
      : "r"(h2));
}


// Shared loads at a 32-bit shared address plus a compile-time byte offset,
// ordered after the mbarrier waits (all are volatile asm).
template <int OFF> __device__ __forceinline__ float4 lds128i(uint32_t a) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4+%5];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(a), "n"(OFF));
  return v;
}
template <int OFF> __device__ __forceinline__ uint2 lds64i(uint32_t a) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0,%1}, [%2+%3];" : "=r"(v.x), "=r"(v.y) : "r"(a), "n"(OFF));
  return v;
}
template <int I, int N, class F> __device__ __forceinline__ void static_for(F &&f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for<I + 1, N>(f);
  }
}

constexpr float MAGIC = 12582912.0f;      // 1.5 * 2^23
constexpr uint32_t MAGIC_BITS = 0x4B400000u;

// exact reference position for (dx, dz): ((dx*c)*cxt + (dz*s)*zf) + cx.
// ZF: 0 no z-factor, 1 z-factor, 2 z-factor and x-tilt (t1 carries *cos_xt)
template <int ZF>
__device__ __forceinline__ float ref_x(float t1, float dz, float s, float zf, float cx) {
  float t2 = __fmul_rn(dz, s);
  if (ZF) t2 = __fmul_rn(t2, zf);
  return __fadd_rn(__fadd_rn(t1, t2), cx);
}

template <int STORE, int S, int K, int TX, int NT, int VPS, int NSTAGE, int ZF>
struct FastCfg {
  static constexpr int SP = S / 2;           // row pairs per tile
  static constexpr int OZG = NT / TX;        // depth groups of consumer threads
  static constexpr int TZ = OZG * K;         // tile depth
  static constexpr int NTHR = NT + 32;       // consumers + one producer warp
  static constexpr int NSTAGE_ = NSTAGE, NT_ = NT;
  static constexpr int EB = STORE == TG_STORE_FP32 ? 16 : 8;
  static constexpr int WMAX = ((TX + TZ * (ZF ? 2 : 1) + 8) + 1) & ~1;  // window elements, even
  static constexpr int SLOT = SP * WMAX * EB;                             // bytes per view
  static constexpr int BUF = NSTAGE * VPS * SLOT;
  static_assert(VPS * SP <= 32, "one copy per producer lane");
  static size_t smem(int nviews) { return BUF + 8 * (size_t)nviews + 16 * NSTAGE + 16 + 64; }
};

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void consumer_sync(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}
// try_wait that lets the hardware suspend the thread (up to hint_ns) until the
// phase completes, instead of returning at once
__device__ __forceinline__ bool mbar_try_wait_sleep(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on an mbarrier phase: sleeps in try_wait, gives up after limit_ns
// of wall time (BpArgs::wait_limit_ns, 2 s by default: a stage never
// legitimately takes that long) or, when abort is given, as soon as another warp
// of the CTA has given up.
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t parity, volatile int *abort, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    if (mbar_try_wait_sleep(bar, parity, 20000u)) return true;
    if ((abort && *abort) || globaltimer_ns() - t0 > limit_ns) return false;
  }
}

// Warp-specialised pipeline: warp NT/32 (the producer) copies each stage's
// per-view row windows with cp.async.bulk, one copy per lane, completing on
// full[b]; consumer warps wait on full[b], accumulate, and release the buffer
// on empty[b].  NSTAGE buffers of VPS views form a ring.
// Shared-memory layout of a CTA: the stage ring, the per-view windows (sized
// for max_views) and the 2*NSTAGE mbarriers.
template <class C> struct SmemLayout {
  unsigned char *bufs;
  int *win_k0, *win_n;
  uint64_t *full, *empty;
  __device__ SmemLayout(unsigned char *sm, int max_views) {
    bufs = sm;
    win_k0 = reinterpret_cast<int *>(sm + C::BUF);
    win_n = win_k0 + max_views;
    uint64_t *bars = reinterpret_cast<uint64_t *>(
        (reinterpret_cast<uintptr_t>(win_n + max_views) + 15) & ~(uintptr_t)15);
    full = bars;
    empty = bars + C::NSTAGE_;
  }
};

// One output tile (S slices x TX columns x TZ depths) of one series.  gst is the
// CTA's running stage count: ring slots and mbarrier phases continue across the
// tiles a persistent CTA processes.  Returns false on abort.
// Producer state that outlives a tile: issued = 1 + the global index of the last
// stage whose copies were issued; skipped = a stage left out by the test hook (-1).
struct ProducerState { int issued = 0, skipped = -1; };

template <int STORE, int S, int K, int TX, int NT, int VPS, int NSTAGE, int ZF>
__device__ __forceinline__ bool bp_tile(const BpArgs &a, int bx, int by, int bz, unsigned char *sm,
                                        const SmemLayout<FastCfg<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>> &L,
                                        int &gst, volatile int *s_abort_p, ProducerState &ps) {
  using C = FastCfg<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>;
  constexpr int SP = C::SP, OZG = C::OZG, TZ = C::TZ, EB = C::EB, WMAX = C::WMAX, SLOT = C::SLOT;
  unsigned char *bufs = L.bufs;
  int *win_k0 = L.win_k0, *win_n = L.win_n;
  uint64_t *full = L.full, *empty = L.empty;
  volatile int &s_abort = *s_abort_p;

  const int tid = threadIdx.x;
  const int ox0 = bx * TX, oz0 = by * TZ, iy0 = bz * S;
  const int oxlo = ox0, oxhi = min(ox0 + TX, a.onx) - 1;
  const int ozlo = oz0, ozhi = min(oz0 + TZ, a.onz) - 1;

  // ---- per-view windows of this tile (x is monotone in dx and dz: corners bound it)
  for (int v = tid; v < a.nviews; v += C::NTHR) {
    float4 g = __ldg(&a.vg[v]);
    float t1l = __fmul_rn(__fsub_rn((float)oxlo, a.ocx), g.x);
    float t1h = __fmul_rn(__fsub_rn((float)oxhi, a.ocx), g.x);
    if (ZF == 2) {  // x-tilt: (dx*cos_t)*cos_xt
      t1l = __fmul_rn(t1l, g.w);
      t1h = __fmul_rn(t1h, g.w);
    }
    float dzl = __fsub_rn((float)ozlo, a.cz), dzh = __fsub_rn((float)ozhi, a.cz);
    float x0 = ref_x<ZF>(t1l, dzl, g.y, g.z, a.cx), x1 = ref_x<ZF>(t1l, dzh, g.y, g.z, a.cx);
    float x2 = ref_x<ZF>(t1h, dzl, g.y, g.z, a.cx), x3 = ref_x<ZF>(t1h, dzh, g.y, g.z, a.cx);
    float xmn = fminf(fminf(x0, x1), fminf(x2, x3)), xmx = fmaxf(fmaxf(x0, x1), fmaxf(x2, x3));
    int kmin = (int)floorf(xmn), kmax = (int)floorf(xmx);
    if (STORE != TG_STORE_FP32) {  // the FMA positions may floor one element beyond the corners
      kmin -= 1;
      kmax += 1;
    }
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
  __syncthreads();

  const int nst = (a.nviews + VPS - 1) / VPS;
  const int g0 = gst;  // global index of this tile's first stage
  gst += nst;
  if (tid >= NT) {
    // ---------------- producer warp ----------------
    const int lane = tid - NT;
    const uint8_t *pairs = reinterpret_cast<const uint8_t *>(a.pairs);
    const int jp0 = iy0 / 2;
    for (int st = 0; st < nst; ++st) {
      const int g = g0 + st, b = g % NSTAGE;
      bool go = g < NSTAGE || wait_phase(smem_u32(&empty[b]), ((g / NSTAGE) - 1) & 1, &s_abort, a.wait_limit_ns);
      // one decision for the whole warp: no lane may leave while others reach the
      // warp-wide reduction below
      go = __all_sync(0xffffffffu, go && !s_abort);
      if (!go) {
        if (lane == 0) s_abort = 1;
        return false;
      }
      if (st == a.fault_skip_stage) {  // test hook: no expect_tx, no copy -> full[b] never completes
        ps.skipped = g;
        continue;
      }
      const int v0 = st * VPS, nv = min(VPS, a.nviews - v0);
      const bool mine = lane < nv * SP;
      const int vi = lane / SP, sp = lane % SP, v = v0 + vi;
      const uint32_t bytes = mine ? (uint32_t)(win_n[v] * EB) : 0u;
      const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
      if (lane == 0) {
        fence_proxy_async();  // order the consumers' reads of buffer b before the refill
        mbar_expect_tx(smem_u32(&full[b]), total);
      }
      __syncwarp();
      if (mine) {
        const uint8_t *src =
            pairs + (((size_t)v * a.rows_alloc + jp0 + sp) * a.PW + (size_t)(win_k0[v] + a.padL)) * EB;
        const uint32_t dst = smem_u32(bufs) + (b * VPS + vi) * SLOT + sp * WMAX * EB;
        bulk_g2s(dst, src, bytes, smem_u32(&full[b]));
      }
      ps.issued = g + 1;
    }
    return true;
  }

  // ---------------- consumer warps ----------------
  const int tx = tid % TX, tzg = tid / TX;
  const int ox = min(ox0 + tx, a.onx - 1);
  // FP32: accumulators of slices (2sp, 2sp+1) packed for the f32x2 pipe;
  // FP16/BF16: one f32 accumulator per slice
  constexpr int NACC = STORE == TG_STORE_FP32 ? 1 : S;
  constexpr int NACC2 = STORE == TG_STORE_FP32 ? SP : 1;
  float acc[NACC][K];
  uint64_t acc2[NACC2][K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
#pragma unroll
    for (int s = 0; s < NACC; ++s) acc[s][j] = 0.0f;
#pragma unroll
    for (int s = 0; s < NACC2; ++s) acc2[s][j] = 0ull;
  }
  const float dx = __fsub_rn((float)ox, a.ocx);
  float dz[K];
#pragma unroll
  for (int j = 0; j < K; ++j) dz[j] = __fsub_rn((float)min(oz0 + tzg + j * OZG, a.onz - 1), a.cz);

  bool ok = true;
  for (int st = 0; st < nst && ok; ++st) {
    const int g = g0 + st, b = g % NSTAGE;
    if (!wait_phase(smem_u32(&full[b]), (g / NSTAGE) & 1, &s_abort, a.wait_limit_ns)) {
      s_abort = 1;
      ok = false;
      break;
    }
    const int v0 = st * VPS, nv = min(VPS, a.nviews - v0);
#pragma unroll
    for (int vi = 0; vi < VPS; ++vi) {
      if (vi < nv) {
        const int v = v0 + vi;
        const float4 g = __ldg(&a.vg[v]);
        // (dx*cos_t)*cos_xt; without x-tilt (ZF < 2) cos_xt is 1 and the product dx*cos_t
        const float t1 = ZF == 2 ? __fmul_rn(__fmul_rn(dx, g.x), g.w) : __fmul_rn(dx, g.x);
        // half staging (a tolerance path): one FMA per position, x within an ulp of the
        // reference's; linear interpolation is continuous, so a floor moved by it
        // changes the sample by at most the rounding of x
        const float t1c = __fadd_rn(t1, a.cx);
        const float szf = ZF ? __fmul_rn(g.y, g.z) : g.y;
        const int k0 = win_k0[v];
        // shared address of element k of this view's slot: bits(tt)*EB + adj
        const uint32_t adj = smem_u32(bufs) + (uint32_t)((b * VPS + vi) * SLOT) -
                             (MAGIC_BITS + (uint32_t)k0) * (uint32_t)EB;
#pragma unroll
        for (int j = 0; j < K; ++j) {
          const float x = STORE == TG_STORE_FP32 ? ref_x<ZF>(t1, dz[j], g.y, g.z, a.cx) : fmaf(dz[j], szf, t1c);
          const float tt = __fadd_rd(x, MAGIC);  // MAGIC + floor(x), exactly
          const float f0 = __fsub_rn(x, __fsub_rn(tt, MAGIC));
          const uint32_t bits = __float_as_uint(tt);
          const uint32_t addr = bits * (uint32_t)EB + adj;
          if constexpr (STORE == TG_STORE_FP32) {
            const bool in = (bits - MAGIC_BITS) <= (uint32_t)(a.nx - 2);
            const float f = in ? f0 : 0.0f;
            const float omf = __fsub_rn(1.0f, f);
            const uint64_t omf2 = pk2(omf, omf), ff2 = pk2(f, f);
            static_for<0, SP>([&](auto spc) {
              constexpr int sp = decltype(spc)::value;
              // (a0, a1, b0, b1): RN(RN(a*(1-f)) + RN(b*f)) for both slices.  The
              // products use the f32x2 pipe; the sums stay scalar so that no
              // multiply is contracted into them.
              const float4 e = lds128i<sp * WMAX * 16>(addr);
              const float2 p = up2(mul2(pk2(e.x, e.y), omf2));
              const float2 q = up2(mul2(pk2(e.z, e.w), ff2));
              acc2[sp][j] = add2(acc2[sp][j], pk2(__fadd_rn(p.x, q.x), __fadd_rn(p.y, q.y)));
            });
          } else if constexpr (STORE == TG_STORE_FP16) {
            const __half2 f2 = __float2half2_rn(f0);
            static_for<0, SP>([&](auto spc) {
              constexpr int sp = decltype(spc)::value;
              const uint2 e = lds64i<sp * WMAX * 8>(addr);
              const __half2 r = __hfma2(f2, *reinterpret_cast<const __half2 *>(&e.y),
                                        *reinterpret_cast<const __half2 *>(&e.x));
              add2_f32_f16(acc[2 * sp][j], acc[2 * sp + 1][j], *reinterpret_cast<const uint32_t *>(&r));
            });
          } else {
            const __nv_bfloat162 f2 = __float2bfloat162_rn(f0);
            static_for<0, SP>([&](auto spc) {
              constexpr int sp = decltype(spc)::value;
              const uint2 e = lds64i<sp * WMAX * 8>(addr);
              const __nv_bfloat162 r = __hfma2(f2, *reinterpret_cast<const __nv_bfloat162 *>(&e.y),
                                               *reinterpret_cast<const __nv_bfloat162 *>(&e.x));
              add2_f32_bf16(acc[2 * sp][j], acc[2 * sp + 1][j], *reinterpret_cast<const uint32_t *>(&r));
            });
          }
        }
      }
    }
    __syncwarp();
    if ((tid & 31) == 0) mbar_arrive(smem_u32(&empty[b]));  // this warp is done with buffer b
  }
  __syncwarp();       // lanes that left the loop at different stages reconverge
  consumer_sync(NT);  // all consumers past the loop (buffers free, abort flag settled)
  if (s_abort) {
    if (tid == 0) atomicOr(a.err, 1);
    return false;
  }

  // ---- epilogue: 1/N, output transform or SIRT update, per-slice partial stats
  const int oxr = ox0 + tx;
  const bool xok = oxr < a.onx;
  float *red = reinterpret_cast<float *>(sm);  // staging buffers are free now
  const int tile = bx + by * a.nbx;
  auto acc_at = [&](int s, int j) {
    if constexpr (STORE == TG_STORE_FP32) {
      const float2 p = up2(acc2[s / 2][j]);
      return (s & 1) ? p.y : p.x;
    } else {
      return acc[s < NACC ? s : 0][j];
    }
  };
  if (a.mode == 2) {
    // SIRT update vol += relax * v.  The old values of SG slices (8 values) are
    // loaded together before any of their stores: a store through vol could
    // alias a later load as far as the compiler knows, which would otherwise
    // make each of the S*K updates wait for its own round trip to HBM.
    constexpr int SG = 1;
    const int ozt = oz0 + tzg, zstep = OZG * a.onx;  // depth j of a slice: + j * zstep
#pragma unroll
    for (int s0 = 0; s0 < S; s0 += SG) {
      float old[SG][K];
      float *rows[SG];
#pragma unroll
      for (int g = 0; g < SG; ++g) {
        rows[g] = a.vol + ((size_t)(iy0 + s0 + g) * a.onz + ozt) * a.onx + oxr;
        const bool yok = xok && iy0 + s0 + g < a.ny;
#pragma unroll
        for (int j = 0; j < K; ++j) old[g][j] = (yok && ozt + j * OZG < a.onz) ? rows[g][j * zstep] : 0.0f;
      }
#pragma unroll
      for (int g = 0; g < SG; ++g) {
        const bool yok = xok && iy0 + s0 + g < a.ny;
#pragma unroll
        for (int j = 0; j < K; ++j)
          if (yok && ozt + j * OZG < a.onz)
            rows[g][j * zstep] = __fadd_rn(old[g][j], __fmul_rn(a.relax, __fmul_rn(acc_at(s0 + g, j), a.inv_n)));
      }
    }
    return true;
  }
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
        const float v = __fmul_rn(acc_at(s, j), a.inv_n);
        if (a.mode == 0) {
          const float y = __fadd_rn(__fmul_rn(__fmul_rn(v, a.dw), a.os), a.oa);
          a.vol[idx] = y;
          mn = fminf(mn, y);
          mx = fmaxf(mx, y);
          sum += (double)y;
        } else {  // mode 1
          a.vol[idx] = v;
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
    consumer_sync(NT);
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
      a.partial[(size_t)(iy0 + tid) * a.ntiles_xz + tile] = p;
    }
  }
  return true;
}

template <class C> __device__ __forceinline__ void init_ring(const SmemLayout<C> &L, volatile int *s_abort) {
  if (threadIdx.x == 0) {
    for (int b = 0; b < C::NSTAGE_; ++b) {
      mbar_init(smem_u32(&L.full[b]), 1);
      mbar_init(smem_u32(&L.empty[b]), C::NT_ / 32);
    }
    fence_mbar_init();
    *s_abort = 0;
  }
}

// The producer leaves no copy landing in shared memory after the CTA exits
// (only possible after an abort): a bounded wait, which an abort does not cut
// short, on each of the last NSTAGE stages it issued (a stage it left out by the
// test hook has no copy in flight).  Within the last NSTAGE issued stages every
// barrier serves one stage, so its parity identifies that stage's phase.
template <class C> __device__ __forceinline__ void drain_ring(const SmemLayout<C> &L, const ProducerState &ps,
                                                              volatile int *s_abort, uint64_t limit_ns) {
  if (threadIdx.x == C::NT_ && *s_abort)
    for (int g = max(0, ps.issued - C::NSTAGE_); g < ps.issued; ++g)
      if (g != ps.skipped) wait_phase(smem_u32(&L.full[g % C::NSTAGE_]), (g / C::NSTAGE_) & 1, nullptr, limit_ns);
}

// One launch per series: grid = tiles of that series.
template <int STORE, int S, int K, int TX, int NT, int VPS, int NSTAGE, int ZF>
__global__ void __launch_bounds__(NT + 32) bp_fast_kernel(const __grid_constant__ BpArgs a) {
  using C = FastCfg<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ volatile int s_abort;
  const SmemLayout<C> L(sm, a.nviews);
  init_ring(L, &s_abort);
  int gst = 0;
  ProducerState ps;
  bp_tile<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>(a, blockIdx.x, blockIdx.y, blockIdx.z, sm, L, gst, &s_abort, ps);
  drain_ring(L, ps, &s_abort, a.wait_limit_ns);
}

// Persistent launch over the tiles of many series: each CTA takes the next
// tile of the queue (longest series first) until it is empty.  Each tile's
// arithmetic is the same as in the per-series kernel, so every series' result
// does not depend on what else is in the batch.
// Resident CTAs per SM: the per-series kernel's 32-accumulator shapes fit three
// 288-thread (five 160-thread) CTAs in the register file; without a bound the
// tile loop's extra state takes this kernel to 84-96 registers and two (four)
// CTAs, a third less throughput.  The bound keeps the per-series occupancy.
template <int S, int K, int NT> constexpr int batch_min_ctas() {
  return S * K > 32 ? 1 : NT == 256 ? 3 : 5;
}
template <int STORE, int S, int K, int TX, int NT, int VPS, int NSTAGE, int ZF>
__global__ void __launch_bounds__(NT + 32, (batch_min_ctas<S, K, NT>())) bp_batch_kernel(const BpArgs *__restrict__ jobs, int njobs,
                                                           int ntiles, int *counter, int max_views) {
  using C = FastCfg<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ volatile int s_abort;
  __shared__ int4 s_tile;  // (tile, series, index inside the series, -)
  __shared__ __align__(16) BpArgs s_args;
  const SmemLayout<C> L(sm, max_views);
  init_ring(L, &s_abort);
  int gst = 0;
  ProducerState ps;
  uint64_t limit_ns = 2000000000ull;
  for (;;) {
    if (threadIdx.x == 0) {
      const int t = atomicAdd(counter, 1);
      int lo = 0, hi = njobs - 1;  // last series whose first tile is <= t
      while (t < ntiles && lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&jobs[mid].tile0) <= t) lo = mid;
        else hi = mid - 1;
      }
      s_tile = make_int4(t, lo, t < ntiles ? t - __ldg(&jobs[lo].tile0) : 0, 0);
    }
    __syncthreads();
    const int4 T = s_tile;
    if (T.x >= ntiles || s_abort) break;
    {
      const uint32_t *src = reinterpret_cast<const uint32_t *>(&jobs[T.y]);
      uint32_t *dst = reinterpret_cast<uint32_t *>(const_cast<BpArgs *>(&s_args));
      for (int i = threadIdx.x; i < (int)(sizeof(BpArgs) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const int nbx = s_args.nbx, nxz = s_args.ntiles_xz;
    const int bx = T.z % nbx, by = (T.z % nxz) / nbx, bz = T.z / nxz;
    limit_ns = s_args.wait_limit_ns;
    if (!bp_tile<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>(s_args, bx, by, bz, sm, L, gst, &s_abort, ps)) {
      s_abort = 1;
    }
  }
  drain_ring(L, ps, &s_abort, limit_ns);
}



// ---- variant table (tile shapes the autotuner chooses from) ----
struct FastVariant { int S, K, TX, NT, VPS, NSTAGE; const char *name; };
static const FastVariant kFast[] = {
    {8, 4, 32, 128, 2, 4, "S8K4TX32NT128V2N4"},
    {8, 4, 32, 128, 4, 3, "S8K4TX32NT128V4N3"},
    {8, 4, 32, 256, 2, 4, "S8K4TX32NT256V2N4"},
    {8, 4, 64, 256, 2, 4, "S8K4TX64NT256V2N4"},
    {16, 2, 32, 128, 2, 4, "S16K2TX32NT128V2N4"},
    {16, 2, 32, 256, 2, 4, "S16K2TX32NT256V2N4"},
    {8, 8, 32, 128, 2, 4, "S8K8TX32NT128V2N4"},
    {8, 8, 32, 256, 2, 4, "S8K8TX32NT256V2N4"},
    {8, 4, 32, 256, 4, 3, "S8K4TX32NT256V4N3"},
    {8, 4, 32, 256, 8, 2, "S8K4TX32NT256V8N2"},
    {8, 4, 32, 256, 8, 3, "S8K4TX32NT256V8N3"},
    {8, 4, 64, 256, 4, 3, "S8K4TX64NT256V4N3"},
    {16, 2, 64, 256, 4, 3, "S16K2TX64NT256V4N3"},
    {16, 2, 32, 256, 4, 3, "S16K2TX32NT256V4N3"},
};
constexpr int MAX_S = 16;  // rows per tile of the widest variant (sizes the staging buffer)
int bp_fast_variants() { return (int)(sizeof(kFast) / sizeof(kFast[0])); }
const char *bp_fast_variant_name(int v) { return kFast[v].name; }
int bp_fast_row_align() { return MAX_S; }

template <int STORE, int S, int K, int TX, int NT, int VPS, int NSTAGE, int ZF>
static int launch_fast_t(const BpArgs &a0, cudaStream_t st, int *ntiles) {
  using C = FastCfg<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>;
  auto kern = bp_fast_kernel<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>;
  size_t smem = C::smem(a0.nviews);
  if (smem > 220 * 1024) return TG_ERR_UNSUPPORTED;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(bp_fast)");
  dim3 grid((a0.onx + TX - 1) / TX, (a0.onz + C::TZ - 1) / C::TZ, (a0.ny + S - 1) / S);
  BpArgs a = a0;
  a.nbx = grid.x;
  a.ntiles_xz = grid.x * grid.y;
  if (ntiles) *ntiles = grid.x * grid.y;
  kern<<<grid, C::NTHR, smem, st>>>(a);
  return TG_OK;
}

template <int STORE, int S, int K, int TX, int NT, int VPS, int NSTAGE, int ZF>
static int launch_batch_t(const BatchLaunch &bl, cudaStream_t st) {
  using C = FastCfg<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>;
  auto kern = bp_batch_kernel<STORE, S, K, TX, NT, VPS, NSTAGE, ZF>;
  size_t smem = C::smem(bl.max_views);
  if (smem > 220 * 1024) return TG_ERR_UNSUPPORTED;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(bp_batch)");
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, C::NTHR, smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  const int grid = std::max(1, std::min(bl.ntiles, nsm * std::max(1, per_sm)));
  e = cudaMemsetAsync(bl.counter, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(tile counter)");
  kern<<<grid, C::NTHR, smem, st>>>(bl.jobs, bl.njobs, bl.ntiles, bl.counter, bl.max_views);
  return TG_OK;
}

template <int STORE, int ZF>
static int launch_fast_v(const BpArgs &a, int variant, cudaStream_t st, int *ntiles) {
  switch (variant) {
    case 0: return launch_fast_t<STORE, 8, 4, 32, 128, 2, 4, ZF>(a, st, ntiles);
    case 1: return launch_fast_t<STORE, 8, 4, 32, 128, 4, 3, ZF>(a, st, ntiles);
    case 2: return launch_fast_t<STORE, 8, 4, 32, 256, 2, 4, ZF>(a, st, ntiles);
    case 3: return launch_fast_t<STORE, 8, 4, 64, 256, 2, 4, ZF>(a, st, ntiles);
    case 4: return launch_fast_t<STORE, 16, 2, 32, 128, 2, 4, ZF>(a, st, ntiles);
    case 5: return launch_fast_t<STORE, 16, 2, 32, 256, 2, 4, ZF>(a, st, ntiles);
    case 6: return launch_fast_t<STORE, 8, 8, 32, 128, 2, 4, ZF>(a, st, ntiles);
    case 7: return launch_fast_t<STORE, 8, 8, 32, 256, 2, 4, ZF>(a, st, ntiles);
    case 8: return launch_fast_t<STORE, 8, 4, 32, 256, 4, 3, ZF>(a, st, ntiles);
    case 9: return launch_fast_t<STORE, 8, 4, 32, 256, 8, 2, ZF>(a, st, ntiles);
    case 10: return launch_fast_t<STORE, 8, 4, 32, 256, 8, 3, ZF>(a, st, ntiles);
    case 12: return launch_fast_t<STORE, 16, 2, 64, 256, 4, 3, ZF>(a, st, ntiles);
    case 13: return launch_fast_t<STORE, 16, 2, 32, 256, 4, 3, ZF>(a, st, ntiles);
    default: return launch_fast_t<STORE, 8, 4, 64, 256, 4, 3, ZF>(a, st, ntiles);
  }
}

template <int STORE, int ZF>
static int launch_batch_v(const BatchLaunch &bl, int variant, cudaStream_t st) {
  switch (variant) {
    case 0: return launch_batch_t<STORE, 8, 4, 32, 128, 2, 4, ZF>(bl, st);
    case 1: return launch_batch_t<STORE, 8, 4, 32, 128, 4, 3, ZF>(bl, st);
    case 2: return launch_batch_t<STORE, 8, 4, 32, 256, 2, 4, ZF>(bl, st);
    case 3: return launch_batch_t<STORE, 8, 4, 64, 256, 2, 4, ZF>(bl, st);
    case 4: return launch_batch_t<STORE, 16, 2, 32, 128, 2, 4, ZF>(bl, st);
    case 5: return launch_batch_t<STORE, 16, 2, 32, 256, 2, 4, ZF>(bl, st);
    case 6: return launch_batch_t<STORE, 8, 8, 32, 128, 2, 4, ZF>(bl, st);
    case 7: return launch_batch_t<STORE, 8, 8, 32, 256, 2, 4, ZF>(bl, st);
    case 8: return launch_batch_t<STORE, 8, 4, 32, 256, 4, 3, ZF>(bl, st);
    case 9: return launch_batch_t<STORE, 8, 4, 32, 256, 8, 2, ZF>(bl, st);
    case 10: return launch_batch_t<STORE, 8, 4, 32, 256, 8, 3, ZF>(bl, st);
    case 12: return launch_batch_t<STORE, 16, 2, 64, 256, 4, 3, ZF>(bl, st);
    case 13: return launch_batch_t<STORE, 16, 2, 32, 256, 4, 3, ZF>(bl, st);
    default: return launch_batch_t<STORE, 8, 4, 64, 256, 4, 3, ZF>(bl, st);
  }
}

int launch_bp_batch(const BatchLaunch &bl, int store, bool zf, int variant, cudaStream_t st) {
  if (variant < 0 || variant >= bp_fast_variants()) variant = 0;
  if (store == TG_STORE_FP32)
    return zf ? launch_batch_v<TG_STORE_FP32, 1>(bl, variant, st) : launch_batch_v<TG_STORE_FP32, 0>(bl, variant, st);
  if (store == TG_STORE_FP16)
    return zf ? launch_batch_v<TG_STORE_FP16, 1>(bl, variant, st) : launch_batch_v<TG_STORE_FP16, 0>(bl, variant, st);
  return zf ? launch_batch_v<TG_STORE_BF16, 1>(bl, variant, st) : launch_batch_v<TG_STORE_BF16, 0>(bl, variant, st);
}

void bp_fast_tile_shape(int variant, int *S, int *TX, int *TZ) {
  const FastVariant &f = kFast[variant < 0 || variant >= bp_fast_variants() ? 0 : variant];
  *S = f.S;
  *TX = f.TX;
  *TZ = (f.NT / f.TX) * f.K;
}

int bp_fast_ntiles(const BpArgs &a, int variant) {
  const FastVariant &f = kFast[variant];
  int tz = (f.NT / f.TX) * f.K;
  return ((a.onx + f.TX - 1) / f.TX) * ((a.onz + tz - 1) / tz);
}

template <int STORE>
static int launch_fast_z(const BpArgs &a, int zf, int variant, cudaStream_t st, int *ntiles) {
  return zf == 2 ? launch_fast_v<STORE, 2>(a, variant, st, ntiles)
                 : zf ? launch_fast_v<STORE, 1>(a, variant, st, ntiles) : launch_fast_v<STORE, 0>(a, variant, st, ntiles);
}

int launch_bp_fast(const BpArgs &a, int store, int zf, int variant, cudaStream_t st, int *ntiles) {
  if (variant < 0 || variant >= bp_fast_variants()) variant = 0;
  if (store == TG_STORE_FP32) return launch_fast_z<TG_STORE_FP32>(a, zf, variant, st, ntiles);
  if (store == TG_STORE_FP16) return launch_fast_z<TG_STORE_FP16>(a, zf, variant, st, ntiles);
  return launch_fast_z<TG_STORE_BF16>(a, zf, variant, st, ntiles);
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
    if (a.has_local) use_l = local_corr(a.loc, v, oxc, iy, a.ny, ldx, ldy);
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
  if (a.mode == 2) {  // vol += relax * v: the K old values are loaded before any store
    float old[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const int oz = oz0 + tzg + j * OZG;
      old[j] = (xok && oz < a.onz) ? a.vol[((size_t)iy * a.onz + oz) * a.onx + ox] : 0.0f;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const int oz = oz0 + tzg + j * OZG;
      if (xok && oz < a.onz)
        a.vol[((size_t)iy * a.onz + oz) * a.onx + ox] = __fadd_rn(old[j], __fmul_rn(a.relax, __fmul_rn(acc[j], a.inv_n)));
    }
    return;
  }
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
      } else {  // mode 1
        a.vol[idx] = v;
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
