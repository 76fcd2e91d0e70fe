// session.cu -- C ABI of libtiltgpu: planning, device residency and the
// stage sequence of one reconstruction.
//
// The stage order is main() of apps/tilt/src/main.rs:607-1093:
//   log10 (608-613) -> per-view means (616-623) -> R-weighting (638-646)
//   -> cosine stretch (648-653) -> WBP (1002-1090) | SIRT (919-975)
//   -> fake SIRT (955-962, 976-1001) -> output transform and header stats.
// Geometry (tilt/x-tilt sin & cos, z-factor, stretch factors, centres) is
// computed on the host in the reference's f32 expressions, so the device
// makes the same sampling decisions as the reference.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "session_impl.h"

namespace tg {

static thread_local std::string g_err;
void set_error(const std::string &m) { g_err = m; }
int cuda_fail(cudaError_t e, const char *what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? TG_ERR_OOM : TG_ERR_CUDA;
}
int device_error_status(int word) {
  if (word & 1) { set_error("a bounded device wait timed out"); return TG_ERR_TIMEOUT; }
  if (word & 4) {
    set_error("a filtered projection or SIRT residual exceeds the FP16 staging range (|v| >= 65520); "
              "the SIRT run diverges or the data need FP32/BF16 staging");
    return TG_ERR_RANGE;
  }
  set_error("staging window outside the padded row (internal error)");
  return TG_ERR_CUDA;
}

static const float PI_F = 3.14159265358979323846f;  // std::f32::consts::PI

// Per-view geometry exactly as ProjParams is built (main.rs:683-700).
struct HostView { float cos_t, sin_t, cos_xt, sin_xt, zf; };

static std::vector<HostView> host_views(int nviews, const float *ang, const float *xt, int nxt,
                                        const float *zf, int nzf) {
  std::vector<HostView> v(nviews);
  for (int i = 0; i < nviews; ++i) {
    volatile float rad = ang[i] * PI_F / 180.0f;  // (deg*PI)/180 in f32
    float xdeg = (xt && i < nxt) ? xt[i] : 0.0f;
    volatile float xrad = xdeg * PI_F / 180.0f;
    v[i].cos_t = cosf(rad);
    v[i].sin_t = sinf(rad);
    v[i].cos_xt = cosf(xrad);
    v[i].sin_xt = sinf(xrad);
    v[i].zf = (zf && i < nzf) ? zf[i] : 1.0f;
  }
  return v;
}

// Exact f32 sample position (main.rs:1015-1021).
static inline float ref_x_host(float dx, float dz, const HostView &h, float cx) {
  volatile float t1 = dx * h.cos_t;
  volatile float t1b = t1 * h.cos_xt;
  volatile float t2 = dz * h.sin_t;
  volatile float t2b = t2 * h.zf;
  volatile float s = t1b + t2b;
  return s + cx;
}

// Radial weight table, apps/tilt/src/main.rs:348-369 (f32 expressions).
void weight_table(int n, float cutoff, float falloff, int efs, int hamming, float *wt) {
  size_t filter_nxc = efs > 0 ? (size_t)efs : (size_t)(n / 2 + 1);
  for (int i = 0; i < n; ++i) {
    int fb = i <= n / 2 ? i : n - i;
    volatile float w = (float)fb / (float)filter_nxc;
    float weight;
    if (hamming) {
      float h;
      if (cutoff > 1e-12f && w <= cutoff) {
        volatile float arg = PI_F * w;
        volatile float arg2 = arg / cutoff;
        volatile float c = cosf(arg2);
        volatile float m = 0.46f * c;
        h = 0.54f + m;
      } else if (w > cutoff) {
        h = 0.0f;
      } else {
        h = 1.0f;
      }
      weight = w * h;
    } else if (w <= cutoff) {
      weight = w;
    } else {
      volatile float d = w - cutoff;
      volatile float num = -d * d;
      volatile float den0 = 2.0f * falloff;
      volatile float den = den0 * falloff;
      volatile float q = num / den;
      weight = w * expf(q);
    }
    wt[i] = weight;
  }
}

// ---------------------------------------------------------------------------
// Autotuned tile variant per (nx, onx, onz, nviews, storage, zf), process-wide.
// ---------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int, int, int, int>, int> g_tune;

}  // namespace tg

using namespace tg;

namespace tg {

// Sessions of the server allocate stream-ordered from its pool (a free does not
// synchronise the device); a dry session only counts the bytes it would take.
template <class T> static int dalloc(tg_session *s, T **p, size_t bytes) {
  if (s->dry) {
    *p = nullptr;
    s->dev_bytes += bytes;
    return TG_OK;
  }
  if (s->fail_alloc) {
    *p = nullptr;
    set_error("device allocation failed (injected)");
    return TG_ERR_OOM;
  }
  cudaError_t e = s->pool ? cudaMallocFromPoolAsync((void **)p, std::max<size_t>(bytes, 16), s->pool, s->own_st)
                          : cudaMalloc((void **)p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) {
    char buf[128];
    snprintf(buf, sizeof buf, "cudaMalloc(%zu bytes)", bytes);
    return cuda_fail(e, buf);
  }
  s->dev_bytes += bytes;
  return TG_OK;
}

static void free_session(tg_session *s) {
  if (!s) return;
  if (s->pool) {  // stream-ordered on the session's own stream
    free_session_async(s, s->own_st);
    return;
  }
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->sirt_exec) cudaGraphExecDestroy(s->sirt_exec);
  void *ptrs[] = {s->d_raw, s->d_logd, s->d_means, s->d_vol, s->d_sino, s->d_tmp, s->d_volg, s->d_volh, s->d_maxbits, s->d_mpart, s->d_pairs,
                  s->d_part, s->d_slice_stats, s->d_stats3, s->d_vg, s->d_vg2, s->d_weights,
                  s->d_conv, s->d_stretch, s->d_tw, s->d_err, s->d_lvinfo, s->d_lgoff, s->d_lxs,
                  s->d_lys, s->d_lgdx, s->d_lgdy, s->d_ltab, s->d_xtb, s->d_lbnd, s->d_half};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (auto &e : s->ev)
    if (e) cudaEventDestroy(e);
  if (s->own_st) cudaStreamDestroy(s->own_st);
  delete s;
}

void free_session_async(tg_session *s, cudaStream_t after) {
  if (s->sirt_exec) cudaGraphExecDestroy(s->sirt_exec);  // freed on completion if in flight
  void *ptrs[] = {s->d_raw, s->d_logd, s->d_means, s->d_vol, s->d_sino, s->d_tmp, s->d_volg, s->d_volh, s->d_maxbits, s->d_mpart, s->d_pairs,
                  s->d_part, s->d_slice_stats, s->d_stats3, s->d_vg, s->d_vg2, s->d_weights,
                  s->d_conv, s->d_stretch, s->d_tw, s->d_err, s->d_lvinfo, s->d_lgoff, s->d_lxs,
                  s->d_lys, s->d_lgdx, s->d_lgdy, s->d_ltab, s->d_xtb, s->d_lbnd, s->d_half};
  for (void *p : ptrs)
    if (p) cudaFreeAsync(p, after);
  for (auto &e : s->ev)
    if (e) cudaEventDestroy(e);
  if (s->own_st) cudaStreamDestroy(s->own_st);
  delete s;
}

// load_local_alignment (apps/tilt/src/main.rs:232-307) into flat device arrays
static int upload_local(tg_session *s, const float *rows, int nrows, std::vector<float4> &vg2) {
  std::vector<int4> vinfo(s->nviews, make_int4(0, 0, 0, 0));
  std::vector<int> goff(s->nviews, 0);
  std::vector<float> xs_all, ys_all, gdx, gdy;
  std::vector<std::vector<int>> by_view(s->nz);
  for (int i = 0; i < nrows; ++i) {
    long v = (long)rows[i * 5];
    if (v >= 0 && v < s->nz) by_view[v].push_back(i);
  }
  auto dedup = [](std::vector<float> &v) {
    std::vector<float> out;
    for (float e : v)
      if (out.empty() || !(fabsf(e - out.back()) < 0.01f)) out.push_back(e);
    v.swap(out);
  };
  for (int vi = 0; vi < s->nviews; ++vi) {
    auto &idx = by_view[vi];
    if (idx.empty()) continue;
    std::vector<float> xs, ys;
    for (int i : idx) { xs.push_back(rows[i * 5 + 1]); ys.push_back(rows[i * 5 + 2]); }
    std::stable_sort(xs.begin(), xs.end());
    dedup(xs);
    std::stable_sort(ys.begin(), ys.end());
    dedup(ys);
    int nx = (int)xs.size(), ny = (int)ys.size();
    std::vector<float> dxg((size_t)nx * ny, 0.f), dyg((size_t)nx * ny, 0.f);
    for (int i : idx) {
      float px = rows[i * 5 + 1], py = rows[i * 5 + 2];
      int ix = 0, iy = 0;
      for (int k = 0; k < nx; ++k) if (fabsf(xs[k] - px) < 0.01f) { ix = k; break; }
      for (int k = 0; k < ny; ++k) if (fabsf(ys[k] - py) < 0.01f) { iy = k; break; }
      dxg[(size_t)iy * nx + ix] = rows[i * 5 + 3];
      dyg[(size_t)iy * nx + ix] = rows[i * 5 + 4];
    }
    float lx = 0.f, ly = 0.f;
    for (float d : dxg) lx = std::max(lx, fabsf(d));
    for (float d : dyg) ly = std::max(ly, fabsf(d));
    vg2[vi].y = lx;
    vg2[vi].z = ly;
    vinfo[vi] = make_int4((int)xs_all.size(), nx, (int)ys_all.size(), ny);
    goff[vi] = (int)gdx.size();
    xs_all.insert(xs_all.end(), xs.begin(), xs.end());
    ys_all.insert(ys_all.end(), ys.begin(), ys.end());
    gdx.insert(gdx.end(), dxg.begin(), dxg.end());
    gdy.insert(gdy.end(), dyg.begin(), dyg.end());
  }
  int rc;
  if ((rc = dalloc(s, &s->d_lvinfo, vinfo.size() * sizeof(int4)))) return rc;
  if ((rc = dalloc(s, &s->d_lgoff, goff.size() * sizeof(int)))) return rc;
  if ((rc = dalloc(s, &s->d_lxs, xs_all.size() * sizeof(float)))) return rc;
  if ((rc = dalloc(s, &s->d_lys, ys_all.size() * sizeof(float)))) return rc;
  if ((rc = dalloc(s, &s->d_lgdx, gdx.size() * sizeof(float)))) return rc;
  if ((rc = dalloc(s, &s->d_lgdy, gdy.size() * sizeof(float)))) return rc;
  if (s->dry) return TG_OK;
  if (s->pool) TG_CUDA(cudaStreamSynchronize(s->own_st));  // the stream-ordered allocations exist
  TG_CUDA(cudaMemcpy(s->d_lvinfo, vinfo.data(), vinfo.size() * sizeof(int4), cudaMemcpyHostToDevice));
  TG_CUDA(cudaMemcpy(s->d_lgoff, goff.data(), goff.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (!xs_all.empty()) TG_CUDA(cudaMemcpy(s->d_lxs, xs_all.data(), xs_all.size() * sizeof(float), cudaMemcpyHostToDevice));
  if (!ys_all.empty()) TG_CUDA(cudaMemcpy(s->d_lys, ys_all.data(), ys_all.size() * sizeof(float), cudaMemcpyHostToDevice));
  if (!gdx.empty()) TG_CUDA(cudaMemcpy(s->d_lgdx, gdx.data(), gdx.size() * sizeof(float), cudaMemcpyHostToDevice));
  if (!gdy.empty()) TG_CUDA(cudaMemcpy(s->d_lgdy, gdy.data(), gdy.size() * sizeof(float), cudaMemcpyHostToDevice));
  return TG_OK;
}

LocalDev local_dev(tg_session *s) {
  LocalDev L{};
  L.vinfo = s->d_lvinfo;
  L.goff = s->d_lgoff;
  L.xs = s->d_lxs;
  L.ys = s->d_lys;
  L.gdx = s->d_lgdx;
  L.gdy = s->d_lgdy;
  L.table = s->d_ltab;
  L.table_nx = s->onx;
  return L;
}

BpArgs bp_args(tg_session *s, int mode) {
  BpArgs a{};
  a.pairs = s->d_pairs;
  a.vg = s->d_vg;
  a.vg2 = s->d_vg2;
  a.vol = s->d_vol;
  a.partial = s->d_part;
  a.err = s->d_err;
  a.nx = s->nx;
  a.ny = s->ny;
  a.nviews = s->nviews;
  a.onx = s->onx;
  a.onz = s->onz;
  a.PW = s->PW;
  a.padL = s->padL;
  a.rows_alloc = s->rows_alloc;
  a.cx = s->cx;
  a.cz = s->cz;
  a.ocx = s->ocx;
  a.inv_n = s->inv_n;
  a.dw = s->o.densweight;
  a.os = s->o.outscale;
  a.oa = s->o.outadd;
  a.relax = s->o.sirt_relax;
  a.mode = mode;
  a.has_local = s->has_local ? 1 : 0;
  a.loc = local_dev(s);
  a.wait_limit_ns = s->wait_limit_ns;
  a.fault_skip_stage = s->fault_skip_stage;
  return a;
}

FilterArgs filter_args(tg_session *s, bool residual) {
  FilterArgs f{};
  f.in = s->d_logd ? s->d_logd : s->d_raw;
  f.sub = residual ? s->d_sino : nullptr;
  f.out = s->d_pairs;
  f.weights = s->o.no_weight ? nullptr : s->d_weights;
  f.tw = s->d_tw;
  f.tw2 = s->has_tw2 ? s->d_tw + s->nx : nullptr;
  f.conv_h = s->use_conv ? s->d_conv : nullptr;
  f.stretch = residual ? nullptr : s->d_stretch;
  f.fill = s->d_means;
  f.nx = s->nx;
  f.ny = s->ny;
  f.nviews = s->nviews;
  f.rows_alloc = s->rows_alloc;
  f.PW = s->PW;
  f.padL = s->padL;
  f.fill_mode = s->o.gpu_compat ? TG_FILL_ZERO : s->o.fill_mode;
  f.cubic = s->o.cosine_cubic;
  f.fmt = s->fmt;
  f.store = s->store;
  f.inv_n = 1.0f / (float)s->nx;
  f.plan = s->plan;
  f.err = s->d_err;
  return f;
}

int launch_bp(tg_session *s, int mode, int *ntiles) {
  BpArgs a = bp_args(s, mode);
  if (s->fast) return launch_bp_fast(a, s->store, fast_zf(s), s->variant < 0 ? 0 : s->variant, s->st, ntiles);
  if (s->xt_split) {  // per-row view sums, then the two-row blend of every voxel
    BpArgs r = bp_args(s, 1);
    r.vol = s->xtb;
    int rc = launch_bp_fast(r, s->store, fast_zf(s), s->variant < 0 ? 0 : s->variant, s->st, nullptr);
    if (rc != TG_OK) return rc;
    return launch_xt_blend(a, s->xtb, s->sin_xt_common, s->st, ntiles);
  }
  if (s->xt_fast) return launch_bp_xtilt(a, s->store, s->st, ntiles);
  return launch_bp_general(a, s->store, s->st, ntiles);
}

// Times each fast tile variant once on (the first 64 slices of) this series and
// keeps the fastest (process-wide cache keyed by the series shape).
int autotune(tg_session *s) {
  if (!s->fast && !s->xt_split) { s->variant = 0; return TG_OK; }
  if (const char *env = getenv("TG_BP_VARIANT")) {  // fixed tile shape (profiling, tuning)
    int v = atoi(env);
    if (v >= 0 && v < bp_fast_variants()) { s->variant = v; return TG_OK; }
  }
  auto key = std::make_tuple(s->nx, s->onx, s->onz, s->nviews, s->store, fast_zf(s), s->ny >= 64 ? 64 : s->ny);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) { s->variant = it->second; return TG_OK; }
  }
  int best = 0;
  float best_ms = 1e30f;
  cudaEvent_t e0, e1;
  TG_CUDA(cudaEventCreate(&e0));
  TG_CUDA(cudaEventCreate(&e1));
  for (int v = 0; v < bp_fast_variants(); ++v) {
    BpArgs a = bp_args(s, 1);
    a.wait_limit_ns = 2000000000ull;  // tuning never runs the test hook
    a.fault_skip_stage = -1;
    // the first 64 slices (every tile shape's rows divide 64): the time per update does
    // not depend on the slice, and a one-shot reconstruction should not pay for tuning
    // that is longer than the reconstruction itself
    a.ny = std::min(a.ny, 64);
    if (s->xt_split) a.vol = s->xtb;
    int nt = 0;
    // warm + timed launch (mode 1 writes the volume, which is rewritten afterwards)
    if (launch_bp_fast(a, s->store, fast_zf(s), v, s->st, &nt) != TG_OK) continue;
    cudaEventRecord(e0, s->st);
    launch_bp_fast(a, s->store, fast_zf(s), v, s->st, &nt);
    cudaEventRecord(e1, s->st);
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) { best_ms = ms; best = v; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  TG_CUDA(cudaGetLastError());
  s->variant = best;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[key] = best;
  return TG_OK;
}

int tune_lookup(tg_session *s) {
  if (!s->fast && !s->xt_split) return 0;
  if (const char *env = getenv("TG_BP_VARIANT")) {
    int v = atoi(env);
    if (v >= 0 && v < bp_fast_variants()) return v;
  }
  auto key = std::make_tuple(s->nx, s->onx, s->onz, s->nviews, s->store, fast_zf(s), s->ny >= 64 ? 64 : s->ny);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(key);
  return it != g_tune.end() ? it->second : -1;
}

FpArgs fp_args(tg_session *s) {
  FpArgs f{};
  f.vol = s->d_vol;
  f.sino = s->d_sino;
  f.vg = s->d_vg;
  f.vg2 = s->d_vg2;
  f.nx = s->nx;
  f.ny = s->ny;
  f.nviews = s->nviews;
  f.nviews_all = s->nviews;
  f.onx = s->onx;
  f.onz = s->onz;
  f.cx = s->cx;
  f.cz = s->cz;
  f.ocx = s->ocx;
  f.has_local = s->has_local;
  f.loc = local_dev(s);
  f.fast = s->fp_fast;
  f.volg = s->d_volg;
  f.sin_xt_common = s->sin_xt_common;
  f.volh = s->d_volh;
  f.maxbits = s->d_maxbits;
  f.variant = s->fp_variant;
  f.lbnd = s->d_lbnd;
  return f;
}

int stage_front(tg_session *s, int *launches) {
  // every run starts from the uploaded projections: log10 into d_logd (--log) and the
  // per-view means, as main.rs:608-623 does before each reconstruction
  launch_log_means(s->d_raw, s->d_logd, s->nx * s->ny, s->nz, s->d_mpart, s->means_pinned ? nullptr : s->d_means,
                   s->st);
  *launches += 2;
  launch_filter(filter_args(s, false), s->st);
  *launches += 1;
  TG_CUDA(cudaGetLastError());
  return TG_OK;
}

int stage_finish(tg_session *s, int mode0, int ntiles, int *launches) {
  for (int k = 0; k < fake_passes(s); ++k) {
    launch_lowpass(s->d_vol, s->d_tmp, s->onx, s->onz, s->ny, s->st);
    *launches += 3;
  }
  if (mode0 == 1) {
    launch_transform_stats(s->d_vol, s->onx, s->onz, s->ny, s->o.densweight, s->o.outscale, s->o.outadd,
                           s->d_part, &ntiles, s->st);
    *launches += 1;
  }
  launch_stats_reduce(s->d_part, s->ny, ntiles, s->onx * s->onz, s->d_slice_stats, s->d_stats3, s->st);
  *launches += 2;
  TG_CUDA(cudaGetLastError());
  return TG_OK;
}

}  // namespace tg

extern "C" {

int tg_abi_version(void) { return TG_ABI_VERSION; }
const char *tg_last_error(void) { return tg::g_err.c_str(); }

const char *tg_status_string(int st) {
  switch (st) {
    case TG_OK: return "ok";
    case TG_ERR_INVALID_ARG: return "invalid argument";
    case TG_ERR_OOM: return "out of device memory";
    case TG_ERR_CUDA: return "CUDA error";
    case TG_ERR_TIMEOUT: return "device wait timed out";
    case TG_ERR_BUDGET: return "over memory budget";
    case TG_ERR_UNSUPPORTED: return "unsupported";
    case TG_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case TG_ERR_PANIC: return "input on which the reference panics";
    case TG_ERR_NOT_READY: return "not ready";
    case TG_ERR_NOT_FOUND: return "not found";
    case TG_ERR_CANCELLED: return "cancelled";
    case TG_ERR_RANGE: return "value beyond the FP16 staging range";
    default: return "unknown status";
  }
}

void tg_options_default(tg_options *o) {
  memset(o, 0, sizeof *o);
  o->radial_cutoff = 0.35f;
  o->radial_falloff = 0.05f;
  o->fill_mode = TG_FILL_MEAN;
  o->max_cosine_tilt = 80.0f;
  o->sirt_relax = 1.0f;
  o->densweight = 1.0f;
  o->outscale = 1.0f;
  o->outadd = 0.0f;
  o->storage = TG_STORE_FP32;
  o->use_graphs = 1;
}

int tg_session_create(const tg_geometry *g, const tg_options *opt, tg_session **out) {
  return tg::session_create_ex(g, opt, nullptr, false, false, out);
}

}  // extern "C"

// pool: allocate stream-ordered from it; dry: compute sizes only (no device
// work; the returned object holds dev_bytes and must be freed with
// session_discard); fail_alloc: fault-injection hook (the first allocation fails).
int tg::session_create_ex(const tg_geometry *g, const tg_options *opt, cudaMemPool_t pool, bool dry,
                          bool fail_alloc, tg_session **out) {
  if (!g || !opt || !out) { set_error("null argument"); return TG_ERR_INVALID_ARG; }
  *out = nullptr;
  if (g->nx < 2 || g->ny < 1 || g->nz < 1 || g->nx > 65536 || g->ny > 65535 || g->nz > 4096) {
    set_error("unsupported projection dimensions (need nx>=2)");
    return TG_ERR_INVALID_ARG;
  }
  if (g->n_angles < 1 || !g->angles) { set_error("no tilt angles"); return TG_ERR_INVALID_ARG; }
  if (opt->storage < 0 || opt->storage > 2) { set_error("bad storage"); return TG_ERR_INVALID_ARG; }
  {
    const int onx = g->out_nx > 0 ? g->out_nx : g->nx, onz = g->out_nz > 0 ? g->out_nz : g->nx;
    if (onx > 65536 || onz > 65536) { set_error("output too large"); return TG_ERR_INVALID_ARG; }
    // non-finite geometry would put sample positions outside every staged window
    auto finite = [](const float *a, int n) {
      for (int i = 0; a && i < n; ++i)
        if (!std::isfinite(a[i])) return false;
      return true;
    };
    if (!finite(g->angles, g->n_angles) || !finite(g->xtilt, g->n_xtilt) ||
        !finite(g->zfactor, g->n_zfactor) || (g->local && !finite(g->local, 5 * g->n_local))) {
      set_error("non-finite tilt, x-tilt, z-factor or local-alignment value");
      return TG_ERR_INVALID_ARG;
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("no CUDA device");
    return TG_ERR_NO_DEVICE;
  }
  if (opt->device < 0 || opt->device >= ndev) { set_error("bad device ordinal"); return TG_ERR_INVALID_ARG; }
  int major = 0;
  TG_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, opt->device));
  if (major != 10) { set_error("libtiltgpu is built for sm_100a only"); return TG_ERR_NO_DEVICE; }
  TG_CUDA(cudaSetDevice(opt->device));

  tg_session *s = new tg_session();
  s->pool = pool;
  s->dry = dry;
  s->fail_alloc = fail_alloc;
  s->o = *opt;
  s->dev = opt->device;
  s->nx = g->nx;
  s->ny = g->ny;
  s->nz = g->nz;
  s->onx = g->out_nx > 0 ? g->out_nx : g->nx;
  s->onz = g->out_nz > 0 ? g->out_nz : g->nx;
  s->nviews = std::min(g->n_angles, g->nz);  // tilt_angles.iter().take(nz)
  s->store = opt->storage;
  if (opt->gpu_compat) s->store = TG_STORE_FP32;
  s->has_local = !opt->gpu_compat && g->has_local;
  s->cx = (float)s->nx / 2.0f;
  s->cz = (float)s->onz / 2.0f;
  s->ocx = (float)s->onx / 2.0f;
  s->inv_n = 1.0f / (float)s->nz;
  int rc = TG_OK;
  auto fail = [&](int r) { free_session(s); return r; };

  // per-view geometry
  std::vector<HostView> hv;
  if (opt->gpu_compat)
    hv = host_views(s->nviews, g->angles, nullptr, 0, nullptr, 0);
  else
    hv = host_views(s->nviews, g->angles, g->xtilt, g->n_xtilt, g->zfactor, g->n_zfactor);
  std::vector<float4> vg(s->nviews), vg2(s->nviews);
  float zsmax = 0.f;
  bool xt_any = false;
  for (int i = 0; i < s->nviews; ++i) {
    vg[i] = make_float4(hv[i].cos_t, hv[i].sin_t, hv[i].zf, hv[i].cos_xt);
    vg2[i] = make_float4(hv[i].sin_xt, 0.f, 0.f, 0.f);
    if (hv[i].zf != 1.0f) s->zf_any = true;
    if (hv[i].sin_xt != 0.0f || hv[i].cos_xt != 1.0f) xt_any = true;
    zsmax = std::max(zsmax, fabsf(hv[i].sin_t * hv[i].zf));
  }
  s->fast = !s->has_local && !xt_any && zsmax <= 2.0f && fabsf(zsmax) == zsmax;
  {
    // the fast reprojector needs cos(tilt)*cos(x-tilt) > 0.05 in every view, and
    // x-tilts whose row offsets are either zero or clearly above the reference's
    // 1e-6 one-row threshold (|sin| >= 1e-5 with |dx| >= 0.5)
    bool ok = !s->has_local;
    for (int i = 0; i < s->nviews; ++i) {
      ok &= hv[i].cos_t * hv[i].cos_xt > 0.05f;
      ok &= hv[i].sin_xt == 0.0f || fabsf(hv[i].sin_xt) >= 1e-5f;
    }
    s->fp_fast = !ok ? 0 : xt_any ? 2 : 1;
    s->xt_common = s->nviews > 0;
    for (int i = 0; i < s->nviews; ++i) s->xt_common &= hv[i].sin_xt == hv[0].sin_xt;
    if (s->xt_common) s->sin_xt_common = hv[0].sin_xt;
  }
  if (s->zf_any && zsmax > 2.0f) s->fast = false;
  // one x-tilt for every view: the fast kernel's per-row sums, blended per voxel
  s->xt_split = !s->fast && !s->has_local && xt_any && s->xt_common && !opt->exact_xtilt &&
                zsmax <= 2.0f && fabsf(zsmax) == zsmax && !getenv("TG_BP_GENERAL");
  if (!s->fast && !s->xt_split && !s->has_local && zsmax <= 2.0f && !getenv("TG_BP_GENERAL")) {
    float msx = 0.0f, mext = 0.0f;
    bool ok = true;
    for (int i = 0; i < s->nviews; ++i) {
      ok &= hv[i].cos_t * hv[i].cos_xt > 0.0f;
      msx = std::max(msx, fabsf(hv[i].sin_xt));
      mext = std::max(mext, 31.0f * fabsf(hv[i].cos_t * hv[i].cos_xt) + 15.0f * fabsf(hv[i].sin_t * hv[i].zf));
    }
    s->xt_fast = ok && bp_xtilt_supported(s->onx, msx, mext);
  }
  s->fmt = s->fast || s->xt_split ? FMT_ROWPAIR : FMT_SINGLE;

  // cosine stretch factors (main.rs:446-460); the reference indexes
  // tilt_angles[p] for every section p < nz and panics if the file is short.
  std::vector<float> stretch(s->nviews, 0.0f);
  bool any_stretch = false;
  if (!opt->no_cosine_stretch) {
    if (g->n_angles < g->nz) {
      set_error("cosine stretch needs one tilt angle per section (the reference panics here)");
      return fail(TG_ERR_PANIC);
    }
    for (int p = 0; p < s->nviews; ++p) {
      float angle_abs = fabsf(g->angles[p]);
      if (angle_abs > opt->max_cosine_tilt) continue;
      volatile float rad = g->angles[p] * PI_F / 180.0f;
      float cos_t = cosf(rad);
      if (fabsf(cos_t) < 1e-6f) continue;
      stretch[p] = 1.0f / cos_t;
      any_stretch = true;
    }
  }

  // row padding so every staged window lies inside the row (exact corners)
  {
    int kmin = 0, kmax = s->nx - 1;
    float dxs[2] = {0.0f - s->ocx, (float)(s->onx - 1) - s->ocx};
    float dzs[2] = {0.0f - s->cz, (float)(s->onz - 1) - s->cz};
    for (int i = 0; i < s->nviews; ++i)
      for (float dx : dxs)
        for (float dz : dzs) {
          float x = ref_x_host(dx, dz, hv[i], s->cx);
          kmin = std::min(kmin, (int)floorf(x));
          kmax = std::max(kmax, (int)floorf(x));
        }
    int needL = std::max(0, -kmin), needR = std::max(0, kmax - (s->nx - 1));
    s->padL = ((needL + 3) + 1) & ~1;
    int padR = needR + 6;
    s->PW = (s->padL + s->nx + padR + 1) & ~1;
  }
  const int ra = bp_fast_row_align();  // a tile's row pairs never pass the allocation
  s->rows_alloc = s->fmt == FMT_ROWPAIR ? ((s->ny + ra - 1) / ra) * (ra / 2) : s->ny;

  // FFT plan or circulant fallback
  s->use_conv = !fft_plan(s->nx, &s->plan);
  if (s->nx * 16 > 200 * 1024) { set_error("rows wider than 12800 are not supported"); return fail(TG_ERR_UNSUPPORTED); }

  cudaError_t ce = cudaSuccess;
  if (!dry) {
    ce = cudaStreamCreateWithFlags(&s->own_st, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(cuda_fail(ce, "cudaStreamCreate"));
    s->st = s->own_st;
    for (auto &e : s->ev)
      if ((ce = cudaEventCreate(&e)) != cudaSuccess) return fail(cuda_fail(ce, "cudaEventCreate"));
  }

  const size_t nproj = (size_t)s->nx * s->ny * s->nz;
  const size_t nvol = (size_t)s->onx * s->onz * s->ny;
  s->pairs_bytes = (size_t)s->nviews * s->rows_alloc * s->PW * elem_bytes(s->fmt, s->store);
  // partial-stat capacity: the largest tile count of any kernel that may run
  int ntiles = 64;
  {
    BpArgs a{};
    a.onx = s->onx;
    a.onz = s->onz;
    for (int v = 0; v < bp_fast_variants(); ++v) ntiles = std::max(ntiles, bp_fast_ntiles(a, v));
    ntiles = std::max(ntiles, ((s->onx + 31) / 32) * ((s->onz + 15) / 16));
  }
  s->ntiles_cap = ntiles;
  if ((rc = dalloc(s, &s->d_raw, nproj * 4)) || (rc = dalloc(s, &s->d_means, (size_t)s->nz * 4)) ||
      (rc = dalloc(s, &s->d_mpart, (size_t)s->nz * 32 * 8)) || (rc = dalloc(s, &s->d_vol, nvol * 4)) ||
      (rc = dalloc(s, &s->d_pairs, s->pairs_bytes)) ||
      (rc = dalloc(s, &s->d_part, (size_t)s->ny * ntiles * sizeof(StatPartial))) ||
      (rc = dalloc(s, &s->d_slice_stats, (size_t)s->ny * 12)) || (rc = dalloc(s, &s->d_stats3, 16)) ||
      (rc = dalloc(s, &s->d_vg, (size_t)s->nviews * 16)) || (rc = dalloc(s, &s->d_vg2, (size_t)s->nviews * 16)) ||
      (rc = dalloc(s, &s->d_weights, (size_t)s->nx * 4)) || (rc = dalloc(s, &s->d_tw, (size_t)s->nx * 16)) ||
      (rc = dalloc(s, &s->d_stretch, (size_t)s->nviews * 4)) || (rc = dalloc(s, &s->d_err, 16)))
    return fail(rc);
  if (opt->log_transform && (rc = dalloc(s, &s->d_logd, nproj * 4))) return fail(rc);
  if (!opt->gpu_compat && opt->sirt_iters > 0 && (rc = dalloc(s, &s->d_sino, nproj * 4))) return fail(rc);
  if (!opt->gpu_compat && opt->fake_sirt > 0 && (rc = dalloc(s, &s->d_tmp, nvol * 4))) return fail(rc);
  if (const char *e = getenv("TG_FP_VARIANT")) s->fp_variant = atoi(e) & 15;
  // half staging forms reproject from an FP16 copy unless variant bit 3 asks for FP32
  const bool half_fp = s->store != TG_STORE_FP32 && !(s->fp_variant & 8);
  if (!opt->gpu_compat && opt->sirt_iters > 0 && half_fp &&
      (s->fp_fast == 1 || (s->fp_fast == 2 && s->xt_common))) {
    const int G = fp_half_rows(s->fp_variant);
    const size_t ng = (size_t)((s->ny + G - 1) / G) * G * s->onz * s->onx;
    if ((rc = dalloc(s, &s->d_volh, ng * 2)) || (rc = dalloc(s, &s->d_maxbits, 16))) return fail(rc);
  } else if (!opt->gpu_compat && opt->sirt_iters > 0 && s->fp_fast == 2 && s->xt_common && (s->fp_variant & 2)) {
    const int G = fp_group_rows(s->fp_variant);
    const size_t ng = (size_t)((s->ny + G - 1) / G) * G * s->onz * s->onx;
    if ((rc = dalloc(s, &s->d_volg, ng * 4))) return fail(rc);
    s->volg_elems = ng;
  } else if (!opt->gpu_compat && opt->sirt_iters > 0 && s->fp_fast == 1 && (s->fp_variant & 2)) {
    const int G = fp_group_rows(s->fp_variant);
    const size_t ng = (size_t)((s->ny + G - 1) / G) * G * s->onz * s->onx;
    if ((rc = dalloc(s, &s->d_volg, ng * 4))) return fail(rc);
    s->volg_elems = ng;
  }
  if (s->xt_split) {
    // the row sums may live in the reprojector's FP32 copy: it is rebuilt from the
    // volume before every reprojection and is dead while the back-projection runs
    if (s->volg_elems >= nvol) s->xtb = s->d_volg;
    else if ((rc = dalloc(s, &s->d_xtb, nvol * 4))) return fail(rc);
    else s->xtb = s->d_xtb;
  }
  if (s->has_local && (rc = upload_local(s, g->local, g->local ? g->n_local : 0, vg2))) return fail(rc);
  // corrections per (view, slice, column): 8 bytes each, filled below
  if (s->has_local && (rc = dalloc(s, &s->d_lbnd, (size_t)s->nviews * ((s->ny + LB_TILE - 1) / LB_TILE) *
                                                      s->onx * sizeof(float2))))
    return fail(rc);
  if (s->has_local && (rc = dalloc(s, &s->d_ltab, (size_t)s->nviews * s->ny * s->onx * sizeof(float2))))
    return fail(rc);
  if (dry) {
    if (s->use_conv) s->dev_bytes += (size_t)s->nx * 4;
    *out = s;
    return TG_OK;
  }
  if (pool && (ce = cudaStreamSynchronize(s->st)) != cudaSuccess) return fail(cuda_fail(ce, "sync"));
  // zero the staging buffer once: rows past ny stay zero
  if ((ce = cudaMemsetAsync(s->d_pairs, 0, s->pairs_bytes, s->st)) != cudaSuccess) return fail(cuda_fail(ce, "memset"));
  if ((ce = cudaMemsetAsync(s->d_err, 0, 16, s->st)) != cudaSuccess) return fail(cuda_fail(ce, "memset"));

  std::vector<float> wt(s->nx);
  weight_table(s->nx, opt->radial_cutoff, opt->radial_falloff, opt->exact_filter_size, opt->hamming, wt.data());
  // [0, nx): exp(-2 pi i k/nx); [nx, 2 nx - 1): the register-resident kernel's
  // per-pass table, for the widths that have that kernel
  std::vector<float2> tw(2 * (size_t)s->nx, make_float2(0.0f, 0.0f)), tw2;
  for (int k = 0; k < s->nx; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)s->nx;
    tw[k] = make_float2((float)cos(a), (float)sin(a));
  }
  s->has_tw2 = p2_twiddle_table(s->nx, tw2);
  std::copy(tw2.begin(), tw2.end(), tw.begin() + s->nx);
  if (s->use_conv) {
    // h[m] = (1/n) * sum_k w[k] exp(2 pi i k m / n)  (w real and even)
    std::vector<float> h(s->nx);
    for (int m = 0; m < s->nx; ++m) {
      double acc = 0.0;
      for (int k = 0; k < s->nx; ++k) acc += (double)wt[k] * cos(2.0 * M_PI * (double)k * m / s->nx);
      h[m] = (float)(acc / s->nx);
    }
    if ((rc = dalloc(s, &s->d_conv, (size_t)s->nx * 4))) return fail(rc);
    if ((ce = cudaMemcpyAsync(s->d_conv, h.data(), h.size() * 4, cudaMemcpyHostToDevice, s->st)))
      return fail(cuda_fail(ce, "copy"));
  }
  // on the session's stream (after its stream-ordered allocations); pageable
  // sources have been staged when each call returns; synchronised below
  if ((ce = cudaMemcpyAsync(s->d_weights, wt.data(), wt.size() * 4, cudaMemcpyHostToDevice, s->st)) ||
      (ce = cudaMemcpyAsync(s->d_tw, tw.data(), tw.size() * 8, cudaMemcpyHostToDevice, s->st)) ||
      (ce = cudaMemcpyAsync(s->d_vg, vg.data(), vg.size() * 16, cudaMemcpyHostToDevice, s->st)) ||
      (ce = cudaMemcpyAsync(s->d_vg2, vg2.data(), vg2.size() * 16, cudaMemcpyHostToDevice, s->st)) ||
      (ce = cudaMemcpyAsync(s->d_stretch, stretch.data(), stretch.size() * 4, cudaMemcpyHostToDevice, s->st)))
    return fail(cuda_fail(ce, "cudaMemcpy(setup)"));
  if (!any_stretch) {
    if (pool) cudaFreeAsync(s->d_stretch, s->st);
    else cudaFree(s->d_stretch);
    s->d_stretch = nullptr;
  }
  if (s->has_local) {
    launch_local_table(local_dev(s), s->nviews, s->ny, s->onx, s->d_ltab, s->st);
    launch_local_bounds(s->d_ltab, s->nviews, s->ny, s->onx, s->d_lbnd, s->st);
  }
  if ((ce = cudaStreamSynchronize(s->st)) != cudaSuccess) return fail(cuda_fail(ce, "sync"));
  *out = s;
  return TG_OK;
}

void tg::session_discard(tg_session *s) { free_session(s); }

extern "C" {

int tg_upload_projections(tg_session *s, const float *host, size_t n) {
  if (!s || !host) return TG_ERR_INVALID_ARG;
  if (n != (size_t)s->nx * s->ny * s->nz) { set_error("projection count mismatch"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(s->dev));
  TG_CUDA(cudaMemcpyAsync(s->d_raw, host, n * 4, cudaMemcpyHostToDevice, s->st));
  s->uploaded = true;
  return TG_OK;
}

int tg_set_projections_device(tg_session *s, const float *dev, size_t n) {
  if (!s || !dev) return TG_ERR_INVALID_ARG;
  if (n != (size_t)s->nx * s->ny * s->nz) { set_error("projection count mismatch"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(s->dev));
  TG_CUDA(cudaMemcpyAsync(s->d_raw, dev, n * 4, cudaMemcpyDeviceToDevice, s->st));
  s->uploaded = true;
  return TG_OK;
}

namespace tg {
// n SIRT iterations (main.rs:919-975) on the session's stream: reprojection,
// residual R-weighting, relaxed back-projection update; one CUDA graph per
// iteration, captured on first use, when the session uses graphs
int sirt_iterations(tg_session *s, int n) {
  auto one_iter = [&]() -> int {
    s->iter_launches = launch_reproject(fp_args(s), s->st) + 1 + bp_launch_count(s);
    launch_filter(filter_args(s, true), s->st);
    return launch_bp(s, 2, nullptr);
  };
  if (n <= 0) return TG_OK;
  if (s->o.use_graphs) {
    if (!s->sirt_exec) {
      cudaGraph_t graph;
      TG_CUDA(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeRelaxed));
      int r2 = one_iter();
      cudaError_t ec = cudaStreamEndCapture(s->st, &graph);
      if (r2 != TG_OK) return r2;
      if (ec != cudaSuccess) return cuda_fail(ec, "cudaStreamEndCapture");
      ec = cudaGraphInstantiate(&s->sirt_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ec != cudaSuccess) return cuda_fail(ec, "cudaGraphInstantiate");
    }
    for (int it = 0; it < n; ++it) TG_CUDA(cudaGraphLaunch(s->sirt_exec, s->st));
  } else {
    for (int it = 0; it < n; ++it) {
      const int rc = one_iter();
      if (rc != TG_OK) return rc;
    }
  }
  return TG_OK;
}
}  // namespace tg

int tg_reconstruct(tg_session *s) {
  if (!s) return TG_ERR_INVALID_ARG;
  if (!s->uploaded) { set_error("no projections uploaded"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(s->dev));
  (void)cudaGetLastError();  // a stale error of an earlier, unrelated call must not fail this run
  int rc, launches = 0, ntiles = 0;
  if (s->variant < 0 && (rc = autotune(s)) != TG_OK) return rc;
  const int iters = sirt_iters(s);
  s->timed = false;
  s->sirt_done = -1;  // closes a SIRT run in steps
  TG_CUDA(cudaEventRecord(s->ev[0], s->st));
  {
    NvtxRange r("tg.filter");
    if ((rc = stage_front(s, &launches)) != TG_OK) return rc;
  }
  TG_CUDA(cudaEventRecord(s->ev[1], s->st));
  const int mode0 = first_mode(s);
  {
    NvtxRange r("tg.backproject");
    if ((rc = launch_bp(s, mode0, &ntiles)) != TG_OK) return rc;
  }
  launches += bp_launch_count(s);
  TG_CUDA(cudaGetLastError());
  TG_CUDA(cudaEventRecord(s->ev[2], s->st));
  if (iters > 0) {
    NvtxRange r("tg.sirt");
    if ((rc = sirt_iterations(s, iters)) != TG_OK) return rc;
    launches += s->iter_launches * iters;  // counted when the iteration was issued or captured
  }
  TG_CUDA(cudaEventRecord(s->ev[3], s->st));
  {
    NvtxRange r("tg.finish");
    if ((rc = stage_finish(s, mode0, ntiles, &launches)) != TG_OK) return rc;
  }
  TG_CUDA(cudaEventRecord(s->ev[4], s->st));
  s->info = tg_run_info{};
  s->info.passes = 1 + iters;
  s->info.updates = (double)s->onx * s->onz * s->ny * s->nviews * (1.0 + 2.0 * iters);
  s->info.kernel_launches = launches;
  s->timed = true;
  return TG_OK;
}

int tg_sirt_begin(tg_session *s) {
  if (!s) return TG_ERR_INVALID_ARG;
  if (!s->uploaded) { set_error("no projections uploaded"); return TG_ERR_INVALID_ARG; }
  if (sirt_iters(s) <= 0) { set_error("the session runs no SIRT iterations"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(s->dev));
  (void)cudaGetLastError();
  int rc, launches = 0;
  if (s->variant < 0 && (rc = autotune(s)) != TG_OK) return rc;
  s->timed = false;
  s->sirt_done = -1;
  if ((rc = stage_front(s, &launches)) != TG_OK) return rc;
  if ((rc = launch_bp(s, first_mode(s), nullptr)) != TG_OK) return rc;  // mode 1: raw sums, no statistics
  TG_CUDA(cudaGetLastError());
  s->sirt_done = 0;
  return TG_OK;
}

int tg_sirt_iterate(tg_session *s, int32_t n) {
  if (!s || n < 0) return TG_ERR_INVALID_ARG;
  if (s->sirt_done < 0) { set_error("no SIRT run open (tg_sirt_begin or tg_sirt_restore first)"); return TG_ERR_INVALID_ARG; }
  if (s->sirt_done + n > sirt_iters(s)) {
    set_error("more SIRT iterations than the session's sirt_iters");
    return TG_ERR_INVALID_ARG;
  }
  TG_CUDA(cudaSetDevice(s->dev));
  const int rc = sirt_iterations(s, n);
  if (rc != TG_OK) return rc;
  s->sirt_done += n;
  return TG_OK;
}

int tg_sirt_end(tg_session *s) {
  if (!s) return TG_ERR_INVALID_ARG;
  if (s->sirt_done < 0) { set_error("no SIRT run open"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(s->dev));
  int launches = 0;
  const int rc = stage_finish(s, first_mode(s), 0, &launches);
  if (rc != TG_OK) return rc;
  s->sirt_done = -1;
  return TG_OK;
}

int tg_sirt_save(tg_session *s, float *host_volume, int32_t *iterations_done) {
  if (!s || !host_volume) return TG_ERR_INVALID_ARG;
  if (s->sirt_done < 0) { set_error("no SIRT run open"); return TG_ERR_INVALID_ARG; }
  const int rc = tg_synchronize(s);
  if (rc != TG_OK) return rc;
  TG_CUDA(cudaMemcpy(host_volume, s->d_vol, (size_t)s->onx * s->onz * s->ny * 4, cudaMemcpyDeviceToHost));
  if (iterations_done) *iterations_done = s->sirt_done;
  return TG_OK;
}

int tg_sirt_restore(tg_session *s, const float *host_volume, int32_t iterations_done) {
  if (!s || !host_volume || iterations_done < 0) return TG_ERR_INVALID_ARG;
  if (!s->uploaded) { set_error("no projections uploaded"); return TG_ERR_INVALID_ARG; }
  if (sirt_iters(s) <= 0 || iterations_done > sirt_iters(s)) {
    set_error("iteration count outside the session's SIRT run");
    return TG_ERR_INVALID_ARG;
  }
  TG_CUDA(cudaSetDevice(s->dev));
  (void)cudaGetLastError();
  int rc;
  if (s->variant < 0 && (rc = autotune(s)) != TG_OK) return rc;
  s->timed = false;
  // the log and the per-view means the iterations read (main.rs:608-623)
  launch_log_means(s->d_raw, s->d_logd, s->nx * s->ny, s->nz, s->d_mpart, s->means_pinned ? nullptr : s->d_means,
                   s->st);
  TG_CUDA(cudaMemcpyAsync(s->d_vol, host_volume, (size_t)s->onx * s->onz * s->ny * 4, cudaMemcpyHostToDevice,
                          s->st));
  TG_CUDA(cudaStreamSynchronize(s->st));  // the pageable source may be reused on return
  s->sirt_done = iterations_done;
  return TG_OK;
}

int tg_synchronize(tg_session *s) {
  if (!s) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(s->dev));
  TG_CUDA(cudaStreamSynchronize(s->st));
  int err[4] = {0, 0, 0, 0};
  TG_CUDA(cudaMemcpy(err, s->d_err, 16, cudaMemcpyDeviceToHost));
  if (err[0]) {
    cudaMemsetAsync(s->d_err, 0, 16, s->st);
    return device_error_status(err[0]);
  }
  if (s->timed) {  // stage times of the last tg_reconstruct (not recorded for batched runs)
    float t[4] = {0, 0, 0, 0};
    TG_CUDA(cudaEventElapsedTime(&t[0], s->ev[0], s->ev[4]));
    TG_CUDA(cudaEventElapsedTime(&t[1], s->ev[0], s->ev[1]));
    TG_CUDA(cudaEventElapsedTime(&t[2], s->ev[1], s->ev[2]));
    TG_CUDA(cudaEventElapsedTime(&t[3], s->ev[2], s->ev[3]));
    s->info.ms_total = t[0];
    s->info.ms_filter = t[1];
    s->info.ms_backproject = t[2];
    s->info.ms_reproject = t[3];
  }
  return TG_OK;
}

int tg_download_slices(tg_session *s, int32_t y0, int32_t y1, float *host_out, tg_stats *stats) {
  if (!s || y0 < 0 || y1 > s->ny || y0 > y1 || (!host_out && y1 > y0)) return TG_ERR_INVALID_ARG;
  int rc = tg_synchronize(s);
  if (rc != TG_OK) return rc;
  size_t sl = (size_t)s->onx * s->onz;
  if (y1 > y0)
    TG_CUDA(cudaMemcpyAsync(host_out, s->d_vol + (size_t)y0 * sl, (size_t)(y1 - y0) * sl * 4,
                            cudaMemcpyDeviceToHost, s->st));
  TG_CUDA(cudaStreamSynchronize(s->st));
  if (stats) return tg_get_stats(s, stats);
  return TG_OK;
}

int tg_download_slices_async(tg_session *s, int32_t y0, int32_t y1, float *host_out) {
  if (!s || y0 < 0 || y1 > s->ny || y0 > y1 || (!host_out && y1 > y0)) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(s->dev));
  const size_t sl = (size_t)s->onx * s->onz;
  if (y1 > y0)
    TG_CUDA(cudaMemcpyAsync(host_out, s->d_vol + (size_t)y0 * sl, (size_t)(y1 - y0) * sl * 4,
                            cudaMemcpyDeviceToHost, s->st));
  return TG_OK;
}

int tg_upload_sections(tg_session *s, int32_t z0, int32_t z1, const float *host) {
  if (!s || z0 < 0 || z1 > s->nz || z0 > z1 || (!host && z1 > z0)) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(s->dev));
  const size_t sec = (size_t)s->nx * s->ny;
  if (z1 > z0)
    TG_CUDA(cudaMemcpyAsync(s->d_raw + (size_t)z0 * sec, host, (size_t)(z1 - z0) * sec * 4,
                            cudaMemcpyHostToDevice, s->st));
  s->uploaded = true;
  return TG_OK;
}

int tg_download_slices_f16_async(tg_session *s, int32_t y0, int32_t y1, uint16_t *host_out) {
  if (!s || y0 < 0 || y1 > s->ny || y0 > y1 || (!host_out && y1 > y0)) return TG_ERR_INVALID_ARG;
  if (y1 == y0) return TG_OK;
  TG_CUDA(cudaSetDevice(s->dev));
  const size_t sl = (size_t)s->onx * s->onz, n = (size_t)(y1 - y0) * sl;
  if (n * 2 > s->half_cap) {  // grows once for a caller's fixed chunk size
    TG_CUDA(cudaStreamSynchronize(s->st));
    if (s->d_half) cudaFree(s->d_half);
    s->d_half = nullptr;
    s->half_cap = 0;
    cudaError_t e = cudaMalloc(&s->d_half, n * 2);
    if (e != cudaSuccess) { s->d_half = nullptr; return cuda_fail(e, "cudaMalloc(half staging)"); }
    s->half_cap = n * 2;
  }
  launch_to_half(s->d_vol + (size_t)y0 * sl, s->d_half, n, s->st);
  TG_CUDA(cudaGetLastError());
  TG_CUDA(cudaMemcpyAsync(host_out, s->d_half, n * 2, cudaMemcpyDeviceToHost, s->st));
  return TG_OK;
}

int tg_host_alloc(size_t bytes, void **out) {
  if (!out) return TG_ERR_INVALID_ARG;
  *out = nullptr;
  if (bytes == 0) return TG_OK;
  TG_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocPortable));
  return TG_OK;
}

int tg_host_free(void *p) {
  if (p) TG_CUDA(cudaFreeHost(p));
  return TG_OK;
}

int tg_get_stats(tg_session *s, tg_stats *stats) {
  if (!s || !stats) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(s->dev));
  float t[3];
  TG_CUDA(cudaMemcpyAsync(t, s->d_stats3, 12, cudaMemcpyDeviceToHost, s->st));
  TG_CUDA(cudaStreamSynchronize(s->st));
  stats->amin = t[0];
  stats->amax = t[1];
  stats->amean = t[2];
  return TG_OK;
}

const float *tg_volume_device(tg_session *s) { return s ? s->d_vol : nullptr; }

int tg_session_last_run(tg_session *s, tg_run_info *info) {
  if (!s || !info) return TG_ERR_INVALID_ARG;
  *info = s->info;
  return TG_OK;
}

int tg_session_dims(tg_session *s, int32_t *onx, int32_t *onz, int32_t *ony) {
  if (!s) return TG_ERR_INVALID_ARG;
  if (onx) *onx = s->onx;
  if (onz) *onz = s->onz;
  if (ony) *ony = s->ny;
  return TG_OK;
}

size_t tg_session_device_bytes(tg_session *s) { return s ? s->dev_bytes : 0; }

int tg_session_set_stream(tg_session *s, void *stream) {
  if (!s) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(s->dev));
  TG_CUDA(cudaStreamSynchronize(s->st));
  // a captured SIRT graph stays valid: graphs are launched on whichever stream is current
  s->st = stream ? (cudaStream_t)stream : s->own_st;
  return TG_OK;
}

int tg_session_destroy(tg_session *s) {
  if (!s) return TG_ERR_INVALID_ARG;
  cudaSetDevice(s->dev);
  free_session(s);
  return TG_OK;
}

// ---- tg_session internals exposed to the other translation units ----
int tg_session_kernel_info(tg_session *s, int32_t *fast, int32_t *variant, int32_t *fmt,
                           int32_t *padL, int32_t *PW) {
  if (!s) return TG_ERR_INVALID_ARG;
  // 2: staged x-tilt kernel, 3: fast kernel's row sums + blend, 0: general kernel
  if (fast) *fast = s->fast ? 1 : s->xt_split ? 3 : s->xt_fast ? 2 : 0;
  if (variant) *variant = s->variant;
  if (fmt) *fmt = s->fmt;
  if (padL) *padL = s->padL;
  if (PW) *PW = s->PW;
  return TG_OK;
}

int tg_session_view_sums(tg_session *s, double *sums) {
  if (!s || !sums) return TG_ERR_INVALID_ARG;
  if (!s->uploaded) { set_error("no projections uploaded"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(s->dev));
  double *d = nullptr;
  TG_CUDA(cudaMallocAsync((void **)&d, (size_t)s->nz * sizeof(double), s->st));
  launch_log_means(s->d_raw, s->d_logd, s->nx * s->ny, s->nz, s->d_mpart, nullptr, s->st);
  launch_view_sums(s->d_mpart, s->nz, d, s->st);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(sums, d, (size_t)s->nz * sizeof(double), cudaMemcpyDeviceToHost, s->st);
  cudaFreeAsync(d, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  return e == cudaSuccess ? TG_OK : cuda_fail(e, "tg_session_view_sums");
}

int tg_session_set_view_means(tg_session *s, const float *means) {
  if (!s) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(s->dev));
  if (!means) {
    s->means_pinned = false;
    return TG_OK;
  }
  TG_CUDA(cudaMemcpyAsync(s->d_means, means, (size_t)s->nz * sizeof(float), cudaMemcpyHostToDevice, s->st));
  TG_CUDA(cudaStreamSynchronize(s->st));
  s->means_pinned = true;
  return TG_OK;
}

int tg_session_inject_wait_fault(tg_session *s, int32_t skip_stage, uint32_t wait_limit_us) {
  if (!s) return TG_ERR_INVALID_ARG;
  if (!s->fast && !s->xt_split) {
    set_error("the session does not use the pipelined back-projector");
    return TG_ERR_UNSUPPORTED;
  }
  TG_CUDA(cudaSetDevice(s->dev));
  TG_CUDA(cudaStreamSynchronize(s->st));
  s->fault_skip_stage = skip_stage < 0 ? -1 : skip_stage;
  s->wait_limit_ns = wait_limit_us ? (unsigned long long)wait_limit_us * 1000ull : 2000000000ull;
  if (s->sirt_exec) {  // captured iterations hold the old arguments: capture again
    cudaGraphExecDestroy(s->sirt_exec);
    s->sirt_exec = nullptr;
  }
  return TG_OK;
}

int tg_session_set_variant(tg_session *s, int32_t variant) {
  if (!s || variant < -1 || variant >= bp_fast_variants()) return TG_ERR_INVALID_ARG;
  s->variant = variant;
  return TG_OK;
}

const char *tg_variant_name(int32_t v) {
  return (v >= 0 && v < bp_fast_variants()) ? bp_fast_variant_name(v) : "general";
}

// ---- the reference's GPU seam (apps/tilt/src/gpu.rs) ----
}  // extern "C"

struct tg_gpu_session {
  tg_session *s = nullptr;
  bool done = false;
  size_t out_nx = 0, out_nz = 0, in_ny = 0;
};

extern "C" {

int tg_gpu_session_new(const float *proj, const float *cs, size_t in_nx, size_t in_ny, size_t n_projs,
                       size_t out_nx, size_t out_nz, int32_t device, tg_gpu_session **out) {
  if (!proj || !cs || !out || n_projs == 0 || in_nx < 2 || in_ny == 0 || out_nx == 0 || out_nz == 0)
    return TG_ERR_INVALID_ARG;
  *out = nullptr;
  // the caller passes (cos, sin) pairs; recover angles is not needed: build a
  // session in --gpu semantics and overwrite its per-view geometry.
  std::vector<float> ang(n_projs, 0.0f);
  tg_geometry g{};
  g.nx = (int)in_nx;
  g.ny = (int)in_ny;
  g.nz = (int)n_projs;
  g.out_nx = (int)out_nx;
  g.out_nz = (int)out_nz;
  g.n_angles = (int)n_projs;
  g.angles = ang.data();
  tg_options o;
  tg_options_default(&o);
  o.no_weight = 1;          // the projections arrive filtered and stretched
  o.no_cosine_stretch = 1;
  o.gpu_compat = 1;
  o.device = device;
  tg_session *s = nullptr;
  int rc = tg_session_create(&g, &o, &s);
  if (rc != TG_OK) return rc;
  std::vector<float4> vg(n_projs);
  for (size_t i = 0; i < n_projs; ++i) vg[i] = make_float4(cs[2 * i], cs[2 * i + 1], 1.0f, 1.0f);
  // the padding was planned for angle 0; re-plan it for the given (cos, sin)
  {
    int kmin = 0, kmax = s->nx - 1;
    float dxs[2] = {0.0f - s->ocx, (float)(s->onx - 1) - s->ocx};
    float dzs[2] = {0.0f - s->cz, (float)(s->onz - 1) - s->cz};
    for (size_t i = 0; i < n_projs; ++i)
      for (float dx : dxs)
        for (float dz : dzs) {
          HostView h{cs[2 * i], cs[2 * i + 1], 1.0f, 0.0f, 1.0f};
          float x = ref_x_host(dx, dz, h, s->cx);
          kmin = std::min(kmin, (int)floorf(x));
          kmax = std::max(kmax, (int)floorf(x));
        }
    int needL = std::max(0, -kmin), needR = std::max(0, kmax - (s->nx - 1));
    int padL = ((needL + 3) + 1) & ~1;
    int PW = (padL + s->nx + needR + 6 + 1) & ~1;
    if (PW != s->PW || padL != s->padL) {
      cudaFree(s->d_pairs);
      s->padL = padL;
      s->PW = PW;
      s->pairs_bytes = (size_t)s->nviews * s->rows_alloc * s->PW * elem_bytes(s->fmt, s->store);
      cudaError_t e = cudaMalloc(&s->d_pairs, s->pairs_bytes);
      if (e != cudaSuccess) { s->d_pairs = nullptr; tg_session_destroy(s); return cuda_fail(e, "cudaMalloc"); }
      cudaMemset(s->d_pairs, 0, s->pairs_bytes);
    }
  }
  cudaError_t e = cudaMemcpy(s->d_vg, vg.data(), vg.size() * 16, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { tg_session_destroy(s); return cuda_fail(e, "cudaMemcpy"); }
  rc = tg_upload_projections(s, proj, in_nx * in_ny * n_projs);
  if (rc != TG_OK) { tg_session_destroy(s); return rc; }
  tg_gpu_session *gs = new tg_gpu_session();
  gs->s = s;
  gs->out_nx = out_nx;
  gs->out_nz = out_nz;
  gs->in_ny = in_ny;
  *out = gs;
  return TG_OK;
}

int tg_gpu_session_reconstruct_row(tg_gpu_session *gs, size_t iy, float *out) {
  if (!gs || !out || iy >= gs->in_ny) return TG_ERR_INVALID_ARG;
  tg_session *s = gs->s;
  if (!gs->done) {
    // all rows in one launch on the first call; later calls read the resident volume
    s->o.densweight = 1.0f;
    s->o.outscale = 1.0f;
    s->o.outadd = 0.0f;
    int rc = tg_reconstruct(s);
    if (rc != TG_OK) return rc;
    gs->done = true;
  }
  return tg_download_slices(s, (int)iy, (int)iy + 1, out, nullptr);
}

void tg_gpu_session_free(tg_gpu_session *gs) {
  if (!gs) return;
  tg_session_destroy(gs->s);
  delete gs;
}

int tg_apply_rweighting(float *proj, size_t in_nx, size_t in_ny, size_t nz, float cutoff, float falloff,
                        int32_t efs, int32_t hamming, int32_t device) {
  if (!proj || in_nx < 2 || in_ny == 0 || nz == 0) return TG_ERR_INVALID_ARG;
  std::vector<float> ang(nz, 0.0f);
  tg_geometry g{};
  g.nx = (int)in_nx;
  g.ny = (int)in_ny;
  g.nz = (int)nz;
  g.out_nx = 2;
  g.out_nz = 2;
  g.n_angles = (int)nz;
  g.angles = ang.data();
  tg_options o;
  tg_options_default(&o);
  o.radial_cutoff = cutoff;
  o.radial_falloff = falloff;
  o.exact_filter_size = efs;
  o.hamming = hamming;
  o.no_cosine_stretch = 1;
  o.device = device;
  o.fill_mode = TG_FILL_ZERO;
  tg_session *s = nullptr;
  int rc = tg_session_create(&g, &o, &s);
  if (rc != TG_OK) return rc;
  // SINGLE FP32 staging with no padding holds (row[k], row[k+1]) pairs;
  // element k's first value is the filtered sample.
  cudaFree(s->d_pairs);
  s->fmt = FMT_SINGLE;
  s->padL = 0;
  s->PW = (int)in_nx;
  s->rows_alloc = (int)in_ny;
  s->pairs_bytes = (size_t)nz * in_ny * in_nx * 8;
  cudaError_t e = cudaMalloc(&s->d_pairs, s->pairs_bytes);
  if (e != cudaSuccess) { s->d_pairs = nullptr; tg_session_destroy(s); return cuda_fail(e, "cudaMalloc"); }
  rc = tg_upload_projections(s, proj, in_nx * in_ny * nz);
  if (rc == TG_OK) {
    launch_filter(filter_args(s, false), s->st);
    std::vector<float2> tmp((size_t)nz * in_ny * in_nx);
    e = cudaMemcpyAsync(tmp.data(), s->d_pairs, s->pairs_bytes, cudaMemcpyDeviceToHost, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    if (e != cudaSuccess) rc = cuda_fail(e, "filter");
    else
      for (size_t r = 0; r < nz * in_ny; ++r)  // element k holds (row[k], row[k+1])
        for (size_t k = 0; k < in_nx; ++k)
          proj[r * in_nx + k] = k + 1 < in_nx ? tmp[r * in_nx + k].x : tmp[r * in_nx + in_nx - 2].y;
  }
  tg_session_destroy(s);
  return rc;
}

int tg_synth_projections(const tg_phantom_spec *spec, const float *angles, float *out, int32_t is_device,
                         int32_t device) {
  if (!spec || !angles || !out) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(device));
  cudaStream_t st;
  TG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  size_t n = (size_t)spec->nx * spec->ny * spec->nz;
  float *d = out;
  if (!is_device) {
    cudaError_t e = cudaMalloc(&d, n * 4);
    if (e != cudaSuccess) { cudaStreamDestroy(st); return cuda_fail(e, "cudaMalloc"); }
  }
  int rc = synth_projections(spec, angles, d, st);
  if (rc == TG_OK && !is_device) {
    cudaError_t e = cudaMemcpy(out, d, n * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemcpy");
  }
  if (!is_device) cudaFree(d);
  cudaStreamDestroy(st);
  return rc;
}

}  // extern "C"
