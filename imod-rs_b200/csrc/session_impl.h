// session_impl.h -- the session object and the stage helpers shared by the
// per-series C ABI (session.cu) and the batched launch (batch.cu).
#pragma once
#include <cstring>
#include <tuple>
#include <vector>

#include "tg_internal.h"

using tg::StatPartial;
using tg::FftPlanDev;
using tg::FMT_ROWPAIR;

struct tg_session {  // one tilt series resident on a device
  int nx = 0, ny = 0, nz = 0, onx = 0, onz = 0, nviews = 0;
  tg_options o{};
  bool has_local = false, fast = true, zf_any = false;
  bool xt_fast = false;  // not fast: x-tilt back-projection with staged rows instead of the general kernel
  // x-tilt shared by all views: the fast kernel sums every projection row over the
  // views into xtb, then launch_xt_blend blends two rows per voxel into the volume
  bool xt_split = false;
  float *xtb = nullptr;    // row sums (d_xtb, or the reprojector's FP32 copy, which is dead then)
  float *d_xtb = nullptr;
  int fp_fast = 0;  // reprojector: 0 general, 1 fast (no x-tilt), 2 fast with x-tilt
  bool xt_common = false;  // every view has the same x-tilt (blended copy for the reprojector)
  float sin_xt_common = 0.0f;
  // reprojector variant bits (FpArgs::variant; TG_FP_VARIANT overrides): 16 rows per thread and
  // the interleaved copy (FP32 SIRT at 1024 wide, 61 views, x-tilt 1.5: 0.487 s vs 0.545 s with 8 rows)
  int fp_variant = 3;
  float *d_volg = nullptr;  // interleaved copy of the volume for the reprojector
  size_t volg_elems = 0;
  void *d_volh = nullptr;   // FP16 interleaved copy (half staging forms)
  unsigned *d_maxbits = nullptr;
  int fmt = FMT_ROWPAIR, store = TG_STORE_FP32;
  int padL = 0, PW = 0, rows_alloc = 0, variant = -1, ntiles_cap = 0;
  int dev = 0;
  cudaStream_t st = nullptr, own_st = nullptr;
  // d_raw: the projections as uploaded (never modified); d_logd: their log10 (--log),
  // rewritten by every reconstruction so each run repeats the reference's whole path
  float *d_raw = nullptr, *d_logd = nullptr, *d_means = nullptr, *d_vol = nullptr, *d_sino = nullptr, *d_tmp = nullptr;
  double *d_mpart = nullptr;
  void *d_pairs = nullptr;
  size_t pairs_bytes = 0;
  void *d_half = nullptr;   // mode-12 download staging (tg_download_slices_f16_async), grown on demand
  size_t half_cap = 0;
  StatPartial *d_part = nullptr;
  float *d_slice_stats = nullptr, *d_stats3 = nullptr;
  float4 *d_vg = nullptr, *d_vg2 = nullptr;
  float *d_weights = nullptr, *d_conv = nullptr, *d_stretch = nullptr;
  float2 *d_tw = nullptr;  // 2 nx: plain twiddles, then the register-resident filter's per-pass table
  bool has_tw2 = false;
  int *d_err = nullptr;
  int4 *d_lvinfo = nullptr;
  int *d_lgoff = nullptr;
  float *d_lxs = nullptr, *d_lys = nullptr, *d_lgdx = nullptr, *d_lgdy = nullptr;
  float2 *d_ltab = nullptr;  // local corrections per (view, slice, column)
  float2 *d_lbnd = nullptr;  // their dx range per (view, slice tile, column): FpArgs::lbnd
  FftPlanDev plan{};
  bool use_conv = false;
  bool uploaded = false;
  bool timed = false;  // ev[] were recorded by the last tg_reconstruct
  size_t dev_bytes = 0;
  tg_run_info info{};
  cudaEvent_t ev[6] = {};
  cudaGraphExec_t sirt_exec = nullptr;
  // view means given by the caller (tg_session_set_view_means): a Y slab of a series
  // sharded over GPUs fills with the whole series' means
  bool means_pinned = false;
  // bounded-wait settings of the fast back-projector (tg_session_inject_wait_fault)
  unsigned long long wait_limit_ns = 2000000000ull;
  int fault_skip_stage = -1;
  int iter_launches = 0;  // kernels of one SIRT iteration
  int sirt_done = -1;     // SIRT in steps: iterations done since tg_sirt_begin/restore (-1: none open)
  float cx = 0, cz = 0, ocx = 0, inv_n = 0;
  cudaMemPool_t pool = nullptr;  // stream-ordered allocations (server sessions)
  bool dry = false, fail_alloc = false;
};

namespace tg {

int session_create_ex(const tg_geometry *g, const tg_options *opt, cudaMemPool_t pool, bool dry,
                      bool fail_alloc, tg_session **out);
void session_discard(tg_session *s);
// frees the session's device memory stream-ordered after the work queued on `after`
void free_session_async(tg_session *s, cudaStream_t after);
LocalDev local_dev(tg_session *s);
BpArgs bp_args(tg_session *s, int mode);
FilterArgs filter_args(tg_session *s, bool residual);
FpArgs fp_args(tg_session *s);
int launch_bp(tg_session *s, int mode, int *ntiles);
inline int bp_launch_count(const tg_session *s) { return s->xt_split ? 2 : 1; }
// position form of the fast kernel: 2 with x-tilt (row sums), else whether z-factors apply
inline int fast_zf(const tg_session *s) { return s->xt_split ? 2 : s->zf_any ? 1 : 0; }
int autotune(tg_session *s);
// the tile variant already tuned for this shape (or pinned by TG_BP_VARIANT), else -1
int tune_lookup(tg_session *s);
// log10 + per-view means, then the filter stage of the WBP pass
int stage_front(tg_session *s, int *launches);
// fake-SIRT passes, output transform (when the volume was stored raw) and statistics;
// bp_ntiles: partial-stat tiles written by the back-projection in mode 0
int stage_finish(tg_session *s, int mode0, int bp_ntiles, int *launches);
inline int sirt_iters(const tg_session *s) { return s->o.gpu_compat ? 0 : s->o.sirt_iters; }
inline int fake_passes(const tg_session *s) { return s->o.gpu_compat ? 0 : s->o.fake_sirt; }
inline int first_mode(const tg_session *s) { return (sirt_iters(s) > 0 || fake_passes(s) > 0) ? 1 : 0; }

// One persistent back-projection launch per (storage, z-factor) group of
// fast-path series, on b->st; other series get their own launch.  ntiles[i]
// receives the partial-stat tile count written for ss[i] (used when
// modes[i] == 0).  Job and tile tables are copied stream-ordered, so calls may
// follow each other on the same stream without waiting.
int batch_bp(tg_batch *b, const std::vector<tg_session *> &ss, const std::vector<int> &modes,
             std::vector<int> &ntiles, int *launches);

}  // namespace tg

namespace tg {
// One SIRT round over many series: grouped launches from tables in one device
// buffer (round.cu).  key identifies the member list and settings the tables
// were built for; exec holds the round captured as a graph, once replayed.
struct RoundPlan {
  std::vector<uint64_t> key;
  std::vector<unsigned char> host;
  unsigned char *dev = nullptr;
  size_t cap = 0;
  struct Fp { int key, njobs, nabs, ncopy, nfp; size_t jobs, abs, copy, fpb; };
  struct Fi { int n, fmt, store, njobs, nblk; size_t jobs, blk; };
  struct Bp { int store, zf, variant, njobs, ntiles, max_views; size_t jobs, counter; };
  std::vector<Fp> fp;
  std::vector<Fi> fi;
  std::vector<Bp> bp;
  std::vector<tg_session *> fp_single, fi_single, bp_single;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;  // kernels of one issue
};
int round_plan_build(RoundPlan &p, const std::vector<tg_session *> &ss, const std::vector<uint64_t> &key,
                     cudaStream_t st);
int round_plan_issue(RoundPlan &p, cudaStream_t st);
int round_plan_launch_graph(RoundPlan &p, cudaStream_t st);
void round_plan_release(RoundPlan &p, cudaStream_t st);
void round_plan_signature(const std::vector<tg_session *> &ss, std::vector<uint64_t> &key);
}  // namespace tg

struct tg_batch {
  int dev = 0;
  cudaStream_t st = nullptr;
  std::vector<tg_session *> sess;
  tg::BpArgs *d_jobs = nullptr;
  size_t jobs_cap = 0;
  int *d_counter = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  tg_run_info info{};
  int rounds = 0, persistent_launches = 0;
  uint64_t generation = 1;  // changes with the member list (plan keys)
  tg::RoundPlan plan;       // the SIRT rounds' plan and graph
  int graph_launches = 0;   // rounds of the last reconstruction replayed from a graph
};
