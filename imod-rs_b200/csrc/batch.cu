// batch.cu -- many tilt series reconstructed together.
//
// Each series keeps its own session (buffers, filter stage, SIRT reprojection).
// The back-projection passes of all series that take the fast kernel and
// share a staging precision run as ONE persistent launch per round: round 0
// is every series' WBP pass, round r the r-th SIRT update of the series that
// still iterate.  The tile queue is ordered longest series first so the last
// tiles to finish are short ones.  A tile's arithmetic does not depend on the
// batch, so each series' volume is bit-identical to its stand-alone result.
#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "session_impl.h"

using namespace tg;

namespace tg {

// One persistent launch per (storage, z-factor, tile variant) group of fast-path
// series, each series keeping the tile shape tuned for it; other series get
// their own launch.  ntiles[i] receives the partial-stat
// tile count written for ss[i] (used when modes[i] == 0).
int batch_bp(tg_batch *b, const std::vector<tg_session *> &ss, const std::vector<int> &modes,
             std::vector<int> &ntiles, int *launches) {
  ntiles.assign(ss.size(), 0);
  std::map<std::tuple<int, int, int>, std::vector<int>> groups;
  for (size_t i = 0; i < ss.size(); ++i) {
    if (ss[i]->fast)
      groups[std::make_tuple(ss[i]->store, ss[i]->zf_any ? 1 : 0, std::max(0, ss[i]->variant))].push_back((int)i);
    else {
      int rc = launch_bp(ss[i], modes[i], &ntiles[i]);
      if (rc != TG_OK) return rc;
      *launches += bp_launch_count(ss[i]);
    }
  }
  for (auto &kv : groups) {
    std::vector<int> &idx = kv.second;
    // longest series (most views) first in the tile queue
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return ss[x]->nviews > ss[y]->nviews; });
    const int variant = std::get<2>(kv.first);
    int S, TX, TZ;
    bp_fast_tile_shape(variant, &S, &TX, &TZ);
    std::vector<BpArgs> jobs;
    long long total = 0;
    int max_views = 1;
    for (int i : idx) {
      BpArgs a = bp_args(ss[i], modes[i]);
      a.nbx = (a.onx + TX - 1) / TX;
      const int nbz = (a.onz + TZ - 1) / TZ, nby = (a.ny + S - 1) / S;
      a.ntiles_xz = a.nbx * nbz;
      a.tile0 = (int)total;
      total += (long long)a.ntiles_xz * nby;
      ntiles[i] = a.ntiles_xz;
      jobs.push_back(a);
      max_views = std::max(max_views, a.nviews);
    }
    if (total >= (1ll << 31) - (1ll << 20)) { set_error("too many tiles in one batch"); return TG_ERR_UNSUPPORTED; }
    if (jobs.size() > b->jobs_cap) {
      cudaFree(b->d_jobs);  // synchronises: earlier launches may still read the table
      b->jobs_cap = std::max<size_t>(std::max<size_t>(jobs.size(), 64), 2 * b->jobs_cap);
      TG_CUDA(cudaMalloc(&b->d_jobs, b->jobs_cap * sizeof(BpArgs)));
    }
    // stream-ordered after the previous launch that read the table; the pageable
    // source has been staged when the call returns
    TG_CUDA(cudaMemcpyAsync(b->d_jobs, jobs.data(), jobs.size() * sizeof(BpArgs), cudaMemcpyHostToDevice, b->st));
    BatchLaunch bl{};
    bl.jobs = b->d_jobs;
    bl.njobs = (int)jobs.size();
    bl.ntiles = (int)total;
    bl.counter = b->d_counter;
    bl.max_views = max_views;
    int rc = launch_bp_batch(bl, std::get<0>(kv.first), std::get<1>(kv.first) != 0, variant, b->st);
    if (rc != TG_OK) return rc;
    TG_CUDA(cudaGetLastError());
    ++*launches;
    ++b->persistent_launches;
  }
  return TG_OK;
}

}  // namespace tg

extern "C" {

int tg_batch_create(int32_t device, tg_batch **out) {
  if (!out) return TG_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("no CUDA device"); return TG_ERR_NO_DEVICE; }
  if (device < 0 || device >= ndev) { set_error("bad device ordinal"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(device));
  tg_batch *b = new tg_batch();
  b->dev = device;
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess ||
      (e = cudaMalloc(&b->d_counter, sizeof(int))) != cudaSuccess) {
    int rc = cuda_fail(e, "tg_batch_create");
    if (b->st) cudaStreamDestroy(b->st);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    delete b;
    return rc;
  }
  *out = b;
  return TG_OK;
}

int tg_batch_add(tg_batch *b, tg_session *s) {
  if (!b || !s) return TG_ERR_INVALID_ARG;
  if (s->dev != b->dev) { set_error("session and batch are on different devices"); return TG_ERR_INVALID_ARG; }
  if (std::find(b->sess.begin(), b->sess.end(), s) != b->sess.end()) return TG_OK;
  b->sess.push_back(s);
  ++b->generation;
  return TG_OK;
}

int tg_batch_clear(tg_batch *b) {
  if (!b) return TG_ERR_INVALID_ARG;
  b->sess.clear();
  ++b->generation;
  return TG_OK;
}

int tg_batch_reconstruct(tg_batch *b) {
  if (!b) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(b->dev));
  (void)cudaGetLastError();  // a stale error of an earlier, unrelated call must not fail this run
  for (tg_session *s : b->sess)
    if (!s->uploaded) { set_error("a session in the batch has no projections"); return TG_ERR_INVALID_ARG; }
  int rc, launches = 0;
  // every session's work goes on the batch stream (its own stream is restored at the end)
  std::vector<cudaStream_t> saved;
  for (tg_session *s : b->sess) {
    saved.push_back(s->st);
    TG_CUDA(cudaStreamSynchronize(s->st));
    s->st = b->st;
  }
  auto restore = [&]() {
    for (size_t i = 0; i < b->sess.size(); ++i) b->sess[i]->st = saved[i];
  };
  for (tg_session *s : b->sess)
    if (s->variant < 0 && (rc = autotune(s)) != TG_OK) { restore(); return rc; }
  b->persistent_launches = 0;
  if (cudaEventRecord(b->ev0, b->st) != cudaSuccess) { restore(); return cuda_fail(cudaGetLastError(), "event"); }
  // round 0: filter every series, then one back-projection round
  std::vector<int> modes, nt0, nt;
  for (tg_session *s : b->sess) {
    if ((rc = stage_front(s, &launches)) != TG_OK) { restore(); return rc; }
    modes.push_back(first_mode(s));
  }
  if ((rc = batch_bp(b, b->sess, modes, nt0, &launches)) != TG_OK) { restore(); return rc; }
  int max_it = 0;
  for (tg_session *s : b->sess) max_it = std::max(max_it, sirt_iters(s));
  // round r: the r-th SIRT update of every series that still iterates, as one
  // plan of grouped launches (round.cu); rounds with the same members replay the
  // plan's CUDA graph
  b->graph_launches = 0;
  for (int r = 1; r <= max_it; ++r) {
    NvtxRange nv("tg.batch.sirt_round");
    std::vector<tg_session *> act;
    bool graphs = true;
    for (tg_session *s : b->sess)
      if (sirt_iters(s) >= r) {
        act.push_back(s);
        graphs &= s->o.use_graphs != 0;
      }
    std::vector<uint64_t> key{b->generation, (uint64_t)act.size()};
    for (tg_session *s : act) key.push_back((uint64_t)(uintptr_t)s);
    round_plan_signature(act, key);
    if (key != b->plan.key && (rc = round_plan_build(b->plan, act, key, b->st)) != TG_OK) { restore(); return rc; }
    rc = graphs ? round_plan_launch_graph(b->plan, b->st) : round_plan_issue(b->plan, b->st);
    if (rc != TG_OK) { restore(); return rc; }
    if (graphs) ++b->graph_launches;
    launches += b->plan.launches;
    b->persistent_launches += (int)b->plan.bp.size();
  }
  double updates = 0.0;
  for (size_t i = 0; i < b->sess.size(); ++i) {
    tg_session *s = b->sess[i];
    if ((rc = stage_finish(s, modes[i], nt0[i], &launches)) != TG_OK) { restore(); return rc; }
    const int it = sirt_iters(s);
    s->info = tg_run_info{};
    s->timed = false;
    s->info.passes = 1 + it;
    s->info.updates = (double)s->onx * s->onz * s->ny * s->nviews * (1.0 + 2.0 * it);
    updates += s->info.updates;
  }
  cudaError_t e = cudaEventRecord(b->ev1, b->st);
  restore();
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  // later work of a session on its own stream must wait for the batch
  for (tg_session *s : b->sess)
    if (s->st != b->st) TG_CUDA(cudaStreamWaitEvent(s->st, b->ev1, 0));
  b->info = tg_run_info{};
  b->info.updates = updates;
  b->info.passes = 1 + max_it;
  b->info.kernel_launches = launches;
  b->rounds = 1 + max_it;
  return TG_OK;
}

int tg_batch_synchronize(tg_batch *b) {
  if (!b) return TG_ERR_INVALID_ARG;
  TG_CUDA(cudaSetDevice(b->dev));
  TG_CUDA(cudaStreamSynchronize(b->st));
  for (tg_session *s : b->sess) {
    int err[4] = {0, 0, 0, 0};
    TG_CUDA(cudaMemcpy(err, s->d_err, 16, cudaMemcpyDeviceToHost));
    if (err[0]) {
      cudaMemset(s->d_err, 0, 16);
      return device_error_status(err[0]);
    }
  }
  float ms = 0.f;
  TG_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->info.ms_total = ms;
  return TG_OK;
}

int tg_batch_last_run(tg_batch *b, tg_run_info *info) {
  if (!b || !info) return TG_ERR_INVALID_ARG;
  *info = b->info;
  return TG_OK;
}

// Plan of the last batched reconstruction's SIRT rounds (tests and profiling):
// rounds replayed from a CUDA graph, grouped reprojection and filter launches,
// kernels per round.
int tg_batch_plan_info(tg_batch *b, int32_t *graph_rounds, int32_t *fp_groups, int32_t *filter_groups,
                       int32_t *round_launches) {
  if (!b) return TG_ERR_INVALID_ARG;
  if (graph_rounds) *graph_rounds = b->graph_launches;
  if (fp_groups) *fp_groups = (int32_t)b->plan.fp.size();
  if (filter_groups) *filter_groups = (int32_t)b->plan.fi.size();
  if (round_launches) *round_launches = b->plan.launches;
  return TG_OK;
}

int tg_batch_destroy(tg_batch *b) {
  if (!b) return TG_ERR_INVALID_ARG;
  cudaSetDevice(b->dev);
  round_plan_release(b->plan, b->st);
  cudaStreamSynchronize(b->st);
  cudaFree(b->d_jobs);
  cudaFree(b->d_counter);
  cudaEventDestroy(b->ev0);
  cudaEventDestroy(b->ev1);
  cudaStreamDestroy(b->st);
  delete b;
  return TG_OK;
}

}  // extern "C"
