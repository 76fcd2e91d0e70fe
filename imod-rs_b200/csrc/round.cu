// round.cu -- one SIRT round over many series as a plan of grouped launches,
// replayable as a CUDA graph.
//
// A round takes every member series one SIRT iteration further (the loop body
// of apps/tilt/src/main.rs:919-975): reprojection, residual R-weighting, and
// the relaxed back-projection update.  The plan groups the members:
//   * reprojection: each series' own launches (or, on request, series with the
//     same form share one launch per phase over a block table);
//   * residual filter: series with the same register-resident FFT width,
//     staging format and precision share one launch;
//   * back-projection: one persistent launch per (precision, z-factor, tile
//     variant) group with a longest-first tile queue, as in batch_bp;
// series that fit no group (local alignment, general kernels, other widths)
// get their own launches inside the same plan.  Each group kernel runs the
// per-series body on each block's own series, so every series' result is the
// same as when it runs alone.
//
// All tables live in one device buffer written before the launches, so the
// launches alone can be captured: a plan whose member list and settings come
// round after round unchanged is captured once and replayed with
// cudaGraphLaunch.
#include <stdlib.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "session_impl.h"

namespace tg {

namespace {
size_t append(std::vector<unsigned char> &h, const void *p, size_t bytes) {
  const size_t off = (h.size() + 15) & ~(size_t)15;
  h.resize(off + bytes);
  if (bytes) memcpy(h.data() + off, p, bytes);
  return off;
}
}  // namespace

void round_plan_release(RoundPlan &p, cudaStream_t st) {
  if (p.exec) cudaGraphExecDestroy(p.exec);  // an executing graph is freed when it completes
  p.exec = nullptr;
  if (p.dev) cudaFreeAsync(p.dev, st);
  p.dev = nullptr;
  p.cap = 0;
  p.key.clear();
  p.fp.clear();
  p.fi.clear();
  p.bp.clear();
  p.fp_single.clear();
  p.fi_single.clear();
  p.bp_single.clear();
  p.host.clear();
}

// Builds the plan for `ss` (one SIRT update each) and writes its tables to the
// device on `st` (stream-ordered after earlier users of the buffer).
int round_plan_build(RoundPlan &p, const std::vector<tg_session *> &ss, const std::vector<uint64_t> &key,
                     cudaStream_t st) {
  if (p.exec) {
    cudaGraphExecDestroy(p.exec);
    p.exec = nullptr;
  }
  p.key = key;
  p.host.clear();
  p.fp.clear();
  p.fi.clear();
  p.bp.clear();
  p.fp_single.clear();
  p.fi_single.clear();
  p.bp_single.clear();
  p.launches = 0;
  // reprojection groups
  std::map<int, std::vector<FpArgs>> fpg;
  // Reprojection: every series' own kernels inside the round (its arguments are
  // kernel parameters, used straight from the constant bank), by default.  The
  // grouped form (TG_ROUND_FP_BATCH=1: one launch per phase over a block table,
  // arguments read into registers from shared memory) launches less but measured
  // slower on the 64-series mix (FP16 2.93e12 vs 3.17e12, FP32 1.76e12 vs 2.07e12
  // updates/s): these kernels are issue-bound, and the argument registers cost
  // occupancy.
  const bool fp_grouped = getenv("TG_ROUND_FP_BATCH") != nullptr;
  for (tg_session *s : ss) {
    FpArgs a = fp_args(s);
    const int k = fp_grouped ? fp_batch_key(a) : -1;
    if (k < 0) p.fp_single.push_back(s);
    else fpg[k].push_back(a);
  }
  for (auto &kv : fpg) {
    RoundPlan::Fp g{};
    g.key = kv.first;
    g.njobs = (int)kv.second.size();
    std::vector<int> ba(1, 0), bc(1, 0), bf(1, 0);
    for (const FpArgs &a : kv.second) {
      int na, nc, nf;
      fp_batch_blocks(a, g.key, &na, &nc, &nf);
      ba.push_back(ba.back() + na);
      bc.push_back(bc.back() + nc);
      bf.push_back(bf.back() + nf);
    }
    g.nabs = ba.back();
    g.ncopy = bc.back();
    g.nfp = bf.back();
    g.jobs = append(p.host, kv.second.data(), kv.second.size() * sizeof(FpArgs));
    g.abs = append(p.host, ba.data(), ba.size() * sizeof(int));
    g.copy = append(p.host, bc.data(), bc.size() * sizeof(int));
    g.fpb = append(p.host, bf.data(), bf.size() * sizeof(int));
    p.fp.push_back(g);
  }
  // residual filter groups
  std::map<std::tuple<int, int, int>, std::vector<FilterArgs>> fig;
  for (tg_session *s : ss) {
    FilterArgs f = filter_args(s, true);
    const int n = filter_batch_width(f);
    if (n == 0) p.fi_single.push_back(s);
    else fig[std::make_tuple(n, f.fmt, f.store)].push_back(f);
  }
  for (auto &kv : fig) {
    RoundPlan::Fi g{};
    g.n = std::get<0>(kv.first);
    g.fmt = std::get<1>(kv.first);
    g.store = std::get<2>(kv.first);
    g.njobs = (int)kv.second.size();
    std::vector<int> b(1, 0);
    for (const FilterArgs &f : kv.second) b.push_back(b.back() + ((f.ny + 1) / 2) * f.nviews);
    g.nblk = b.back();
    g.jobs = append(p.host, kv.second.data(), kv.second.size() * sizeof(FilterArgs));
    g.blk = append(p.host, b.data(), b.size() * sizeof(int));
    p.fi.push_back(g);
  }
  // back-projection groups (batch_bp's grouping, SIRT update mode)
  std::map<std::tuple<int, int, int>, std::vector<tg_session *>> bpg;
  for (tg_session *s : ss) {
    if (s->fast) bpg[std::make_tuple(s->store, s->zf_any ? 1 : 0, std::max(0, s->variant))].push_back(s);
    else p.bp_single.push_back(s);
  }
  for (auto &kv : bpg) {
    std::vector<tg_session *> &mem = kv.second;
    std::stable_sort(mem.begin(), mem.end(), [](tg_session *x, tg_session *y) { return x->nviews > y->nviews; });
    RoundPlan::Bp g{};
    g.store = std::get<0>(kv.first);
    g.zf = std::get<1>(kv.first);
    g.variant = std::get<2>(kv.first);
    int S, TX, TZ;
    bp_fast_tile_shape(g.variant, &S, &TX, &TZ);
    std::vector<BpArgs> jobs;
    long long total = 0;
    g.max_views = 1;
    for (tg_session *s : mem) {
      BpArgs a = bp_args(s, 2);
      a.nbx = (a.onx + TX - 1) / TX;
      const int nbz = (a.onz + TZ - 1) / TZ, nby = (a.ny + S - 1) / S;
      a.ntiles_xz = a.nbx * nbz;
      a.tile0 = (int)total;
      total += (long long)a.ntiles_xz * nby;
      jobs.push_back(a);
      g.max_views = std::max(g.max_views, a.nviews);
    }
    if (total >= (1ll << 31) - (1ll << 20)) { set_error("too many tiles in one round"); return TG_ERR_UNSUPPORTED; }
    g.ntiles = (int)total;
    g.njobs = (int)jobs.size();
    g.jobs = append(p.host, jobs.data(), jobs.size() * sizeof(BpArgs));
    const int zero = 0;
    g.counter = append(p.host, &zero, sizeof(int));
    p.bp.push_back(g);
  }
  // tables -> device (the pageable source is staged when the call returns)
  if (p.host.size() > p.cap) {
    if (p.dev) cudaFreeAsync(p.dev, st);
    p.dev = nullptr;
    p.cap = 0;
    const size_t cap = std::max<size_t>(p.host.size() * 2, 4096);
    TG_CUDA(cudaMallocAsync((void **)&p.dev, cap, st));
    p.cap = cap;
  }
  if (!p.host.empty()) TG_CUDA(cudaMemcpyAsync(p.dev, p.host.data(), p.host.size(), cudaMemcpyHostToDevice, st));
  return TG_OK;
}

// The plan's launches on `st` (capturable: no allocation, no host copy).
int round_plan_issue(RoundPlan &p, cudaStream_t st) {
  int launches = 0;
  unsigned char *d = p.dev;
  for (const RoundPlan::Fp &g : p.fp)
    launches += launch_reproject_batch(g.key, reinterpret_cast<const FpArgs *>(d + g.jobs), g.njobs,
                                       reinterpret_cast<const int *>(d + g.abs), g.nabs,
                                       reinterpret_cast<const int *>(d + g.copy), g.ncopy,
                                       reinterpret_cast<const int *>(d + g.fpb), g.nfp, st);
  for (tg_session *s : p.fp_single) launches += launch_reproject(fp_args(s), st);
  for (const RoundPlan::Fi &g : p.fi) {
    FilterBatchDev fb{reinterpret_cast<const FilterArgs *>(d + g.jobs), reinterpret_cast<const int *>(d + g.blk),
                      g.njobs};
    launch_filter_batch(g.n, g.fmt, g.store, fb, g.nblk, st);
    ++launches;
  }
  for (tg_session *s : p.fi_single) {
    launch_filter(filter_args(s, true), st);
    ++launches;
  }
  for (const RoundPlan::Bp &g : p.bp) {
    BatchLaunch bl{};
    bl.jobs = reinterpret_cast<const BpArgs *>(d + g.jobs);
    bl.njobs = g.njobs;
    bl.ntiles = g.ntiles;
    bl.counter = reinterpret_cast<int *>(d + g.counter);
    bl.max_views = g.max_views;
    const int rc = launch_bp_batch(bl, g.store, g.zf != 0, g.variant, st);
    if (rc != TG_OK) return rc;
    ++launches;
  }
  for (tg_session *s : p.bp_single) {
    const cudaStream_t own = s->st;
    s->st = st;
    const int rc = launch_bp(s, 2, nullptr);
    s->st = own;
    if (rc != TG_OK) return rc;
    launches += bp_launch_count(s);
  }
  TG_CUDA(cudaGetLastError());
  p.launches = launches;
  return TG_OK;
}

// Captures the plan's launches once; later calls replay the graph.
int round_plan_launch_graph(RoundPlan &p, cudaStream_t st) {
  if (!p.exec) {
    cudaGraph_t graph;
    TG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    const int rc = round_plan_issue(p, st);
    const cudaError_t ec = cudaStreamEndCapture(st, &graph);
    if (rc != TG_OK) {
      if (ec == cudaSuccess) cudaGraphDestroy(graph);
      return rc;
    }
    if (ec != cudaSuccess) return cuda_fail(ec, "cudaStreamEndCapture(round)");
    const cudaError_t ei = cudaGraphInstantiate(&p.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      p.exec = nullptr;
      return cuda_fail(ei, "cudaGraphInstantiate(round)");
    }
  }
  TG_CUDA(cudaGraphLaunch(p.exec, st));
  return TG_OK;
}

// Plan key of a member list: what the plan's tables depend on besides the
// members' device buffers (fixed for a session's lifetime).
void round_plan_signature(const std::vector<tg_session *> &ss, std::vector<uint64_t> &key) {
  for (tg_session *s : ss) {
    key.push_back((uint64_t)s->variant);
    key.push_back((uint64_t)s->fp_variant);
  }
}

}  // namespace tg
