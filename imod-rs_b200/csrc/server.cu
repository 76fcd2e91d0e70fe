// server.cu -- request loop with continuous batching over one device.
//
// Threads: any number of client threads call tg_server_submit / poll / wait;
// an admission thread creates the sessions of admitted jobs and starts their
// copies in; the device thread issues the rounds and collects finished jobs.
// Streams: `cs` runs the rounds (filter, reprojection, batched back-projection,
// statistics), `us` copies projections in, `ds` copies volumes and statistics
// out, `fs` returns memory to the pool.
//
//   1. (device thread) finished jobs -- their copy-out event has completed --
//      report DONE/FAILED and their memory is freed stream-ordered on `fs`;
//   2. (admission thread) first-in first-out: a job is admitted while the
//      device bytes of the running jobs plus its own stay within the budget and
//      fewer than max_active run; a job that does not fit yet may be passed by
//      later ones for at most kMaxBypassMs, then it holds the line.  Its session
//      allocates from the server's pool and its projections copy in on `us`;
//   3. (device thread) a round: every running job whose projections have
//      arrived takes one step (round 0: log/means, filter, WBP; round r:
//      reproject, residual filter, SIRT update) and all back-projections of the
//      round go into one persistent launch (batch_bp).  A job that took its last
//      step gets its output transform and statistics on `cs`, then its copy-out
//      on `ds`.  At most two rounds are queued ahead of the device.
// A job's arithmetic is the same as tg_reconstruct on its own (the batched
// back-projection is bit-identical per tile), so results do not depend on
// the mix.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "session_impl.h"

using namespace tg;

namespace {

struct SJob {
  uint64_t id = 0, tag = 0;
  tg_geometry g{};
  tg_options o{};
  std::vector<float> angles, xtilt, zfactor, local;
  const float *h_proj = nullptr;
  size_t n = 0;
  float *h_out = nullptr;
  int state = TG_JOB_QUEUED, status = TG_OK;
  size_t est = 0, held = 0;
  tg_session *s = nullptr;
  int rounds_total = 0, rounds_done = 0, mode0 = 0, nt0 = 0;
  bool finishing = false;
  cudaEvent_t ev_up = nullptr, ev_fin = nullptr, ev_dl = nullptr;
  int slot = -1;
  double t_submit = -1, t_admit = -1, t_done = -1, updates = 0;
  int oom_retries = 0;
  double retry_at = 0;  // server clock before which an OOM-requeued job is not retried
  tg_stats stats{};
  std::string message;  // why a failed job failed
};

constexpr int kSlotBytes = 32;           // 3 floats of statistics, then the 4-int device error word
constexpr double kMaxBypassMs = 2000.0;  // how long a waiting job may be passed by later ones
constexpr int kMaxOomRetries = 50;       // admissions retried after a device allocation failure

}  // namespace

struct tg_server {
  int dev = 0;
  size_t budget = 0;
  int max_active = 64;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_done, cv_admit;
  std::map<uint64_t, std::shared_ptr<SJob>> jobs;
  std::deque<std::shared_ptr<SJob>> pending;
  std::deque<std::shared_ptr<SJob>> admitted;   // created and copying in; the device thread takes them
  std::vector<std::shared_ptr<SJob>> active;    // device thread only
  int n_running = 0;                            // admitted and not yet ended
  uint64_t next_id = 1;
  bool stop = false, admit_done = false;
  std::thread th, th_admit;
  cudaStream_t cs = nullptr, us = nullptr, ds = nullptr, fs = nullptr;
  cudaMemPool_t pool = nullptr;
  tg_batch batch;
  RoundPlan plan, scratch;    // SIRT rounds: the captured plan, and the plan of the last round
  uint64_t graph_rounds = 0;  // device thread only
  unsigned char *h_slots = nullptr;
  std::vector<int> free_slots;                  // guarded by mu
  std::mutex ev_mu;                             // guards event_pool
  std::deque<cudaEvent_t> event_pool;
  std::deque<std::pair<cudaEvent_t, cudaEvent_t>> rounds_in_flight;  // device thread only
  std::vector<cudaEvent_t> timing_pool;                              // device thread only
  // counters (guarded by mu)
  uint64_t submitted = 0, completed = 0, failed = 0, rounds = 0, bp_launches = 0, oom_requeues = 0;
  size_t used = 0, peak = 0;
  double updates_done = 0, gpu_round_ms = 0, host_round_ms = 0, host_admit_ms = 0;
  int inject_alloc = 0, inject_admit = 0;

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

double host_ms(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

cudaEvent_t take_event(tg_server *sv) {
  {
    std::lock_guard<std::mutex> lk(sv->ev_mu);
    if (!sv->event_pool.empty()) {
      cudaEvent_t e = sv->event_pool.back();
      sv->event_pool.pop_back();
      return e;
    }
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  return e;
}

void give_event(tg_server *sv, cudaEvent_t &e) {
  if (e) {
    std::lock_guard<std::mutex> lk(sv->ev_mu);
    sv->event_pool.push_back(e);
  }
  e = nullptr;
}

cudaEvent_t take_timing_event(tg_server *sv) {
  if (!sv->timing_pool.empty()) {
    cudaEvent_t e = sv->timing_pool.back();
    sv->timing_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

// Ends a job (either server thread; mu must not be held).  Its memory is freed
// on fs, a stream of its own so that frees do not queue behind other jobs'
// copies: at once after a completed copy-out, and -- when the job ends early --
// after everything queued so far on cs and us, which may still use it.
void end_job(tg_server *sv, const std::shared_ptr<SJob> &j, int status) {
  if (status != TG_OK) j->message = tg_last_error();
  if (j->s) {
    if (!j->finishing) {
      for (cudaStream_t st : {sv->cs, sv->us}) {
        cudaEvent_t e = take_event(sv);
        if (e && cudaEventRecord(e, st) == cudaSuccess) cudaStreamWaitEvent(sv->fs, e, 0);
        else cudaStreamSynchronize(st);
        give_event(sv, e);
      }
    }
    free_session_async(j->s, sv->fs);
    j->s = nullptr;
  }
  give_event(sv, j->ev_up);
  give_event(sv, j->ev_fin);
  give_event(sv, j->ev_dl);
  std::lock_guard<std::mutex> lk(sv->mu);
  if (j->slot >= 0) sv->free_slots.push_back(j->slot);
  j->slot = -1;
  if (j->state == TG_JOB_RUNNING) --sv->n_running;
  sv->used -= j->held;
  j->held = 0;
  j->t_done = sv->now_ms();
  j->status = status;
  j->state = status == TG_OK ? TG_JOB_DONE : TG_JOB_FAILED;
  if (status == TG_OK) {
    ++sv->completed;
    sv->updates_done += j->updates;
  } else {
    ++sv->failed;
  }
  sv->cv_done.notify_all();
  sv->cv_admit.notify_all();
}

void drop_active(tg_server *sv, const std::shared_ptr<SJob> &j) {
  for (size_t i = 0; i < sv->active.size(); ++i)
    if (sv->active[i] == j) {
      sv->active.erase(sv->active.begin() + i);
      return;
    }
}

// 1. finished copies
void collect(tg_server *sv) {
  for (size_t i = 0; i < sv->active.size();) {
    std::shared_ptr<SJob> j = sv->active[i];
    if (!j->finishing) { ++i; continue; }
    cudaError_t q = cudaEventQuery(j->ev_dl);
    if (q == cudaErrorNotReady) { ++i; continue; }
    int st = TG_OK;
    if (q != cudaSuccess) {
      st = cuda_fail(q, "server copy-out");
    } else {
      const unsigned char *slot = sv->h_slots + (size_t)j->slot * kSlotBytes;
      const float *f = reinterpret_cast<const float *>(slot);
      const int *err = reinterpret_cast<const int *>(slot + 16);
      j->stats.amin = f[0];
      j->stats.amax = f[1];
      j->stats.amean = f[2];
      if (err[0]) st = device_error_status(err[0]);
    }
    sv->active.erase(sv->active.begin() + i);
    end_job(sv, j, st);
  }
}

// 2. admission thread: session creation overlaps the rounds
void admit_loop(tg_server *sv) {
  cudaSetDevice(sv->dev);
  for (;;) {
    std::shared_ptr<SJob> j;
    bool refuse = false, fail_alloc = false;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      size_t pick = 0;
      auto choose = [&]() {
        if (sv->pending.empty() || sv->n_running >= sv->max_active || sv->free_slots.empty()) return false;
        const double now = sv->now_ms();
        for (size_t k = 0; k < sv->pending.size(); ++k) {
          const std::shared_ptr<SJob> &c = sv->pending[k];
          if (c->retry_at <= now && (sv->inject_admit > 0 || sv->used + c->est <= sv->budget)) {
            pick = k;
            return true;
          }
          if (now - c->t_submit > kMaxBypassMs) return false;  // it holds the line
        }
        return false;
      };
      while (!sv->stop && !choose()) sv->cv_admit.wait_for(lk, std::chrono::milliseconds(2));
      if (sv->stop) break;
      j = sv->pending[pick];
      sv->pending.erase(sv->pending.begin() + pick);
      if (sv->inject_admit > 0) {
        --sv->inject_admit;
        refuse = true;
      } else {
        if (sv->inject_alloc > 0) {
          --sv->inject_alloc;
          fail_alloc = true;
        }
        j->held = j->est;  // reserved now, corrected to the session's bytes below
        sv->used += j->held;
        sv->peak = std::max(sv->peak, sv->used);
        ++sv->n_running;
        j->slot = sv->free_slots.back();
        sv->free_slots.pop_back();
        j->state = TG_JOB_RUNNING;
        j->t_admit = sv->now_ms();
      }
    }
    if (refuse) {
      set_error("admission refused (injected)");
      end_job(sv, j, TG_ERR_BUDGET);
      continue;
    }
    const auto t_adm = std::chrono::steady_clock::now();
    NvtxRange nv("tg.server.admit");
    tg_session *s = nullptr;
    int rc = session_create_ex(&j->g, &j->o, sv->pool, false, fail_alloc, &s);
    if (rc == TG_ERR_OOM && !fail_alloc && j->oom_retries < kMaxOomRetries) {
      // the budget admitted it but the pool could not map the memory yet (frees
      // in flight, fragmentation): give unused memory back, requeue the job at
      // the head and retry it shortly
      (void)cudaGetLastError();
      ++j->oom_retries;
      cudaStreamSynchronize(sv->fs);
      cudaMemPoolTrimTo(sv->pool, 0);
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->used -= j->held;
      j->held = 0;
      --sv->n_running;
      sv->free_slots.push_back(j->slot);
      j->slot = -1;
      j->state = TG_JOB_QUEUED;
      j->t_admit = -1;
      j->retry_at = sv->now_ms() + 5.0;
      sv->pending.push_front(j);
      ++sv->oom_requeues;
      continue;
    }
    if (rc != TG_OK) {
      end_job(sv, j, rc);
      continue;
    }
    j->s = s;
    s->st = sv->cs;
    s->variant = tune_lookup(s);
    if (s->variant < 0) s->variant = s->fast || s->xt_split ? 8 : 0;  // S8K4TX32NT256V4N3: best or near on the measured shapes
    j->ev_up = take_event(sv);
    j->ev_fin = take_event(sv);
    j->ev_dl = take_event(sv);
    if (!j->ev_up || !j->ev_fin || !j->ev_dl) {
      set_error("server out of events");
      end_job(sv, j, TG_ERR_CUDA);
      continue;
    }
    cudaError_t e = cudaMemcpyAsync(s->d_raw, j->h_proj, j->n * 4, cudaMemcpyHostToDevice, sv->us);
    if (e == cudaSuccess) e = cudaEventRecord(j->ev_up, sv->us);
    if (e != cudaSuccess) {
      end_job(sv, j, cuda_fail(e, "server copy-in"));
      continue;
    }
    s->uploaded = true;
    j->rounds_total = 1 + sirt_iters(s);
    j->updates = (double)s->onx * s->onz * s->ny * s->nviews * (1.0 + 2.0 * sirt_iters(s));
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->used += s->dev_bytes;
    sv->used -= j->held;
    j->held = s->dev_bytes;
    sv->peak = std::max(sv->peak, sv->used);
    sv->host_admit_ms += host_ms(t_adm);
    sv->admitted.push_back(j);
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->admit_done = true;
}

// 3. one round over every running job whose projections have arrived
bool run_round(tg_server *sv) {
  while (!sv->rounds_in_flight.empty() && cudaEventQuery(sv->rounds_in_flight.front().second) != cudaErrorNotReady) {
    auto pr = sv->rounds_in_flight.front();
    sv->rounds_in_flight.pop_front();
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->gpu_round_ms += ms;
    }
    sv->timing_pool.push_back(pr.first);
    sv->timing_pool.push_back(pr.second);
  }
  if (sv->rounds_in_flight.size() >= 2) return false;
  std::vector<std::shared_ptr<SJob>> ready;
  for (auto &j : sv->active) {
    if (j->finishing || j->rounds_done >= j->rounds_total) continue;
    if (j->rounds_done == 0 && cudaEventQuery(j->ev_up) == cudaErrorNotReady) continue;
    ready.push_back(j);
  }
  if (ready.empty()) return false;
  const auto t_host = std::chrono::steady_clock::now();
  NvtxRange nv("tg.server.round");
  cudaEvent_t r0 = take_timing_event(sv);
  if (r0) cudaEventRecord(r0, sv->cs);
  // jobs in their first round: log/means, filter, one WBP back-projection launch;
  // jobs in SIRT rounds: one plan of grouped launches (round.cu), replayed from its
  // CUDA graph while the same jobs keep iterating together
  std::vector<tg_session *> first, iter;
  std::vector<int> modes, nt;
  std::vector<uint64_t> key;
  int launches = 0, rc = TG_OK;
  for (auto &j : ready) {
    tg_session *s = j->s;
    if (j->rounds_done == 0) {
      cudaStreamWaitEvent(sv->cs, j->ev_up, 0);
      if (rc == TG_OK) rc = stage_front(s, &launches);
      modes.push_back(first_mode(s));
      first.push_back(s);
    } else {
      iter.push_back(s);
      key.push_back(j->id);
    }
  }
  sv->batch.persistent_launches = 0;
  if (rc == TG_OK && !iter.empty()) {
    round_plan_signature(iter, key);
    if (key == sv->plan.key) {
      rc = round_plan_launch_graph(sv->plan, sv->cs);
      ++sv->graph_rounds;
    } else if (key == sv->scratch.key) {  // the same jobs a second round in a row: capture
      std::swap(sv->plan, sv->scratch);
      rc = round_plan_launch_graph(sv->plan, sv->cs);
      ++sv->graph_rounds;
    } else {
      rc = round_plan_build(sv->scratch, iter, key, sv->cs);
      if (rc == TG_OK) rc = round_plan_issue(sv->scratch, sv->cs);
    }
    const RoundPlan &p = key == sv->plan.key ? sv->plan : sv->scratch;
    launches += p.launches;
    sv->batch.persistent_launches += (int)p.bp.size();
  }
  if (rc == TG_OK && !first.empty()) rc = batch_bp(&sv->batch, first, modes, nt, &launches);
  if (rc != TG_OK) {  // a launch could not be issued: the round's jobs fail, the others go on
    for (auto &j : ready) {
      drop_active(sv, j);
      end_job(sv, j, rc);
    }
    (void)cudaGetLastError();
    if (r0) sv->timing_pool.push_back(r0);
    return true;
  }
  for (size_t i = 0, fi = 0; i < ready.size(); ++i) {
    std::shared_ptr<SJob> j = ready[i];
    tg_session *s = j->s;
    if (j->rounds_done == 0) {
      j->mode0 = modes[fi];
      j->nt0 = nt[fi];
      ++fi;
    }
    if (++j->rounds_done < j->rounds_total) continue;
    rc = stage_finish(s, j->mode0, j->nt0, &launches);
    cudaError_t e = rc == TG_OK ? cudaEventRecord(j->ev_fin, sv->cs) : cudaErrorUnknown;
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sv->ds, j->ev_fin, 0);
    const size_t nvol = (size_t)s->onx * s->onz * s->ny;
    unsigned char *slot = sv->h_slots + (size_t)j->slot * kSlotBytes;
    if (e == cudaSuccess && j->h_out) e = cudaMemcpyAsync(j->h_out, s->d_vol, nvol * 4, cudaMemcpyDeviceToHost, sv->ds);
    if (e == cudaSuccess) e = cudaMemcpyAsync(slot, s->d_stats3, 12, cudaMemcpyDeviceToHost, sv->ds);
    if (e == cudaSuccess) e = cudaMemcpyAsync(slot + 16, s->d_err, 16, cudaMemcpyDeviceToHost, sv->ds);
    if (e == cudaSuccess) e = cudaEventRecord(j->ev_dl, sv->ds);
    if (e != cudaSuccess) {
      drop_active(sv, j);
      end_job(sv, j, rc != TG_OK ? rc : cuda_fail(e, "server finish"));
      continue;
    }
    j->finishing = true;
  }
  cudaEvent_t r1 = take_timing_event(sv);
  if (r0 && r1 && cudaEventRecord(r1, sv->cs) == cudaSuccess) {
    sv->rounds_in_flight.push_back({r0, r1});
  } else {  // no event to bound the queue: wait for the round
    cudaStreamSynchronize(sv->cs);
    if (r0) sv->timing_pool.push_back(r0);
    if (r1) sv->timing_pool.push_back(r1);
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->host_round_ms += host_ms(t_host);
  ++sv->rounds;
  sv->bp_launches += sv->batch.persistent_launches;
  return true;
}

void device_loop(tg_server *sv) {
  cudaSetDevice(sv->dev);
  for (;;) {
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      while (!sv->admitted.empty()) {
        sv->active.push_back(sv->admitted.front());
        sv->admitted.pop_front();
      }
      if (sv->stop && sv->admit_done) {
        while (!sv->pending.empty()) {  // dropped before admission
          std::shared_ptr<SJob> j = sv->pending.front();
          sv->pending.pop_front();
          j->state = TG_JOB_FAILED;
          j->status = TG_ERR_CANCELLED;
          j->message = "cancelled by tg_server_destroy";
          j->t_done = sv->now_ms();
          ++sv->failed;
        }
        sv->cv_done.notify_all();
        if (sv->active.empty()) break;
      }
    }
    collect(sv);
    if (!run_round(sv)) std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
  round_plan_release(sv->plan, sv->cs);
  round_plan_release(sv->scratch, sv->cs);
  cudaStreamSynchronize(sv->cs);
  cudaStreamSynchronize(sv->us);
  cudaStreamSynchronize(sv->ds);
  cudaStreamSynchronize(sv->fs);
}

}  // namespace

extern "C" {

int tg_server_create(int32_t device, uint64_t budget_bytes, int32_t max_active, tg_server **out) {
  if (!out) return TG_ERR_INVALID_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { set_error("no CUDA device"); return TG_ERR_NO_DEVICE; }
  if (device < 0 || device >= ndev) { set_error("bad device ordinal"); return TG_ERR_INVALID_ARG; }
  TG_CUDA(cudaSetDevice(device));
  std::unique_ptr<tg_server> sv(new tg_server());
  sv->dev = device;
  sv->max_active = max_active > 0 ? max_active : 64;
  if (budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    TG_CUDA(cudaMemGetInfo(&fr, &tot));
    budget_bytes = (uint64_t)(0.8 * (double)fr);
  }
  sv->budget = budget_bytes;
  sv->t0 = std::chrono::steady_clock::now();
  cudaError_t e;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  uint64_t keep = UINT64_MAX;
  int no = 0;
  if ((e = cudaStreamCreateWithFlags(&sv->cs, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&sv->us, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&sv->ds, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&sv->fs, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaMemPoolCreate(&sv->pool, &props)) != cudaSuccess ||
      (e = cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess ||
      // no hidden cross-stream waits: memory is reused once its free has completed
      (e = cudaMemPoolSetAttribute(sv->pool, cudaMemPoolReuseAllowInternalDependencies, &no)) != cudaSuccess ||
      (e = cudaMalloc(&sv->batch.d_counter, sizeof(int))) != cudaSuccess ||
      (e = cudaHostAlloc((void **)&sv->h_slots, (size_t)sv->max_active * kSlotBytes, cudaHostAllocDefault)) !=
          cudaSuccess) {
    int rc = cuda_fail(e, "tg_server_create");
    if (sv->cs) cudaStreamDestroy(sv->cs);
    if (sv->us) cudaStreamDestroy(sv->us);
    if (sv->ds) cudaStreamDestroy(sv->ds);
    if (sv->fs) cudaStreamDestroy(sv->fs);
    if (sv->pool) cudaMemPoolDestroy(sv->pool);
    if (sv->batch.d_counter) cudaFree(sv->batch.d_counter);
    return rc;
  }
  sv->batch.dev = device;
  sv->batch.st = sv->cs;
  for (int i = sv->max_active - 1; i >= 0; --i) sv->free_slots.push_back(i);
  tg_server *p = sv.release();
  p->th = std::thread(device_loop, p);
  p->th_admit = std::thread(admit_loop, p);
  *out = p;
  return TG_OK;
}

int tg_server_submit(tg_server *sv, const tg_job *job, uint64_t *id) {
  if (!sv || !job || !id) return TG_ERR_INVALID_ARG;
  const tg_geometry &g = job->geometry;
  if (!job->projections || job->n_projections != (size_t)g.nx * g.ny * g.nz || g.nx < 1 || g.ny < 1 || g.nz < 1) {
    set_error("projection count mismatch");
    return TG_ERR_INVALID_ARG;
  }
  auto j = std::make_shared<SJob>();
  j->angles.assign(g.angles, g.angles + (g.angles ? g.n_angles : 0));
  if (g.xtilt) j->xtilt.assign(g.xtilt, g.xtilt + g.n_xtilt);
  if (g.zfactor) j->zfactor.assign(g.zfactor, g.zfactor + g.n_zfactor);
  if (g.local) j->local.assign(g.local, g.local + 5 * (size_t)g.n_local);
  j->g = g;
  j->g.angles = j->angles.empty() ? nullptr : j->angles.data();
  j->g.xtilt = j->xtilt.empty() ? nullptr : j->xtilt.data();
  j->g.zfactor = j->zfactor.empty() ? nullptr : j->zfactor.data();
  j->g.local = j->local.empty() ? nullptr : j->local.data();
  j->o = job->options;
  j->o.device = sv->dev;
  j->o.use_graphs = 0;
  j->h_proj = job->projections;
  j->n = job->n_projections;
  j->h_out = job->volume_out;
  j->tag = job->tag;
  // size (and validate) the job with a dry session: no device work
  tg_session *dry = nullptr;
  int rc = session_create_ex(&j->g, &j->o, nullptr, true, false, &dry);
  if (rc != TG_OK) return rc;
  j->est = dry->dev_bytes;
  session_discard(dry);
  std::lock_guard<std::mutex> lk(sv->mu);
  if (sv->stop) { set_error("server is shutting down"); return TG_ERR_CANCELLED; }
  if (j->est > sv->budget) {
    set_error("job needs more device memory than the server's budget");
    return TG_ERR_BUDGET;
  }
  j->id = sv->next_id++;
  j->t_submit = sv->now_ms();
  sv->jobs[j->id] = j;
  sv->pending.push_back(j);
  ++sv->submitted;
  sv->cv_admit.notify_all();
  *id = j->id;
  return TG_OK;
}

static void fill_result(const SJob &j, tg_job_result *r) {
  r->state = j.state;
  r->status = j.status;
  r->stats = j.stats;
  r->rounds = j.rounds_total;
  r->submit_ms = j.t_submit;
  r->admit_ms = j.t_admit;
  r->done_ms = j.t_done;
  r->updates = j.updates;
  r->device_bytes = j.held ? j.held : j.est;
  r->tag = j.tag;
  snprintf(r->message, sizeof r->message, "%s", j.message.c_str());
}

int tg_server_poll(tg_server *sv, uint64_t id, tg_job_result *out) {
  if (!sv || !out) return TG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) return TG_ERR_NOT_FOUND;
  fill_result(*it->second, out);
  return TG_OK;
}

int tg_server_wait(tg_server *sv, uint64_t id, int32_t timeout_ms, tg_job_result *out) {
  if (!sv) return TG_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) return TG_ERR_NOT_FOUND;
  std::shared_ptr<SJob> j = it->second;
  auto ended = [&] { return j->state == TG_JOB_DONE || j->state == TG_JOB_FAILED; };
  if (timeout_ms < 0) sv->cv_done.wait(lk, ended);
  else if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ended)) {
    if (out) fill_result(*j, out);
    return TG_ERR_NOT_READY;
  }
  if (out) fill_result(*j, out);
  return TG_OK;
}

int tg_server_release(tg_server *sv, uint64_t id) {
  if (!sv) return TG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(id);
  if (it == sv->jobs.end()) return TG_ERR_NOT_FOUND;
  if (it->second->state != TG_JOB_DONE && it->second->state != TG_JOB_FAILED) return TG_ERR_NOT_READY;
  sv->jobs.erase(it);
  return TG_OK;
}

int tg_server_get_info(tg_server *sv, tg_server_info *out) {
  if (!sv || !out) return TG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  *out = tg_server_info{};
  out->submitted = sv->submitted;
  out->completed = sv->completed;
  out->failed = sv->failed;
  out->queued = sv->pending.size();
  uint64_t running = 0;
  for (auto &kv : sv->jobs) running += kv.second->state == TG_JOB_RUNNING;
  out->running = running;
  out->budget_bytes = sv->budget;
  out->bytes_in_use = sv->used;
  out->bytes_peak = sv->peak;
  out->rounds = sv->rounds;
  out->bp_launches = sv->bp_launches;
  out->updates_done = sv->updates_done;
  out->oom_requeues = sv->oom_requeues;
  out->gpu_round_ms = sv->gpu_round_ms;
  out->host_round_ms = sv->host_round_ms;
  out->host_admit_ms = sv->host_admit_ms;
  return TG_OK;
}

int tg_server_inject(tg_server *sv, int32_t fault, int32_t count) {
  if (!sv || count < 0) return TG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  if (fault == TG_FAULT_ALLOC) sv->inject_alloc = count;
  else if (fault == TG_FAULT_ADMIT) sv->inject_admit = count;
  else return TG_ERR_INVALID_ARG;
  return TG_OK;
}

int tg_submit(tg_server *sv, const tg_job *job, uint64_t *id) { return tg_server_submit(sv, job, id); }
int tg_poll(tg_server *sv, uint64_t id, tg_job_result *out) { return tg_server_poll(sv, id, out); }

int tg_server_destroy(tg_server *sv) {
  if (!sv) return TG_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
    sv->cv_admit.notify_all();
  }
  if (sv->th_admit.joinable()) sv->th_admit.join();
  if (sv->th.joinable()) sv->th.join();
  cudaSetDevice(sv->dev);
  for (cudaEvent_t e : sv->event_pool) cudaEventDestroy(e);
  for (auto &pr : sv->rounds_in_flight) {
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  for (cudaEvent_t e : sv->timing_pool) cudaEventDestroy(e);
  cudaFree(sv->batch.d_jobs);
  cudaFree(sv->batch.d_counter);
  cudaFreeHost(sv->h_slots);
  cudaStreamDestroy(sv->cs);
  cudaStreamDestroy(sv->us);
  cudaStreamDestroy(sv->ds);
  cudaStreamDestroy(sv->fs);
  cudaMemPoolDestroy(sv->pool);
  delete sv;
  return TG_OK;
}

}  // extern "C"
