// The request loop: continuous batching of force and step requests for boxes
// of different sizes on one GPU.
//
// Clients submit requests (tpm_server_submit) from any thread; one worker
// thread owns every CUDA call. Each loop of the worker
//   * admits queued requests in arrival order while their device footprint
//     (tpm_estimate_bytes) fits under the HBM cap and in the device's free
//     memory, skipping over requests that do not fit yet so that small boxes
//     are not held behind a large one;
//   * gives each admitted request a context, reused from a pool of idle
//     contexts of the same mesh size when one exists, and uploads its
//     particles (pinned staging when the caller's buffers are pageable);
//   * launches the next step (a captured step graph, or the captured force
//     graph for a force request) of every active request whose previous
//     launch has finished: requests progress independently, so work from
//     requests admitted at different times overlaps on the device;
//   * retires finished requests: results to the caller's buffers, context
//     back to the pool, timestamps recorded.
// Device state (particles, mesh, tree, graphs) stays resident between the
// steps of a request. A request's result does not depend on what else is in
// flight: each context has its own buffers, stream and graphs.
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "ctx.cuh"

using namespace tpm;

namespace {

using Clock = std::chrono::steady_clock;

enum Phase { kQueued = 0, kRunning, kDraining, kDone, kFailed };

struct Req {
  int64_t id = 0;
  tpm_request r;
  int phase = kQueued;
  int status = 0;
  std::string error;
  double t_submit = 0, t_admit = 0, t_done = 0;
  int64_t bytes = 0;
  // running state
  tpm_ctx *ctx = nullptr;
  int step = 0;           // steps launched so far
  bool inflight = false;  // a launch not yet seen finished
  cudaEvent_t ev = nullptr;
  // pinned staging for pageable caller buffers
  void *stage = nullptr;
  size_t stage_bytes = 0;
  bool out_pinned[3] = {true, true, true};
};

struct PoolEntry {
  tpm_ctx *ctx;
  int64_t bytes;
  double last_used;
};

bool is_pinned(const void *p) {
  if (!p) return true;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

struct tpm_server {
  int device = 0;
  int64_t cap = 0;
  int max_active = 0;
  Clock::time_point t0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_submit, cv_done;
  bool stop = false;
  int64_t next_id = 1;
  std::deque<Req *> incoming;             // submitted, not yet seen by the worker
  std::map<int64_t, Req *> all;           // every request by id
  // worker-only state
  std::vector<Req *> queue;               // waiting for admission, arrival order
  std::vector<Req *> active;
  std::vector<PoolEntry> pool;            // idle contexts
  int64_t bytes_active = 0, bytes_pool = 0;
  int64_t stats[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // [0] done [1] failed [2] peak active [3] peak bytes [4] contexts created
  // [5] contexts reused [6] contexts evicted [7] admissions deferred for memory

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

void finish(tpm_server *s, Req *q, int status, const char *msg) {
  std::lock_guard<std::mutex> lk(s->mu);
  q->status = status;
  if (status) {
    q->phase = kFailed;
    q->error = msg ? msg : "";
    s->stats[1]++;
  } else {
    q->phase = kDone;
    s->stats[0]++;
  }
  q->t_done = s->now();
  s->cv_done.notify_all();
}

void release_ctx(tpm_server *s, Req *q) {
  if (q->ctx) {
    s->pool.push_back(PoolEntry{q->ctx, q->bytes, s->now()});
    s->bytes_pool += q->bytes;
    s->bytes_active -= q->bytes;
    q->ctx = nullptr;
  }
  if (q->ev) cudaEventDestroy(q->ev);
  q->ev = nullptr;
  if (q->stage) cudaFreeHost(q->stage);
  q->stage = nullptr;
}

void evict_one(tpm_server *s) {
  // the least recently used idle context
  auto it = std::min_element(s->pool.begin(), s->pool.end(),
                             [](const PoolEntry &a, const PoolEntry &b) { return a.last_used < b.last_used; });
  if (it == s->pool.end()) return;
  tpm_destroy(it->ctx);
  s->bytes_pool -= it->bytes;
  s->pool.erase(it);
  s->stats[6]++;
}

// A context for q from the pool (same mesh size, enough capacity) or new.
int acquire_ctx(tpm_server *s, Req *q) {
  const tpm_request &r = q->r;
  for (size_t i = 0; i < s->pool.size(); i++) {
    PoolEntry &p = s->pool[i];
    if (p.ctx->prm.n_mesh == r.params.n_mesh && p.ctx->cap >= r.np) {
      q->ctx = p.ctx;
      q->bytes = p.bytes;
      s->bytes_pool -= p.bytes;
      s->pool.erase(s->pool.begin() + i);
      s->stats[5]++;
      return tpm_set_params(q->ctx, &r.params);
    }
  }
  tpm_ctx *c = nullptr;
  int rc = tpm_create(&r.params, s->device, &c);
  if (rc) return rc;
  q->ctx = c;
  q->bytes = ctx_bytes(r.params.n_mesh, r.np);
  s->stats[4]++;
  return 0;
}

// Uploads the particles and prepares the per-request event and staging.
int start(tpm_server *s, Req *q) {
  const tpm_request &r = q->r;
  tpm_ctx *c = q->ctx;
  CK(cudaEventCreateWithFlags(&q->ev, cudaEventDisableTiming));
  size_t nb = sizeof(float) * 3 * (size_t)r.np;
  bool in_pinned = is_pinned(r.pos) && is_pinned(r.vel);
  q->out_pinned[0] = is_pinned(r.pos_out);
  q->out_pinned[1] = is_pinned(r.vel_out);
  q->out_pinned[2] = is_pinned(r.force_out);
  bool need_stage = !in_pinned || !q->out_pinned[0] || !q->out_pinned[1] || !q->out_pinned[2];
  if (need_stage) {
    q->stage_bytes = 3 * nb;
    CK(cudaMallocHost(&q->stage, q->stage_bytes));
  }
  const uint32_t *pos = r.pos;
  const float *vel = r.vel;
  if (!in_pinned) {
    memcpy(q->stage, r.pos, nb);
    pos = (const uint32_t *)q->stage;
    if (r.vel) {
      memcpy((char *)q->stage + nb, r.vel, nb);
      vel = (const float *)((char *)q->stage + nb);
    }
  }
  int rc = tpm_load_fixed(c, r.np, pos, vel, TPM_MEM_HOST);
  if (rc) return rc;
  if (r.nsteps == 0) return ensure_graph(c, kGraphAll);
  return ensure_graph(c, kGraphStep);
}

// Launches the next unit of work of q (one step, or the force evaluation).
int launch_next(tpm_server *s, Req *q) {
  (void)s;
  const tpm_request &r = q->r;
  tpm_ctx *c = q->ctx;
  if (r.nsteps == 0) {
    CK(cudaGraphLaunch(c->graphs[kGraphAll].exec, c->st));
  } else {
    if (c->prm.law == TPM_LAW_REFERENCE) {
      // TreeAndPreFoFmain's opening-angle schedule (Cosmos/globalT.c:41-44)
      tpm_params p = c->prm;
      p.theta = theta_schedule(q->step);
      if (p.theta != c->prm.theta) {
        int rc = tpm_set_params(c, &p);
        if (!rc) rc = ensure_graph(c, kGraphStep);
        if (rc) return rc;
      }
    }
    int rc = step_factors(c, &r.cosmo, r.anow + (float)q->step * r.astep, r.astep, c->hfac);
    if (rc) return rc;
    CK(cudaGraphLaunch(c->graphs[kGraphStep].exec, c->st));
  }
  CK(cudaEventRecord(q->ev, c->st));
  q->step++;
  q->inflight = true;
  return 0;
}

// Results to the caller: device -> pinned (theirs or the staging) copies.
int drain(tpm_server *s, Req *q) {
  (void)s;
  const tpm_request &r = q->r;
  tpm_ctx *c = q->ctx;
  size_t nb = sizeof(float) * 3 * (size_t)r.np;
  if (r.force_out) {
    int rc = launch_finish(c, c->st);
    if (rc) return rc;
    void *dst = q->out_pinned[2] ? (void *)r.force_out : (char *)q->stage + 2 * nb;
    CK(cudaMemcpyAsync(dst, c->fout, nb, cudaMemcpyDeviceToHost, c->st));
  }
  if (r.pos_out) {
    void *dst = q->out_pinned[0] ? (void *)r.pos_out : q->stage;
    CK(cudaMemcpyAsync(dst, c->pos, nb, cudaMemcpyDeviceToHost, c->st));
  }
  if (r.vel_out) {
    void *dst = q->out_pinned[1] ? (void *)r.vel_out : (char *)q->stage + nb;
    CK(cudaMemcpyAsync(dst, c->vel, nb, cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaEventRecord(q->ev, c->st));
  q->inflight = true;
  return 0;
}

void copy_out_staged(Req *q) {
  const tpm_request &r = q->r;
  size_t nb = sizeof(float) * 3 * (size_t)r.np;
  if (r.pos_out && !q->out_pinned[0]) memcpy(r.pos_out, q->stage, nb);
  if (r.vel_out && !q->out_pinned[1]) memcpy(r.vel_out, (char *)q->stage + nb, nb);
  if (r.force_out && !q->out_pinned[2]) memcpy(r.force_out, (char *)q->stage + 2 * nb, nb);
}

bool try_admit(tpm_server *s, Req *q) {
  int64_t need = ctx_bytes(q->r.params.n_mesh, q->r.np);
  // an idle context of this mesh with the capacity is reused without new memory
  bool reusable = false;
  for (const PoolEntry &p : s->pool)
    if (p.ctx->prm.n_mesh == q->r.params.n_mesh && p.ctx->cap >= q->r.np) reusable = true;
  if (!reusable) {
    while (s->bytes_active + s->bytes_pool + need > s->cap && !s->pool.empty()) evict_one(s);
    if (s->bytes_active + s->bytes_pool + need > s->cap) return false;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
      const int64_t margin = 512ll << 20;
      while ((int64_t)fr < need + margin && !s->pool.empty()) {
        evict_one(s);
        cudaMemGetInfo(&fr, &tot);
      }
      if ((int64_t)fr < need + margin) return false;
    }
  }
  int rc = acquire_ctx(s, q);
  if (!rc) {
    s->bytes_active += q->bytes;
    q->t_admit = s->now();
    rc = start(s, q);
  }
  if (rc) {
    std::string m = last_error_string();
    if (q->ctx) {
      tpm_destroy(q->ctx);
      s->bytes_active -= q->bytes;
      q->ctx = nullptr;
    }
    if (q->ev) cudaEventDestroy(q->ev);
    q->ev = nullptr;
    if (q->stage) cudaFreeHost(q->stage);
    q->stage = nullptr;
    finish(s, q, rc, m.c_str());
    return true;  // consumed (failed)
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    q->phase = kRunning;
  }
  s->active.push_back(q);
  s->stats[2] = std::max<int64_t>(s->stats[2], (int64_t)s->active.size());
  s->stats[3] = std::max<int64_t>(s->stats[3], s->bytes_active + s->bytes_pool);
  return true;
}

void worker_main(tpm_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->incoming.empty() && s->queue.empty() && s->active.empty()) {
        if (s->stop) break;
        s->cv_submit.wait_for(lk, std::chrono::milliseconds(5));
      }
      while (!s->incoming.empty()) {
        s->queue.push_back(s->incoming.front());
        s->incoming.pop_front();
      }
    }
    bool progressed = false;
    // admission, arrival order, skipping what does not fit yet
    for (size_t i = 0; i < s->queue.size();) {
      if ((int)s->active.size() >= s->max_active) break;
      Req *q = s->queue[i];
      if (try_admit(s, q)) {
        s->queue.erase(s->queue.begin() + i);
        progressed = true;
      } else {
        s->stats[7]++;
        i++;
      }
    }
    // launches and completions
    for (size_t i = 0; i < s->active.size();) {
      Req *q = s->active[i];
      int rc = 0;
      bool retired = false;
      if (q->inflight) {
        cudaError_t e = cudaEventQuery(q->ev);
        if (e == cudaErrorNotReady) {
          i++;
          continue;
        }
        q->inflight = false;
        progressed = true;
        if (e != cudaSuccess) {
          rc = fail(TPM_E_CUDA, "request %lld: %s", (long long)q->id, cudaGetErrorString(e));
        } else if (q->phase == kDraining) {
          copy_out_staged(q);
          release_ctx(s, q);
          finish(s, q, 0, nullptr);
          retired = true;
        } else {
          rc = finish_forces(q->ctx, TPM_PART_ALL, true, false);
          if (!rc && q->r.nsteps > 0) q->ctx->parts_valid = TPM_PART_ALL;
        }
      }
      if (!retired && !rc && !q->inflight) {
        int total = q->r.nsteps > 0 ? q->r.nsteps : 1;
        if (q->step < total) {
          rc = launch_next(s, q);
        } else {
          {
            std::lock_guard<std::mutex> lk(s->mu);
            q->phase = kDraining;
          }
          rc = drain(s, q);
        }
        progressed = true;
      }
      if (rc) {
        std::string m = last_error_string();
        if (q->ctx) cudaStreamSynchronize(q->ctx->st);
        // a context that saw a device error is not reused
        if (q->ctx) {
          tpm_destroy(q->ctx);
          s->bytes_active -= q->bytes;
          q->ctx = nullptr;
        }
        release_ctx(s, q);
        finish(s, q, rc, m.c_str());
        retired = true;
      }
      if (retired) {
        s->active.erase(s->active.begin() + i);
      } else {
        i++;
      }
    }
    if (!progressed && !s->active.empty()) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  for (PoolEntry &p : s->pool) tpm_destroy(p.ctx);
  s->pool.clear();
}

}  // namespace

extern "C" {

int tpm_server_create(int device, int64_t hbm_cap_bytes, int32_t max_active, tpm_server **out) {
  if (!out || hbm_cap_bytes <= 0 || max_active <= 0) return fail(TPM_E_ARG, "bad arguments to tpm_server_create");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return fail(TPM_E_NODEV, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return fail(TPM_E_ARG, "device %d out of range", device);
  tpm_server *s = new tpm_server();
  s->device = device;
  s->cap = hbm_cap_bytes;
  s->max_active = max_active;
  s->t0 = Clock::now();
  s->worker = std::thread(worker_main, s);
  *out = s;
  return 0;
}

int tpm_server_submit(tpm_server *s, const tpm_request *req, int64_t *id) {
  if (!s || !req || !id) return fail(TPM_E_ARG, "NULL argument");
  int rc = check_params(&req->params);
  if (rc) return rc;
  if (req->np <= 0 || req->np > 0xffffffffll - 64 || !req->pos || req->nsteps < 0)
    return fail(TPM_E_ARG, "bad request: np, pos or nsteps");
  if (req->nsteps > 0 && !(req->anow > 0.f && req->astep >= 0.f)) return fail(TPM_E_ARG, "bad request: anow/astep");
  if (ctx_bytes(req->params.n_mesh, req->np) > s->cap)
    return fail(TPM_E_NOMEM, "request needs %lld bytes, above the server's cap",
                (long long)ctx_bytes(req->params.n_mesh, req->np));
  Req *q = new Req();
  q->r = *req;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    delete q;
    return fail(TPM_E_STATE, "server is shutting down");
  }
  q->id = s->next_id++;
  q->t_submit = s->now();
  s->all[q->id] = q;
  s->incoming.push_back(q);
  *id = q->id;
  s->cv_submit.notify_one();
  return 0;
}

int tpm_server_info(tpm_server *s, int64_t id, tpm_request_info *out) {
  if (!s || !out) return fail(TPM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return fail(TPM_E_ARG, "unknown request %lld", (long long)id);
  const Req *q = it->second;
  out->state = q->phase == kQueued ? TPM_REQ_QUEUED
               : q->phase == kDone ? TPM_REQ_DONE
               : q->phase == kFailed ? TPM_REQ_FAILED
                                     : TPM_REQ_ACTIVE;
  out->status = q->status;
  out->t_submit = q->t_submit;
  out->t_admit = q->t_admit;
  out->t_done = q->t_done;
  out->device_bytes = q->bytes;
  return 0;
}

int tpm_server_wait(tpm_server *s, int64_t id, double timeout_s) {
  if (!s) return fail(TPM_E_ARG, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  auto pending = [&]() {
    if (id >= 0) {
      auto it = s->all.find(id);
      return it != s->all.end() && it->second->phase != kDone && it->second->phase != kFailed;
    }
    for (auto &kv : s->all)
      if (kv.second->phase != kDone && kv.second->phase != kFailed) return true;
    return false;
  };
  if (id >= 0 && s->all.find(id) == s->all.end()) return fail(TPM_E_ARG, "unknown request %lld", (long long)id);
  auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
  while (pending()) {
    if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout && pending())
      return fail(TPM_E_STATE, "timed out waiting for request %lld", (long long)id);
  }
  if (id >= 0) {
    const Req *q = s->all[id];
    if (q->phase == kFailed) return fail(q->status, "request %lld failed: %s", (long long)id, q->error.c_str());
  }
  return 0;
}

int tpm_server_stats(tpm_server *s, int64_t *out, int n) {
  if (!s || !out) return fail(TPM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  int k = n < 8 ? n : 8;
  for (int i = 0; i < k; i++) out[i] = s->stats[i];
  return k;
}

int tpm_server_destroy(tpm_server *s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_submit.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  for (auto &kv : s->all) delete kv.second;
  delete s;
  return 0;
}

}  // extern "C"
