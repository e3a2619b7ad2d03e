// The request loop: continuous batching of force and step requests for boxes
// of different sizes on one GPU.
//
// Clients submit requests (tpm_server_submit) from any thread. Two threads
// serve them:
//   * the admission thread takes queued requests in arrival order while their
//     device footprint (tpm_estimate_bytes) fits under the HBM cap and in the
//     device's free memory, skipping over requests that do not fit yet so
//     that small boxes are not held behind a large one. It gives each
//     admitted request a context, reused from a pool of idle contexts of the
//     same mesh size when one exists, uploads its particles (pinned staging
//     when the caller's buffers are pageable) and captures its graph, then
//     hands it to the launch thread. Creating a context, its first upload and
//     its capture take 10-60 ms; the launch thread keeps stepping the active
//     requests meanwhile.
//   * the launch thread launches the next step (a captured step graph, or the
//     captured force graph for a force request) of every active request whose
//     previous launch has finished: requests progress independently, so work
//     from requests admitted at different times overlaps on the device. It
//     retires finished requests: results to the caller's buffers, context
//     back to the pool, timestamps recorded.
// The two threads share the pool, the byte accounting and the hand-over list
// under the server's mutex, held for bookkeeping only, never across a CUDA
// call. Each context belongs to one thread at a time. Graph capture runs in
// the relaxed mode, so the launch thread's calls are legal during a capture.
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

constexpr int kNStats = 12;

int64_t usec_since(Clock::time_point t) {
  return std::chrono::duration_cast<std::chrono::microseconds>(Clock::now() - t).count();
}

enum Phase { kQueued = 0, kRunning, kDraining, kDone, kFailed };

struct Req {
  tpm_server *srv = nullptr;
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
  // the contexts' device buffers: claimed from the driver in large blocks,
  // kept across requests
  DeviceArena *arena = nullptr;
  std::thread admitter, launcher;
  // guards every field below except queue and active
  std::mutex mu;
  std::condition_variable cv_submit;  // wakes the admission thread: a request arrived or one retired
  std::condition_variable cv_ready;   // wakes the launch thread: a request was admitted
  std::condition_variable cv_done;    // wakes clients in tpm_server_wait
  bool stop = false;
  bool admit_done = false;                // the admission thread has left
  int64_t next_id = 1;
  std::deque<Req *> incoming;             // submitted, not yet seen by the admission thread
  std::map<int64_t, Req *> all;           // every request by id
  std::vector<Req *> ready;               // admitted, not yet taken by the launch thread
  int completions = 0;                    // launches seen finished by the stream callbacks
  std::vector<PoolEntry> pool;            // idle contexts
  int64_t bytes_active = 0, bytes_pool = 0;
  int live = 0;                           // requests ready or active
  int64_t stats[kNStats] = {};
  // [0] done [1] failed [2] peak active [3] peak bytes [4] contexts created
  // [5] contexts reused [6] contexts evicted [7] admissions deferred for memory
  // admission thread time, microseconds: [8] making or re-parameterising
  // contexts [9] uploading particles [10] capturing graphs [11] reserving
  // memory (evictions included); tpm_server_stats adds [12] the arena's bytes
  // admission-thread only
  std::vector<Req *> queue;               // waiting for admission, arrival order
  // launch-thread only
  std::vector<Req *> active;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// Records q's outcome. A request that was handed to the launch thread
// (retiring) frees its slot and wakes the admission thread.
void finish(tpm_server *s, Req *q, int status, const char *msg, bool retiring) {
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
  if (retiring) {
    s->live--;
    s->cv_submit.notify_one();
  }
  s->cv_done.notify_all();
}

// q's context back to the pool (a device error destroys it instead), its
// event and staging freed.
void release_ctx(tpm_server *s, Req *q, bool broken) {
  if (q->ctx) {
    if (broken) tpm_destroy(q->ctx);
    std::lock_guard<std::mutex> lk(s->mu);
    if (!broken) {
      s->pool.push_back(PoolEntry{q->ctx, q->bytes, s->now()});
      s->bytes_pool += q->bytes;
    }
    s->bytes_active -= q->bytes;
    q->ctx = nullptr;
  }
  if (q->ev) cudaEventDestroy(q->ev);
  q->ev = nullptr;
  if (q->stage) cudaFreeHost(q->stage);
  q->stage = nullptr;
}

// Takes the least recently used idle context out of the pool; the caller
// holds s->mu and destroys the context after releasing it.
tpm_ctx *take_lru(tpm_server *s) {
  auto it = std::min_element(s->pool.begin(), s->pool.end(),
                             [](const PoolEntry &a, const PoolEntry &b) { return a.last_used < b.last_used; });
  if (it == s->pool.end()) return nullptr;
  tpm_ctx *c = it->ctx;
  s->bytes_pool -= it->bytes;
  s->pool.erase(it);
  s->stats[6]++;
  return c;
}

// Reserves q's device bytes: an idle context of the same mesh size and
// enough capacity (no new memory), else room under the cap, evicting idle
// contexts least recently used first. False when q does not fit yet.
bool reserve(tpm_server *s, Req *q) {
  const tpm_request &r = q->r;
  const int64_t need = ctx_bytes(r.params.n_mesh, r.np);
  std::vector<tpm_ctx *> evicted;
  bool fits = true;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (size_t i = 0; i < s->pool.size(); i++) {
      PoolEntry &p = s->pool[i];
      if (p.ctx->prm.n_mesh == r.params.n_mesh && p.ctx->cap >= r.np) {
        q->ctx = p.ctx;
        q->bytes = p.bytes;
        s->bytes_pool -= p.bytes;
        s->bytes_active += p.bytes;
        s->pool.erase(s->pool.begin() + i);
        s->stats[5]++;
        return true;
      }
    }
    while (s->bytes_active + s->bytes_pool + need > s->cap && !s->pool.empty()) evicted.push_back(take_lru(s));
    if (s->bytes_active + s->bytes_pool + need > s->cap) {
      fits = false;
    } else {
      q->bytes = need;
      s->bytes_active += need;
    }
  }
  for (tpm_ctx *c : evicted) tpm_destroy(c);
  if (!fits) return false;
  // the device's free memory too (other processes share the GPU), beside
  // what the arena holds unused
  const int64_t margin = 512ll << 20;
  size_t fr = 0, tot = 0;
  auto available = [&]() {
    int64_t reserved = 0, in_use = 0;
    arena_usage(s->arena, &reserved, &in_use);
    return (int64_t)fr + (reserved - in_use);
  };
  while (cudaMemGetInfo(&fr, &tot) == cudaSuccess && available() < need + margin) {
    tpm_ctx *c = nullptr;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      c = take_lru(s);
      if (!c) {
        s->bytes_active -= need;
        q->bytes = 0;
        return false;
      }
    }
    tpm_destroy(c);
  }
  return true;
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
  Clock::time_point t = Clock::now();
  int rc = tpm_load_fixed(c, r.np, pos, vel, TPM_MEM_HOST);
  if (rc) return rc;
  int64_t t_load = usec_since(t);
  t = Clock::now();
  rc = ensure_graph(c, r.nsteps == 0 ? kGraphAll : kGraphStep);
  std::lock_guard<std::mutex> lk(s->mu);
  s->stats[9] += t_load;
  s->stats[10] += usec_since(t);
  return rc;
}

// Runs on the CUDA callback thread when a launch of q has finished: wakes
// the launch thread. Every context's stream is synchronized before the
// context is destroyed, so no callback outlives the server.
void CUDART_CB on_launch_done(void *p) {
  tpm_server *s = static_cast<Req *>(p)->srv;
  std::lock_guard<std::mutex> lk(s->mu);
  s->completions++;
  s->cv_ready.notify_one();
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
  CK(cudaLaunchHostFunc(c->st, on_launch_done, q));
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
  CK(cudaLaunchHostFunc(c->st, on_launch_done, q));
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

// Admits q: reserve its bytes, take or create its context, upload, capture,
// hand it to the launch thread. False when q does not fit yet; true when q
// was consumed, admitted or failed.
bool try_admit(tpm_server *s, Req *q) {
  Clock::time_point t = Clock::now();
  bool fits = reserve(s, q);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats[11] += usec_since(t);
  }
  if (!fits) return false;
  t = Clock::now();
  int rc = 0;
  bool created = false;
  if (q->ctx) {
    rc = tpm_set_params(q->ctx, &q->r.params);
  } else {
    rc = create_ctx(&q->r.params, s->device, s->arena, &q->ctx);
    created = !rc;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (created) s->stats[4]++;
    s->stats[8] += usec_since(t);
    q->t_admit = s->now();
  }
  if (!rc) rc = start(s, q);
  if (rc) {
    std::string m = last_error_string();
    if (!q->ctx) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->bytes_active -= q->bytes;
    }
    release_ctx(s, q, true);
    q->bytes = 0;
    if (rc == TPM_E_NOMEM) {
      // out of device memory (the free ranges too fragmented, or another
      // process took the memory): the idle contexts go back to the arena and
      // q waits for a retry, unless nothing else holds memory
      std::vector<tpm_ctx *> idle;
      bool others;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        while (tpm_ctx *c = take_lru(s)) idle.push_back(c);
        others = s->live > 0 || !idle.empty();
      }
      for (tpm_ctx *c : idle) tpm_destroy(c);
      if (others) return false;
    }
    finish(s, q, rc, m.c_str(), false);
    return true;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  q->phase = kRunning;
  s->ready.push_back(q);
  s->live++;
  s->stats[2] = std::max<int64_t>(s->stats[2], (int64_t)s->live);
  s->stats[3] = std::max<int64_t>(s->stats[3], s->bytes_active + s->bytes_pool);
  s->cv_ready.notify_one();
  return true;
}

void admit_main(tpm_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      while (!s->incoming.empty()) {
        s->queue.push_back(s->incoming.front());
        s->incoming.pop_front();
      }
      if (s->queue.empty()) {
        if (s->stop) break;
        s->cv_submit.wait_for(lk, std::chrono::milliseconds(5));
        continue;
      }
    }
    // arrival order, skipping what does not fit yet
    bool admitted = false;
    for (size_t i = 0; i < s->queue.size();) {
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->live >= s->max_active) break;
      }
      if (try_admit(s, s->queue[i])) {
        s->queue.erase(s->queue.begin() + i);
        admitted = true;
      } else {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stats[7]++;
        i++;
      }
    }
    if (!admitted) {
      // until a request retires (a slot or memory freed) or arrives
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->incoming.empty()) s->cv_submit.wait_for(lk, std::chrono::milliseconds(2));
    }
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->admit_done = true;
  s->cv_ready.notify_all();
}

void launch_main(tpm_server *s) {
  cudaSetDevice(s->device);
  for (;;) {
    {
      // sleep until a request is admitted or a launch finishes; the timeout
      // only bounds the wait should a callback never come
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->ready.empty() && s->completions == 0) {
        if (s->active.empty() && s->admit_done) break;
        s->cv_ready.wait_for(lk, std::chrono::milliseconds(2));
      }
      s->completions = 0;
      for (Req *q : s->ready) s->active.push_back(q);
      s->ready.clear();
    }
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
        if (e != cudaSuccess) {
          rc = fail(TPM_E_CUDA, "request %lld: %s", (long long)q->id, cudaGetErrorString(e));
        } else if (q->phase == kDraining) {
          copy_out_staged(q);
          release_ctx(s, q, false);
          finish(s, q, 0, nullptr, true);
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
      }
      if (rc) {
        std::string m = last_error_string();
        if (q->ctx) cudaStreamSynchronize(q->ctx->st);
        // a context that saw a device error is not reused
        release_ctx(s, q, true);
        finish(s, q, rc, m.c_str(), true);
        retired = true;
      }
      if (retired) {
        s->active.erase(s->active.begin() + i);
      } else {
        i++;
      }
    }
  }
  std::vector<PoolEntry> idle;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    idle.swap(s->pool);
    s->bytes_pool = 0;
  }
  for (PoolEntry &p : idle) tpm_destroy(p.ctx);
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
  s->arena = arena_create(device, 0);
  s->admitter = std::thread(admit_main, s);
  s->launcher = std::thread(launch_main, s);
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
  q->srv = s;
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
  int64_t all[kNStats + 1];
  for (int i = 0; i < kNStats; i++) all[i] = s->stats[i];
  arena_usage(s->arena, &all[kNStats], nullptr);
  int k = n < kNStats + 1 ? n : kNStats + 1;
  for (int i = 0; i < k; i++) out[i] = all[i];
  return k;
}

int tpm_server_reserve(tpm_server *s, int64_t bytes) {
  if (!s || bytes < 0) return fail(TPM_E_ARG, "bad arguments to tpm_server_reserve");
  if (bytes > s->cap) return fail(TPM_E_ARG, "reserve of %lld bytes above the server's cap", (long long)bytes);
  CK(cudaSetDevice(s->device));
  CK(arena_reserve(s->arena, bytes));
  return 0;
}

int tpm_server_destroy(tpm_server *s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_submit.notify_all();
  }
  if (s->admitter.joinable()) s->admitter.join();
  if (s->launcher.joinable()) s->launcher.join();
  // every context is destroyed by now: the arena's blocks go back to the driver
  arena_destroy(s->arena);
  for (auto &kv : s->all) delete kv.second;
  delete s;
  return 0;
}

}  // extern "C"
