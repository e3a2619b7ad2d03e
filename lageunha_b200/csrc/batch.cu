// Captured force evaluations and ensembles of boxes.
//
// A context's force evaluation (or its whole global step) is captured once
// into a CUDA graph and replayed while its buffers and parameters stay the
// same (tpm_ctx::gen and np). The step graph reads its evolution factors from
// device words that a copy node at its head fills from pinned host memory, so
// one graph serves every step. Error words travel back through a copy node
// at its tail.
//
// An ensemble (tpm_batch) is one graph per kind, launched once per call: the
// boxes' stages up to the tree groups run as parallel branches (sort,
// deposit, FFT, gradient, tree build, one stream per box), then ONE walk
// launch takes the groups of every box from a per-box offset table, then the
// boxes' kicks/drift and error copies run as parallel branches again. Boxes of
// different particle counts and mesh sizes mix freely; each keeps its own
// device state between launches. Boxes whose force laws differ cannot share
// the walk's table: such an ensemble is built from the boxes' own graphs
// side by side instead.
#include <string.h>

#include <vector>

#include "ctx.cuh"

using namespace tpm;

namespace {

void drop_graph(CapturedGraph &gr) {
  if (gr.exec) cudaGraphExecDestroy(gr.exec);
  if (gr.graph) cudaGraphDestroy(gr.graph);
  gr.exec = nullptr;
  gr.graph = nullptr;
  gr.gen = 0;
  gr.np = -1;
}

int capture_body(tpm_ctx *c, int kind) {
  cudaStream_t st = c->st;
  if (kind == kGraphStep) {
    CK(cudaMemcpyAsync(c->dfac, c->hfac, sizeof(double) * kFacWords, cudaMemcpyHostToDevice, st));
    int rc = launch_drag(c, st, 1.f, c->dfac);
    if (!rc) rc = enqueue_forces(c, TPM_PART_ALL, st, false);
    if (!rc) rc = launch_kick(c, st, 0.f, 0.f, c->dfac);
    if (!rc) rc = launch_drift(c, st, 0.0, c->dfac);
    if (rc) return rc;
  } else {
    int rc = enqueue_forces(c, (unsigned)kind, st, false);
    if (rc) return rc;
  }
  CK(cudaMemcpyAsync(c->herr, c->err, sizeof(uint32_t) * 8, cudaMemcpyDeviceToHost, st));
  return 0;
}

}  // namespace

int tpm::ensure_graph(tpm_ctx *c, int kind) {
  CapturedGraph &gr = c->graphs[kind];
  if (gr.exec && gr.gen == c->gen && gr.np == c->np) return 0;
  drop_graph(gr);
  CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeRelaxed));
  int rc = capture_body(c, kind);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->st, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(TPM_E_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&gr.exec, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(TPM_E_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
  }
  gr.graph = g;
  gr.gen = c->gen;
  gr.np = c->np;
  return 0;
}

// ------------------------------------------------------------------ ensembles
struct tpm_batch {
  std::vector<tpm_ctx *> boxes;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  // the one-walk form: box records, group offsets, next-group counter
  WalkBox *dboxes = nullptr;
  uint32_t *gprefix = nullptr;
  uint32_t *gnext = nullptr;
  std::vector<cudaEvent_t> fork;  // [0] the fork, [1] after the walk, then 2 per box
  bool fused = false;
  // the ensemble graph per kind, with the box graphs' (gen, np) it was built on
  cudaGraphExec_t exec[kNGraphs] = {};
  std::vector<uint64_t> sig_gen[kNGraphs];
  std::vector<int64_t> sig_np[kNGraphs];
  float last_ms = 0.f;
};

namespace {

// Whether the boxes can share one walk: same law, softening, split and cut.
bool shares_law(const tpm_batch *b) {
  const tpm_params &p0 = b->boxes[0]->prm;
  for (const tpm_ctx *c : b->boxes) {
    const tpm_params &p = c->prm;
    if (p.law != p0.law || p.epsilon != p0.epsilon || p.rs_split != p0.rs_split || p.rsphere != p0.rsphere)
      return false;
  }
  return true;
}

// The ensemble graph of one walk over all boxes, by multi-stream capture.
int capture_fused(tpm_batch *b, int kind, cudaGraph_t *out) {
  int nb = (int)b->boxes.size();
  std::vector<WalkBox> hb(nb);
  for (int i = 0; i < nb; i++) hb[i] = ctx_walk_box(b->boxes[i]);
  CK(cudaMemcpy(b->dboxes, hb.data(), sizeof(WalkBox) * nb, cudaMemcpyHostToDevice));
  unsigned parts = kind == kGraphStep ? TPM_PART_ALL : (unsigned)kind;
  const tpm_ctx *c0 = b->boxes[0];
  CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeRelaxed));
  int rc = 0;
  cudaEventRecord(b->fork[0], b->st);
  for (int i = 0; i < nb && !rc; i++) {
    tpm_ctx *c = b->boxes[i];
    cudaStreamWaitEvent(c->st, b->fork[0], 0);
    if (kind == kGraphStep) {
      if (cudaMemcpyAsync(c->dfac, c->hfac, sizeof(double) * kFacWords, cudaMemcpyHostToDevice, c->st) != cudaSuccess)
        rc = fail(TPM_E_CUDA, "factor copy capture failed");
      if (!rc) rc = launch_drag(c, c->st, 1.f, c->dfac);
    }
    if (!rc) rc = enqueue_forces(c, parts, c->st, false, false);
    cudaEventRecord(b->fork[2 + 2 * i], c->st);
    cudaStreamWaitEvent(b->st, b->fork[2 + 2 * i], 0);
  }
  if (!rc && (parts & TPM_PART_TREE))
    tree_walk_multi(b->dboxes, nb, b->gprefix, b->gnext, c0->tb.stack, c0->tb.stack_words, c0->tb.counters, c0->law,
                    c0->prm.rsphere, b->st);
  cudaEventRecord(b->fork[1], b->st);
  for (int i = 0; i < nb && !rc; i++) {
    tpm_ctx *c = b->boxes[i];
    cudaStreamWaitEvent(c->st, b->fork[1], 0);
    if (kind == kGraphStep) {
      rc = launch_kick(c, c->st, 0.f, 0.f, c->dfac);
      if (!rc) rc = launch_drift(c, c->st, 0.0, c->dfac);
    }
    if (!rc && cudaMemcpyAsync(c->herr, c->err, sizeof(uint32_t) * 8, cudaMemcpyDeviceToHost, c->st) != cudaSuccess)
      rc = fail(TPM_E_CUDA, "error copy capture failed");
    cudaEventRecord(b->fork[3 + 2 * i], c->st);
    cudaStreamWaitEvent(b->st, b->fork[3 + 2 * i], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->st, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(TPM_E_CUDA, "ensemble capture failed: %s", cudaGetErrorString(e));
  *out = g;
  return 0;
}

int ensure_batch_graph(tpm_batch *b, int kind) {
  bool fresh = b->exec[kind] != nullptr;
  for (size_t i = 0; i < b->boxes.size() && fresh; i++)
    fresh = b->sig_gen[kind][i] == b->boxes[i]->gen && b->sig_np[kind][i] == b->boxes[i]->np;
  if (fresh) return 0;
  b->fused = shares_law(b);
  if (b->fused) {
    cudaGraph_t g = nullptr;
    int rc = capture_fused(b, kind, &g);
    if (rc) return rc;
    if (b->exec[kind]) cudaGraphExecDestroy(b->exec[kind]);
    b->exec[kind] = nullptr;
    cudaError_t e = cudaGraphInstantiate(&b->exec[kind], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(TPM_E_CUDA, "ensemble graph instantiation failed: %s", cudaGetErrorString(e));
    b->sig_gen[kind].resize(b->boxes.size());
    b->sig_np[kind].resize(b->boxes.size());
    for (size_t i = 0; i < b->boxes.size(); i++) {
      b->sig_gen[kind][i] = b->boxes[i]->gen;
      b->sig_np[kind][i] = b->boxes[i]->np;
    }
    return 0;
  }
  for (tpm_ctx *c : b->boxes) {
    int rc = ensure_graph(c, kind);
    if (rc) return rc;
  }
  if (b->exec[kind]) cudaGraphExecDestroy(b->exec[kind]);
  b->exec[kind] = nullptr;
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  for (tpm_ctx *c : b->boxes) {
    cudaGraphNode_t node;
    cudaError_t e = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, c->graphs[kind].graph);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return fail(TPM_E_CUDA, "cudaGraphAddChildGraphNode: %s", cudaGetErrorString(e));
    }
  }
  cudaError_t e = cudaGraphInstantiate(&b->exec[kind], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(TPM_E_CUDA, "ensemble graph instantiation failed: %s", cudaGetErrorString(e));
  b->sig_gen[kind].resize(b->boxes.size());
  b->sig_np[kind].resize(b->boxes.size());
  for (size_t i = 0; i < b->boxes.size(); i++) {
    b->sig_gen[kind][i] = b->boxes[i]->gen;
    b->sig_np[kind][i] = b->boxes[i]->np;
  }
  return 0;
}

int run_batch(tpm_batch *b, int kind) {
  CK(cudaSetDevice(b->device));
  for (tpm_ctx *c : b->boxes)
    if (c->np <= 0) return fail(TPM_E_STATE, "a box of the ensemble has no particles");
  int rc = ensure_batch_graph(b, kind);
  if (rc) return rc;
  // work queued on the boxes' own streams comes first
  for (tpm_ctx *c : b->boxes) CK(cudaStreamSynchronize(c->st));
  CK(cudaEventRecord(b->t0, b->st));
  CK(cudaGraphLaunch(b->exec[kind], b->st));
  CK(cudaEventRecord(b->t1, b->st));
  CK(cudaEventSynchronize(b->t1));
  CK(cudaEventElapsedTime(&b->last_ms, b->t0, b->t1));
  unsigned parts = kind == kGraphStep ? 0u : (unsigned)kind;
  int first = 0;
  for (tpm_ctx *c : b->boxes) {
    int r = finish_forces(c, kind == kGraphStep ? TPM_PART_ALL : parts, true, false);
    if (kind == kGraphStep) c->parts_valid = 0;  // the drift moved the particles
    if (r && !first) first = r;
  }
  return first;
}

}  // namespace

extern "C" {

int tpm_batch_create(tpm_ctx *const *boxes, int32_t nbox, tpm_batch **out) {
  if (!out || !boxes || nbox <= 0) return fail(TPM_E_ARG, "bad arguments to tpm_batch_create");
  *out = nullptr;
  for (int i = 0; i < nbox; i++) {
    if (!boxes[i]) return fail(TPM_E_ARG, "box %d is NULL", i);
    if (boxes[i]->device != boxes[0]->device) return fail(TPM_E_ARG, "boxes on different devices");
    for (int j = 0; j < i; j++)
      if (boxes[j] == boxes[i]) return fail(TPM_E_ARG, "box %d repeated", i);
  }
  tpm_batch *b = new tpm_batch();
  b->boxes.assign(boxes, boxes + nbox);
  b->device = boxes[0]->device;
  cudaSetDevice(b->device);
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->t0) != cudaSuccess || cudaEventCreate(&b->t1) != cudaSuccess) {
    tpm_batch_destroy(b);
    return fail(TPM_E_CUDA, "stream/event creation failed");
  }
  b->fork.assign(2 + 2 * (size_t)nbox, nullptr);
  for (cudaEvent_t &e : b->fork)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      tpm_batch_destroy(b);
      return fail(TPM_E_CUDA, "event creation failed");
    }
  if (cudaMalloc(&b->dboxes, sizeof(WalkBox) * nbox) != cudaSuccess ||
      cudaMalloc(&b->gprefix, sizeof(uint32_t) * (nbox + 1)) != cudaSuccess ||
      cudaMalloc(&b->gnext, sizeof(uint32_t)) != cudaSuccess) {
    tpm_batch_destroy(b);
    return fail(TPM_E_NOMEM, "allocation of the ensemble tables failed");
  }
  *out = b;
  return 0;
}

int tpm_batch_destroy(tpm_batch *b) {
  if (!b) return 0;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  for (cudaGraphExec_t &x : b->exec)
    if (x) cudaGraphExecDestroy(x);
  for (cudaEvent_t e : b->fork)
    if (e) cudaEventDestroy(e);
  if (b->dboxes) cudaFree(b->dboxes);
  if (b->gprefix) cudaFree(b->gprefix);
  if (b->gnext) cudaFree(b->gnext);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->t1) cudaEventDestroy(b->t1);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return 0;
}

int tpm_batch_compute(tpm_batch *b, unsigned parts) {
  if (!b) return fail(TPM_E_ARG, "batch is NULL");
  parts &= TPM_PART_ALL;
  if (!parts) return fail(TPM_E_ARG, "no force part requested");
  return run_batch(b, (int)parts);
}

int tpm_batch_step(tpm_batch *b, const tpm_cosmology *cosmo, const float *anow, const float *astep) {
  if (!b || !cosmo || !anow || !astep) return fail(TPM_E_ARG, "bad arguments to tpm_batch_step");
  // the previous launch has finished (run_batch waits), so the pinned factor
  // words are free to change
  for (size_t i = 0; i < b->boxes.size(); i++) {
    int rc = step_factors(b->boxes[i], cosmo, anow[i], astep[i], b->boxes[i]->hfac);
    if (rc) return rc;
  }
  return run_batch(b, kGraphStep);
}

int tpm_batch_time(tpm_batch *b, float *ms) {
  if (!b || !ms) return fail(TPM_E_ARG, "NULL argument");
  *ms = b->last_ms;
  return 0;
}

int tpm_graph_compute(tpm_ctx *c, unsigned parts) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  parts &= TPM_PART_ALL;
  if (!parts) return fail(TPM_E_ARG, "no force part requested");
  CK(cudaSetDevice(c->device));
  int rc = ensure_graph(c, (int)parts);
  if (rc) return rc;
  CK(cudaGraphLaunch(c->graphs[parts].exec, c->st));
  CK(cudaStreamSynchronize(c->st));
  return finish_forces(c, parts, true, false);
}

}  // extern "C"
