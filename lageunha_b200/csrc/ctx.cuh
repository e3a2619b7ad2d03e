// The engine context (one periodic box on one GPU) shared by the translation
// units that drive it: engine.cu (the plain C ABI), step.cu (the global step),
// batch.cu (captured graphs, ensembles) and server.cu (the request loop).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "engine_internal.cuh"
#include "tpm_engine.h"

namespace tpm {

enum Stage { kStSort = 0, kStDeposit, kStFft, kStFda4, kStTreeBuild, kStTreeWalk, kStFinish, kNStages };

// Graphs a context keeps: one force evaluation per part mask (1..3) and one
// global step (drag, forces, kick, drift), each valid for the buffers and
// parameters it was captured with.
enum GraphKind { kGraphPm = 1, kGraphTree = 2, kGraphAll = 3, kGraphStep = 4, kNGraphs = 5 };

struct CapturedGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t gen = 0;
  int64_t np = -1;
};

// Per-box evolution factors as the step graph reads them:
// [0] fact1 (drag), [1] fact2 (kicks), [2] pfact (drift), [3] unused.
constexpr int kFacWords = 4;

}  // namespace tpm

struct tpm_ctx {
  tpm_params prm;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[tpm::kNStages + 1];
  // the PM chain of an evaluation that has both parts runs on st_pm, forked
  // after the sort and joined before the walk, beside the tree build on st
  cudaStream_t st_pm = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool overlapped = false;  // the last timed evaluation ran the two chains side by side
  // streamed evaluations (tpm_stream_submit / tpm_stream_wait): two slots of
  // positions and forces, a copy-in and a copy-out stream
  struct {
    cudaStream_t in = nullptr, out = nullptr;
    uint32_t *pos[2] = {nullptr, nullptr};
    float *force[2] = {nullptr, nullptr};
    int64_t cap = 0;
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_comp[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
    uint32_t *herr = nullptr;      // pinned, [2][8]: each slot's error flags
    int64_t ticket[2] = {-1, -1};  // the submission a slot holds
    bool pending[2] = {false, false};
    int64_t next = 0;
  } sp;
  // particles
  int64_t np = 0, cap = 0;
  uint32_t *pos = nullptr;
  float *vel = nullptr;
  uint64_t *key = nullptr, *key_alt = nullptr;
  uint32_t *val = nullptr, *val_alt = nullptr;
  uint32_t *perm = nullptr;  // sorted -> caller index (one of val/val_alt)
  uint64_t *skey = nullptr;  // sorted keys (one of key/key_alt)
  uint32_t *spos = nullptr;
  float *fpm = nullptr, *ftree = nullptr;  // sorted order
  float *fout = nullptr;                   // caller order scratch
  void *stage = nullptr;                   // record staging for the Lagrangian layout
  size_t stage_bytes = 0;
  tpm::SortScratch ss;
  // mesh
  tpm::MeshGeom g;
  tpm::FftPlan fp;
  float *rho = nullptr;
  float2 *spec = nullptr;
  float *phi = nullptr;
  CUtensorMap tmap2, tmap4;  // potential boxes for the 4- and 8-point gradients
  // the half-cell-shifted grid of the interlaced deposit (Gaussian law)
  float *rho2 = nullptr;
  float2 *spec2 = nullptr;
  float *phi2 = nullptr;
  CUtensorMap tmap4b;
  float *gt = nullptr;       // tabulated influence function of the pair
  float gt_rs = -1.f;        // split scale gt was computed for
  uint32_t *tile_start = nullptr;
  // tree
  tpm::TreeBuffers tb;
  uint32_t *cube_start = nullptr;
  int64_t ncubes = 0;
  tpm::LawTable law;
  int law_n = -1;
  float law_eps = -1, law_rs = -1, law_rsphere = -1;
  int law_kind = -1;
  uint32_t *err = nullptr;
  // power spectrum of the mass assignment (tpm_set_power_spectrum)
  bool measure_pk = false;
  double *pk_acc = nullptr;  // device [2][n+1]
  // launch shapes (tpm_autotune): 0 = the built-in choice
  int tune_fft_px = 0, tune_fft_tx = 0;
  int tune_group_level = 2;  // groups live in cubes of 2^level cells
  int tune_group_max = 32;   // targets per warp group
  // graphs: gen counts every change of buffers or parameters baked into a
  // captured launch; herr/hfac are pinned host words the graphs copy through
  uint64_t gen = 1;
  tpm::CapturedGraph graphs[tpm::kNGraphs];
  uint32_t *herr = nullptr;  // pinned [8]
  double *hfac = nullptr;    // pinned [kFacWords]
  double *dfac = nullptr;    // device [kFacWords]
  // where the device buffers come from: the request loop's arena, or
  // cudaMalloc (nullptr)
  tpm::DeviceArena *arena = nullptr;
  // bookkeeping
  unsigned parts_valid = 0;
  float stage_ms[tpm::kNStages];
  int64_t launches = 0;
  int64_t counters[7] = {0, 0, 0, 0, 0, 0, 0};
};

namespace tpm {

// Sets the thread's error message and returns code.
int fail(int code, const char *fmt, ...);
const std::string &last_error_string();

#define CK(call)                                                                                      \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      return ::tpm::fail(e_ == cudaErrorMemoryAllocation ? TPM_E_NOMEM : TPM_E_CUDA, "%s: %s (%s:%d)", \
                         #call, cudaGetErrorString(e_), __FILE__, __LINE__);                          \
  } while (0)

// Enqueues one force evaluation of the loaded particles on st (no host
// synchronisation); with timing, records the stage events. walk == false
// stops before the tree walk (the tree and the groups are built): an
// ensemble walks all its boxes in one launch.
int enqueue_forces(tpm_ctx *c, unsigned parts, cudaStream_t st, bool timing, bool walk = true);
// The walk record of the context's current buffers.
WalkBox ctx_walk_box(const tpm_ctx *c);
// After the stream has finished an evaluation: checks the device error words
// (from c->err, or from the pinned copy when from_host), and on success marks
// the parts valid and reads the tree counters.
int finish_forces(tpm_ctx *c, unsigned parts, bool from_host, bool timing);
// v *= fact1; v += fact2 F; x += v pfact. With fac != nullptr the factors are
// read on the device from fac[0..2] (the step graph); else the scalars apply.
int launch_drag(tpm_ctx *c, cudaStream_t st, float fact1, const double *fac);
int launch_kick(tpm_ctx *c, cudaStream_t st, float f2pm, float f2tree, const double *fac);
int launch_drift(tpm_ctx *c, cudaStream_t st, double pfact, const double *fac);
// k_finish into c->fout: the summed forces in the caller's particle order.
int launch_finish(tpm_ctx *c, cudaStream_t st);
// grows the particle buffers to np (frees the loaded particles if it must)
int ensure_particles_for(tpm_ctx *c, int64_t np);
// the same into `out` with the given parts
int launch_finish_to(tpm_ctx *c, cudaStream_t st, unsigned parts, float *out);
// releases the buffers, streams and events of the streamed evaluations
// (tpm_stream_*), after waiting for them
void free_stream_state(tpm_ctx *c);
// Device bytes a context of this mesh and particle capacity allocates.
int64_t ctx_bytes(int n_mesh, int64_t np);
// tpm_create with the context's device buffers taken from an arena (nullptr:
// cudaMalloc). A context in an arena must not join an ensemble: it drains
// only its own streams before it releases a buffer.
int create_ctx(const tpm_params *params, int device, DeviceArena *arena, tpm_ctx **out);
// Parameter validation of tpm_create / tpm_set_params (sets the error).
int check_params(const tpm_params *p);
// The reference's opening-angle schedule (Cosmos/globalT.c:41-44).
float theta_schedule(int stepcount);
// Makes c->graphs[kind] current (captures it again after a change).
int ensure_graph(tpm_ctx *c, int kind);
// Host-side evolution factors of one step (fact1, fact2, pfact).
int step_factors(const tpm_ctx *c, const tpm_cosmology *cosmo, float anow, float astep, double fac[kFacWords]);

}  // namespace tpm
