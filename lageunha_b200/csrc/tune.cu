// The autotuner: launch shapes picked by timing them on the context's own
// particles.
//
//   TPM_TUNE_FFT     pencils per block of the x passes and kx columns per
//                    block of the y/z passes (results do not change: every
//                    pencil is transformed by the same arithmetic);
//   TPM_TUNE_GROUPS  targets per warp group (16 or 32) and the cube size the
//                    groups are cut from (4 or 8 cells). A group opens a node
//                    if any of its targets would, so this changes the tree
//                    force within its error, not the algorithm.
// Each candidate runs its stage three times after one warm-up, timed with
// CUDA events on the context's stream; the fastest median wins and stays in
// the context (tpm_get_tuning / tpm_set_tuning carry it to boxes of the same
// size).
#include <algorithm>
#include <vector>

#include "ctx.cuh"

using namespace tpm;

namespace {

template <class F>
float time_median(cudaStream_t st, F &&run, int reps = 3) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  run();
  std::vector<float> ms;
  for (int r = 0; r < reps; r++) {
    cudaEventRecord(a, st);
    run();
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    ms.push_back(t);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  std::sort(ms.begin(), ms.end());
  return ms[ms.size() / 2];
}

void poisson(tpm_ctx *c) {
  const MeshGeom &g = c->g;
  bool il = c->prm.law == TPM_LAW_GAUSSIAN;
  launch_poisson(g, c->fp, c->rho, c->spec, c->phi, c->prm.law, c->prm.efold, c->prm.rs_split, c->st, nullptr,
                 il ? c->rho2 : nullptr, il ? c->spec2 : nullptr, il ? c->phi2 : nullptr, il ? c->gt : nullptr,
                 c->tune_fft_px, c->tune_fft_tx);
}

TreeParams tree_params(const tpm_ctx *c) {
  TreeParams tp;
  tp.n = (uint32_t)c->g.n;
  tp.sub_bits = c->g.sub_bits;
  tp.theta2 = c->prm.theta * c->prm.theta;
  tp.rsphere = c->prm.rsphere;
  tp.cell_per_unit = (float)((double)c->g.n / 4294967296.0);
  tp.mass = c->prm.particle_mass;
  tp.group_max = c->tune_group_max;
  return tp;
}

void groups_and_walk(tpm_ctx *c) {
  TreeParams tp = tree_params(c);
  const MeshGeom &g = c->g;
  int glev = c->tune_group_level;
  cudaMemsetAsync(c->tb.counters, 0, sizeof(uint32_t) * 16, c->st);
  tree_groups(tp, c->skey, c->np, c->tb, c->cube_start, 1ll << (3 * (g.cbits - glev)), 3 * (g.sub_bits + glev), c->st,
              nullptr);
  tree_walk(tp, c->spos, c->np, c->tb, c->law, c->ftree, c->err, c->st, nullptr);
}

}  // namespace

extern "C" {

int tpm_get_tuning(const tpm_ctx *c, tpm_tuning *out) {
  if (!c || !out) return fail(TPM_E_ARG, "NULL argument");
  out->fft_pencils_x = c->tune_fft_px;
  out->fft_cols = c->tune_fft_tx;
  out->group_level = c->tune_group_level;
  out->group_max = c->tune_group_max;
  out->ms_fft = out->ms_walk = out->ms_fft_default = out->ms_walk_default = 0.f;
  return 0;
}

int tpm_set_tuning(tpm_ctx *c, const tpm_tuning *t) {
  if (!c || !t) return fail(TPM_E_ARG, "NULL argument");
  if (t->fft_pencils_x < 0 || t->fft_pencils_x > 64 || t->fft_cols < 0 || t->fft_cols > 32 ||
      (t->group_level != 2 && t->group_level != 3) || t->group_max < 1 || t->group_max > 32)
    return fail(TPM_E_ARG, "tuning values out of range");
  c->tune_fft_px = t->fft_pencils_x;
  c->tune_fft_tx = t->fft_cols;
  c->tune_group_level = t->group_level;
  c->tune_group_max = t->group_max;
  c->gen++;
  return 0;
}

int tpm_autotune(tpm_ctx *c, unsigned what, tpm_tuning *out) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  CK(cudaSetDevice(c->device));
  // one evaluation leaves sorted keys, the mesh and the tree in place
  int rc = enqueue_forces(c, TPM_PART_ALL, c->st, false);
  if (!rc) rc = finish_forces(c, TPM_PART_ALL, false, false);
  if (rc) return rc;
  tpm_tuning res;
  tpm_get_tuning(c, &res);
  if (what & TPM_TUNE_FFT) {
    const int pxs[] = {0, 2, 4, 8, 16, 32, 64};
    const int txs[] = {0, 1, 2, 4, 8, 16};
    c->tune_fft_px = c->tune_fft_tx = 0;
    float best = time_median(c->st, [&] { poisson(c); });
    res.ms_fft_default = best;
    int bpx = 0, btx = 0;
    for (int px : pxs)
      for (int tx : txs) {
        if (px == 0 && tx == 0) continue;
        c->tune_fft_px = px;
        c->tune_fft_tx = tx;
        float t = time_median(c->st, [&] { poisson(c); });
        if (t < best) {
          best = t;
          bpx = px;
          btx = tx;
        }
      }
    c->tune_fft_px = bpx;
    c->tune_fft_tx = btx;
    res.fft_pencils_x = bpx;
    res.fft_cols = btx;
    res.ms_fft = best;
  }
  if (what & TPM_TUNE_GROUPS) {
    c->tune_group_level = 2;
    c->tune_group_max = 32;
    float best = time_median(c->st, [&] { groups_and_walk(c); });
    res.ms_walk_default = best;
    int blev = 2, bmax = 32;
    const int levs[] = {2, 3};
    const int maxs[] = {16, 32};
    for (int lev : levs)
      for (int gm : maxs) {
        if (lev == 2 && gm == 32) continue;
        c->tune_group_level = lev;
        c->tune_group_max = gm;
        float t = time_median(c->st, [&] { groups_and_walk(c); });
        if (t < best) {
          best = t;
          blev = lev;
          bmax = gm;
        }
      }
    c->tune_group_level = blev;
    c->tune_group_max = bmax;
    res.group_level = blev;
    res.group_max = bmax;
    res.ms_walk = best;
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  // the trial runs left the forces of other shapes behind
  c->parts_valid = 0;
  c->gen++;
  uint32_t herr = 0;
  CK(cudaMemcpy(&herr, c->err, sizeof(herr), cudaMemcpyDeviceToHost));
  if (herr) return fail(TPM_E_CUDA, "device error flags 0x%x during tuning", herr);
  if (out) *out = res;
  return 0;
}

}  // extern "C"
