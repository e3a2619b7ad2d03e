// TreePM force engine: context, orchestration and the C ABI of
// include/tpm_engine.h.
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "tpm_engine.h"
#include "engine_internal.cuh"
#include "ctx.cuh"

namespace tpm {
int ewald_force(const uint32_t *pos, int64_t np, int n, float eps, int64_t nt, const int64_t *targets_host,
                double *out_host, cudaStream_t st);
int64_t walk_stack_words();
}  // namespace tpm

using namespace tpm;

static thread_local std::string g_err;

// TPM_DEBUG_SYNC=1 synchronises and checks after every stage of a force
// evaluation, so a failing kernel is reported by stage name.
static bool debug_sync() {
  static int v = -1;
  if (v < 0) {
    const char *s = getenv("TPM_DEBUG_SYNC");
    v = (s && s[0] == '1') ? 1 : 0;
  }
  return v == 1;
}

void tpm::set_last_error(const char *msg) { g_err = msg; }

int tpm::fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

const std::string &tpm::last_error_string() { return g_err; }

static cudaError_t stage_check(cudaStream_t st, const char *name) {
  cudaError_t e = cudaGetLastError();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (e == cudaSuccess && debug_sync() && cudaStreamIsCapturing(st, &cs) == cudaSuccess &&
      cs == cudaStreamCaptureStatusNone)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) fprintf(stderr, "tpm: stage %s failed: %s\n", name, cudaGetErrorString(e));
  return e;
}

extern "C" {

void tpm_default_params(tpm_params *p, int32_t n_mesh) {
  p->n_mesh = n_mesh;
  p->law = TPM_LAW_REFERENCE;
  p->theta = 0.3f;
  p->rsphere = 4.0f;
  p->epsilon = 0.1f;
  p->efold = 0.9f;
  p->rs_split = 1.25f;
  p->particle_mass = 1.0f;
}

const char *tpm_last_error(void) { return g_err.c_str(); }
const char *tpm_version(void) { return "lageunha_b200 tpm_engine 0.1 (sm_100a)"; }

}  // extern "C"

int tpm::check_params(const tpm_params *p) {
  if (!p) return fail(TPM_E_ARG, "params is NULL");
  if (p->n_mesh < 16 || p->n_mesh > 4096) return fail(TPM_E_ARG, "n_mesh %d outside [16, 4096]", p->n_mesh);
  if (p->law != TPM_LAW_REFERENCE && p->law != TPM_LAW_GAUSSIAN) return fail(TPM_E_ARG, "unknown law %d", p->law);
  if (!(p->theta > 0.f && p->theta < 1.f)) return fail(TPM_E_ARG, "theta %g outside (0,1)", p->theta);
  if (!(p->rsphere > 0.f && p->rsphere <= 6.0f)) return fail(TPM_E_ARG, "rsphere %g outside (0, 6]", p->rsphere);
  // pairs are taken at their minimum image, so the cutoff sphere must fit in
  // half the box
  if (p->rsphere * 2.f >= (float)p->n_mesh) return fail(TPM_E_ARG, "rsphere %g too large for n_mesh %d", p->rsphere, p->n_mesh);
  if (!(p->epsilon >= 0.f)) return fail(TPM_E_ARG, "epsilon %g < 0", p->epsilon);
  if (p->law == TPM_LAW_GAUSSIAN && !(p->rs_split > 0.f)) return fail(TPM_E_ARG, "rs_split must be > 0");
  if (!(p->particle_mass > 0.f)) return fail(TPM_E_ARG, "particle_mass must be > 0");
  return 0;
}

// ------------------------------------------------------------------ law table
// Residual short-range law f(r)/N^2 and its tables. OST/Model4TreeForce.c:
// 48-91 tabulates {-f/r, -(f'r - f)/(2 r^3), -(f''r^2 - 3f'r + 3f)/(2 r^5)}
// linearly at r = i*6/4096 (central differences of step 0.1*6/4096) and the
// walk interpolates at r. The engine keeps the same three columns of the same
// law but on grids uniform in log r^2 (indexed by the float bits of r^2, no
// square root in the walk): -f/r on a fine grid (kLogMantissa bits per
// octave), the two node columns on a coarse one (kPcMantissa bits).
static const double kPmFit[8] = {1.0 / 256.0 / 256.0, 0.78224E+00, 0.37971E-06, -0.60338E+00,
                                 -0.34419E-07, -0.39741E+01, -0.10607E+01, -0.38145E+00};

static double law_f(int kind, double r, float eps, double rs, double LL) {
  double soft = r / pow(r * r + (double)(eps * eps), 1.5);
  double longr;
  if (kind == TPM_LAW_REFERENCE) {
    // PMFITPARA fit of the reference's PM force (Model4TreeForce.c:92-116)
    const double *P = kPmFit;
    double t = cosh(P[1] * r);
    longr = 1.0 / (r * r) * tanh(P[1] * r) - P[1] / (t * t * r) - 2.0 * P[2] / P[0] * r * exp(P[3] * r * r) -
            2.0 * P[2] * P[3] / P[0] * r * r * r * exp(P[3] * r * r) +
            P[4] / P[0] * (1.0 + P[5] * r * r + P[6] * r * r * r * r) * exp(P[7] * r * r);
  } else {
    // force of a Gaussian-filtered point mass, filter exp(-k^2 rs^2)
    double u = r / (2.0 * rs);
    longr = (erf(u) - 2.0 * u / sqrt(M_PI) * exp(-u * u)) / (r * r);
  }
  return (soft - longr) / LL;
}

// cudaFree waits for the whole device before it returns memory; a range of
// the context's arena can go to another context at once, so a context in an
// arena drains its own streams before it releases a buffer.
static void quiesce(tpm_ctx *c) {
  if (!c->arena) return;
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->st_pm) cudaStreamSynchronize(c->st_pm);
  if (c->sp.in) cudaStreamSynchronize(c->sp.in);
  if (c->sp.out) cudaStreamSynchronize(c->sp.out);
}

static int build_law(tpm_ctx *c) {
  const tpm_params &p = c->prm;
  if (c->law.tlog && c->law_n == p.n_mesh && c->law_eps == p.epsilon && c->law_kind == p.law &&
      c->law_rs == p.rs_split && c->law_rsphere == p.rsphere)
    return 0;
  // the tables are per unit LL (= N^2): the walk scales each box's forces by
  // its own 1/N^2, so boxes of every mesh size share one table
  const double LL = 1.0;
  // the reference's derivative step: a tenth of its table spacing 6/4096
  const double dr = 0.1 * 6.0 / 4096.0;
  const double rs2 = (double)p.rsphere * (double)p.rsphere;
  // the reference law keeps its per-pair test r <= rsphere, so its column
  // continues past the cut (the last bin before the cut interpolates the law
  // itself); the Gaussian law's column is zero from the cut on, so the pair
  // term ramps to zero over the last bin and the walk needs no pair test
  const int hard_cut = p.law == TPM_LAW_GAUSSIAN ? 0 : 1;
  auto at_bits = [](uint32_t bits) {
    float sf;
    memcpy(&sf, &bits, 4);
    return (double)sf;
  };
  // the particle-particle column -f/r on the log-spaced grid of
  // s = r^2 + kLogR2Floor, held at its value at r = 2^-10 cells below that
  // (the reference's table is flat below its first entry, r = 6/4096, and
  // its fitted long-range law does not vanish at r = 0)
  std::vector<float2> tlog(kLogEntries + 1);
  {
    std::vector<double> v(kLogEntries + 1);
    for (int k = 0; k <= kLogEntries; k++) {
      double s = at_bits((uint32_t)(kLogBase + k) << kLogShift);
      double r2 = s - (double)kLogR2Floor, r = std::max(sqrt(std::max(r2, 0.0)), 0.0009765625);
      v[k] = (r2 >= rs2 && !hard_cut) ? 0.0 : -(law_f(p.law, r, p.epsilon, p.rs_split, LL) / r);
    }
    for (int k = 0; k < kLogEntries; k++) {
      double s0 = at_bits((uint32_t)(kLogBase + k) << kLogShift);
      double s1 = at_bits((uint32_t)(kLogBase + k + 1) << kLogShift);
      double slope = (v[k + 1] - v[k]) / (s1 - s0);
      tlog[k] = make_float2((float)(v[k] - slope * s0), (float)slope);
    }
    tlog[kLogEntries] = make_float2(0.f, 0.f);
    // the first entry from which the column is zero: the walk reads no entry
    // at or beyond it (the values there are zero anyway)
    int k0 = kLogEntries;
    while (k0 > 0 && v[k0 - 1] == 0.0) k0--;
    c->law.cut_bits = (uint32_t)(kLogBase + k0) << kLogShift;
  }
  // the node terms' derivative columns (Model4TreeForce.c:48-91:
  // -(f'r - f)/(2 r^3) and -(f''r^2 - 3f'r + 3f)/(2 r^5), central
  // differences) on the coarse log grid of r^2; the node test r <= rsphere is
  // always made, so the columns continue past the cut
  std::vector<float4> tpc(kPcEntries + 1);
  {
    std::vector<double> f2(kPcEntries + 1), f3(kPcEntries + 1);
    for (int k = 0; k <= kPcEntries; k++) {
      double s = at_bits((uint32_t)(kPcBase + k) << kPcShift), r = sqrt(s);
      double fm2 = law_f(p.law, r - 2 * dr, p.epsilon, p.rs_split, LL);
      double fm1 = law_f(p.law, r - dr, p.epsilon, p.rs_split, LL);
      double fr = law_f(p.law, r, p.epsilon, p.rs_split, LL);
      double fp1 = law_f(p.law, r + dr, p.epsilon, p.rs_split, LL);
      double fp2 = law_f(p.law, r + 2 * dr, p.epsilon, p.rs_split, LL);
      double fp = (fp1 - fm1) / (dr + dr);
      double fpp = (fp2 - 2 * fr + fm2) / (4 * dr * dr);
      f2[k] = -(0.5 * (fp * r - fr) / r / r / r);
      f3[k] = -(0.5 * (fpp * r * r - 3 * fp * r + 3 * fr) / r / r / r / r / r);
    }
    const double sc = (double)(1 << kPcMantissa);
    for (int k = 0; k < kPcEntries; k++) {
      double d2 = (f2[k + 1] - f2[k]) * sc, d3 = (f3[k + 1] - f3[k]) * sc;
      tpc[k] = make_float4((float)(f2[k] - d2), (float)d2, (float)(f3[k] - d3), (float)d3);
    }
    tpc[kPcEntries] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (c->law.tlog || c->law.tpc) {
    CK(cudaStreamSynchronize(c->st));
    quiesce(c);
  }
  dfree(c->arena, c->law.tlog);
  dfree(c->arena, c->law.tpc);
  c->law.tlog = nullptr;
  c->law.tpc = nullptr;
  CK(dmalloc(c->arena, &c->law.tlog, sizeof(float2) * (kLogEntries + 1)));
  CK(cudaMemcpy(c->law.tlog, tlog.data(), sizeof(float2) * (kLogEntries + 1), cudaMemcpyHostToDevice));
  CK(dmalloc(c->arena, &c->law.tpc, sizeof(float4) * (kPcEntries + 1)));
  CK(cudaMemcpy(c->law.tpc, tpc.data(), sizeof(float4) * (kPcEntries + 1), cudaMemcpyHostToDevice));
  c->law.hard_cut = hard_cut;
  c->law_n = p.n_mesh;
  c->law_eps = p.epsilon;
  c->law_kind = p.law;
  c->law_rs = p.rs_split;
  c->law_rsphere = p.rsphere;
  c->gen++;
  return 0;
}

// ------------------------------------------------------------------ buffers
static void free_mesh2(tpm_ctx *c) {
  quiesce(c);
  dfree(c->arena, c->rho2);
  dfree(c->arena, c->spec2);
  dfree(c->arena, c->phi2);
  dfree(c->arena, c->gt);
  c->rho2 = nullptr;
  c->spec2 = nullptr;
  c->phi2 = nullptr;
  c->gt = nullptr;
  c->gt_rs = -1.f;
}

// The second (half-cell-shifted) grid of the Gaussian law's interlaced PM and
// the pair's influence function for the current split scale.
static int ensure_mesh2(tpm_ctx *c) {
  if (c->prm.law != TPM_LAW_GAUSSIAN) return 0;
  const MeshGeom &g = c->g;
  if (c->rho2) {
    if (c->gt_rs != c->prm.rs_split) {
      launch_green_opt(c->gt, g.n, (double)c->prm.rs_split, c->st);
      CK(cudaGetLastError());
      c->gt_rs = c->prm.rs_split;
      c->gen++;
    }
    return 0;
  }
  CK(dmalloc(c->arena, &c->gt, sizeof(float) * (int64_t)g.n * g.hx * g.n));
  launch_green_opt(c->gt, g.n, (double)c->prm.rs_split, c->st);
  CK(cudaGetLastError());
  c->gt_rs = c->prm.rs_split;
  int64_t n3 = (int64_t)g.n * g.n * g.n;
  CK(dmalloc(c->arena, &c->rho2, sizeof(float) * n3));
  CK(dmalloc(c->arena, &c->spec2, sizeof(float2) * g.spec_elems));
  CK(dmalloc(c->arena, &c->phi2, sizeof(float) * (int64_t)g.px * g.py * g.pz));
  CK(cudaMemsetAsync(c->phi2, 0, sizeof(float) * (int64_t)g.px * g.py * g.pz, c->st));
  if (make_phi_tensor_map(g, c->phi2, 4, &c->tmap4b) != 0) return fail(TPM_E_CUDA, "cuTensorMapEncodeTiled failed");
  c->gen++;
  return 0;
}

static void free_mesh(tpm_ctx *c) {
  free_mesh2(c);
  dfree(c->arena, c->pk_acc);
  c->pk_acc = nullptr;
  c->measure_pk = false;
  dfree(c->arena, c->rho);
  dfree(c->arena, c->spec);
  dfree(c->arena, c->phi);
  dfree(c->arena, c->tile_start);
  dfree(c->arena, c->cube_start);
  dfree(c->arena, c->tb.cube_node);
  dfree(c->arena, c->tb.start_cube);
  c->tb.cube_node = c->tb.start_cube = nullptr;
  c->tb.ncubes4 = 0;
  fft_plan_free(c->fp);
  c->rho = nullptr;
  c->spec = nullptr;
  c->phi = nullptr;
  c->tile_start = nullptr;
  c->cube_start = nullptr;
}

static int alloc_mesh(tpm_ctx *c) {
  // buffers about to be freed may still be read by queued work
  CK(cudaStreamSynchronize(c->st));
  free_mesh(c);
  c->g = make_geom(c->prm.n_mesh);
  const MeshGeom &g = c->g;
  int64_t n3 = (int64_t)g.n * g.n * g.n;
  CK(dmalloc(c->arena, &c->rho, sizeof(float) * n3));
  CK(dmalloc(c->arena, &c->spec, sizeof(float2) * g.spec_elems));
  CK(dmalloc(c->arena, &c->phi, sizeof(float) * (int64_t)g.px * g.py * g.pz));
  CK(cudaMemsetAsync(c->phi, 0, sizeof(float) * (int64_t)g.px * g.py * g.pz, c->st));
  uint32_t ntiles = 1u << (3 * (g.cbits - 3));
  CK(dmalloc(c->arena, &c->tile_start, sizeof(uint32_t) * (ntiles + 1)));
  c->ncubes = 1ll << (3 * (g.cbits - 2));
  CK(dmalloc(c->arena, &c->cube_start, sizeof(uint32_t) * (c->ncubes + 1)));
  c->tb.ncubes4 = c->ncubes;
  CK(dmalloc(c->arena, &c->tb.cube_node, sizeof(uint32_t) * c->ncubes));
  CK(dmalloc(c->arena, &c->tb.start_cube, sizeof(uint32_t) * (c->ncubes + 1)));
  CK(fft_plan_init(c->fp, g.n, c->st, c->arena));
  if (make_phi_tensor_map(g, c->phi, 2, &c->tmap2) != 0 || make_phi_tensor_map(g, c->phi, 4, &c->tmap4) != 0)
    return fail(TPM_E_CUDA, "cuTensorMapEncodeTiled failed");
  CK(cudaGetLastError());
  // the set-up kernels ran on the context stream, ahead of any evaluation
  c->gen++;
  return 0;
}

static void free_particles(tpm_ctx *c) {
  void *ps[] = {c->pos, c->vel, c->key, c->key_alt, c->val, c->val_alt, c->spos, c->fpm, c->ftree, c->fout,
                c->ss.hist, c->ss.dtotal, c->tb.start, c->tb.count, c->tb.child, c->tb.nchild, c->tb.level, c->tb.geo,
                c->tb.mom0, c->tb.mom1, c->tb.mom2, c->tb.walkA, c->tb.walkB, c->tb.tile_sum, c->tb.groups};
  quiesce(c);
  for (void *p : ps)
    dfree(c->arena, p);
  c->pos = nullptr;
  c->vel = nullptr;
  c->key = c->key_alt = nullptr;
  c->val = c->val_alt = nullptr;
  c->spos = nullptr;
  c->fpm = c->ftree = c->fout = nullptr;
  c->ss.hist = nullptr;
  c->ss.dtotal = nullptr;
  c->tb.start = c->tb.count = c->tb.child = c->tb.nchild = nullptr;
  c->tb.level = nullptr;
  c->tb.geo = nullptr;
  c->tb.mom0 = c->tb.mom1 = c->tb.mom2 = nullptr;
  c->tb.walkA = c->tb.walkB = nullptr;
  c->tb.tile_sum = nullptr;
  c->tb.groups = nullptr;
  c->cap = 0;
}

static int ensure_particles(tpm_ctx *c, int64_t np) {
  if (np <= c->cap) return 0;
  CK(cudaStreamSynchronize(c->st));
  free_particles(c);
  c->gen++;
  int64_t cap = np;
  CK(dmalloc(c->arena, &c->pos, sizeof(uint32_t) * 3 * cap));
  CK(dmalloc(c->arena, &c->vel, sizeof(float) * 3 * cap));
  CK(dmalloc(c->arena, &c->key, sizeof(uint64_t) * cap));
  CK(dmalloc(c->arena, &c->key_alt, sizeof(uint64_t) * cap));
  CK(dmalloc(c->arena, &c->val, sizeof(uint32_t) * cap));
  CK(dmalloc(c->arena, &c->val_alt, sizeof(uint32_t) * cap));
  CK(dmalloc(c->arena, &c->spos, sizeof(uint32_t) * 3 * cap));
  CK(dmalloc(c->arena, &c->fpm, sizeof(float) * 3 * cap));
  CK(dmalloc(c->arena, &c->ftree, sizeof(float) * 3 * cap));
  CK(dmalloc(c->arena, &c->fout, sizeof(float) * 3 * cap));
  int64_t ntiles = sort_tiles(cap);
  CK(dmalloc(c->arena, &c->ss.hist, sizeof(uint32_t) * 256 * (ntiles + 1)));
  CK(dmalloc(c->arena, &c->ss.dtotal, sizeof(uint32_t) * 256));
  c->ss.cap_tiles = ntiles;
  // tree: every node holds >= 1 particle and every inner node >= 10, so the
  // node count is bounded by the leaves (<= np) plus the inner nodes
  int64_t cap_nodes = cap + cap / 4 + 64;
  TreeBuffers &tb = c->tb;
  tb.cap_nodes = cap_nodes;
  CK(dmalloc(c->arena, &tb.start, sizeof(uint32_t) * cap_nodes));
  CK(dmalloc(c->arena, &tb.count, sizeof(uint32_t) * cap_nodes));
  CK(dmalloc(c->arena, &tb.child, sizeof(uint32_t) * cap_nodes));
  CK(dmalloc(c->arena, &tb.nchild, sizeof(uint32_t) * cap_nodes));
  CK(dmalloc(c->arena, &tb.level, sizeof(uint8_t) * cap_nodes));
  CK(dmalloc(c->arena, &tb.geo, sizeof(uint4) * cap_nodes));
  CK(dmalloc(c->arena, &tb.mom0, sizeof(float4) * cap_nodes));
  CK(dmalloc(c->arena, &tb.mom1, sizeof(float4) * cap_nodes));
  CK(dmalloc(c->arena, &tb.mom2, sizeof(float4) * cap_nodes));
  CK(dmalloc(c->arena, &tb.walkA, sizeof(uint4) * 2 * cap_nodes));
  CK(dmalloc(c->arena, &tb.walkB, sizeof(uint4) * cap_nodes));
  int64_t ts = (cap_nodes + 1023) / 1024 + 16;
  int64_t need_groups = 2 * c->ncubes + (c->ncubes + 4095) / 4096 + 16;
  if (ts < need_groups) ts = need_groups;
  tb.cap_tiles = ts;
  CK(dmalloc(c->arena, &tb.tile_sum, sizeof(uint32_t) * ts));
  tb.cap_groups = cap / 1 + c->ncubes + 16;
  CK(dmalloc(c->arena, &tb.groups, sizeof(uint32_t) * 2 * tb.cap_groups));
  c->cap = cap;
  return 0;
}

// ------------------------------------------------------------------ kernels
namespace {

__global__ void k_decode_lagrangian(const uint8_t *__restrict__ rec, int64_t np, int64_t stride, int64_t oi,
                                    int64_t op, int64_t ov, int n, uint32_t *__restrict__ pos,
                                    float *__restrict__ vel) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t *r = rec + i * stride;
    uint64_t idx;
    memcpy(&idx, r + oi, 8);
    idx = (idx << 8) >> 8;  // PINDX: drop the flag byte (eunha.h:1212)
    float off[3];
    memcpy(off, r + op, 12);
    uint64_t N = (uint64_t)n;
    uint64_t grid[3] = {idx % N, (idx % (N * N)) / N, idx / (N * N)};
    for (int a = 0; a < 3; a++) {
      // XofP: fmod(offset + grid + N, N) (eunha.h:1228-1232), then fixed point
      double x = fmod((double)off[a] + (double)grid[a] + (double)n, (double)n);
      double fr = x / (double)n;
      fr -= floor(fr);
      double u = rint(fr * 4294967296.0);
      if (u >= 4294967296.0) u = 0.0;
      pos[3 * i + a] = (uint32_t)(unsigned long long)u;
    }
    if (ov >= 0) {
      float v[3];
      memcpy(v, r + ov, 12);
      vel[3 * i + 0] = v[0];
      vel[3 * i + 1] = v[1];
      vel[3 * i + 2] = v[2];
    } else {
      vel[3 * i + 0] = vel[3 * i + 1] = vel[3 * i + 2] = 0.f;
    }
  }
}

__global__ void k_store_vel(const float *__restrict__ vel, int64_t np, int64_t stride, int64_t ov,
                            uint8_t *__restrict__ rec) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    memcpy(rec + i * stride + ov, vel + 3 * i, 12);
  }
}

__global__ void k_finish(const uint32_t *__restrict__ perm, int64_t np, const float *__restrict__ fpm,
                         const float *__restrict__ ftree, unsigned parts, float *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    float f[3] = {0.f, 0.f, 0.f};
    if (parts & TPM_PART_PM)
      for (int a = 0; a < 3; a++) f[a] += fpm[3 * i + a];
    if (parts & TPM_PART_TREE)
      for (int a = 0; a < 3; a++) f[a] += ftree[3 * i + a];
    int64_t j = perm[i];
    out[3 * j + 0] = f[0];
    out[3 * j + 1] = f[1];
    out[3 * j + 2] = f[2];
  }
}

// v += fact2_pm F_pm + fact2_tree F_tree, in the caller's particle order. The
// step graph passes fac (fac[1] = fact2 for both parts, each part applied if
// it was evaluated).
__global__ void k_kick(const uint32_t *__restrict__ perm, int64_t np, const float *__restrict__ fpm,
                       const float *__restrict__ ftree, float f2pm, float f2tree, float *__restrict__ vel,
                       const double *__restrict__ fac, unsigned parts) {
  if (fac) {
    float f2 = (float)fac[1];
    f2pm = (parts & TPM_PART_PM) ? f2 : 0.f;
    f2tree = (parts & TPM_PART_TREE) ? f2 : 0.f;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = perm[i];
    for (int a = 0; a < 3; a++) {
      float v = vel[3 * j + a];
      if (f2pm != 0.f) v += f2pm * fpm[3 * i + a];
      if (f2tree != 0.f) v += f2tree * ftree[3 * i + a];
      vel[3 * j + a] = v;
    }
  }
}

// x += v * pfact (cells) in FP64, onto the exact periodic fixed point.
__global__ void k_drift(uint32_t *__restrict__ pos, const float *__restrict__ vel, int64_t np, double pfact,
                        double units_per_cell, const double *__restrict__ fac) {
  if (fac) pfact = fac[2];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * np; i += (int64_t)gridDim.x * blockDim.x) {
    double d = (double)vel[i] * pfact * units_per_cell;
    double m = fmod(d, 4294967296.0);
    long long s = llrint(m);
    pos[i] = pos[i] + (uint32_t)(unsigned long long)s;
  }
}

// Hubble drag v *= fact1 (HubbleDragDM, Cosmos/globalT.c:102-110).
__global__ void k_drag(float *__restrict__ vel, int64_t n3, float f, const double *__restrict__ fac) {
  if (fac) f = (float)fac[0];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x)
    vel[i] *= f;
}

int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 32) b = 148 * 32;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

int tpm::launch_finish(tpm_ctx *c, cudaStream_t st) {
  k_finish<<<grid_for(c->np), 256, 0, st>>>(c->perm, c->np, c->fpm, c->ftree, TPM_PART_ALL, c->fout);
  CK(cudaGetLastError());
  return 0;
}

int tpm::ensure_particles_for(tpm_ctx *c, int64_t np) { return ensure_particles(c, np); }

int tpm::launch_finish_to(tpm_ctx *c, cudaStream_t st, unsigned parts, float *out) {
  k_finish<<<grid_for(c->np), 256, 0, st>>>(c->perm, c->np, c->fpm, c->ftree, parts, out);
  CK(cudaGetLastError());
  return 0;
}

WalkBox tpm::ctx_walk_box(const tpm_ctx *c) {
  TreeParams tp;
  tp.n = (uint32_t)c->g.n;
  tp.sub_bits = c->g.sub_bits;
  tp.theta2 = c->prm.theta * c->prm.theta;
  tp.rsphere = c->prm.rsphere;
  tp.cell_per_unit = (float)((double)c->g.n / 4294967296.0);
  tp.mass = c->prm.particle_mass;
  return walk_box(tp, c->spos, c->tb, c->ftree, c->err);
}

int64_t tpm::ctx_bytes(int n_mesh, int64_t np) {
  // the allocations of tpm_create, alloc_mesh and ensure_particles
  MeshGeom g = make_geom(n_mesh);
  int64_t n3 = (int64_t)g.n * g.n * g.n;
  // both grids of the interlaced pair (the Gaussian law's second grid)
  int64_t mesh = 2 * (4 * n3 + 8 * g.spec_elems + 4 * (int64_t)g.px * g.py * g.pz) + 4 * g.spec_elems;
  int64_t ntiles = 1ll << (3 * (g.cbits - 3)), ncubes = 1ll << (3 * (g.cbits - 2));
  mesh += 4 * (ntiles + 1) + 3 * 4 * (ncubes + 1) + 8 * (int64_t)(n_mesh + n_mesh / 2 + 1);
  int64_t parts = np * (12 + 12 + 8 + 8 + 4 + 4 + 12 + 12 + 12 + 12) + 4 * 256 * (sort_tiles(np) + 1) + 1024;
  int64_t cap_nodes = np + np / 4 + 64;
  int64_t tree = cap_nodes * (4 + 4 + 4 + 4 + 1 + 16 + 3 * 16 + 32 + 16);
  int64_t ts = (cap_nodes + 1023) / 1024 + 16, need = 2 * ncubes + (ncubes + 4095) / 4096 + 16;
  tree += 4 * (ts > need ? ts : need) + 8 * (np + ncubes + 16);
  int64_t fixed = 4 * walk_stack_words() + 8 * 4097 + 16 * 4096 + 4096;
  return mesh + parts + tree + fixed;
}

int tpm::launch_drag(tpm_ctx *c, cudaStream_t st, float fact1, const double *fac) {
  k_drag<<<grid_for(3 * c->np), 256, 0, st>>>(c->vel, 3 * c->np, fact1, fac);
  CK(cudaGetLastError());
  return 0;
}

int tpm::launch_kick(tpm_ctx *c, cudaStream_t st, float f2pm, float f2tree, const double *fac) {
  k_kick<<<grid_for(c->np), 256, 0, st>>>(c->perm, c->np, c->fpm, c->ftree, f2pm, f2tree, c->vel, fac,
                                          TPM_PART_ALL);
  CK(cudaGetLastError());
  return 0;
}

int tpm::launch_drift(tpm_ctx *c, cudaStream_t st, double pfact, const double *fac) {
  double upc = 4294967296.0 / (double)c->prm.n_mesh;
  k_drift<<<grid_for(3 * c->np), 256, 0, st>>>(c->pos, c->vel, c->np, pfact, upc, fac);
  CK(cudaGetLastError());
  return 0;
}

extern "C" {

int tpm_device_count(void) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return ndev;
}

int tpm_create(const tpm_params *params, int device, tpm_ctx **out) {
  return tpm::create_ctx(params, device, nullptr, out);
}

}  // extern "C"

int tpm::create_ctx(const tpm_params *params, int device, DeviceArena *arena, tpm_ctx **out) {
  if (!out) return fail(TPM_E_ARG, "out is NULL");
  *out = nullptr;
  int rc = check_params(params);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return fail(TPM_E_NODEV, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return fail(TPM_E_ARG, "device %d out of range", device);
  CK(cudaSetDevice(device));
  tpm_ctx *c = new tpm_ctx();
  c->prm = *params;
  c->device = device;
  c->arena = arena;
  memset(c->stage_ms, 0, sizeof(c->stage_ms));
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(TPM_E_CUDA, "cudaStreamCreate failed");
  }
  for (int i = 0; i <= kNStages; i++) cudaEventCreate(&c->ev[i]);
  {
    if (cudaStreamCreateWithFlags(&c->st_pm, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
      tpm_destroy(c);
      return fail(TPM_E_CUDA, "stream or event creation failed");
    }
  }
  // the allocations below are mirrored by ctx_bytes()
  if (dmalloc(c->arena, &c->err, sizeof(uint32_t) * 8) != cudaSuccess ||
      dmalloc(c->arena, &c->tb.counters, sizeof(uint32_t) * 16) != cudaSuccess ||
      dmalloc(c->arena, &c->tb.level_range, sizeof(uint32_t) * 2 * (kAxisBits + 2)) != cudaSuccess ||
      dmalloc(c->arena, &c->tb.walkbox, sizeof(WalkBox)) != cudaSuccess) {
    tpm_destroy(c);
    return fail(TPM_E_NOMEM, "cudaMalloc of context scratch failed");
  }
  c->tb.stack_words = walk_stack_words();
  if (dmalloc(c->arena, &c->tb.stack, sizeof(uint32_t) * c->tb.stack_words) != cudaSuccess) {
    tpm_destroy(c);
    return fail(TPM_E_NOMEM, "cudaMalloc of walk stacks failed");
  }
  if (cudaMallocHost(&c->herr, sizeof(uint32_t) * 8) != cudaSuccess ||
      cudaMallocHost(&c->hfac, sizeof(double) * kFacWords) != cudaSuccess ||
      dmalloc(c->arena, &c->dfac, sizeof(double) * kFacWords) != cudaSuccess) {
    tpm_destroy(c);
    return fail(TPM_E_NOMEM, "allocation of step scratch failed");
  }
  memset(c->herr, 0, sizeof(uint32_t) * 8);
  memset(c->hfac, 0, sizeof(double) * kFacWords);
  cudaMemsetAsync(c->err, 0, sizeof(uint32_t) * 8, c->st);
  rc = alloc_mesh(c);
  if (!rc) rc = ensure_mesh2(c);
  if (!rc) rc = build_law(c);
  if (rc) {
    std::string m = g_err;
    tpm_destroy(c);
    return fail(rc, "%s", m.c_str());
  }
  *out = c;
  return 0;
}

extern "C" {

int tpm_destroy(tpm_ctx *c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  quiesce(c);
  free_stream_state(c);
  free_particles(c);
  free_mesh(c);
  dfree(c->arena, c->law.tlog);
  dfree(c->arena, c->law.tpc);
  dfree(c->arena, c->err);
  dfree(c->arena, c->tb.counters);
  dfree(c->arena, c->tb.level_range);
  dfree(c->arena, c->tb.walkbox);
  dfree(c->arena, c->tb.stack);
  dfree(c->arena, c->stage);
  for (CapturedGraph &gr : c->graphs) {
    if (gr.exec) cudaGraphExecDestroy(gr.exec);
    if (gr.graph) cudaGraphDestroy(gr.graph);
  }
  if (c->herr) cudaFreeHost(c->herr);
  if (c->hfac) cudaFreeHost(c->hfac);
  dfree(c->arena, c->dfac);
  for (int i = 0; i <= kNStages; i++)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->st_pm) cudaStreamDestroy(c->st_pm);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return 0;
}

int tpm_set_params(tpm_ctx *c, const tpm_params *p) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  int rc = check_params(p);
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  bool remesh = p->n_mesh != c->prm.n_mesh;
  if (memcmp(p, &c->prm, sizeof(*p)) != 0) c->gen++;
  c->prm = *p;
  if (remesh) {
    CK(cudaStreamSynchronize(c->st));
    free_particles(c);
    c->np = 0;
    rc = alloc_mesh(c);
    if (rc) return rc;
  }
  rc = ensure_mesh2(c);
  if (rc) return rc;
  c->parts_valid = 0;
  return build_law(c);
}

int tpm_get_params(const tpm_ctx *c, tpm_params *out) {
  if (!c || !out) return fail(TPM_E_ARG, "NULL argument");
  *out = c->prm;
  return 0;
}

void *tpm_stream(tpm_ctx *c) { return c ? (void *)c->st : nullptr; }

static cudaMemcpyKind kind_in(int mem) { return mem == TPM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice; }
static cudaMemcpyKind kind_out(int mem) { return mem == TPM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost; }

int tpm_load_fixed(tpm_ctx *c, int64_t np, const uint32_t *pos, const float *vel, int mem) {
  if (!c || !pos || np <= 0) return fail(TPM_E_ARG, "bad arguments to tpm_load_fixed");
  if (np > 0xffffffffll - 64) return fail(TPM_E_ARG, "np %lld too large", (long long)np);
  CK(cudaSetDevice(c->device));
  int rc = ensure_particles(c, np);
  if (rc) return rc;
  c->np = np;
  CK(cudaMemcpyAsync(c->pos, pos, sizeof(uint32_t) * 3 * np, kind_in(mem), c->st));
  if (vel)
    CK(cudaMemcpyAsync(c->vel, vel, sizeof(float) * 3 * np, kind_in(mem), c->st));
  else
    CK(cudaMemsetAsync(c->vel, 0, sizeof(float) * 3 * np, c->st));
  c->parts_valid = 0;
  return 0;
}

static int ensure_stage(tpm_ctx *c, size_t bytes) {
  if (bytes <= c->stage_bytes) return 0;
  if (c->stage) quiesce(c);
  dfree(c->arena, c->stage);
  c->stage = nullptr;
  c->stage_bytes = 0;
  CK(dmalloc(c->arena, &c->stage, bytes));
  c->stage_bytes = bytes;
  return 0;
}

int tpm_load_lagrangian(tpm_ctx *c, int64_t np, const void *particles, int64_t stride, int64_t off_indx,
                        int64_t off_pos, int64_t off_vel, int mem) {
  if (!c || !particles || np <= 0 || stride < 20 || off_indx < 0 || off_pos < 0 || off_indx + 8 > stride ||
      off_pos + 12 > stride || (off_vel >= 0 && off_vel + 12 > stride))
    return fail(TPM_E_ARG, "bad arguments to tpm_load_lagrangian");
  CK(cudaSetDevice(c->device));
  int rc = ensure_particles(c, np);
  if (rc) return rc;
  c->np = np;
  const uint8_t *src = (const uint8_t *)particles;
  if (mem != TPM_MEM_DEVICE) {
    rc = ensure_stage(c, (size_t)np * stride);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->stage, particles, (size_t)np * stride, cudaMemcpyHostToDevice, c->st));
    src = (const uint8_t *)c->stage;
  }
  k_decode_lagrangian<<<grid_for(np), 256, 0, c->st>>>(src, np, stride, off_indx, off_pos, off_vel,
                                                       c->prm.n_mesh, c->pos, c->vel);
  CK(cudaGetLastError());
  c->parts_valid = 0;
  return 0;
}

}  // extern "C"

int tpm::enqueue_forces(tpm_ctx *c, unsigned parts, cudaStream_t st, bool timing, bool walk) {
  const MeshGeom &g = c->g;
  int64_t np = c->np;
  c->launches = 0;
  CK(cudaMemsetAsync(c->err, 0, sizeof(uint32_t) * 8, st));
  if (timing) CK(cudaEventRecord(c->ev[0], st));
  // ---- sort
  launch_make_keys(c->pos, np, (uint32_t)g.n, g.sub_bits, c->key, c->val, st);
  uint64_t *k = c->key;
  uint32_t *v = c->val;
  uint64_t *kalt = c->key_alt;
  uint32_t *valt = c->val_alt;
  radix_sort_pairs(&k, &v, kalt, valt, np, kKeyBits, c->ss, st, &c->launches);
  c->skey = k;
  c->perm = v;
  launch_gather_pos(c->pos, c->perm, np, c->spos, st);
  c->launches += 2;
  CK(stage_check(st, "sort"));
  if (timing) CK(cudaEventRecord(c->ev[1], st));
  // ---- PM: with both parts, on st_pm beside the tree build
  bool split = (parts & TPM_PART_PM) && (parts & TPM_PART_TREE);
  c->overlapped = split;
  cudaStream_t pst = st;
  if (split) {
    CK(cudaEventRecord(c->ev_fork, st));
    CK(cudaStreamWaitEvent(c->st_pm, c->ev_fork, 0));
    pst = c->st_pm;
  }
  if (parts & TPM_PART_PM) {
    uint32_t ntiles = 1u << (3 * (g.cbits - 3));
    launch_range_table(c->skey, np, 3 * (g.sub_bits + 3), ntiles, c->tile_start, pst);
    CK(cudaMemsetAsync(c->rho, 0, sizeof(float) * (int64_t)g.n * g.n * g.n, pst));
    const bool il = c->prm.law == TPM_LAW_GAUSSIAN;  // interlaced pair of grids
    if (il) CK(cudaMemsetAsync(c->rho2, 0, sizeof(float) * (int64_t)g.n * g.n * g.n, pst));
    launch_tsc_deposit(g, c->spos, c->tile_start, c->prm.particle_mass, c->rho, pst, il ? c->rho2 : nullptr);
    c->launches += 2;
    CK(stage_check(pst, "deposit"));
    if (timing) CK(cudaEventRecord(c->ev[2], pst));
    double *pk = c->measure_pk ? c->pk_acc : nullptr;
    if (pk) CK(cudaMemsetAsync(pk, 0, sizeof(double) * 2 * (g.n + 1), pst));
    if (il)
      launch_poisson(g, c->fp, c->rho, c->spec, c->phi, c->prm.law, c->prm.efold, c->prm.rs_split, pst,
                     &c->launches, c->rho2, c->spec2, c->phi2, c->gt, c->tune_fft_px, c->tune_fft_tx, pk);
    else
      launch_poisson(g, c->fp, c->rho, c->spec, c->phi, c->prm.law, c->prm.efold, c->prm.rs_split, pst,
                     &c->launches, nullptr, nullptr, nullptr, nullptr, c->tune_fft_px, c->tune_fft_tx, pk);
    CK(stage_check(pst, "fft"));
    if (timing) CK(cudaEventRecord(c->ev[3], pst));
    // the reference law keeps the reference's 4-point gradient; the Gaussian
    // law uses the 8-point one on both interlaced grids and averages
    if (c->prm.law == TPM_LAW_REFERENCE) {
      launch_fda4(g, &c->tmap2, 2, c->spos, c->tile_start, c->fpm, c->err, pst);
      c->launches += 1;
    } else {
      launch_fda4_pair(g, &c->tmap4, &c->tmap4b, c->spos, c->tile_start, c->fpm, c->err, pst);
      c->launches += 1;
    }
    CK(stage_check(pst, "fda4"));
    if (timing) CK(cudaEventRecord(c->ev[4], pst));
  } else if (timing) {
    for (int i = 2; i <= 4; i++) CK(cudaEventRecord(c->ev[i], pst));
  }
  if (split) CK(cudaEventRecord(c->ev_join, pst));
  // ---- tree
  if (parts & TPM_PART_TREE) {
    TreeParams tp;
    tp.n = (uint32_t)g.n;
    tp.sub_bits = g.sub_bits;
    tp.theta2 = c->prm.theta * c->prm.theta;
    tp.rsphere = c->prm.rsphere;
    tp.cell_per_unit = (float)((double)g.n / 4294967296.0);
    tp.mass = c->prm.particle_mass;
    tp.group_max = c->tune_group_max;
    tree_build(tp, c->skey, c->spos, np, c->tb, c->err, st, &c->launches);
    CK(cudaMemsetAsync(c->tb.counters, 0, sizeof(uint32_t) * 16, st));
    int glev = c->tune_group_level;
    int64_t gcubes = 1ll << (3 * (g.cbits - glev));
    tree_groups(tp, c->skey, np, c->tb, c->cube_start, gcubes, 3 * (g.sub_bits + glev), st, &c->launches);
    CK(stage_check(st, "tree_build"));
    // the walk takes every SM: it starts once the PM chain is done too (the
    // tree_build stage of an overlapped evaluation ends with both chains)
    if (split) {
      CK(cudaStreamWaitEvent(st, c->ev_join, 0));
      split = false;
    }
    if (timing) CK(cudaEventRecord(c->ev[5], st));
    if (walk) tree_walk(tp, c->spos, np, c->tb, c->law, c->ftree, c->err, st, &c->launches);
    CK(stage_check(st, "tree_walk"));
    if (timing) CK(cudaEventRecord(c->ev[6], st));
  } else if (timing) {
    for (int i = 5; i <= 6; i++) CK(cudaEventRecord(c->ev[i], st));
  }
  if (split) CK(cudaStreamWaitEvent(st, c->ev_join, 0));
  if (timing) CK(cudaEventRecord(c->ev[7], st));
  CK(cudaGetLastError());
  return 0;
}

int tpm::finish_forces(tpm_ctx *c, unsigned parts, bool from_host, bool timing) {
  uint32_t herr[8];
  if (from_host) {
    memcpy(herr, c->herr, sizeof(herr));
  } else {
    CK(cudaMemcpyAsync(herr, c->err, sizeof(herr), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  if (herr[0]) {
    c->parts_valid = 0;
    if (herr[0] & kErrNodeOverflow) return fail(TPM_E_OVERFLOW, "tree node capacity exceeded");
    if (herr[0] & kErrStackOverflow) return fail(TPM_E_OVERFLOW, "tree-walk stack overflow");
    if (herr[0] & kErrTmaTimeout) return fail(TPM_E_CUDA, "TMA load timed out in fda4");
    return fail(TPM_E_CUDA, "device error flags 0x%x", herr[0]);
  }
  if (timing) {
    for (int s = 0; s < kNStages; s++) {
      // beside the PM chain, the tree build starts at the end of the sort
      int s0 = (s == kStTreeBuild && c->overlapped) ? kStDeposit : s;
      float ms = 0;
      cudaEventElapsedTime(&ms, c->ev[s0], c->ev[s + 1]);
      c->stage_ms[s] = ms;
    }
    // counters: nodes, pp, pc, groups
    uint32_t hc[12];
    uint32_t lr[2 * (kAxisBits + 2)];
    CK(cudaMemcpy(hc, c->tb.counters, sizeof(hc), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(lr, c->tb.level_range, sizeof(lr), cudaMemcpyDeviceToHost));
    uint32_t nn = 0;
    for (int l = 0; l <= kAxisBits; l++)
      if (lr[2 * l + 1] > nn) nn = lr[2 * l + 1];
    c->counters[0] = (parts & TPM_PART_TREE) ? nn : 0;
    c->counters[1] = (int64_t)(((uint64_t)hc[3] << 32) | hc[2]);
    c->counters[2] = (int64_t)(((uint64_t)hc[5] << 32) | hc[4]);
    c->counters[3] = hc[0];
    c->counters[4] = (int64_t)(((uint64_t)hc[7] << 32) | hc[6]);
    c->counters[5] = (int64_t)(((uint64_t)hc[9] << 32) | hc[8]);
    c->counters[6] = hc[10];
  }
  c->parts_valid = parts & TPM_PART_ALL;
  return 0;
}

extern "C" {

int tpm_compute_forces(tpm_ctx *c, unsigned parts) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  if ((parts & TPM_PART_ALL) == 0) return fail(TPM_E_ARG, "no force part requested");
  CK(cudaSetDevice(c->device));
  int rc = enqueue_forces(c, parts, c->st, true);
  if (rc) return rc;
  return finish_forces(c, parts, false, true);
}

int tpm_read_forces(tpm_ctx *c, float *out, int mem) {
  if (!c || !out) return fail(TPM_E_ARG, "NULL argument");
  if (!c->parts_valid) return fail(TPM_E_STATE, "no forces computed");
  CK(cudaSetDevice(c->device));
  // device memory takes the scatter to caller order directly; host memory
  // gets it through the context's buffer
  float *dst = mem == TPM_MEM_DEVICE ? out : c->fout;
  k_finish<<<grid_for(c->np), 256, 0, c->st>>>(c->perm, c->np, c->fpm, c->ftree, c->parts_valid, dst);
  CK(cudaGetLastError());
  if (dst != out) CK(cudaMemcpyAsync(out, c->fout, sizeof(float) * 3 * c->np, kind_out(mem), c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int tpm_kick(tpm_ctx *c, float fact2_pm, float fact2_tree) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  if (!c->parts_valid) return fail(TPM_E_STATE, "no forces computed");
  if (!(c->parts_valid & TPM_PART_PM)) fact2_pm = 0.f;
  if (!(c->parts_valid & TPM_PART_TREE)) fact2_tree = 0.f;
  CK(cudaSetDevice(c->device));
  return launch_kick(c, c->st, fact2_pm, fact2_tree, nullptr);
}

int tpm_drift(tpm_ctx *c, double pfact) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  CK(cudaSetDevice(c->device));
  int rc = launch_drift(c, c->st, pfact, nullptr);
  c->parts_valid = 0;
  return rc;
}

int tpm_read_velocities(tpm_ctx *c, float *out, int mem) {
  if (!c || !out) return fail(TPM_E_ARG, "NULL argument");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(out, c->vel, sizeof(float) * 3 * c->np, kind_out(mem), c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int tpm_read_positions(tpm_ctx *c, uint32_t *out, int mem) {
  if (!c || !out) return fail(TPM_E_ARG, "NULL argument");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(out, c->pos, sizeof(uint32_t) * 3 * c->np, kind_out(mem), c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

static int store_velocities(tpm_ctx *c, void *particles, int64_t stride, int64_t off_vel, int mem,
                            bool stage_holds_records) {
  if (!c || !particles || off_vel < 0 || off_vel + 12 > stride) return fail(TPM_E_ARG, "bad arguments");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  CK(cudaSetDevice(c->device));
  int64_t np = c->np;
  if (mem == TPM_MEM_DEVICE) {
    k_store_vel<<<grid_for(np), 256, 0, c->st>>>(c->vel, np, stride, off_vel, (uint8_t *)particles);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->st));
    return 0;
  }
  // the velocities go into a device copy of the record array, which then
  // replaces the caller's records: fields other than vx,vy,vz keep the
  // values of that copy
  int rc = ensure_stage(c, (size_t)np * stride);
  if (rc) return rc;
  if (!stage_holds_records)
    CK(cudaMemcpyAsync(c->stage, particles, (size_t)np * stride, cudaMemcpyHostToDevice, c->st));
  k_store_vel<<<grid_for(np), 256, 0, c->st>>>(c->vel, np, stride, off_vel, (uint8_t *)c->stage);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(particles, c->stage, (size_t)np * stride, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int tpm_store_lagrangian_velocities(tpm_ctx *c, void *particles, int64_t stride, int64_t off_vel, int mem) {
  return store_velocities(c, particles, stride, off_vel, mem, false);
}

int tpm_sync(tpm_ctx *c) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// ---- drop-in forms
int tpm_pmmain(tpm_ctx *c, void *dm, int64_t np, float fact2) {
  int rc = tpm_load_lagrangian(c, np, dm, 32, 0, 8, 20, TPM_MEM_HOST);
  if (!rc) rc = tpm_compute_forces(c, TPM_PART_PM);
  if (!rc) rc = tpm_kick(c, fact2, 0.f);
  if (!rc) rc = store_velocities(c, dm, 32, 20, TPM_MEM_HOST, true);
  return rc;
}

int tpm_treecorrection(tpm_ctx *c, void *tdm, int64_t np, float fact2) {
  int rc = tpm_load_lagrangian(c, np, tdm, 40, 8, 16, 28, TPM_MEM_HOST);
  if (!rc) rc = tpm_compute_forces(c, TPM_PART_TREE);
  if (!rc) rc = tpm_kick(c, 0.f, fact2);
  if (!rc) rc = store_velocities(c, tdm, 40, 28, TPM_MEM_HOST, true);
  return rc;
}

int tpm_treemain(tpm_ctx *c, void *tdm, int64_t np, float fact2, int stepcount) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  tpm_params p = c->prm;
  // Treemain.c:598-601
  p.theta = theta_schedule(stepcount);
  int rc = tpm_set_params(c, &p);
  if (!rc) rc = tpm_treecorrection(c, tdm, np, fact2);
  return rc;
}

int tpm_ewald(tpm_ctx *c, int64_t nt, const int64_t *targets, double *out) {
  if (!c || !targets || !out || nt <= 0) return fail(TPM_E_ARG, "bad arguments to tpm_ewald");
  if (c->np <= 0) return fail(TPM_E_STATE, "no particles loaded");
  for (int64_t i = 0; i < nt; i++)
    if (targets[i] < 0 || targets[i] >= c->np) return fail(TPM_E_ARG, "target index out of range");
  CK(cudaSetDevice(c->device));
  int rc = ewald_force(c->pos, c->np, c->prm.n_mesh, c->prm.epsilon, nt, targets, out, c->st);
  if (rc) return fail(TPM_E_CUDA, "Ewald kernels failed: %s", cudaGetErrorString(cudaGetLastError()));
  return 0;
}

int tpm_stage_times(tpm_ctx *c, float *ms, int n) {
  if (!c || !ms) return fail(TPM_E_ARG, "NULL argument");
  int k = n < kNStages ? n : kNStages;
  for (int i = 0; i < k; i++) ms[i] = c->stage_ms[i];
  return k;
}

int tpm_counters(tpm_ctx *c, int64_t *out, int n) {
  if (!c || !out) return fail(TPM_E_ARG, "NULL argument");
  int k = n < 7 ? n : 7;
  for (int i = 0; i < k; i++) out[i] = c->counters[i];
  return k;
}

int64_t tpm_launch_count(tpm_ctx *c) { return c ? c->launches : 0; }

int64_t tpm_estimate_bytes(int32_t n_mesh, int64_t np) {
  if (n_mesh < 16 || n_mesh > 4096 || np <= 0) return -1;
  return ctx_bytes(n_mesh, np);
}

int tpm_read_order(tpm_ctx *c, uint64_t *keys, uint32_t *perm) {
  if (!c) return fail(TPM_E_ARG, "ctx is NULL");
  if (!c->parts_valid || !c->perm) return fail(TPM_E_STATE, "no forces computed");
  CK(cudaSetDevice(c->device));
  if (keys) CK(cudaMemcpyAsync(keys, c->skey, sizeof(uint64_t) * c->np, cudaMemcpyDeviceToHost, c->st));
  if (perm) CK(cudaMemcpyAsync(perm, c->perm, sizeof(uint32_t) * c->np, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int tpm_read_mesh(tpm_ctx *c, int which, float *out) {
  if (!c || !out) return fail(TPM_E_ARG, "NULL argument");
  if (!(c->parts_valid & TPM_PART_PM)) return fail(TPM_E_STATE, "no PM evaluation");
  CK(cudaSetDevice(c->device));
  const MeshGeom &g = c->g;
  int64_t n = g.n;
  if (which == TPM_MESH_DENSITY) {
    CK(cudaMemcpyAsync(out, c->rho, sizeof(float) * n * n * n, cudaMemcpyDeviceToHost, c->st));
  } else if (which == TPM_MESH_POTENTIAL) {
    // interior of the ghosted potential: n rows of n per z plane at offset kGhost
    for (int64_t z = 0; z < n; z++)
      CK(cudaMemcpy2DAsync(out + z * n * n, sizeof(float) * n,
                           c->phi + kGhost + (int64_t)g.px * (kGhost + (int64_t)g.py * (kGhost + z)),
                           sizeof(float) * g.px, sizeof(float) * n, n, cudaMemcpyDeviceToHost, c->st));
  } else {
    return fail(TPM_E_ARG, "unknown mesh %d", which);
  }
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

}  // extern "C"
