// The GOTPM global step around the force evaluation: the evolution factors
// of an expanding background and the drag / kick / drift sequence.
//
// Reference: GetEvolFactor and GetFact1/GetFact2 (Cosmos/CosmosEvolFactor.c:
// 26-65,230-255) on HofEz/ap/gzDE (Cosmos/FLRW.c:27-71), integrated with the
// Numerical-Recipes Simpson/Romberg rules of Cosmos/mynr.c:10-86; the step of
// GOTPM_Cosmos_GlobalT (Cosmos/globalT.c:221-305): PM_PULL_AND_PUSH (Hubble
// drag v *= fact1, pmmain kick), TreeAndPreFoFmain (theta schedule, tree kick
// with fact2), onestepforwardposition (x += v * pfact, Cosmos/stepevolv.c:
// 19-29). The scalars are computed in float with the reference's mixed
// float/double expressions so that they agree with it bit for bit.
#include <math.h>
#include <string.h>

#include "ctx.cuh"

namespace {

struct Cosmo {
  float omep, omeplam, wlam0, wlam1, amax;
};

typedef float (*CFunc)(const Cosmo &, float);

float wlambda(const Cosmo &c, float red) { return c.wlam0 + c.wlam1 * red / (1 + red); }

float de_func(const Cosmo &c, float tau) {
  float red;
  if (tau == 0)
    red = 1.e20;
  else
    red = 1 / tau - 1;
  float result = 3 * (1 + wlambda(c, red)) * (1 + red);
  return result;
}

// Trapezoid refinement: stage n of the extended trapezoidal rule. The
// reference keeps the running sum in ONE static variable for every
// integration (Cosmos/mynr.c:67-85), so when a1ap's integrand itself
// integrates the dark-energy density (w1 != 0), the inner integration
// overwrites the outer one's running sum. That sharing is reproduced here:
// the factors must agree with the reference's for every cosmology it accepts.
thread_local float g_trap_sum = 0.f;

struct Trapzd {
  float step(CFunc f, const Cosmo &c, float a, float b, int n) {
    float &s = g_trap_sum;
    if (a == b) return 0.0;
    if (n == 1) return (s = 0.5 * (b - a) * (f(c, a) + f(c, b)));
    int it = 1;
    for (int j = 1; j < n - 1; j++) it <<= 1;
    float tnm = it;
    float del = (b - a) / tnm;
    float x = a + 0.5 * del;
    float sum = 0.0;
    for (int j = 1; j <= it; j++, x += del) sum += f(c, x);
    s = 0.5 * (s + (b - a) * sum / tnm);
    return s;
  }
};

// Simpson's rule by trapezoid refinement, relative tolerance 1e-4, 20 stages
float qsimp(CFunc f, const Cosmo &c, float a, float b) {
  const double eps = 1.0e-4;
  if (a == b) return 0.0;
  Trapzd tz;
  float ost = -1.0e30, os = -1.0e30;
  for (int j = 1; j <= 20; j++) {
    float st = tz.step(f, c, a, b, j);
    float s = (4.0 * st - ost) / 3.0;
    if (fabs(s - os) <= eps * fabs(os)) return s;
    os = s;
    ost = st;
  }
  return 0.0;
}

// Neville polynomial extrapolation to x through n points (1-based arrays)
void polint(const float *xa, const float *ya, int n, float x, float *y, float *dy) {
  int ns = 1;
  float c[8], d[8];
  float dif = fabs(x - xa[1]);
  for (int i = 1; i <= n; i++) {
    float dift = fabs(x - xa[i]);
    if (dift < dif) {
      ns = i;
      dif = dift;
    }
    c[i] = ya[i];
    d[i] = ya[i];
  }
  *y = ya[ns--];
  for (int m = 1; m < n; m++) {
    for (int i = 1; i <= n - m; i++) {
      float ho = xa[i] - x, hp = xa[i + m] - x;
      float w = c[i + 1] - d[i];
      float den = ho - hp;
      if (den == 0.0f) den = 1e-30f;
      den = w / den;
      d[i] = hp * den;
      c[i] = ho * den;
    }
    *y += (*dy = (2 * ns < (n - m) ? c[ns + 1] : d[ns--]));
  }
}

// Romberg integration, relative tolerance 1e-6, order 5, 20 stages
float qromb(CFunc f, const Cosmo &c, float a, float b) {
  const double eps = 1.0e-6;
  const int K = 5, JMAX = 20;
  float s[JMAX + 2], h[JMAX + 2];
  Trapzd tz;
  h[1] = 1.0;
  for (int j = 1; j <= JMAX; j++) {
    s[j] = tz.step(f, c, a, b, j);
    if (j >= K) {
      float ss, dss;
      polint(&h[j - K], &s[j - K], K, 0.0, &ss, &dss);
      if (fabs(dss) < eps * fabs(ss)) return ss;
    }
    s[j + 1] = s[j];
    h[j + 1] = 0.25 * h[j];
  }
  return 0.0;
}

float gz_de(const Cosmo &c, float anow) {
  float integral;
  if (c.wlam0 == -1 && c.wlam1 == 0) return 1;
  if (c.wlam1 == 0) return pow(c.amax / anow, 3. * (1 + c.wlam0));
  if (anow == c.amax) {
    integral = 0;
  } else if (anow == 0) {
    integral = qsimp(de_func, c, 0, 1);
  } else {
    float tau = anow / c.amax;
    if (tau < 0.8)
      integral = qsimp(de_func, c, tau, 1);
    else
      integral = qromb(de_func, c, tau, 1);
  }
  integral = exp(integral);
  return integral;
}

float hof_ez(const Cosmo &c, float anow) {
  float red = c.amax / anow - 1;
  float zp1 = red + 1;
  return sqrt(zp1 * zp1 * zp1 * c.omep + zp1 * zp1 * (1 - c.omep - c.omeplam) + c.omeplam * gz_de(c, anow));
}

float ap(const Cosmo &c, float anow) {
  float red = c.amax / anow - 1;
  float hofez = hof_ez(c, anow);
  float result = sqrt(8. * M_PI / 3. / (c.amax * c.omep) / ((red + 1) * (red + 1)) * hofez * hofez);
  return result;
}

float a1ap(const Cosmo &c, float a) { return 1. / (a * ap(c, a)); }

float get_fact2(const Cosmo &c, int nx, float a1, float a2) {
  float res1 = 1. / (a2 * a2 * ap(c, a2));
  float res2 = qsimp(a1ap, c, a1, a2);
  return res1 * res2 * nx;
}

float get_fact1(const Cosmo &c, float a1, float a2) {
  float h1 = hof_ez(c, a1);
  float h2 = hof_ez(c, a2);
  return (a1 * a1 * a1 * h1) / (a2 * a2 * a2 * h2);
}

}  // namespace

extern "C" {

int tpm_evol_factors(const tpm_cosmology *cosmo, int32_t nx, float anow, float astep, tpm_evolfact *out) {
  if (!cosmo || !out || nx <= 0 || !(anow > 0.f) || !(astep >= 0.f) || !(cosmo->amax > 0.f) ||
      !(cosmo->omep > 0.f)) {
    tpm::set_last_error("bad arguments to tpm_evol_factors");
    return TPM_E_ARG;
  }
  Cosmo c{cosmo->omep, cosmo->omeplam, cosmo->wlam0, cosmo->wlam1, cosmo->amax};
  tpm_evolfact e;
  e.afact = 0.f;
  e.bfact = 0.f;
  e.fact1 = get_fact1(c, anow - 0.5 * astep, anow + 0.5 * astep);
  e.fact2 = get_fact2(c, nx, anow - 0.5 * astep, anow + 0.5 * astep);
  e.pfact = astep * nx;
  e.fact1_push = get_fact1(c, anow, anow + 0.5 * astep);
  e.fact1_pull = get_fact1(c, anow - 0.5 * astep, anow);
  e.fact2_push = get_fact2(c, nx, anow, anow + 0.5 * astep);
  e.fact2_pull = get_fact2(c, nx, anow - 0.5 * astep, anow);
  // fda4's PUSH branch divides fact2_push by GetFact1(anow, anow + astep/2)
  // (Cosmos/fda4.c:49-54)
  *out = e;
  return 0;
}

int tpm_hubble_drag(tpm_ctx *ctx, float fact1) {
  if (!ctx) return tpm::fail(TPM_E_ARG, "ctx is NULL");
  if (ctx->np <= 0) return tpm::fail(TPM_E_STATE, "no particles loaded");
  CK(cudaSetDevice(ctx->device));
  return tpm::launch_drag(ctx, ctx->st, fact1, nullptr);
}

int tpm_step(tpm_ctx *ctx, const tpm_cosmology *cosmo, float anow, float astep, int32_t stepcount) {
  if (!ctx || !cosmo) return tpm::fail(TPM_E_ARG, "tpm_step: NULL argument");
  tpm_params p;
  int rc = tpm_get_params(ctx, &p);
  if (rc) return rc;
  tpm_evolfact e;
  rc = tpm_evol_factors(cosmo, p.n_mesh, anow, astep, &e);
  if (rc) return rc;
  if (p.law == TPM_LAW_REFERENCE) {
    float th = tpm::theta_schedule(stepcount);
    if (th != p.theta) {
      p.theta = th;
      rc = tpm_set_params(ctx, &p);
      if (rc) return rc;
    }
  }
  // KICK status: drag with fact1, both kicks with fact2 (fda4.c:60-61,
  // indT.h:104-117), then the drift
  rc = tpm_hubble_drag(ctx, e.fact1);
  if (!rc) rc = tpm_compute_forces(ctx, TPM_PART_ALL);
  if (!rc) rc = tpm_kick(ctx, e.fact2, e.fact2);
  if (!rc) rc = tpm_drift(ctx, e.pfact);
  return rc;
}

int tpm_status_factors(const tpm_evolfact *e, int32_t status, float *drag, float *pm_kick, float *tree_kick) {
  if (!e || (status != TPM_KICK && status != TPM_PULL && status != TPM_PUSH)) {
    tpm::set_last_error("bad arguments to tpm_status_factors");
    return TPM_E_ARG;
  }
  float f1, f2;
  if (status == TPM_PUSH) {
    // fda4 divides fact2_push by GetFact1(anow, anow + astep/2), the same
    // float call that made fact1_push
    f1 = e->fact1_push;
    f2 = e->fact2_push / e->fact1_push;
  } else if (status == TPM_PULL) {
    f1 = e->fact1_pull;
    f2 = e->fact2_pull;
  } else {
    f1 = e->fact1;
    f2 = e->fact2;
  }
  if (drag) *drag = f1;
  if (pm_kick) *pm_kick = f2;
  if (tree_kick) *tree_kick = e->fact2;
  return 0;
}

int tpm_status_kick(tpm_ctx *ctx, const tpm_cosmology *cosmo, float anow, float astep, int32_t status) {
  if (!ctx || !cosmo) return tpm::fail(TPM_E_ARG, "tpm_status_kick: NULL argument");
  if (ctx->np <= 0) return tpm::fail(TPM_E_STATE, "no particles loaded");
  tpm_evolfact e;
  int rc = tpm_evol_factors(cosmo, ctx->prm.n_mesh, anow, astep, &e);
  if (rc) return rc;
  float drag, f2pm, f2tree;
  rc = tpm_status_factors(&e, status, &drag, &f2pm, &f2tree);
  if (rc) return rc;
  // the drag does not move particles: forces of the current positions stay
  // valid across it
  rc = tpm_hubble_drag(ctx, drag);
  if (!rc && (ctx->parts_valid & TPM_PART_ALL) != TPM_PART_ALL) rc = tpm_compute_forces(ctx, TPM_PART_ALL);
  if (!rc) rc = tpm_kick(ctx, f2pm, f2tree);
  return rc;
}

int tpm_global_step(tpm_ctx *ctx, const tpm_cosmology *cosmo, float anow, float astep, int32_t stepcount,
                    int32_t sync) {
  if (!ctx || !cosmo) return tpm::fail(TPM_E_ARG, "tpm_global_step: NULL argument");
  if (!sync) return tpm_step(ctx, cosmo, anow, astep, stepcount);
  tpm_params p;
  int rc = tpm_get_params(ctx, &p);
  if (rc) return rc;
  if (p.law == TPM_LAW_REFERENCE) {
    float th = tpm::theta_schedule(stepcount);
    if (th != p.theta) {
      p.theta = th;
      rc = tpm_set_params(ctx, &p);
      if (rc) return rc;
    }
  }
  // a synchronisation step: PULL (the velocities reach anow), then PUSH on
  // the same positions and forces, then the drift (Cosmos/globalT.c:244-291)
  ctx->parts_valid = 0;
  rc = tpm_status_kick(ctx, cosmo, anow, astep, TPM_PULL);
  if (!rc) rc = tpm_status_kick(ctx, cosmo, anow, astep, TPM_PUSH);
  if (!rc) {
    tpm_evolfact e;
    rc = tpm_evol_factors(cosmo, p.n_mesh, anow, astep, &e);
    if (!rc) rc = tpm_drift(ctx, e.pfact);
  }
  return rc;
}

}  // extern "C"

float tpm::theta_schedule(int stepcount) {
  // TreeAndPreFoFmain (Cosmos/globalT.c:41-44), as TreeMain (Treemain.c:598-601)
  return stepcount < 10 ? 0.3f : (stepcount < 20 ? 0.35f : (stepcount < 60 ? 0.4f : 0.45f));
}

int tpm::step_factors(const tpm_ctx *c, const tpm_cosmology *cosmo, float anow, float astep,
                      double fac[kFacWords]) {
  tpm_evolfact e;
  int rc = tpm_evol_factors(cosmo, c->prm.n_mesh, anow, astep, &e);
  if (rc) return rc;
  fac[0] = (double)e.fact1;
  fac[1] = (double)e.fact2;
  fac[2] = (double)e.pfact;
  fac[3] = 0.0;
  return 0;
}
