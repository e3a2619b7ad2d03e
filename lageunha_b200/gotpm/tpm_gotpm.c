/* GOTPM's three force entry points with the reference's own signatures,
 * backed by the B200 engine (include/tpm_engine.h). Compile this file inside
 * EUNHA's source tree (it includes eunha.h and CosmosEvolFactor.h) in place
 * of the bodies it replaces, and link with lageunha_b200/libtpm_engine.so:
 *
 *   void pmmain(SimParameters *, EvolFact)            Cosmos/pmmain.c:390
 *   void treecorrection(SimParameters *, DeterminedEvolFact *)
 *                                                     Cosmos/treecorrection.c:225
 *   void TreeMain(SimParameters *, DeterminedEvolFact *)
 *                                                     Cosmos/Treemain.c:578-664 (GOTPM)
 *
 * globalT.c and stepevolv.c keep calling them unchanged
 * (Cosmos/globalT.c:85-87,131; Cosmos/indT.h:117; Cosmos/Treemain.c:659).
 * Like the reference, each call reads the particles' Lagrangian index and
 * float offsets (XYZDBL) from the rank's own arrays and adds fact2 * F to
 * vx, vy, vz in place; pmmain applies no drag (PM_PULL_AND_PUSH does that
 * before calling it). One engine context serves the process, created on the
 * first call on device TPM_GOTPM_DEVICE (environment) or MYID modulo the
 * device count, and kept in step with the SimParameters' mesh size, opening
 * angle, rsphere, softening, efold and particle mass. The reference exits on
 * an error; so does this file, after printing tpm_last_error(), unless it is
 * built with TPM_GOTPM_RECORD_ERRORS, which records the status for
 * tpm_gotpm_status() instead (for a harness that must keep running). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mpi.h>

#include "eunha.h"
#include "CosmosEvolFactor.h"
#include "tpm_engine.h"

static tpm_ctx *g_ctx = NULL;
static int g_status = 0;

/* The status of the last call (0 = ok); meaningful with
 * TPM_GOTPM_RECORD_ERRORS, where errors do not end the process. */
int tpm_gotpm_status(void) { return g_status; }

static int gotpm_check(int rc, const char *where) {
  g_status = rc;
  if (rc == TPM_OK) return 0;
  fprintf(stderr, "%s: tpm error %d: %s\n", where, rc, tpm_last_error());
#ifndef TPM_GOTPM_RECORD_ERRORS
  MPI_Finalize();
  exit(99);
#endif
  return rc;
}

/* The engine context for this SimParameters: made on first use, its
 * parameters updated when the caller's change (the reference law: the
 * PMFITPARA residual, psolver's Green's function, the 4-point gradient). */
static tpm_ctx *engine_for(SimParameters *simpar) {
  tpm_params p;
  tpm_default_params(&p, (int32_t)NX(simpar));
  p.law = TPM_LAW_REFERENCE;
  p.theta = THETA(simpar);
  p.rsphere = RSPHERE(simpar);
  p.epsilon = GRV_EPSILON(simpar);
  p.efold = GRV_EFOLD(simpar);
  p.particle_mass = TDM_MASS(simpar, 0);
  if (!g_ctx) {
    int dev;
    const char *env = getenv("TPM_GOTPM_DEVICE");
    int ndev = tpm_device_count();
    if (env && env[0])
      dev = atoi(env);
    else
      dev = ndev > 0 ? MYID(simpar) % ndev : 0;
    if (gotpm_check(tpm_create(&p, dev, &g_ctx), "tpm_create")) return NULL;
    return g_ctx;
  }
  tpm_params cur;
  if (gotpm_check(tpm_get_params(g_ctx, &cur), "tpm_get_params")) return NULL;
  if (memcmp(&cur, &p, sizeof(p)) != 0 && gotpm_check(tpm_set_params(g_ctx, &p), "tpm_set_params")) return NULL;
  return g_ctx;
}

/* Cosmos/pmmain.c:390. The PM kick factor is the one fda4 picks by
 * PMSTATUS (Cosmos/fda4.c:48-62): fact2, fact2_pull, or fact2_push divided
 * by GetFact1(anow, anow + astep/2) (tpm_status_factors). */
void pmmain(SimParameters *simpar, EvolFact evolfact) {
  tpm_evolfact e;
  e.afact = evolfact.afact;
  e.bfact = evolfact.bfact;
  e.pfact = evolfact.pfact;
  e.fact1 = evolfact.fact1;
  e.fact2 = evolfact.fact2;
  e.fact1_push = evolfact.fact1_push;
  e.fact2_push = evolfact.fact2_push;
  e.fact1_pull = evolfact.fact1_pull;
  e.fact2_pull = evolfact.fact2_pull;
  float f2;
  if (gotpm_check(tpm_status_factors(&e, PMSTATUS(simpar), NULL, &f2, NULL), "pmmain")) return;
  tpm_ctx *c = engine_for(simpar);
  if (!c) return;
  gotpm_check(tpm_pmmain(c, DM_BP(simpar), (int64_t)DM_NP(simpar), f2), "tpm_pmmain");
}

/* Cosmos/treecorrection.c:225: v += EvolFactArr[0].fact2 * F_tree
 * (treecorrection.c:227) with the opening angle THETA(simpar). */
void treecorrection(SimParameters *simpar, DeterminedEvolFact *EvolFactArr) {
  tpm_ctx *c = engine_for(simpar);
  if (!c) return;
  gotpm_check(tpm_treecorrection(c, DM_TBP(simpar), (int64_t)DM_NP(simpar), EvolFactArr[0].fact2),
              "tpm_treecorrection");
}

/* Cosmos/Treemain.c:578-664 (GOTPM): the opening-angle schedule of the step
 * count (Treemain.c:598-601), then the tree correction. */
void TreeMain(SimParameters *simpar, DeterminedEvolFact *evolfactor) {
  int s = STEPCOUNT(simpar);
  THETA(simpar) = s < 10 ? 0.3f : (s < 20 ? 0.35f : (s < 60 ? 0.4f : 0.45f));
  treecorrection(simpar, evolfactor);
}
