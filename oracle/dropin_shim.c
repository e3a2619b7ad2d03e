/* Test harness of the legacy-name drop-in (lageunha_b200/gotpm/tpm_gotpm.c)
 * — TEST INFRASTRUCTURE ONLY. It fills a one-rank SimParameters the way the
 * reference's own harness does (oracle/ref_shim.c), lays the particles out
 * as the reference's dmparticletype / treedmparticletype records, and calls
 * the drop-in's pmmain and TreeMain with the reference's signatures, so a
 * test can compare the velocities with those of the reference build. Built
 * by oracle/Makefile against the reference's eunha.h into
 * oracle/_ref/libgotpm_dropin.so, linked with lageunha_b200/libtpm_engine.so. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <mpi.h>

#include "eunha.h"
#include "CosmosEvolFactor.h"

void pmmain(SimParameters *, EvolFact);
void TreeMain(SimParameters *, DeterminedEvolFact *);
int tpm_gotpm_status(void);

static void fill(SimParameters *s, int n, float eps, float theta, float rsphere, float efold, int status,
                 int stepcount) {
  memset(s, 0, sizeof(*s));
  NX(s) = n;
  MYID(s) = 0;
  NID(s) = 1;
  s->bp.dm.mass = 1.0f;
  GRV_EFOLD(s) = efold;
  GRV_EPSILON(s) = eps;
  THETA(s) = theta;
  RSPHERE(s) = rsphere;
  PMSTATUS(s) = status;
  STEPCOUNT(s) = stepcount;
}

static void set_index(indxflag *u, uint64_t idx) { u->indx = idx & ((((uint64_t)1) << 56) - 1); }

/* The drop-in pmmain on 32-byte records; ef = the nine EvolFact fields in
 * their declared order. Returns the drop-in's status. */
int dropin_pmmain(int n, int64_t np, const uint64_t *indx, const float *off, float *vel, const float *ef,
                  int status, float efold, float eps) {
  SimParameters *s = (SimParameters *)calloc(1, sizeof(SimParameters));
  fill(s, n, eps, 0.3f, 4.0f, efold, status, 2);
  dmparticletype *p = (dmparticletype *)calloc((size_t)np, sizeof(dmparticletype));
  for (int64_t i = 0; i < np; i++) {
    set_index(&p[i].u4if, indx[i]);
    p[i].x = off[3 * i];
    p[i].y = off[3 * i + 1];
    p[i].z = off[3 * i + 2];
    p[i].vx = vel[3 * i];
    p[i].vy = vel[3 * i + 1];
    p[i].vz = vel[3 * i + 2];
  }
  DM_NP(s) = np;
  DM_BP(s) = p;
  EvolFact e;
  memcpy(&e, ef, sizeof(e));
  pmmain(s, e);
  for (int64_t i = 0; i < np; i++) {
    vel[3 * i] = p[i].vx;
    vel[3 * i + 1] = p[i].vy;
    vel[3 * i + 2] = p[i].vz;
  }
  free(p);
  free(s);
  return tpm_gotpm_status();
}

/* The drop-in TreeMain on 40-byte records with fact2, at step `stepcount`
 * (its opening-angle schedule). */
int dropin_treemain(int n, int64_t np, const uint64_t *indx, const float *off, float *vel, float fact1, float fact2,
                    int stepcount, float rsphere, float eps) {
  SimParameters *s = (SimParameters *)calloc(1, sizeof(SimParameters));
  fill(s, n, eps, 0.3f, rsphere, 0.9f, KICK, stepcount);
  treedmparticletype *t = (treedmparticletype *)calloc((size_t)np, sizeof(treedmparticletype));
  for (int64_t i = 0; i < np; i++) {
    set_index(&t[i].u4if, indx[i]);
    t[i].x = off[3 * i];
    t[i].y = off[3 * i + 1];
    t[i].z = off[3 * i + 2];
    t[i].vx = vel[3 * i];
    t[i].vy = vel[3 * i + 1];
    t[i].vz = vel[3 * i + 2];
  }
  DM_NP(s) = np;
  DM_TBP(s) = t;
  DeterminedEvolFact ef[1];
  ef[0].fact1 = fact1;
  ef[0].fact2 = fact2;
  TreeMain(s, ef);
  for (int64_t i = 0; i < np; i++) {
    vel[3 * i] = t[i].vx;
    vel[3 * i + 1] = t[i].vy;
    vel[3 * i + 2] = t[i].vz;
  }
  free(t);
  free(s);
  return tpm_gotpm_status();
}
