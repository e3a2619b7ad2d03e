/*
 * Harness that links the reference's own force-path sources into a CPU
 * oracle library (oracle/_ref/libref_{A,B}.so). TEST INFRASTRUCTURE ONLY:
 * tests, the smoke check and bench.py's CPU-baseline leg load it as the
 * checker; the engine never links or calls it.
 *
 * Compiled from the reference tree (not copied):
 *   Cosmos/pmmain.c, Cosmos/psolver.c, Cosmos/fda4.c, Cosmos/treecorrection.c,
 *   Cosmos/BasicCell.c, OST/ost.ver2.c, OST/Model4TreeForce.c,
 *   Timer/timerutil.c, and for the step, snapshot, spectrum and initial
 *   conditions Cosmos/CosmosEvolFactor.c, Cosmos/FLRW.c, Cosmos/mynr.c,
 *   Cosmos/Correlation.c, Params/header.c, Cosmos/CosmosIC/nr.c,
 *   Cosmos/CosmosIC/nrutil.c, Cosmos/CosmosIC/Zeldovich.c,
 *   Cosmos/CosmosIC/TwoLPT.c
 * with -DINTEL -DXYZDBL -DGOTPM (sRules.make:32,46) and -fopenmp.
 *
 * What this file supplies for a single rank on one box:
 *  - MPI: the scalar Reduce/Bcast/Barrier calls of the force path become
 *    copies/no-ops (oracle/stub/mpi.h).
 *  - FFTW-MPI: fftwf_mpi_execute_dft_r2c / _c2r with the reference's plan
 *    flags FFTW_MPI_TRANSPOSED_OUT / _IN (FFT/fft.c:130-146), or without them
 *    for the initial conditions' np/inp plans (FFT/fft.c:81-94): in-place,
 *    unnormalised, rows padded to 2*(nx/2+1) floats, spectrum stored as
 *    [y][z][x/2+1] (the layout psolver indexes, Cosmos/psolver.c:49-72).
 *    The arithmetic is oracle/dft.c in double. The vendored FFTW 3.3.6 is not
 *    built: it needs its configure-generated config.h.
 *  - gmigrate (RkS/gmigrate.c:548-580): with one rank it reduces to
 *    Dump2Outgrid's periodic overlap-add over the 27 box shifts
 *    (RkS/gmigrate.c:212-273).
 *  - PaddingParticles (Cosmos/mpirks.sub.c:14-79 -> RkS/mpirks.c:1058-1198):
 *    with one rank, the periodic images (26 shifts) of every particle that
 *    fall inside [-w, N+w)^3 with w = RSPHERE, flagged BoundaryGhostflag,
 *    positions made absolute (shift2pos) and stored in the float x,y,z slots.
 *  - the side-effect I/O of pmmain (savexzslice, volumeout, CorrMeasure,
 *    Cosmos/pmmain.c:326,453-456,480-481) is skipped.
 *
 * Exported oracle entry points (ref_*) set up a zeroed SimParameters for one
 * rank owning [0,N)^3, run the reference with PMSTATUS = KICK and
 * fact2 = 1 on zero velocities, and read the force back from the velocities
 * (Cosmos/fda4.h:297-299; Cosmos/treecorrection.c:90, OST/ost.ver2.c:273-291).
 */
#include <math.h>
#include <mpi.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "eunha.h"
#include "CosmosEvolFactor.h"
#include "Model4TreeForce.h"
#include "dft.h"

/* ------------------------------------------------------------------ MPI */
static size_t mpi_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR:
    case MPI_BYTE: return 1;
    case MPI_INT:
    case MPI_FLOAT: return 4;
    default: return 8;
  }
}
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c) {
  (void)op; (void)root; (void)c;
  if (s != r) memmove(r, s, (size_t)n * mpi_type_size(t));
  return 0;
}
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  return MPI_Reduce(s, r, n, t, op, 0, c);
}
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c;
  return 0;
}
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }

/* --------------------------------------------------------- FFTW-MPI shim */
struct fftwf_plan_s {
  ptrdiff_t n0, n1, n2; /* z, y, x */
  int natural;          /* 1: the plans without FFTW_MPI_TRANSPOSED_* (FFT/fft.c:81-94, the IC's
                           np/inp): spectrum stored as [z][y][kx] */
};

void fftwf_mpi_execute_dft_r2c(fftwf_plan p, float *in, fftwf_complex *out) {
  ptrdiff_t nz = p->n0, ny = p->n1, nx = p->n2, hx = nx / 2 + 1, mx = 2 * hx;
  int nat = p->natural;
  double *r = (double *)malloc(sizeof(double) * nx * ny * nz);
  double *c = (double *)malloc(sizeof(double) * 2 * hx * ny * nz);
  for (ptrdiff_t k = 0; k < nz; k++)
    for (ptrdiff_t j = 0; j < ny; j++)
      for (ptrdiff_t i = 0; i < nx; i++) r[i + nx * (j + ny * k)] = in[i + mx * (j + ny * k)];
  odft_r2c_3d(nz, ny, nx, r, c);
  float *o = (float *)out;
  /* transposed out: complex element (kx, y, z) at [y][z][kx] */
  for (ptrdiff_t k = 0; k < nz; k++)
    for (ptrdiff_t j = 0; j < ny; j++)
      for (ptrdiff_t i = 0; i < hx; i++) {
        size_t src = 2 * (i + hx * (j + ny * k));
        size_t dst = nat ? src : 2 * (i + hx * (k + nz * j));
        o[dst] = (float)c[src];
        o[dst + 1] = (float)c[src + 1];
      }
  free(r);
  free(c);
}

void fftwf_mpi_execute_dft_c2r(fftwf_plan p, fftwf_complex *in, float *out) {
  ptrdiff_t nz = p->n0, ny = p->n1, nx = p->n2, hx = nx / 2 + 1, mx = 2 * hx;
  int nat = p->natural;
  double *c = (double *)malloc(sizeof(double) * 2 * hx * ny * nz);
  double *r = (double *)malloc(sizeof(double) * nx * ny * nz);
  const float *ci = (const float *)in;
  for (ptrdiff_t k = 0; k < nz; k++)
    for (ptrdiff_t j = 0; j < ny; j++)
      for (ptrdiff_t i = 0; i < hx; i++) {
        size_t dst = 2 * (i + hx * (j + ny * k));
        size_t src = nat ? dst : 2 * (i + hx * (k + nz * j));
        c[dst] = ci[src];
        c[dst + 1] = ci[src + 1];
      }
  odft_c2r_3d(nz, ny, nx, c, r);
  for (ptrdiff_t k = 0; k < nz; k++)
    for (ptrdiff_t j = 0; j < ny; j++)
      for (ptrdiff_t i = 0; i < nx; i++) out[i + mx * (j + ny * k)] = (float)r[i + nx * (j + ny * k)];
  free(c);
  free(r);
}

/* -------------------------------------------------------------- gmigrate */
void gmigrate(GridInfo *ingrid, GridInfo *outgrid, DoDeInfo *ddinfo, int nddinfo) {
  (void)ddinfo; (void)nddinfo;
  ptrdiff_t Nx = ingrid->nx, Ny = ingrid->ny, Nz = ingrid->nz;
  ptrdiff_t inx = ingrid->jx - ingrid->ix + 1, iny = ingrid->jy - ingrid->iy + 1;
  ptrdiff_t onx = outgrid->jx - outgrid->ix + 1, ony = outgrid->jy - outgrid->iy + 1,
            onz = outgrid->jz - outgrid->iz + 1;
  outgrid->npix = onx * ony * onz;
  const DenType *src = (const DenType *)(ingrid + 1);
  DenType *dst = (DenType *)(outgrid + 1);
  for (int sz = -1; sz <= 1; sz++)
    for (int sy = -1; sy <= 1; sy++)
      for (int sx = -1; sx <= 1; sx++) {
        /* the input grid shifted by s*N, overlapped with the output grid */
        ptrdiff_t x0 = ingrid->ix + sx * Nx, x1 = ingrid->jx + sx * Nx;
        ptrdiff_t y0 = ingrid->iy + sy * Ny, y1 = ingrid->jy + sy * Ny;
        ptrdiff_t z0 = ingrid->iz + sz * Nz, z1 = ingrid->jz + sz * Nz;
        if (x0 < outgrid->ix) x0 = outgrid->ix;
        if (y0 < outgrid->iy) y0 = outgrid->iy;
        if (z0 < outgrid->iz) z0 = outgrid->iz;
        if (x1 > outgrid->jx) x1 = outgrid->jx;
        if (y1 > outgrid->jy) y1 = outgrid->jy;
        if (z1 > outgrid->jz) z1 = outgrid->jz;
        if (x1 < x0 || y1 < y0 || z1 < z0) continue;
        for (ptrdiff_t k = z0; k <= z1; k++)
          for (ptrdiff_t j = y0; j <= y1; j++)
            for (ptrdiff_t i = x0; i <= x1; i++) {
              ptrdiff_t io = (i - outgrid->ix) + onx * ((j - outgrid->iy) + ony * (k - outgrid->iz));
              ptrdiff_t ii = (i - sx * Nx - ingrid->ix) +
                             inx * ((j - sy * Ny - ingrid->iy) + iny * (k - sz * Nz - ingrid->iz));
              dst[io] += src[ii];
            }
      }
}

/* ------------------------------------------------------ PaddingParticles */
void PaddingParticles(SimParameters *simpar) {
  double N[3] = {(double)NX(simpar), (double)NY(simpar), (double)NZ(simpar)};
  double w = RSPHERE(simpar);
  NXNY(simpar) = NX(simpar) * NY(simpar);
  ptrdiff_t np = DM_NP(simpar), cap = 1024, n = 0;
  treedmparticletype *pad = (treedmparticletype *)malloc(sizeof(treedmparticletype) * cap);
  treedmparticletype *bp = DM_TBP(simpar);
  for (ptrdiff_t i = 0; i < np; i++) {
    double x[3] = {XofP(simpar, bp + i), YofP(simpar, bp + i), ZofP(simpar, bp + i)};
    for (int s = 0; s < 27; s++) {
      int sh[3] = {s % 3 - 1, (s / 3) % 3 - 1, s / 9 - 1};
      if (sh[0] == 0 && sh[1] == 0 && sh[2] == 0) continue;
      double y[3];
      int inside = 1;
      for (int d = 0; d < 3; d++) {
        y[d] = x[d] + sh[d] * N[d];
        if (!(y[d] >= -w && y[d] < N[d] + w)) inside = 0;
      }
      if (!inside) continue;
      if (n == cap) {
        cap *= 2;
        pad = (treedmparticletype *)realloc(pad, sizeof(treedmparticletype) * cap);
      }
      pad[n] = bp[i];
      pad[n].x = (float)y[0];
      pad[n].y = (float)y[1];
      pad[n].z = (float)y[2];
      CLEAR_FLAG(pad + n);
      SET_FLAG(pad + n, BoundaryGhostflag);
      SET_FLAG(pad + n, DMflag);
      n++;
    }
  }
  DM_TBPP(simpar) = pad;
  DM_NPAD(simpar) = n;
  SPH_NPAD(simpar) = VORO_NPAD(simpar) = STAR_NPAD(simpar) = AGN_NPAD(simpar) = 0;
}

/* ---------------------------------------------- skipped side effects */
/* pmmain calls CorrMeasure after its forward FFT (Cosmos/pmmain.c:480-481);
 * the reference's own function (compiled as ref_corr_measure) runs only
 * when ref_power_spectrum asks for it, and writes pmevol.map in the current
 * directory. */
void ref_corr_measure(SimParameters *simpar, GridInfo *g);
static int g_corr = 0;
static double g_corr_boxsize = 0;
void CorrMeasure(SimParameters *simpar, GridInfo *g) {
  if (!g_corr) return;
  BOXSIZE(simpar) = g_corr_boxsize;
  ref_corr_measure(simpar, g);
}
void savexzslice(SimParameters *simpar, DenType *d) { (void)simpar; (void)d; }
void volumeout(SimParameters *simpar, GridInfo *g, int which) { (void)simpar; (void)g; (void)which; }

/* ------------------------------------------------------- oracle set-up */
extern int initflag; /* Cosmos/treecorrection.c:221: spline table built once */
extern FORCEARRAYTYPE diff[NSPLINE][3], slope[NSPLINE][3]; /* OST/Model4TreeForce.c:14 */
void pmmain(SimParameters *, EvolFact);
void treecorrection(SimParameters *, DeterminedEvolFact *);
void *MakeDenGrid4TSC(SimParameters *, GridInfo *, ptrdiff_t, ptrdiff_t);
void TSC(SimParameters *, GridInfo *);
GridInfo *MakeGrids4FFTWDD(SimParameters *, GridInfo *);
void psolver(SimParameters *, GridInfo *);
void i_force_spline(SimParameters *);

typedef struct {
  SimParameters sim;
  DoDeInfo dd;
  struct fftwf_plan_s fplan, bplan, nfplan, nbplan;
} RefBox;

static RefBox *refbox_new(int n, float efold, float eps, float theta, float rsphere) {
  RefBox *b = (RefBox *)calloc(1, sizeof(RefBox));
  SimParameters *s = &b->sim;
  NX(s) = n;
  s->fftwgrid.gridinfo.ny = n;
  s->fftwgrid.gridinfo.nz = n;
  NXNY(s) = (ptrdiff_t)n * n;
  MYID(s) = 0;
  NID(s) = 1;
  MPI_COMM(s) = MPI_COMM_WORLD;
  LOCAL_NZ(s) = n;
  LOCAL_Z_START(s) = 0;
  LOCAL_GRID_SIZE(s) = (ptrdiff_t)n * n * (n / 2 + 1);
  LOCAL_NY_AFTER_TRANSPOSE(s) = n;
  LOCAL_Y_START_AFTER_TRANSPOSE(s) = 0;
  b->fplan.n0 = b->fplan.n1 = b->fplan.n2 = n;
  b->bplan = b->fplan;
  b->nfplan = b->fplan;
  b->nfplan.natural = 1;
  b->nbplan = b->nfplan;
  FFTW_F_PLAN(s) = &b->fplan;
  FFTW_B_PLAN(s) = &b->bplan;
  FFTW_NF_PLAN(s) = &b->nfplan;
  FFTW_NB_PLAN(s) = &b->nbplan;
  for (int d = 0; d < 3; d++) {
    b->dd.lgroup.r.rmin[d] = 0;
    b->dd.lgroup.r.rmax[d] = n;
  }
  NDDINFO(s) = 1;
  DM_DDINFO(s) = &b->dd;
  TDM_DDINFO(s) = &b->dd;
  s->bp.dm.mass = 1.0f; /* cosmology.c:268 */
  GRV_EFOLD(s) = efold;
  GRV_EPSILON(s) = eps;
  THETA(s) = theta;
  RSPHERE(s) = rsphere;
  PMSTATUS(s) = KICK;
  STEPCOUNT(s) = 100;
  ANOW(s) = 1.0;
  ASTEP(s) = 0.0;
  return b;
}

static void set_index(indxflag *u, uint64_t idx) {
  u->indx = idx & ((((uint64_t)1) << 56) - 1);
}

/* Reference PM force (pmmain with KICK, fact2 = 1) on particles given as
 * Lagrangian index + float offset (XYZDBL, eunha.h:1228-1232). */
int ref_pm_force(int n, int64_t np, const uint64_t *indx, const float *off, float efold,
                 float *force) {
  RefBox *b = refbox_new(n, efold, 0.05f, 0.3f, 4.0f);
  SimParameters *s = &b->sim;
  dmparticletype *p = (dmparticletype *)calloc((size_t)np, sizeof(dmparticletype));
  for (int64_t i = 0; i < np; i++) {
    set_index(&p[i].u4if, indx[i]);
    p[i].x = off[3 * i];
    p[i].y = off[3 * i + 1];
    p[i].z = off[3 * i + 2];
  }
  DM_NP(s) = np;
  DM_BP(s) = p;
  EvolFact ef;
  memset(&ef, 0, sizeof(ef));
  ef.fact2 = 1.0f;
  pmmain(s, ef);
  for (int64_t i = 0; i < np; i++) {
    force[3 * i] = p[i].vx;
    force[3 * i + 1] = p[i].vy;
    force[3 * i + 2] = p[i].vz;
  }
  free(p);
  free(b);
  return 0;
}

/* Reference short-range tree correction (treecorrection, fact2 = 1). */
int ref_tree_force(int n, int64_t np, const uint64_t *indx, const float *off, float theta,
                   float rsphere, float eps, float *force) {
  RefBox *b = refbox_new(n, 0.9f, eps, theta, rsphere);
  SimParameters *s = &b->sim;
  treedmparticletype *p = (treedmparticletype *)calloc((size_t)np, sizeof(treedmparticletype));
  for (int64_t i = 0; i < np; i++) {
    set_index(&p[i].u4if, indx[i]);
    p[i].x = off[3 * i];
    p[i].y = off[3 * i + 1];
    p[i].z = off[3 * i + 2];
  }
  DM_NP(s) = np;
  DM_TBP(s) = p;
  DeterminedEvolFact ef[1];
  ef[0].fact1 = 1.0f;
  ef[0].fact2 = 1.0f;
  initflag = 0; /* rebuild the table for this N and softening */
  treecorrection(s, ef);
  for (int64_t i = 0; i < np; i++) {
    force[3 * i] = p[i].vx;
    force[3 * i + 1] = p[i].vy;
    force[3 * i + 2] = p[i].vz;
  }
  free(p);
  free(b);
  return 0;
}

/* Folded TSC density contrast (mesh - 1), [z][y][x], as it enters the r2c. */
int ref_tsc_density(int n, int64_t np, const uint64_t *indx, const float *off, float *mesh) {
  RefBox *b = refbox_new(n, 0.9f, 0.05f, 0.3f, 4.0f);
  SimParameters *s = &b->sim;
  dmparticletype *p = (dmparticletype *)calloc((size_t)np, sizeof(dmparticletype));
  for (int64_t i = 0; i < np; i++) {
    set_index(&p[i].u4if, indx[i]);
    p[i].x = off[3 * i];
    p[i].y = off[3 * i + 1];
    p[i].z = off[3 * i + 2];
  }
  DM_NP(s) = np;
  DM_BP(s) = p;
  GridInfo *dengrid = (GridInfo *)malloc(sizeof(GridInfo));
  dengrid = (GridInfo *)MakeDenGrid4TSC(s, dengrid, 1, 2);
  TSC(s, dengrid);
  GridInfo *fg = MakeGrids4FFTWDD(s, dengrid);
  const float *d = (const float *)(fg + 1);
  ptrdiff_t mx = 2 * (n / 2 + 1);
  for (ptrdiff_t k = 0; k < n; k++)
    for (ptrdiff_t j = 0; j < n; j++)
      for (ptrdiff_t i = 0; i < n; i++) mesh[i + n * (j + (ptrdiff_t)n * k)] = d[i + mx * (j + n * k)];
  free(fg);
  free(dengrid);
  free(p);
  free(b);
  return 0;
}

/* Potential after psolver and the c2r, [z][y][x] (before the fda4 ghosting). */
int ref_potential(int n, int64_t np, const uint64_t *indx, const float *off, float efold,
                  float *phi) {
  RefBox *b = refbox_new(n, efold, 0.05f, 0.3f, 4.0f);
  SimParameters *s = &b->sim;
  dmparticletype *p = (dmparticletype *)calloc((size_t)np, sizeof(dmparticletype));
  for (int64_t i = 0; i < np; i++) {
    set_index(&p[i].u4if, indx[i]);
    p[i].x = off[3 * i];
    p[i].y = off[3 * i + 1];
    p[i].z = off[3 * i + 2];
  }
  DM_NP(s) = np;
  DM_BP(s) = p;
  GridInfo *dengrid = (GridInfo *)malloc(sizeof(GridInfo));
  dengrid = (GridInfo *)MakeDenGrid4TSC(s, dengrid, 1, 2);
  TSC(s, dengrid);
  GridInfo *fg = MakeGrids4FFTWDD(s, dengrid);
  float *d = (float *)(fg + 1);
  fftwf_mpi_execute_dft_r2c(FFTW_F_PLAN(s), d, (fftwf_complex *)d);
  psolver(s, fg);
  fftwf_mpi_execute_dft_c2r(FFTW_B_PLAN(s), (fftwf_complex *)d, d);
  ptrdiff_t mx = 2 * (n / 2 + 1);
  for (ptrdiff_t k = 0; k < n; k++)
    for (ptrdiff_t j = 0; j < n; j++)
      for (ptrdiff_t i = 0; i < n; i++) phi[i + n * (j + (ptrdiff_t)n * k)] = d[i + mx * (j + n * k)];
  free(fg);
  free(dengrid);
  free(p);
  free(b);
  return 0;
}

/* The short-range force table (OST/Model4TreeForce.c:48-91) for this N and
 * softening: diff and slope, NSPLINE x 3 doubles each. */
int ref_spline_table(int n, float eps, double *diff_out, double *slope_out) {
  RefBox *b = refbox_new(n, 0.9f, eps, 0.3f, 4.0f);
  i_force_spline(&b->sim);
  memcpy(diff_out, diff, sizeof(double) * NSPLINE * 3);
  memcpy(slope_out, slope, sizeof(double) * NSPLINE * 3);
  free(b);
  return 0;
}

int ref_nspline(void) { return NSPLINE; }

/* One PMSTATUS half of the reference's global step on one rank's particles,
 * velocities in and out: PM_PULL_AND_PUSH (Cosmos/globalT.c:113-134: drag
 * v *= fact1 of the status, then the reference's own pmmain, whose fda4
 * picks fact2 by PMSTATUS and divides PUSH's by GetFact1, Cosmos/fda4.c:
 * 48-62), then TreeAndPreFoFmain's tree kick (TREE_HALF, Cosmos/indT.h:
 * 98-118: the full-step fact2 of GetEvolFactor) through the reference's own
 * treecorrection. The drag and the factor selection are restated here
 * because globalT.c does not build on one rank. */
int ref_status_kick(int n, int64_t np, const uint64_t *indx, const float *off, float *vel, float efold,
                    float theta, float rsphere, float eps, float omep, float omeplam, float wlam0, float wlam1,
                    float amax, float anow, float astep, int status) {
  RefBox *b = refbox_new(n, efold, eps, theta, rsphere);
  SimParameters *s = &b->sim;
  OMEP(s) = omep;
  OMEPLAM(s) = omeplam;
  WLAM0(s) = wlam0;
  WLAM1(s) = wlam1;
  AMAX(s) = amax;
  ANOW(s) = anow;
  ASTEP(s) = astep;
  PMSTATUS(s) = status;
  STEPCOUNT(s) = 2;
  EvolFact e = GetEvolFactor(s);
  float vfact1 = status == PUSH ? e.fact1_push : (status == PULL ? e.fact1_pull : e.fact1);
  dmparticletype *p = (dmparticletype *)calloc((size_t)np, sizeof(dmparticletype));
  for (int64_t i = 0; i < np; i++) {
    set_index(&p[i].u4if, indx[i]);
    p[i].x = off[3 * i];
    p[i].y = off[3 * i + 1];
    p[i].z = off[3 * i + 2];
    p[i].vx = vel[3 * i] * vfact1;
    p[i].vy = vel[3 * i + 1] * vfact1;
    p[i].vz = vel[3 * i + 2] * vfact1;
  }
  DM_NP(s) = np;
  DM_BP(s) = p;
  pmmain(s, e);
  treedmparticletype *t = (treedmparticletype *)calloc((size_t)np, sizeof(treedmparticletype));
  for (int64_t i = 0; i < np; i++) {
    t[i].u4if = p[i].u4if;
    t[i].x = p[i].x;
    t[i].y = p[i].y;
    t[i].z = p[i].z;
    t[i].vx = p[i].vx;
    t[i].vy = p[i].vy;
    t[i].vz = p[i].vz;
  }
  DM_TBP(s) = t;
  DeterminedEvolFact ef[1];
  ef[0].fact1 = e.fact1;
  ef[0].fact2 = e.fact2;
  initflag = 0;
  treecorrection(s, ef);
  for (int64_t i = 0; i < np; i++) {
    vel[3 * i] = t[i].vx;
    vel[3 * i + 1] = t[i].vy;
    vel[3 * i + 2] = t[i].vz;
  }
  free(t);
  free(p);
  free(b);
  return 0;
}

/* GetEvolFactor (Cosmos/CosmosEvolFactor.c:230-255) for one cosmology:
 * out = {afact, bfact, pfact, fact1, fact2, fact1_push, fact2_push,
 * fact1_pull, fact2_pull} (the EvolFact field order, CosmosEvolFactor.h:1-6). */
int ref_evol_factors(int n, float omep, float omeplam, float wlam0, float wlam1, float amax, float anow,
                     float astep, float *out) {
  RefBox *b = refbox_new(n, 0.9f, 0.05f, 0.3f, 4.0f);
  SimParameters *s = &b->sim;
  OMEP(s) = omep;
  OMEPLAM(s) = omeplam;
  WLAM0(s) = wlam0;
  WLAM1(s) = wlam1;
  AMAX(s) = amax;
  ANOW(s) = anow;
  ASTEP(s) = astep;
  EvolFact e = GetEvolFactor(s);
  float v[9] = {e.afact, e.bfact, e.pfact, e.fact1, e.fact2, e.fact1_push, e.fact2_push, e.fact1_pull, e.fact2_pull};
  memcpy(out, v, sizeof(v));
  free(b);
  return 0;
}

/* ------------------------------------------------------ snapshot files */
/* Mpi_Basic_Set (MpiAux) is named by Params/header.c but not reached by
 * read_head / write_head. */
void Mpi_Basic_Set(SimParameters *s, MPI_Comm comm) {
  (void)s;
  (void)comm;
  fprintf(stderr, "oracle/_ref: Mpi_Basic_Set is not part of the oracle harness\n");
  abort();
}
void write_head(FILE *, SimParameters *);
void read_head(FILE *, SimParameters *);
void mk_default_param(SimParameters *, char *);

/* One rank's file as jwrite writes it (Cosmos/CosmosRW/kjhrw.c:196-211, GOTPM
 * PMTYPE): write_head, the dmparticletype records (32 bytes each), then the
 * SimParameters struct. */
int ref_write_snapshot(const char *path, int n, int64_t np, const void *records, float omep, float omeplam,
                       float wlam0, float wlam1, float amax, double anow, double astep, float boxsize,
                       float theta, float eps, float rsphere, int stepcount) {
  SimParameters *s = (SimParameters *)calloc(1, sizeof(SimParameters));
  mk_default_param(s, (char *)"WMAP5");
  MYID(s) = 0;
  NID(s) = 1;
  NX(s) = NY(s) = NZ(s) = n;
  NXNY(s) = (ptrdiff_t)n * n;
  OMEP(s) = omep;
  OMEPLAM(s) = omeplam;
  WLAM0(s) = wlam0;
  WLAM1(s) = wlam1;
  AMAX(s) = amax;
  ANOW(s) = anow;
  ASTEP(s) = astep;
  COSBOXSIZE(s) = boxsize;
  THETA(s) = theta;
  GRV_EPSILON(s) = eps;
  RSPHERE(s) = rsphere;
  STEPCOUNT(s) = stepcount;
  DM_NP(s) = np;
  NPSUM(s) = np;
  PTYPE(s) = PMTYPE;
  FILE *fp = fopen(path, "w");
  if (!fp) {
    free(s);
    return -1;
  }
  write_head(fp, s);
  fwrite(records, sizeof(dmparticletype), (size_t)np, fp);
  fwrite(s, sizeof(SimParameters), 1, fp);
  fclose(fp);
  free(s);
  return (int)sizeof(dmparticletype);
}

/* read_head of a file (Params/header.c:72-104): the fields the engine's
 * reader reports, in this order: nx ny nz np_dm np_sph np_star np_agn ptype
 * omep omeplam wlam0 wlam1 amax anow astep theta epsilon rsphere boxsize
 * stepcount. */
int ref_read_head(const char *path, double *out) {
  SimParameters *s = (SimParameters *)calloc(1, sizeof(SimParameters));
  FILE *fp = fopen(path, "r");
  if (!fp) {
    free(s);
    return -1;
  }
  read_head(fp, s);
  fclose(fp);
  double v[20] = {(double)NX(s), (double)NY(s), (double)NZ(s), (double)DM_NP(s), (double)SPH_NP(s),
                  (double)STAR_NP(s), (double)AGN_NP(s), (double)PTYPE(s), OMEP(s), OMEPLAM(s), WLAM0(s),
                  WLAM1(s), AMAX(s), ANOW(s), ASTEP(s), THETA(s), GRV_EPSILON(s), RSPHERE(s),
                  COSBOXSIZE(s), (double)STEPCOUNT(s)};
  memcpy(out, v, sizeof(v));
  free(s);
  return 0;
}

/* The reference's P(k) of a particle set: one pmmain with CorrMeasure on
 * (Cosmos/Correlation.c:13-117); its output is the pmevol.map file it writes
 * in the current directory. */
int ref_power_spectrum(int n, int64_t np, const uint64_t *indx, const float *off, double boxsize, float *force) {
  g_corr = 1;
  g_corr_boxsize = boxsize;
  int rc = ref_pm_force(n, np, indx, off, 0.9f, force);
  g_corr = 0;
  return rc;
}

/* ---------------------------------------------------------- initial conditions
 * The white-noise field of the Zel'dovich initial conditions for one rank:
 * the mode loop of PMSeedForce (Cosmos/CosmosIC/PMSeedForce.c:293-334) with
 * the reference's own gasdev/ran3 (Cosmos/CosmosIC/nr.c:317-384), and its
 * completion of the kx = 0 plane by complex conjugates (PMSeedForce.c:346-399,
 * where the per-rank columns gathered into denpad are, with one rank, the
 * kx = 0 column of den itself). The Fortran amplitude pamp*bpower(rk)/rk^2 of
 * the P(k)-weighted path is passed in as its value per integer
 * k^2 = i^2 + ky^2 + kz^2 (velpot_k2[k2], k2 <= (n/2)^2); iseed >= 0 is the
 * reference's unit-amplitude path, which always runs with seed -1.
 * den: n*n*2*(n/2+1) floats, [z][y][2*(n/2+1)] (the non-transposed layout the
 * IC's plans use). */
float gasdev(long *);
int ref_ic_noise(int n, long iseed, const float *velpot_k2, float *den) {
  ptrdiff_t nx = n, ny = n, nz = n, mx = 2 * (nx / 2 + 1);
  int seedflag = 0;
  if (iseed >= 0) {
    seedflag = 1;
    iseed = -1;
  }
  long iiseed = iseed;
  double rknyq2 = (double)(nx / 2) * (double)(nx / 2);
  for (ptrdiff_t k = 0; k < nz; k++) {
    ptrdiff_t kz = k > nz / 2 ? k - nz : k;
    for (ptrdiff_t j = 0; j < ny; j++) {
      ptrdiff_t ky = j > ny / 2 ? j - ny : j;
      for (ptrdiff_t i = 0; i <= nx / 2; i++) {
        double xksq = (double)(i * i + ky * ky + kz * kz);
        float *d = den + 2 * i + mx * (j + ny * k);
        if (xksq == 0 || xksq > rknyq2) {
          d[0] = 0;
          d[1] = 0;
        } else if (seedflag) {
          d[0] = gasdev(&iiseed);
          d[1] = gasdev(&iiseed);
        } else {
          float velpot = velpot_k2[(ptrdiff_t)xksq];
          d[0] = velpot * gasdev(&iiseed);
          d[1] = velpot * gasdev(&iiseed);
        }
      }
    }
  }
  /* kx = 0 column: (re, im) at den[mx*(j+ny*k)] */
#define C0(j, k) (den + mx * ((j) + ny * (k)))
  for (ptrdiff_t k = 1; k < nz / 2; k++) {
    C0(0, nz - k)[0] = C0(0, k)[0];
    C0(0, nz - k)[1] = -C0(0, k)[1];
    for (ptrdiff_t j = 1; j < ny / 2; j++) {
      C0(ny - j, nz - k)[0] = C0(j, k)[0];
      C0(ny - j, nz - k)[1] = -C0(j, k)[1];
    }
  }
  for (ptrdiff_t j = 1; j < ny / 2; j++) {
    C0(ny - j, 0)[0] = C0(j, 0)[0];
    C0(ny - j, 0)[1] = -C0(j, 0)[1];
  }
  for (ptrdiff_t k = 1; k < nz / 2; k++)
    for (ptrdiff_t j = ny / 2 + 1; j < ny; j++) {
      C0(ny - j, nz - k)[0] = C0(j, k)[0];
      C0(ny - j, nz - k)[1] = -C0(j, k)[1];
    }
#undef C0
  return 0;
}

/* The reference's Zeldovich (Cosmos/CosmosIC/Zeldovich.c:14-100) on one rank:
 * den in/out (the noise field above; left as the potential's spectrum after
 * the fNL/gNL step), fx/fy/fz the displacement fields in the padded real
 * layout [z][y][2*(n/2+1)]. fx/fy/fz are cleared first: the reference fills
 * their spectra for kx < n/2 only (Zeldovich.c:71-88), leaving the kx = n/2
 * plane as it found it. */
void Zeldovich(SimParameters *, DenType *, DenType *, DenType *, DenType *);
int ref_zeldovich(int n, float fnl, float gnl, float *den, float *fx, float *fy, float *fz) {
  RefBox *b = refbox_new(n, 0.9f, 0.05f, 0.3f, 4.0f);
  SimParameters *s = &b->sim;
  FNL(s) = fnl;
  GNL(s) = gnl;
  size_t sz = (size_t)n * n * 2 * (n / 2 + 1);
  memset(fx, 0, sizeof(float) * sz);
  memset(fy, 0, sizeof(float) * sz);
  memset(fz, 0, sizeof(float) * sz);
  Zeldovich(s, den, fx, fy, fz);
  free(b);
  return 0;
}

/* Second-order Lagrangian initial conditions for one rank (PORDER = 2):
 * the reference's TwoLPT (Cosmos/CosmosIC/TwoLPT.c:259-535, its fNL/gNL
 * branch with the box size, Omega_m, amax and growth factor given)
 * on the noise spectrum den1, then per axis the combination amp1*phi1 +
 * amp2*phi2 and the reference's selfdiffphi (TwoLPT.c:17-157), as
 * TwoLPT_GetVR does (Cosmos/CosmosIC/cosmosic.h:141-163): velocities with
 * (vamp1, vamp2) and offsets with (amp1, amp2). vel, off: 3 fields of n^3
 * floats each, [z][y][x]. */
void mpi_fftw_finalize(void) {}
void TwoLPT(SimParameters *, DenType *, DenType *, DenType *, DenType *);
void selfdiffphi(SimParameters *, DenType *, enum dimension);
int ref_two_lpt(int n, const float *den1, float amp1, float amp2, float vamp1, float vamp2, float fnl, float gnl,
                float boxsize, float omep, float amax, float growth, float *vel, float *off) {
  RefBox *b = refbox_new(n, 0.9f, 0.05f, 0.3f, 4.0f);
  SimParameters *s = &b->sim;
  FNL(s) = fnl;
  GNL(s) = gnl;
  COSBOXSIZE(s) = boxsize;
  OMEP(s) = omep;
  AMAX(s) = amax;
  COS_GROWTH(s) = growth;
  size_t sz = (size_t)n * n * 2 * (n / 2 + 1), n3 = (size_t)n * n * n;
  float *d1 = (float *)calloc(sz, sizeof(float)), *d2 = (float *)calloc(sz, sizeof(float));
  float *w1 = (float *)calloc(sz, sizeof(float)), *w2 = (float *)calloc(sz, sizeof(float));
  float *dfr = (float *)calloc(sz, sizeof(float));
  memcpy(d1, den1, sizeof(float) * sz);
  TwoLPT(s, d1, w1, w2, d2);
  for (int pass = 0; pass < 2; pass++) {
    float a1 = pass ? amp1 : vamp1, a2 = pass ? amp2 : vamp2;
    float *out = pass ? off : vel;
    for (int ax = 0; ax < 3; ax++) {
      for (size_t i = 0; i < sz; i++) dfr[i] = a1 * d1[i] + a2 * d2[i];
      selfdiffphi(s, dfr, (enum dimension)(ax + 1));
      memcpy(out + ax * n3, dfr, sizeof(float) * n3);
    }
  }
  free(d1);
  free(d2);
  free(w1);
  free(w2);
  free(dfr);
  free(b);
  return 0;
}
