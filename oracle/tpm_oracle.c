/*
 * CPU oracle for the TreePM force path — TEST INFRASTRUCTURE ONLY (see
 * tpm_oracle.h). A C restatement of the reference's GOTPM force evaluation,
 * written from the reference's source and kept arithmetic-for-arithmetic
 * (same float/double types, same summation orders) so that it can be pinned
 * against the reference compiled under oracle/_ref.
 *
 * Reference files followed (paths inside kjhan0606/LagEunha):
 *   eunha.h:1212,1228-1232           PINDX, XofP/YofP/ZofP (XYZDBL)
 *   Cosmos/pmmain.h:81-159           OMP_Get_TSC_Den (TSC scatter)
 *   Cosmos/pmmain.c:75-185,283-336   padded TSC grid, fold into the FFT slab
 *   Cosmos/psolver.c:13-86           Green's function and k=0
 *   Cosmos/pmmain.c:337-388          ghosted potential for fda4
 *   Cosmos/fda4.h:11-103,276-384     TSC weights, 4-point gradient, kick
 *   OST/Model4TreeForce.c:23-116     PMFITPARA, table, GetPointGrav/GetCellGrav
 *   Cosmos/BasicCell.{h,c}           chaining mesh of CellWidth = 4 buckets
 *   Cosmos/treecorrection.c:53-219,225-475  bucket loop, Dump2Pos/GrvP,
 *                                    DirectSummation
 *   OST/ost.ver2.c:36-196,247-351    divide_node3, Make_Tree3, AddNode,
 *                                    AddPar, nodeopen3, treeforcesearch3
 *   RkS/gmigrate.c:212-273, RkS/mpirks.c:1058-1198  periodic fold / ghosts
 *                                    (single-rank semantics)
 */
#include "tpm_oracle.h"
#include "dft.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NSPLINE_OR 4096
#define RANGE_OR 6
#define CELLWIDTH_OR 4.0L
#define LEAF_MIN_OR 10      /* MIN_CELL_PARTICLE_NUM, OST/ost.h:4 */
#define MINCELLWIDTH_OR 1.E-5 /* OST/ost.h:5 */
#define DIRECTSUM_OR 16     /* Cosmos/treecorrection.c:16 */

static inline int isign_of(double a) { return signbit(a) ? -1 : 1; } /* Cosmos/cosmology.h:1 */

void or_decode(int n, int64_t np, const uint64_t *indx, const float *off, double *pos) {
  uint64_t N = (uint64_t)n, NN = N * N;
  for (int64_t i = 0; i < np; i++) {
    uint64_t id = (indx[i] << 8) >> 8;
    pos[3 * i + 0] = fmod((double)off[3 * i + 0] + (double)(id % N) + (double)n, (double)n);
    pos[3 * i + 1] = fmod((double)off[3 * i + 1] + (double)((id % NN) / N) + (double)n, (double)n);
    pos[3 * i + 2] = fmod((double)off[3 * i + 2] + (double)(id / NN) + (double)n, (double)n);
  }
}

/* ------------------------------------------------------------------ TSC */
/* Scatter into the padded grid [-1, N+1]^3 (pmmain.c:75-110 with bbuffer 1,
 * ubuffer 2), then fold periodically onto a mesh initialised to -1
 * (pmmain.c:304; gmigrate.c:212-273). A particle whose float z equals N is
 * outside every OpenMP z-window (pmmain.c:150-154, pmmain.h:84) and is not
 * deposited, as in the reference. */
int or_tsc_density(int n, int64_t np, const double *pos, float *mesh) {
  ptrdiff_t pn = n + 3;
  float *den = (float *)calloc((size_t)pn * pn * pn, sizeof(float));
  if (!den) return -1;
  const double xs = -1.0;
  for (int64_t p = 0; p < np; p++) {
    float zzp = (float)pos[3 * p + 2];
    if (!(zzp >= 0.0 && zzp < (double)n)) continue;
    float pmas0 = 1.0f;
    float p05 = pmas0 * 0.5;
    double xp = pos[3 * p] - xs, yp = pos[3 * p + 1] - xs, zp = pos[3 * p + 2] - xs;
    ptrdiff_t nearx = (ptrdiff_t)rint(xp), neary = (ptrdiff_t)rint(yp), nearz = (ptrdiff_t)rint(zp);
    double xmin = xp - nearx, ymin = yp - neary, zmin = zp - nearz;
    ptrdiff_t xsign = isign_of(xmin), ysign = isign_of(ymin), zsign = isign_of(zmin);
    ptrdiff_t ii[3] = {nearx, nearx + xsign, nearx - xsign};
    ptrdiff_t jj[3] = {neary, neary + ysign, neary - ysign};
    ptrdiff_t kk[3] = {nearz, nearz + zsign, nearz - zsign};
    float xd1 = fabs(xmin), yd1 = fabs(ymin), zd1 = fabs(zmin);
    float wx[3], wy[3], wz[3];
    wx[0] = (0.75 - xd1 * xd1) * pmas0;
    wy[0] = 0.75 - yd1 * yd1;
    wz[0] = 0.75 - zd1 * zd1;
    wx[2] = p05 * (0.25 + xd1 * (xd1 - 1.));
    wx[1] = wx[2] + pmas0 * xd1;
    wy[2] = 0.5 * (0.25 + yd1 * (yd1 - 1.));
    wy[1] = wy[2] + yd1;
    wz[2] = 0.5 * (0.25 + zd1 * (zd1 - 1.));
    wz[1] = wz[2] + zd1;
    for (int c = 0; c < 3; c++)
      for (int b = 0; b < 3; b++) {
        float wxy[3] = {wx[0] * wy[b], wx[1] * wy[b], wx[2] * wy[b]};
        for (int a = 0; a < 3; a++) den[ii[a] + pn * (jj[b] + pn * kk[c])] += wxy[a] * wz[c];
      }
  }
  size_t nc = (size_t)n * n * n;
  for (size_t i = 0; i < nc; i++) mesh[i] = -1.0f;
  for (int sz = -1; sz <= 1; sz++)
    for (int sy = -1; sy <= 1; sy++)
      for (int sx = -1; sx <= 1; sx++) {
        ptrdiff_t lo[3], hi[3], s[3] = {sx, sy, sz};
        int empty = 0;
        for (int d = 0; d < 3; d++) {
          lo[d] = -1 + s[d] * n;
          hi[d] = (n + 1) + s[d] * n;
          if (lo[d] < 0) lo[d] = 0;
          if (hi[d] > n - 1) hi[d] = n - 1;
          if (hi[d] < lo[d]) empty = 1;
        }
        if (empty) continue;
        for (ptrdiff_t k = lo[2]; k <= hi[2]; k++)
          for (ptrdiff_t j = lo[1]; j <= hi[1]; j++)
            for (ptrdiff_t i = lo[0]; i <= hi[0]; i++)
              mesh[i + n * (j + (ptrdiff_t)n * k)] +=
                  den[(i - sx * n + 1) + pn * ((j - sy * n + 1) + pn * (k - sz * n + 1))];
      }
  free(den);
  return 0;
}

/* ------------------------------------------------------------- Poisson */
/* r2c in the transposed-out layout [y][z][x/2+1] (FFT/fft.c:130-136), the
 * Green's function of psolver.c:49-76, c2r back (fft.c:140-146). The DFT is
 * oracle/dft.c in double with float storage in between, as the harness
 * under oracle/_ref does. */
static void poisson_inplace(int n, float efold, const float *rho, float *phi) {
  ptrdiff_t nx = n, ny = n, nz = n, hx = nx / 2 + 1;
  double *r = (double *)malloc(sizeof(double) * nx * ny * nz);
  double *c = (double *)malloc(sizeof(double) * 2 * hx * ny * nz);
  float *spec = (float *)malloc(sizeof(float) * 2 * hx * ny * nz);
  for (size_t i = 0; i < (size_t)nx * ny * nz; i++) r[i] = rho[i];
  odft_r2c_3d(nz, ny, nx, r, c);
  for (ptrdiff_t k = 0; k < nz; k++)
    for (ptrdiff_t j = 0; j < ny; j++)
      for (ptrdiff_t i = 0; i < hx; i++) {
        size_t s = 2 * (i + hx * (j + ny * k)), d = 2 * (i + hx * (k + nz * j));
        spec[d] = (float)c[s];
        spec[d + 1] = (float)c[s + 1];
      }
  double rnx = nx, rny = ny, rnz = nz;
  ptrdiff_t mx = 2 * hx;
  float xyy = rnx / rny, xyz = rnx / rnz;
  double fact = -1.L / M_PI;
  double sfact = -pow(M_PI * efold / rnx, 2);
  double rngc = rnx * rny * rnz, irngc = 1.L / rngc;
  for (ptrdiff_t j = 0; j < ny; j++) {
    float wy = xyy * j;
    if (wy > rny / 2) wy = wy - rny;
    for (ptrdiff_t k = 0; k < nz; k++) {
      float wz = xyz * k;
      if (wz > rnz / 2) wz = wz - rnz;
      for (ptrdiff_t i = 0; i <= nx / 2; i++) {
        double wave = i * i + wy * wy + wz * wz;
        float *re = spec + 2 * i + mx * (k + nz * j);
        if (wave == 0.L) {
          re[0] = 0;
          re[1] = 0;
        } else {
          double factr = fact / wave;
          double factor = factr * exp(wave * sfact);
          re[0] = factor * re[0] * irngc;
          re[1] = factor * re[1] * irngc;
        }
      }
    }
  }
  for (ptrdiff_t k = 0; k < nz; k++)
    for (ptrdiff_t j = 0; j < ny; j++)
      for (ptrdiff_t i = 0; i < hx; i++) {
        size_t d = 2 * (i + hx * (j + ny * k)), s = 2 * (i + hx * (k + nz * j));
        c[d] = spec[s];
        c[d + 1] = spec[s + 1];
      }
  odft_c2r_3d(nz, ny, nx, c, r);
  for (size_t i = 0; i < (size_t)nx * ny * nz; i++) phi[i] = (float)r[i];
  free(r);
  free(c);
  free(spec);
}

int or_potential(int n, int64_t np, const double *pos, float efold, float *phi) {
  size_t nc = (size_t)n * n * n;
  float *rho = (float *)malloc(sizeof(float) * nc);
  if (!rho) return -1;
  or_tsc_density(n, np, pos, rho);
  poisson_inplace(n, efold, rho, phi);
  free(rho);
  return 0;
}

/* ---------------------------------------------------------------- fda4 */
/* Ghosted potential on [-3, N+3]^3 (pmmain.c:365-382), then per particle the
 * TSC weights, the 4-point gradient at the 27 nodes and their weighted sum
 * (fda4.h:11-103, 276-384; fda4.c:45-46 for ffact1/ffact2), fact2 = 1. */
int or_fda4_force(int n, int64_t np, const double *pos, const float *phi, float *force) {
  ptrdiff_t g = n + 7;
  float *den = (float *)malloc(sizeof(float) * g * g * g);
  if (!den) return -1;
  for (ptrdiff_t k = 0; k < g; k++)
    for (ptrdiff_t j = 0; j < g; j++)
      for (ptrdiff_t i = 0; i < g; i++) {
        ptrdiff_t a = ((i - 3) % n + n) % n, b = ((j - 3) % n + n) % n, c = ((k - 3) % n + n) % n;
        den[i + g * (j + g * k)] = phi[a + n * (b + (ptrdiff_t)n * c)];
      }
  const float ffact1 = (4. / 3.) / 2.;
  const float ffact2 = (-1. / 3.) / 4.;
  const ptrdiff_t mx = g, my = g;
#define DEN(i, j, k) (den[(i) + mx * ((j) + my * (k))])
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < np; p++) {
    double xp = pos[3 * p] + 3.0, yp = pos[3 * p + 1] + 3.0, zp = pos[3 * p + 2] + 3.0;
    int nearx = rint(xp), neary = rint(yp), nearz = rint(zp);
    float xmin = xp - nearx, ymin = yp - neary, zmin = zp - nearz;
    int xsign = isign_of(xmin), ysign = isign_of(ymin), zsign = isign_of(zmin);
    int ii[3] = {nearx, nearx + xsign, nearx - xsign};
    int jj[3] = {neary, neary + ysign, neary - ysign};
    int kk[3] = {nearz, nearz + zsign, nearz - zsign};
    float xd1 = fabs(xmin), yd1 = fabs(ymin), zd1 = fabs(zmin);
    float wx[3], wy[3], wz[3];
    wx[0] = 0.75 - xd1 * xd1;
    wy[0] = 0.75 - yd1 * yd1;
    wz[0] = 0.75 - zd1 * zd1;
    wx[2] = 0.5 * (0.25 + xd1 * (xd1 - 1.));
    wx[1] = wx[2] + xd1;
    wy[2] = 0.5 * (0.25 + yd1 * (yd1 - 1.));
    wy[1] = wy[2] + yd1;
    wz[2] = 0.5 * (0.25 + zd1 * (zd1 - 1.));
    wz[1] = wz[2] + zd1;
    float wxy[9];
    for (int b = 0; b < 3; b++)
      for (int a = 0; a < 3; a++) wxy[a + 3 * b] = wx[a] * wy[b];
    float wt[27], fxs[27], fys[27], fzs[27];
    for (int c = 0; c < 3; c++)
      for (int b = 0; b < 3; b++)
        for (int a = 0; a < 3; a++) {
          int t = a + 3 * b + 9 * c;
          int i = ii[a], j = jj[b], k = kk[c];
          wt[t] = wxy[a + 3 * b] * wz[c];
          fxs[t] = ffact1 * (DEN(i - 1, j, k) - DEN(i + 1, j, k)) + ffact2 * (DEN(i - 2, j, k) - DEN(i + 2, j, k));
          fys[t] = ffact1 * (DEN(i, j - 1, k) - DEN(i, j + 1, k)) + ffact2 * (DEN(i, j - 2, k) - DEN(i, j + 2, k));
          fzs[t] = ffact1 * (DEN(i, j, k - 1) - DEN(i, j, k + 1)) + ffact2 * (DEN(i, j, k - 2) - DEN(i, j, k + 2));
        }
    float fx = wt[0] * fxs[0], fy = wt[0] * fys[0], fz = wt[0] * fzs[0];
    for (int t = 1; t < 27; t++) {
      fx = fx + wt[t] * fxs[t];
      fy = fy + wt[t] * fys[t];
      fz = fz + wt[t] * fzs[t];
    }
    float fact2 = 1.0f;
    float vx = 0, vy = 0, vz = 0;
    vx += fact2 * fx;
    vy += fact2 * fy;
    vz += fact2 * fz;
    force[3 * p] = vx;
    force[3 * p + 1] = vy;
    force[3 * p + 2] = vz;
  }
#undef DEN
  free(den);
  return 0;
}

int or_pm_force(int n, int64_t np, const double *pos, float efold, float *force) {
  size_t nc = (size_t)n * n * n;
  float *phi = (float *)malloc(sizeof(float) * nc);
  if (!phi) return -1;
  or_potential(n, np, pos, efold, phi);
  or_fda4_force(n, np, pos, phi, force);
  free(phi);
  return 0;
}

/* ---------------------------------------------------- short-range law */
/* OST/Model4TreeForce.c:23-32 */
static const double PMFIT[8] = {1.L / 256.L / 256.L, 0.78224E+00L, 0.37971E-06L, -0.60338E+00L,
                                -0.34419E-07L,       -0.39741E+01L, -0.10607E+01L, -0.38145E+00L};

/* f(r) = [r/(r^2+eps^2)^{3/2} - PMfit(r)] / N^2  (Model4TreeForce.c:92-116) */
static double pmcf_or(double r, float eps, double LL) {
  double t = cosh(PMFIT[1] * r);
  /* eps*eps is a float product in the reference (GRV_EPSILON is float) */
  double fr = r / pow(r * r + (eps) * (eps), 1.5L) -
              ((1L / (r * r) * tanh(PMFIT[1] * r) - PMFIT[1] / (t * t * r) -
                2L * PMFIT[2] / PMFIT[0] * r * exp(PMFIT[3] * r * r) -
                2L * PMFIT[2] * PMFIT[3] / PMFIT[0] * r * r * r * exp(PMFIT[3] * r * r) +
                PMFIT[4] / PMFIT[0] * (1L + PMFIT[5] * r * r + PMFIT[6] * r * r * r * r) *
                    exp(PMFIT[7] * r * r)));
  return fr / LL;
}

typedef struct {
  double diff[NSPLINE_OR + 1][3]; /* one spare row: slope(NSPLINE-1) reads row NSPLINE */
  double slope[NSPLINE_OR][3];
  float ran2nran, invran2nran;
} Spline;

/* i_force_spline (Model4TreeForce.c:48-91). The reference computes
 * slope(NSPLINE-1) from the row past the table and then zeroes it; the spare
 * row here is zero and the result is the same. */
static void spline_build(Spline *s, int n, float eps_f) {
  memset(s, 0, sizeof(*s));
  double LL = (double)n * (double)n;
  float eps = eps_f;
  s->ran2nran = (double)RANGE_OR / (double)NSPLINE_OR;
  s->invran2nran = 1. / s->ran2nran;
  double dr = s->ran2nran * 0.1;
  for (int i = 1; i < NSPLINE_OR; i++) {
    double r = (double)(i)*s->ran2nran;
    double rm1 = r - dr, rm2 = r - 2 * dr, rp1 = r + dr, rp2 = r + 2 * dr;
    double fp = (pmcf_or(rp1, eps, LL) - pmcf_or(rm1, eps, LL)) / (dr + dr);
    double fpp = (pmcf_or(rp2, eps, LL) - 2 * pmcf_or(r, eps, LL) + pmcf_or(rm2, eps, LL)) / (4 * dr * dr);
    double fr = pmcf_or(r, eps, LL);
    s->diff[i][0] = -(double)(fr / r);
    s->diff[i][1] = -(double)(0.5L * (fp * r - fr) / r / r / r);
    s->diff[i][2] = -(double)(0.5L * (fpp * r * r - 3 * fp * r + 3 * fr) / r / r / r / r / r);
  }
  for (int i = 0; i < NSPLINE_OR; i++)
    for (int c = 0; c < 3; c++) s->slope[i][c] = (s->diff[i + 1][c] - s->diff[i][c]) / s->ran2nran;
  for (int c = 0; c < 3; c++) {
    s->slope[0][c] = s->slope[1][c];
    s->diff[0][c] = s->diff[1][c];
  }
  for (int c = 0; c < 3; c++) {
    s->diff[NSPLINE_OR - 1][c] = 0;
    s->slope[NSPLINE_OR - 1][c] = 0;
  }
}

int or_nspline(void) { return NSPLINE_OR; }

int or_spline_table(int n, float eps, double *diff, double *slope) {
  Spline *s = (Spline *)malloc(sizeof(Spline));
  if (!s) return -1;
  spline_build(s, n, eps);
  memcpy(diff, s->diff, sizeof(double) * NSPLINE_OR * 3);
  memcpy(slope, s->slope, sizeof(double) * NSPLINE_OR * 3);
  free(s);
  return 0;
}

/* GetPointGrav (Model4TreeForce.c:34-38): no upper clamp. */
static inline float point_grav(const Spline *s, float dist) {
  int ntmp = dist * s->invran2nran;
  float fplmf = s->diff[ntmp][0] + s->slope[ntmp][0] * (dist - ntmp * s->ran2nran);
  return fplmf;
}

/* GetCellGrav (Model4TreeForce.c:39-46). */
static inline void cell_grav(const Spline *s, float dist, float *f1, float *f2, float *f3) {
  int ntmp = dist * s->invran2nran;
  float tmpdist = dist - ntmp * s->ran2nran;
  ntmp = ntmp > NSPLINE_OR - 1 ? NSPLINE_OR - 1 : ntmp;
  *f1 = s->diff[ntmp][0] + s->slope[ntmp][0] * tmpdist;
  *f2 = s->diff[ntmp][1] + s->slope[ntmp][1] * tmpdist;
  *f3 = s->diff[ntmp][2] + s->slope[ntmp][2] * tmpdist;
}

/* ------------------------------------------------------ bucket octree */
/* Threaded octree of one bucket's sources. A link is an int: >= 0 a source
 * particle, < 0 a node (-1 - node index), NIL the end of the thread. */
#define NIL 0x7fffffff
#define NODE_ID(i) (-1 - (i))
#define IS_NODE(l) ((l) < 0)
#define NODE_OF(l) (-1 - (l))

typedef struct {
  double x, y, z;
  float mass;
  int sibling;
} Src;

typedef struct {
  int daughter, sibling;
  double nodesize;
  float mass;
  int nparticle;
  float dist_over_thetasq;
  double monox, monoy, monoz;
  float quad[6], trQ;
} Node;

typedef struct {
  double x, y, z;
  float *axyz;
} Target;

static inline int *sib_of(Src *ptl, Node *nodes, int link) {
  return IS_NODE(link) ? &nodes[NODE_OF(link)].sibling : &ptl[link].sibling;
}

/* divide_node3 (ost.ver2.c:36-144), recursive form. */
static int divide_node(Node *nodes, Src *ptl, int t, int free_node, float thetasq, int variant) {
  Node *T = &nodes[t];
  int plist = T->daughter;
  T->mass = 0;
  T->monox = T->monoy = T->monoz = 0;
  for (int p = plist; p != NIL; p = ptl[p].sibling) {
    float m = ptl[p].mass;
    T->mass += m;
    T->monox += m * ptl[p].x;
    T->monoy += m * ptl[p].y;
    T->monoz += m * ptl[p].z;
  }
  T->monox /= T->mass;
  T->monoy /= T->mass;
  T->monoz /= T->mass;
  {
    double distmax = -1.E20L;
    float q0 = 0, q1 = 0, q2 = 0, q3 = 0, q4 = 0, q5 = 0;
    for (int p = plist; p != NIL; p = ptl[p].sibling) {
      float m = ptl[p].mass;
      double tx = ptl[p].x - T->monox, ty = ptl[p].y - T->monoy, tz = ptl[p].z - T->monoz;
      double d2 = tx * tx + ty * ty + tz * tz;
      distmax = distmax > d2 ? distmax : d2;
      q0 += m * tx * tx;
      q1 += m * ty * ty;
      q2 += m * tz * tz;
      q3 += m * tx * ty;
      q4 += m * tx * tz;
      if (variant == OR_VARIANT_A)
        q5 += m * ty * tx; /* ost.ver2.c:75 as written */
      else
        q5 += m * ty * tz;
    }
    T->nodesize = sqrt(distmax);
    T->quad[0] = q0;
    T->quad[1] = q1;
    T->quad[2] = q2;
    T->quad[3] = q3;
    T->quad[4] = q4;
    T->quad[5] = q5;
    T->trQ = q0 + q1 + q2;
    T->dist_over_thetasq = distmax / thetasq;
  }
  int head[8], cnt[8];
  for (int i = 0; i < 8; i++) {
    head[i] = NIL;
    cnt[i] = 0;
  }
  for (int p = plist; p != NIL;) {
    int mxo = ptl[p].x > T->monox ? 1 : 0;
    int myo = ptl[p].y > T->monoy ? 1 : 0;
    int mzo = ptl[p].z > T->monoz ? 1 : 0;
    int m = mxo + 2 * (myo + 2 * mzo);
    cnt[m]++;
    int next = ptl[p].sibling;
    ptl[p].sibling = head[m];
    head[m] = p;
    p = next;
  }
  int i0;
  for (i0 = 0; i0 < 8; i0++)
    if (cnt[i0] > 0) break;
  int divides = T->nodesize > 0.5L * MINCELLWIDTH_OR;
#define DIVIDE(c) (divides && (c) >= LEAF_MIN_OR)
  int first = free_node, now = free_node;
  if (DIVIDE(cnt[i0]))
    T->daughter = NODE_ID(first);
  else
    T->daughter = head[i0];
  int left = NIL;
  for (int i = 0; i < 8; i++) {
    if (DIVIDE(cnt[i])) {
      nodes[now].daughter = head[i];
      nodes[now].nparticle = cnt[i];
      if (left != NIL) *sib_of(ptl, nodes, left) = NODE_ID(now);
      left = NODE_ID(now);
      now++;
    } else if (cnt[i] > 0) {
      int q = head[i];
      if (left != NIL) *sib_of(ptl, nodes, left) = q;
      for (; q != NIL; q = ptl[q].sibling) left = q;
    }
  }
  /* T may have moved if nodes were reallocated: nodes is fixed-size here */
  *sib_of(ptl, nodes, left) = nodes[t].sibling;
  free_node = now;
  int job = first;
  for (int i = 0; i < 8; i++) {
    if (DIVIDE(cnt[i])) {
      free_node = divide_node(nodes, ptl, job, free_node, thetasq, variant);
      job++;
    }
  }
#undef DIVIDE
  return free_node;
}

/* Make_Tree3 (ost.ver2.c:146-160), RECURSIVE. */
static void make_tree(Node *nodes, Src *ptl, int np, float thetasq, int variant) {
  nodes[0].sibling = NIL;
  for (int i = 0; i < np; i++) ptl[i].sibling = i + 1;
  ptl[np - 1].sibling = NIL;
  nodes[0].daughter = 0;
  nodes[0].nparticle = np;
  divide_node(nodes, ptl, 0, 1, thetasq, variant);
}

/* treeforcesearch3 with nodeopen3/AddNode/AddPar (ost.ver2.c:247-351),
 * vfact2 = 1. */
static void tree_walk(const Spline *s, const Node *nodes, const Src *ptl, Target *p, float rspheresq,
                      int variant) {
  const float vfact2 = 1.0f;
  int ptr = NODE_ID(0);
  while (ptr != NIL) {
    if (IS_NODE(ptr)) {
      const Node *nd = &nodes[NODE_OF(ptr)];
      float ox = p->x - nd->monox, oy = p->y - nd->monoy, oz = p->z - nd->monoz;
      float od2 = ox * ox + oy * oy + oz * oz;
      if (od2 < nd->dist_over_thetasq) {
        ptr = nd->daughter;
      } else {
        float tmpx = (p->x) - (nd->monox), tmpy = (p->y) - (nd->monoy), tmpz = (p->z) - (nd->monoz);
        float dist2 = (tmpx * tmpx + tmpy * tmpy + tmpz * tmpz);
        if (dist2 <= rspheresq) {
          float dist = sqrt(dist2);
          float Qxx = nd->quad[0], Qyy = nd->quad[1], Qzz = nd->quad[2];
          float Qxy = nd->quad[3], Qxz = nd->quad[4], Qyz = nd->quad[5];
          float trQ = nd->trQ;
          float qxx1 = Qxx * tmpx + Qxy * tmpy + Qxz * tmpz;
          float qxx2 = Qxy * tmpx + Qyy * tmpy + Qyz * tmpz;
          float qxx3 = Qxz * tmpx + Qyz * tmpy + Qzz * tmpz;
          float qxy = Qxx * tmpx * tmpx + Qyy * tmpy * tmpy + Qzz * tmpz * tmpz +
                      2 * (Qxy * tmpx * tmpy + Qxz * tmpx * tmpz + Qyz * tmpy * tmpz);
          float f1, f2, f3;
          cell_grav(s, dist, &f1, &f2, &f3);
          float tmptmp = nd->mass * f1 + trQ * f2 + qxy * f3;
          float two2 = 2 * f2;
          if (variant == OR_VARIANT_A) { /* ost.ver2.c:273-275 as written */
            (p->axyz[0]) += vfact2 * (tmpx * tmptmp + qxx1 * two2);
            (p->axyz[0]) += vfact2 * (tmpx * tmptmp + qxx1 * two2);
            (p->axyz[0]) += vfact2 * (tmpx * tmptmp + qxx1 * two2);
          } else {
            (p->axyz[0]) += vfact2 * (tmpx * tmptmp + qxx1 * two2);
            (p->axyz[1]) += vfact2 * (tmpy * tmptmp + qxx2 * two2);
            (p->axyz[2]) += vfact2 * (tmpz * tmptmp + qxx3 * two2);
          }
        }
        ptr = nd->sibling;
      }
    } else {
      const Src *q = &ptl[ptr];
      float tmpx = p->x - q->x, tmpy = p->y - q->y, tmpz = p->z - q->z;
      float dist2 = (tmpx * tmpx + tmpy * tmpy + tmpz * tmpz);
      if (dist2 <= rspheresq) {
        float dist = sqrt(dist2);
        float fplmf = point_grav(s, dist) * q->mass;
        (p->axyz[0]) += tmpx * fplmf * vfact2;
        (p->axyz[1]) += tmpy * fplmf * vfact2;
        (p->axyz[2]) += tmpz * fplmf * vfact2;
      }
      ptr = q->sibling;
    }
  }
}

/* DirectSummation (treecorrection.c:177-219). Variant A adds every target's
 * sum to the first target (pos->axyz); B to each target. */
static void direct_sum(const Spline *s, int ngrv, const Src *g, int npos, Target *pos, float rsphere,
                       int variant) {
  double rspheresq = rsphere * rsphere;
  float vfact2 = 1.0f;
  for (int i = 0; i < npos; i++) {
    float ax = 0, ay = 0, az = 0;
    double px = pos[i].x, py = pos[i].y, pz = pos[i].z;
    for (int j = 0; j < ngrv; j++) {
      double tx = px - g[j].x, ty = py - g[j].y, tz = pz - g[j].z;
      double d2 = tx * tx + ty * ty + tz * tz;
      if (d2 <= rspheresq) {
        float dist = sqrt(d2);
        float f = point_grav(s, dist);
        f = f * g[j].mass;
        ax += tx * f;
        ay += ty * f;
        az += tz * f;
      }
    }
    Target *dst = variant == OR_VARIANT_A ? &pos[0] : &pos[i];
    dst->axyz[0] += vfact2 * ax;
    dst->axyz[1] += vfact2 * ay;
    dst->axyz[2] += vfact2 * az;
  }
}

/* treecorrection (treecorrection.c:225-475) for one rank owning [0,N)^3. */
int or_tree_force(int n, int64_t np, const double *pos, float theta, float rsphere, float eps,
                  int variant, float *force) {
  Spline *s = (Spline *)malloc(sizeof(Spline));
  if (!s) return -1;
  spline_build(s, n, eps);
  float theta2 = theta * theta;
  float rspheresq = rsphere * rsphere;
  double w = rsphere;

  /* ghosts: periodic images inside [-w, N+w)^3, float absolute positions,
   * in particle order then shift order (single-rank ppadding) */
  int64_t gcap = 1024, ng = 0;
  float *gpos = (float *)malloc(sizeof(float) * 3 * gcap);
  for (int64_t i = 0; i < np; i++) {
    for (int sidx = 0; sidx < 27; sidx++) {
      int sh[3] = {sidx % 3 - 1, (sidx / 3) % 3 - 1, sidx / 9 - 1};
      if (!sh[0] && !sh[1] && !sh[2]) continue;
      double y[3];
      int inside = 1;
      for (int d = 0; d < 3; d++) {
        y[d] = pos[3 * i + d] + sh[d] * (double)n;
        if (!(y[d] >= -w && y[d] < n + w)) inside = 0;
      }
      if (!inside) continue;
      if (ng == gcap) {
        gcap *= 2;
        gpos = (float *)realloc(gpos, sizeof(float) * 3 * gcap);
      }
      gpos[3 * ng] = (float)y[0];
      gpos[3 * ng + 1] = (float)y[1];
      gpos[3 * ng + 2] = (float)y[2];
      ng++;
    }
  }

  /* chaining mesh (BasicCell.c:10-42, BasicCell.h:33-63). Each bucket's
   * list is head-inserted: ghosts (reverse order) come first, then the real
   * particles in reverse index order. With OpenMP only buckets with
   * iz < floor((N+8)/4) are linked (BasicCell.c:88-92). */
  double xmin = 0 - CELLWIDTH_OR;
  double xmax = n + CELLWIDTH_OR;
  ptrdiff_t mx = ceil((xmax - xmin) / CELLWIDTH_OR), my = mx, mz = mx;
  int nzlink = (xmax - xmin) / CELLWIDTH_OR;
  ptrdiff_t nb = mx * my * mz;
  int64_t *cnt = (int64_t *)calloc(nb + 1, sizeof(int64_t));
  int64_t nall = np + ng;
  int64_t *bucket_of = (int64_t *)malloc(sizeof(int64_t) * nall);
  for (int64_t i = 0; i < nall; i++) {
    double x, y, z;
    if (i < np) {
      x = pos[3 * i];
      y = pos[3 * i + 1];
      z = pos[3 * i + 2];
    } else {
      x = gpos[3 * (i - np)];
      y = gpos[3 * (i - np) + 1];
      z = gpos[3 * (i - np) + 2];
    }
    ptrdiff_t ix = (x - xmin) / CELLWIDTH_OR, iy = (y - xmin) / CELLWIDTH_OR, iz = (z - xmin) / CELLWIDTH_OR;
    if (iz >= nzlink || ix < 0 || iy < 0 || iz < 0 || ix >= mx || iy >= my) {
      bucket_of[i] = -1;
      continue;
    }
    bucket_of[i] = ix + mx * (iy + my * iz);
    cnt[bucket_of[i] + 1]++;
  }
  for (ptrdiff_t b = 0; b < nb; b++) cnt[b + 1] += cnt[b];
  /* list order inside a bucket: ghosts reversed, then reals reversed */
  int64_t *list = (int64_t *)malloc(sizeof(int64_t) * (nall ? nall : 1));
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * nb);
  for (ptrdiff_t b = 0; b < nb; b++) fill[b] = cnt[b];
  for (int64_t i = nall - 1; i >= np; i--)
    if (bucket_of[i] >= 0) list[fill[bucket_of[i]]++] = i;
  for (int64_t i = np - 1; i >= 0; i--)
    if (bucket_of[i] >= 0) list[fill[bucket_of[i]]++] = i;
  free(fill);

  for (int64_t i = 0; i < 3 * np; i++) force[i] = 0.0f;

#pragma omp parallel
  {
    int64_t cap_src = 0;
    Src *grvp = NULL;
    Node *nodes = NULL;
    Target *tp = NULL;
    int64_t cap_t = 0;
#pragma omp for schedule(dynamic)
    for (ptrdiff_t ii = 0; ii < nb; ii++) {
      ptrdiff_t iz = ii / (mx * my);
      if (iz == mz - 1 || iz == 0) continue;
      ptrdiff_t iy = (ii % (mx * my)) / mx;
      if (iy == my - 1 || iy == 0) continue;
      ptrdiff_t ix = ii % mx;
      if (ix == mx - 1 || ix == 0) continue;
      double cx = CELLWIDTH_OR * (ix - 0.5L) + 0, cy = CELLWIDTH_OR * (iy - 0.5L) + 0,
             cz = CELLWIDTH_OR * (iz - 0.5L) + 0;
      /* Dump2Pos (treecorrection.c:53-98): real particles of this bucket */
      int64_t b0 = cnt[ii], b1 = cnt[ii + 1];
      int64_t npos = 0;
      for (int64_t q = b0; q < b1; q++)
        if (list[q] < np) npos++;
      if (npos == 0) continue;
      if (npos > cap_t) {
        cap_t = npos;
        tp = (Target *)realloc(tp, sizeof(Target) * cap_t);
      }
      npos = 0;
      for (int64_t q = b0; q < b1; q++) {
        int64_t i = list[q];
        if (i >= np) continue;
        tp[npos].x = pos[3 * i] - cx;
        tp[npos].y = pos[3 * i + 1] - cy;
        tp[npos].z = pos[3 * i + 2] - cz;
        tp[npos].axyz = force + 3 * i;
        npos++;
      }
      /* Dump2GrvP (treecorrection.c:99-148): 3x3x3 buckets */
      ptrdiff_t imin = ix - 1 > 0 ? ix - 1 : 0, jmin = iy - 1 > 0 ? iy - 1 : 0, kmin = iz - 1 > 0 ? iz - 1 : 0;
      ptrdiff_t imax = ix + 2 < mx ? ix + 2 : mx, jmax = iy + 2 < my ? iy + 2 : my, kmax = iz + 2 < mz ? iz + 2 : mz;
      int64_t ngrv = 0;
      for (ptrdiff_t k = kmin; k < kmax; k++)
        for (ptrdiff_t j = jmin; j < jmax; j++)
          for (ptrdiff_t i = imin; i < imax; i++) {
            ptrdiff_t b = i + mx * (j + my * k);
            ngrv += cnt[b + 1] - cnt[b];
          }
      if (ngrv + 1 > cap_src) {
        cap_src = ngrv + 1;
        grvp = (Src *)realloc(grvp, sizeof(Src) * cap_src);
        nodes = (Node *)realloc(nodes, sizeof(Node) * cap_src);
      }
      ngrv = 0;
      for (ptrdiff_t k = kmin; k < kmax; k++)
        for (ptrdiff_t j = jmin; j < jmax; j++)
          for (ptrdiff_t i = imin; i < imax; i++) {
            ptrdiff_t b = i + mx * (j + my * k);
            for (int64_t q = cnt[b]; q < cnt[b + 1]; q++) {
              int64_t id = list[q];
              if (id >= np) {
                grvp[ngrv].x = gpos[3 * (id - np)] - cx;
                grvp[ngrv].y = gpos[3 * (id - np) + 1] - cy;
                grvp[ngrv].z = gpos[3 * (id - np) + 2] - cz;
              } else {
                grvp[ngrv].x = pos[3 * id] - cx;
                grvp[ngrv].y = pos[3 * id + 1] - cy;
                grvp[ngrv].z = pos[3 * id + 2] - cz;
              }
              grvp[ngrv].mass = 1.0f;
              ngrv++;
            }
          }
      if (ngrv >= DIRECTSUM_OR) {
        make_tree(nodes, grvp, (int)ngrv, theta2, variant);
        for (int64_t t = 0; t < npos; t++) tree_walk(s, nodes, grvp, &tp[t], rspheresq, variant);
      } else {
        direct_sum(s, (int)ngrv, grvp, (int)npos, tp, rsphere, variant);
      }
    }
    free(grvp);
    free(nodes);
    free(tp);
  }
  free(list);
  free(bucket_of);
  free(cnt);
  free(gpos);
  free(s);
  return 0;
}

/* Exact pairwise sum of the interpolated law within rsphere (minimum image),
 * accumulated in double; no tree. */
int or_direct_short_force(int n, int64_t np, const double *pos, float rsphere, float eps,
                          int64_t nt, const int64_t *targets, double *force) {
  Spline *s = (Spline *)malloc(sizeof(Spline));
  if (!s) return -1;
  spline_build(s, n, eps);
  double r2max = (double)rsphere * rsphere;
#pragma omp parallel for schedule(dynamic)
  for (int64_t t = 0; t < nt; t++) {
    int64_t i = targets[t];
    double f[3] = {0, 0, 0};
    for (int64_t j = 0; j < np; j++) {
      double d[3];
      for (int c = 0; c < 3; c++) {
        d[c] = pos[3 * i + c] - pos[3 * j + c];
        if (d[c] >= 0.5 * n) d[c] -= n;
        if (d[c] < -0.5 * n) d[c] += n;
      }
      double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 > r2max) continue;
      float dist = sqrt(r2);
      double fv = point_grav(s, dist);
      for (int c = 0; c < 3; c++) f[c] += d[c] * fv;
    }
    for (int c = 0; c < 3; c++) force[3 * t + c] = f[c];
  }
  free(s);
  return 0;
}

/* ---------------------------------------------------------------- Ewald */
/* FP64 periodic Ewald sum (new; the reference has none). Force on target i
 *   F_i = sum_j d_ij [erfc(a r)/r^3 + 2a/sqrt(pi) exp(-a^2 r^2)/r^2]      (r < rcut, min image)
 *       + sum_j d_ij [1/(r^2+eps^2)^{3/2} - 1/r^3]                         (softening, r < rcut)
 *       - (4 pi / V) sum_{k != 0} exp(-k^2/4a^2)/k^2 k Im[e^{ik.x_i} conj(S(k))]
 * with d_ij = x_j - x_i, S(k) = sum_j e^{ik.x_j}, V = N^3, then / N^2. */
int or_ewald_force(int n, int64_t np, const double *pos, float eps, int64_t nt,
                   const int64_t *targets, double rcut, double alpha, int kmax, double *force) {
  const double L = n, V = L * L * L, tpi = 6.283185307179586476925286766559;
  double e2 = (double)eps * eps;
  double rc2 = rcut * rcut;
  /* k-space: half space of integer vectors with 0 < |m|^2 <= kmax^2 */
  int M = kmax;
  int nk = 0;
  int *mv = (int *)malloc(sizeof(int) * 3 * (2 * M + 1) * (2 * M + 1) * (2 * M + 1));
  for (int mz = 0; mz <= M; mz++)
    for (int my = -M; my <= M; my++)
      for (int mx = -M; mx <= M; mx++) {
        if (mz == 0 && (my < 0 || (my == 0 && mx <= 0))) continue;
        if (mx * mx + my * my + mz * mz > M * M) continue;
        mv[3 * nk] = mx;
        mv[3 * nk + 1] = my;
        mv[3 * nk + 2] = mz;
        nk++;
      }
  double *S = (double *)calloc(2 * (size_t)nk, sizeof(double));
#pragma omp parallel
  {
    double *Sl = (double *)calloc(2 * (size_t)nk, sizeof(double));
    double *ex = (double *)malloc(sizeof(double) * 2 * (2 * M + 1) * 3);
#pragma omp for schedule(static)
    for (int64_t j = 0; j < np; j++) {
      for (int c = 0; c < 3; c++) {
        double *e = ex + 2 * (2 * M + 1) * c;
        for (int m = -M; m <= M; m++) {
          double ph = tpi * m * pos[3 * j + c] / L;
          e[2 * (m + M)] = cos(ph);
          e[2 * (m + M) + 1] = sin(ph);
        }
      }
      for (int k = 0; k < nk; k++) {
        const double *a = ex + 2 * (mv[3 * k] + M);
        const double *b = ex + 2 * (2 * M + 1) + 2 * (mv[3 * k + 1] + M);
        const double *c = ex + 4 * (2 * M + 1) + 2 * (mv[3 * k + 2] + M);
        double abr = a[0] * b[0] - a[1] * b[1], abi = a[0] * b[1] + a[1] * b[0];
        Sl[2 * k] += abr * c[0] - abi * c[1];
        Sl[2 * k + 1] += abr * c[1] + abi * c[0];
      }
    }
#pragma omp critical
    for (int k = 0; k < 2 * nk; k++) S[k] += Sl[k];
    free(Sl);
    free(ex);
  }
  const double spi = 1.7724538509055160272981674833411;
#pragma omp parallel for schedule(dynamic)
  for (int64_t t = 0; t < nt; t++) {
    int64_t i = targets[t];
    double f[3] = {0, 0, 0};
    for (int64_t j = 0; j < np; j++) {
      if (j == i) continue;
      double d[3];
      for (int c = 0; c < 3; c++) {
        d[c] = pos[3 * j + c] - pos[3 * i + c];
        d[c] -= L * floor(d[c] / L + 0.5);
      }
      double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 >= rc2) continue;
      double r = sqrt(r2);
      double g = erfc(alpha * r) / (r2 * r) + 2 * alpha / spi * exp(-alpha * alpha * r2) / r2;
      g += 1.0 / pow(r2 + e2, 1.5) - 1.0 / (r2 * r);
      for (int c = 0; c < 3; c++) f[c] += d[c] * g;
    }
    for (int k = 0; k < nk; k++) {
      double kv[3] = {tpi * mv[3 * k] / L, tpi * mv[3 * k + 1] / L, tpi * mv[3 * k + 2] / L};
      double k2 = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      double ph = kv[0] * pos[3 * i] + kv[1] * pos[3 * i + 1] + kv[2] * pos[3 * i + 2];
      double cr = cos(ph), ci = sin(ph);
      /* Im[e^{i ph} conj(S)] = ci*Sr - cr*Si */
      double im = ci * S[2 * k] - cr * S[2 * k + 1];
      double w = 2.0 * 4.0 * M_PI / V * exp(-k2 / (4 * alpha * alpha)) / k2 * im; /* x2: half space */
      for (int c = 0; c < 3; c++) f[c] -= w * kv[c];
    }
    double inv = 1.0 / (L * L);
    for (int c = 0; c < 3; c++) force[3 * t + c] = f[c] * inv;
  }
  free(S);
  free(mv);
  return 0;
}
