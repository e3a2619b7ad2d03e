/*
 * CPU oracle for the TreePM force path: a C restatement of the reference's
 * algorithm (kjhan0606/LagEunha, GOTPM build) plus an FP64 periodic Ewald
 * direct sum. TEST INFRASTRUCTURE ONLY: tests/, the smoke check and
 * bench.py's CPU-baseline leg use it as the checker; the engine never links
 * it and has no CPU fallback onto it.
 *
 * Units follow the reference: lengths in mesh cells on a periodic box
 * [0,N)^3, G = particle mass = 1, and every force carries the reference's
 * 1/N^2 factor (Cosmos/psolver.c:28,59-66; OST/Model4TreeForce.c:57,111).
 */
#ifndef TPM_ORACLE_H
#define TPM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Variants of the short-range correction: A reproduces the reference as
 * written, B applies the three one-line fixes (Qyz moment, AddNode y/z,
 * DirectSummation target index). */
enum { OR_VARIANT_A = 0, OR_VARIANT_B = 1 };

/* XYZDBL position decode (eunha.h:1228-1232): fmod(offset + grid + N, N). */
void or_decode(int n, int64_t np, const uint64_t *indx, const float *off, double *pos);

/* TSC density contrast rho - 1 on [z][y][x] (Cosmos/pmmain.h:81-159,
 * Cosmos/pmmain.c:112-185,283-336). */
int or_tsc_density(int n, int64_t np, const double *pos, float *mesh);

/* Potential after the Green's function (Cosmos/psolver.c:13-86) and the c2r,
 * [z][y][x]. */
int or_potential(int n, int64_t np, const double *pos, float efold, float *phi);

/* PM force: TSC, Poisson solve, 4-point gradient and TSC interpolation
 * (Cosmos/pmmain.c:390-527, Cosmos/fda4.h:11-103,276-384). */
int or_pm_force(int n, int64_t np, const double *pos, float efold, float *force);

/* Gradient-only variant of the PM force for a given potential mesh. */
int or_fda4_force(int n, int64_t np, const double *pos, const float *phi, float *force);

/* Short-range law table diff/slope[NSPLINE][3] (OST/Model4TreeForce.c:48-91). */
int or_spline_table(int n, float eps, double *diff, double *slope);
int or_nspline(void);

/* Short-range tree correction (Cosmos/treecorrection.c:225-475,
 * OST/ost.ver2.c:36-351). variant = OR_VARIANT_A or OR_VARIANT_B. */
int or_tree_force(int n, int64_t np, const double *pos, float theta, float rsphere, float eps,
                  int variant, float *force);

/* Exact pairwise short-range sum: every pair within rsphere through the
 * interpolated law (no tree); the limit the tree walk approaches. */
int or_direct_short_force(int n, int64_t np, const double *pos, float rsphere, float eps,
                          int64_t nt, const int64_t *targets, double *force);

/* FP64 periodic Ewald force with Plummer softening eps on the pairs inside
 * the real-space cutoff, for nt target indices, in the reference's units.
 * alpha_cells = Ewald split in cells, kmax = k-space cutoff in units of
 * 2*pi/N. Multithreaded with OpenMP. */
int or_ewald_force(int n, int64_t np, const double *pos, float eps, int64_t nt,
                   const int64_t *targets, double rcut, double alpha, int kmax, double *force);

#ifdef __cplusplus
}
#endif
#endif
