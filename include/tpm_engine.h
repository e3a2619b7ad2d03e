/*
 * tpm_engine.h — C ABI of the B200 TreePM force engine.
 *
 * This is the drop-in boundary for the force evaluation of EUNHA's GOTPM
 * build (kjhan0606/LagEunha). The engine replaces
 *   void pmmain(SimParameters *, EvolFact)                 Cosmos/pmmain.c:390
 *   void treecorrection(SimParameters *, DeterminedEvolFact *)
 *                                                          Cosmos/treecorrection.c:225
 *   void TreeMain(SimParameters *, DeterminedEvolFact *)   Cosmos/Treemain.h:19
 *                                                          (GOTPM body Treemain.c:578-664)
 * and their helpers psolver (Cosmos/psolver.c:13) and fda4 (Cosmos/fda4.c:31).
 * Those take SimParameters; this ABI takes plain pointers and sizes instead,
 * so a caller fills tpm_params from the SimParameters fields it already has
 * (NX, THETA, RSPHERE, GRV_EPSILON, GRV_EFOLD: eunha.h:1033-1090) and hands
 * over the particle array it already owns.
 *
 * Every entry point returns 0 on success or a negative TPM_E* code; the
 * message of the last failure on the calling thread is tpm_last_error().
 * (The reference exits on error: Cosmos/treecorrection.c:245-246.)
 *
 * One tpm_ctx owns one periodic box on one GPU and its own CUDA stream.
 * Calls on one context are not re-entrant; distinct contexts may be used from
 * distinct threads.
 */
#ifndef TPM_ENGINE_H
#define TPM_ENGINE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define TPM_OK 0
#define TPM_E_ARG (-1)      /* bad argument */
#define TPM_E_NOMEM (-2)    /* device allocation failed */
#define TPM_E_CUDA (-3)     /* CUDA runtime or launch failure */
#define TPM_E_STATE (-4)    /* call out of order (e.g. forces before particles) */
#define TPM_E_OVERFLOW (-5) /* a bounded device work queue or stack overflowed */
#define TPM_E_NODEV (-6)    /* no usable CUDA device */

/* ---- force laws ---- */
/* TPM_LAW_REFERENCE: the reference's split. PM Green's function
 *   -1/(pi n^2) exp(-n^2 (pi efold / N)^2) / N^3       (Cosmos/psolver.c:58-72)
 * and the tabulated residual law of OST/Model4TreeForce.c:48-116 (PMFITPARA)
 * cut at rsphere. TPM_LAW_GAUSSIAN: a Gaussian split of scale rs_split cells
 * with the matching erfc short-range law and TSC-deconvolved Green's
 * function (no counterpart in the reference; see tpm_params). */
#define TPM_LAW_REFERENCE 0
#define TPM_LAW_GAUSSIAN 1

/* ---- which parts of the force ---- */
#define TPM_PART_PM 1u
#define TPM_PART_TREE 2u
#define TPM_PART_ALL 3u

/* ---- where a buffer lives ---- */
#define TPM_MEM_HOST 0
#define TPM_MEM_DEVICE 1

typedef struct tpm_params {
  int32_t n_mesh;   /* PM mesh cells per side, NX = NY = NZ (eunha.h:1090) */
  int32_t law;      /* TPM_LAW_* */
  float theta;      /* opening angle THETA (eunha.h:1076); reference default 0.3 */
  float rsphere;    /* short-range cutoff RSPHERE in cells; default 4 */
  float epsilon;    /* Plummer softening GRV_EPSILON in cells */
  float efold;      /* PM split GRV_EFOLD (reference law); default 0.9 */
  float rs_split;   /* Gaussian split scale in cells (TPM_LAW_GAUSSIAN only) */
  float particle_mass; /* particle mass (TDM_MASS); reference runs use 1 */
} tpm_params;

typedef struct tpm_ctx tpm_ctx;

/* Defaults of the reference's parameter file for the GOTPM build
 * (Params/header.c:148-149,501-505,651-653): theta 0.3, rsphere 4,
 * efold 0.9, epsilon 0.1, mass 1. */
void tpm_default_params(tpm_params *p, int32_t n_mesh);

const char *tpm_last_error(void);
const char *tpm_version(void);

/* Number of CUDA devices visible to the process (0 when there is none). */
int tpm_device_count(void);

/* Create a context on CUDA device `device` with capacity for up to np_max
 * particles (device memory is reserved lazily and grown on demand). */
int tpm_create(const tpm_params *params, int device, tpm_ctx **out);
int tpm_destroy(tpm_ctx *ctx);
int tpm_set_params(tpm_ctx *ctx, const tpm_params *params);
int tpm_get_params(const tpm_ctx *ctx, tpm_params *out);

/* ---- particle state ---- */

/* Positions as uint32 fixed point per axis, AoS [np][3]:
 * u = round(frac(x / N) * 2^32), x in cells. vel may be NULL (zeros). */
int tpm_load_fixed(tpm_ctx *ctx, int64_t np, const uint32_t *pos, const float *vel, int mem);

/* Positions in the reference's XYZDBL form (eunha.h:1212,1228-1232): an AoS
 * array of records of `stride` bytes holding a uint64 Lagrangian index
 * (top byte = flags) at byte offset off_indx, float x,y,z offsets at off_pos
 * and float vx,vy,vz at off_vel (off_vel < 0: zero velocities).
 * GOTPM dmparticletype: stride 32, offsets 0, 8, 20 (eunha.h:390-400);
 * treedmparticletype: stride 40, offsets 8, 16, 28 (eunha.h:401-412). */
int tpm_load_lagrangian(tpm_ctx *ctx, int64_t np, const void *particles, int64_t stride,
                        int64_t off_indx, int64_t off_pos, int64_t off_vel, int mem);

/* Evaluate the forces of `parts` (TPM_PART_*) on the loaded particles and
 * keep them on the device. Reference units: F in cells with G = m = 1 carries
 * the reference's 1/N^2 factor. */
int tpm_compute_forces(tpm_ctx *ctx, unsigned parts);

/* Copy the last forces out, AoS [np][3] float, in the caller's particle order. */
int tpm_read_forces(tpm_ctx *ctx, float *out, int mem);

/* v += fact2_pm * F_pm + fact2_tree * F_tree using the last forces
 * (Cosmos/fda4.h:297-299; OST/ost.ver2.c:273-291). */
int tpm_kick(tpm_ctx *ctx, float fact2_pm, float fact2_tree);

/* Drift: x += v * pfact (cells), accumulated in FP64 into the fixed-point
 * positions (Cosmos/stepevolv.c:38-113). */
int tpm_drift(tpm_ctx *ctx, double pfact);

int tpm_read_velocities(tpm_ctx *ctx, float *out, int mem);
int tpm_read_positions(tpm_ctx *ctx, uint32_t *out, int mem);

/* Write the velocities back into a record array of the tpm_load_lagrangian
 * form (only the vx,vy,vz fields are touched). */
int tpm_store_lagrangian_velocities(tpm_ctx *ctx, void *particles, int64_t stride, int64_t off_vel,
                                    int mem);

/* Wait for all work queued on the context's stream. */
int tpm_sync(tpm_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t) so callers can order their own
 * work against it. */
void *tpm_stream(tpm_ctx *ctx);

/* ---- drop-in forms of the reference entry points ---- */

/* pmmain (Cosmos/pmmain.c:390-527) on a GOTPM dmparticletype array:
 * v += fact2 * F_PM. fact2 is the one pmmain's fda4 picks from EvolFact for
 * the current PMSTATUS (Cosmos/fda4.c:48-62). */
int tpm_pmmain(tpm_ctx *ctx, void *dm_particles, int64_t np, float fact2);

/* treecorrection (Cosmos/treecorrection.c:225-475) on a GOTPM
 * treedmparticletype array: v += fact2 * F_tree, fact2 = EvolFactArr[0].fact2
 * (treecorrection.c:227). */
int tpm_treecorrection(tpm_ctx *ctx, void *treedm_particles, int64_t np, float fact2);

/* The GOTPM TreeMain step (Cosmos/Treemain.c:578-664): theta follows the
 * step schedule 0.3 (step < 10), 0.35 (< 20), 0.4 (< 60), 0.45 after
 * (Treemain.c:598-601) and stays set on the context, then treecorrection. */
int tpm_treemain(tpm_ctx *ctx, void *treedm_particles, int64_t np, float fact2, int stepcount);

/* ---- the global step (expanding background) ---- */

/* Cosmology of the background: OMEP, OMEPLAM, WLAM0, WLAM1 and AMAX of the
 * reference's SimParameters (eunha.h:1056-1072). */
typedef struct tpm_cosmology {
  float omep, omeplam, wlam0, wlam1, amax;
} tpm_cosmology;

/* The reference's EvolFact (Cosmos/CosmosEvolFactor.h:1-6); afact and bfact
 * are unused and set to 0. */
typedef struct tpm_evolfact {
  float afact, bfact, pfact;
  float fact1, fact2;
  float fact1_push, fact2_push;
  float fact1_pull, fact2_pull;
} tpm_evolfact;

/* GetEvolFactor (Cosmos/CosmosEvolFactor.c:230-255) for the step from
 * anow - astep/2 to anow + astep/2 on an nx^3 mesh; host only, no GPU. */
int tpm_evol_factors(const tpm_cosmology *cosmo, int32_t nx, float anow, float astep, tpm_evolfact *out);

/* v *= fact1 (HubbleDragDM, Cosmos/globalT.c:102-110). */
int tpm_hubble_drag(tpm_ctx *ctx, float fact1);

/* One GOTPM global step in KICK status (Cosmos/globalT.c:221-305 between
 * synchronisation points): Hubble drag with fact1, PM and tree kicks with
 * fact2, drift with pfact = astep * NX. With the reference law the opening
 * angle follows TreeAndPreFoFmain's step schedule (Cosmos/globalT.c:41-44).
 * The caller advances anow by astep afterwards. */
int tpm_step(tpm_ctx *ctx, const tpm_cosmology *cosmo, float anow, float astep, int32_t stepcount);

/* PMSTATUS of the reference (eunha.h:72-77). */
#define TPM_PUSH 0
#define TPM_PULL 1
#define TPM_KICK 2

/* The factors one status applies (replaces the selections of
 * PM_PULL_AND_PUSH, Cosmos/globalT.c:119-127, fda4, Cosmos/fda4.c:48-62, and
 * TREE_HALF, Cosmos/indT.h:98-118):
 *   drag     KICK fact1, PULL fact1_pull, PUSH fact1_push;
 *   pm_kick  KICK fact2, PULL fact2_pull, PUSH fact2_push / GetFact1(anow,
 *            anow + astep/2), which is fact2_push / fact1_push;
 *   tree_kick  fact2 in every status: TREE_HALF stores the full-step fact2
 *            for PULL and for the PUSH half's KICK call alike.
 * Any output pointer may be NULL. Host only. */
int tpm_status_factors(const tpm_evolfact *e, int32_t status, float *drag, float *pm_kick, float *tree_kick);

/* One status of a global step on the particles the context holds (the body
 * of PM_PULL_AND_PUSH plus TreeAndPreFoFmain's tree kick,
 * Cosmos/globalT.c:113-134,85-87): v *= drag, then v += pm_kick F_pm +
 * tree_kick F_tree with the factors of tpm_status_factors. The forces are
 * evaluated unless the context already holds them for the current positions
 * (the PUSH half of a synchronisation step reuses the PULL half's forces: the
 * positions have not moved). No drift. */
int tpm_status_kick(tpm_ctx *ctx, const tpm_cosmology *cosmo, float anow, float astep, int32_t status);

/* One global step of GOTPM_Cosmos_GlobalT (Cosmos/globalT.c:221-305) with
 * the reference's status sequencing: sync == 0, KICK; sync != 0 (a
 * synchronisation or PreFoF step, flagsyncpdata/flagPreFoF), PULL then
 * PUSH; then the drift with pfact. The opening-angle schedule is tpm_step's.
 * The caller advances anow by astep afterwards. */
int tpm_global_step(tpm_ctx *ctx, const tpm_cosmology *cosmo, float anow, float astep, int32_t stepcount,
                    int32_t sync);

/* ---- captured evaluations and ensembles ---- */

/* tpm_compute_forces replayed from a CUDA graph captured on the first call
 * (and again whenever the particle count, buffers or parameters change): the
 * same kernels and results, one launch, no stage times or counters. No
 * counterpart in the reference, which evaluates one box per process. */
int tpm_graph_compute(tpm_ctx *ctx, unsigned parts);

/* An ensemble of independent boxes (contexts on one device, each with its own
 * particle count, mesh size and parameters). One call evaluates every box
 * through one graph launch built from the boxes' captured graphs, so their
 * kernels overlap on the device, and synchronises once. The boxes stay owned
 * by the caller and must outlive the batch. No counterpart in the reference
 * (one box per MPI job). */
typedef struct tpm_batch tpm_batch;
int tpm_batch_create(tpm_ctx *const *boxes, int32_t nbox, tpm_batch **out);
int tpm_batch_destroy(tpm_batch *batch);
/* Forces of `parts` in every box, as tpm_compute_forces per box. */
int tpm_batch_compute(tpm_batch *batch, unsigned parts);
/* One global step per box (drag, forces, kicks, drift, as tpm_step without
 * the opening-angle schedule), box i at expansion factor anow[i] with step
 * astep[i]. */
int tpm_batch_step(tpm_batch *batch, const tpm_cosmology *cosmo, const float *anow, const float *astep);
/* Device time of the last tpm_batch_compute / tpm_batch_step launch, ms. */
int tpm_batch_time(tpm_batch *batch, float *ms);

/* ---- the autotuner ---- */

/* Launch shapes picked by timing candidates on the context's loaded
 * particles (each three times, median). TPM_TUNE_FFT: pencils per block of
 * the x transforms and kx columns per block of the y/z transforms (forces do
 * not change). TPM_TUNE_GROUPS: targets per warp group (16 or 32) and the
 * cube the groups are cut from (2^group_level cells, 4 or 8); the tree force
 * changes within its error, since a group opens a node if any target would.
 * The choice stays in the context; tpm_set_tuning applies it to other boxes
 * of the same size. 0 in fft_* means the built-in shape. No counterpart in the
 * reference. */
#define TPM_TUNE_FFT 1u
#define TPM_TUNE_GROUPS 2u
typedef struct tpm_tuning {
  int32_t fft_pencils_x, fft_cols;
  int32_t group_level, group_max;
  float ms_fft, ms_fft_default;    /* the chosen and the built-in shape, ms */
  float ms_walk, ms_walk_default;  /* groups + walk, chosen and built-in, ms */
} tpm_tuning;
int tpm_autotune(tpm_ctx *ctx, unsigned what, tpm_tuning *out);
int tpm_get_tuning(const tpm_ctx *ctx, tpm_tuning *out);
int tpm_set_tuning(tpm_ctx *ctx, const tpm_tuning *tuning);

/* ---- the request loop (served solves) ---- */

/* On one device, an admission thread admits requests in arrival order while
 * their device footprint fits under hbm_cap_bytes and in the free HBM
 * (context, upload, graph capture), and a launch thread runs the active
 * requests' steps as they become ready, so requests that arrive while others
 * run overlap with them on the device. Each request's particles, mesh and
 * tree stay on the device between its steps, in buffers taken from the
 * server's device arena. No counterpart in the reference (a batch MPI
 * job). */
typedef struct tpm_server tpm_server;

typedef struct tpm_request {
  tpm_params params;       /* the box's parameters (n_mesh, law, ...) */
  int64_t np;
  const uint32_t *pos;     /* host [np][3] fixed point, valid until done */
  const float *vel;        /* host [np][3] or NULL (zeros) */
  tpm_cosmology cosmo;
  float anow, astep;       /* step k runs at anow + k*astep */
  int32_t nsteps;          /* 0: one force evaluation; n >= 1: n global steps */
  uint32_t *pos_out;       /* host [np][3] or NULL: positions after the steps */
  float *vel_out;          /* host [np][3] or NULL: velocities after the steps */
  float *force_out;        /* host [np][3] or NULL: forces of the last evaluation */
} tpm_request;

#define TPM_REQ_QUEUED 0
#define TPM_REQ_ACTIVE 1
#define TPM_REQ_DONE 2
#define TPM_REQ_FAILED 3

typedef struct tpm_request_info {
  int32_t state;           /* TPM_REQ_* */
  int32_t status;          /* TPM_OK, or the error of a failed request */
  double t_submit, t_admit, t_done;  /* seconds since the server was created */
  int64_t device_bytes;    /* device memory held while active */
} tpm_request_info;

/* Device bytes a context for this mesh and particle count holds. */
int64_t tpm_estimate_bytes(int32_t n_mesh, int64_t np);
int tpm_server_create(int device, int64_t hbm_cap_bytes, int32_t max_active, tpm_server **out);
/* Non-blocking; the request's host buffers must stay valid until it is done. */
int tpm_server_submit(tpm_server *server, const tpm_request *req, int64_t *id);
int tpm_server_info(tpm_server *server, int64_t id, tpm_request_info *out);
/* Waits for request id (id < 0: every request submitted so far). */
int tpm_server_wait(tpm_server *server, int64_t id, double timeout_s);
/* [0] done [1] failed [2] peak active [3] peak device bytes [4] contexts
 * created [5] contexts reused [6] contexts evicted [7] deferred admissions;
 * microseconds the admission thread spent [8] making or re-parameterising
 * contexts [9] uploading particles [10] capturing graphs [11] reserving
 * memory; [12] device bytes the server's arena holds; returns the number of
 * words written (at most 13). */
int tpm_server_stats(tpm_server *server, int64_t *out, int n);
/* Claims device memory for the server's contexts now, so that admissions
 * up to `bytes` (at most the cap) take their buffers without a cudaMalloc.
 * The server otherwise claims memory in 1 GiB blocks as requests need it;
 * it keeps what it claimed until tpm_server_destroy. No reference
 * counterpart: the reference has no request loop. */
int tpm_server_reserve(tpm_server *server, int64_t bytes);
/* Finishes every submitted request, then stops the worker. */
int tpm_server_destroy(tpm_server *server);

/* ---- power spectrum of the mass assignment ---- */

/* With it enabled, every PM evaluation also bins |rho_k|^2 of the forward
 * transform, as the reference's CorrMeasure does after pmmain's forward FFT
 * (Cosmos/pmmain.c:480-481, Cosmos/Correlation.c:13-79): TSC window divided
 * out, kx < N/2, linear sharing between the bins floor(|m|) and its
 * neighbour. Costs one pass of bin additions inside the z transform. */
int tpm_set_power_spectrum(tpm_ctx *ctx, int enable);
/* From the last PM evaluation: P(k) per bin (bin i = |m| in mode numbers,
 * i = 1..N, bin 0 as accumulated), the correlation function xi at i cells,
 * sigma_8 for the box size in Mpc/h and the log slope of xi between 2 and 3
 * cells (Correlation.c:82-103). Fills min(nbins, N+1) entries and returns
 * that count. */
int tpm_power_spectrum(tpm_ctx *ctx, double boxsize, double *pk, double *cor, int32_t nbins, double *sigma8,
                       double *slope);

/* ---- friends-of-friends groups ---- */

/* Groups of particles linked by distance <= link (cells), as the reference's
 * pnew_fof_link grows them (FoF/fof.c:217-290; PreFoF, Cosmos/PreFoF.c:
 * 267-385, uses link 0.2 and at least 20 members). labels[i] (caller order)
 * is the smallest caller index of particle i's group if the group has at
 * least min_members particles, else -1; *ngroups counts those groups. Uses
 * the sort and octree of a force evaluation; the forces held before are
 * dropped. */
int tpm_fof(tpm_ctx *ctx, float link, int32_t min_members, int32_t *labels, int mem, int64_t *ngroups);

/* ---- the reference's snapshot files ---- */

/* What the ASCII header of a GOTPM snapshot says (FILE_HEADER,
 * Params/params.h:500-517, written by jwrite, Cosmos/CosmosRW/kjhrw.c:169).
 * ptype 0: dmparticletype records (32 bytes), 1: treedmparticletype (40). */
typedef struct tpm_snapshot_info {
  int64_t nx, ny, nz;
  int64_t np_dm, np_sph, np_star, np_agn;
  int32_t ptype, record_bytes;
  double anow, astep;
  float omep, omeplam, wlam0, wlam1, amax, boxsize, theta, epsilon, rsphere;
  int32_t stepcount;
  int64_t data_offset;  /* byte offset of the first dark-matter record */
} tpm_snapshot_info;
/* Parses the header (read_head, Params/header.c:72-104). */
int tpm_snapshot_info_read(const char *path, tpm_snapshot_info *info);
/* Reads dark-matter records [first, first + count) as they lie in the file
 * (record_bytes each); they load with tpm_load_lagrangian. */
int tpm_snapshot_read_dm(const char *path, const tpm_snapshot_info *info, void *records, int64_t first,
                         int64_t count);
/* Writes a snapshot the reference's jread accepts: the header lines in the
 * reference's key formats and np_dm dark-matter records (no other species,
 * no trailing parameter struct: jread then decomposes the domain itself). */
int tpm_snapshot_write(const char *path, const tpm_snapshot_info *info, const void *dm_records);

/* ---- diagnostics ---- */

/* FP64 periodic Ewald force (reference units, Plummer softening epsilon on
 * pairs inside the real-space cutoff) on nt target particles given by their
 * caller-order indices; forces [nt][3] double written to out (host). */
int tpm_ewald(tpm_ctx *ctx, int64_t nt, const int64_t *targets, double *out);

/* Per-stage device times (ms) of the last tpm_compute_forces, in the order
 * sort, deposit, fft, fda4, tree_build, tree_walk, finish; returns the
 * number of stages written (<= n). */
int tpm_stage_times(tpm_ctx *ctx, float *ms, int n);

/* Counters of the last force evaluation: [0] tree nodes, [1] particle-
 * particle interactions, [2] particle-node interactions, [3] walk groups,
 * [4] walk iterations, [5] nodes examined by the walk, [6] deepest walk stack. */
int tpm_counters(tpm_ctx *ctx, int64_t *out, int n);

/* Kernel launches issued by the last tpm_compute_forces. */
int64_t tpm_launch_count(tpm_ctx *ctx);

/* The spatial order of the last tpm_compute_forces: sorted 39-bit Morton
 * keys and the permutation (sorted slot -> caller index), np entries each,
 * host memory. Either pointer may be NULL. */
int tpm_read_order(tpm_ctx *ctx, uint64_t *keys, uint32_t *perm);

/* Mesh stages of the last PM evaluation, [z][y][x] n^3 floats, host memory:
 * TPM_MESH_DENSITY is the TSC mass per cell (the reference folds the same
 * mesh minus 1, Cosmos/pmmain.c:304), TPM_MESH_POTENTIAL the potential after
 * the Green's function and the c2r (Cosmos/pmmain.c:492). */
#define TPM_MESH_DENSITY 0
#define TPM_MESH_POTENTIAL 1
int tpm_read_mesh(tpm_ctx *ctx, int which, float *out);

/* ---- allocation-free ordering ---- */

/* ---- Streamed evaluations. A caller that evaluates one particle set after
 * another from host memory (the reference's pmmain/treecorrection callers
 * hand over host arrays every step) can overlap the host copies with the
 * evaluations: tpm_stream_submit queues the copy of `pos` (np x 3 uint32
 * fixed point, host; pinned memory lets the copy run asynchronously), the
 * evaluation of `parts` and the copy of the forces into `forces` (np x 3
 * float, host, caller order), and returns a ticket at once. The copy-in of
 * one submission and the copy-out of another run during the evaluation in
 * between. At most two submissions are in flight: the third call fails with
 * TPM_E_STATE until the first is waited for. Neither buffer may be touched
 * before tpm_stream_wait(ticket) returns; it reports the evaluation's errors.
 * The particles loaded in the context (tpm_load_*) stay as they were, unless
 * a larger np made the context grow its buffers (then load again before
 * tpm_compute_forces); tpm_read_forces has nothing to read afterwards. No
 * counterpart in the reference, which evaluates synchronously. */
int tpm_stream_submit(tpm_ctx *ctx, int64_t np, const uint32_t *pos, float *forces, unsigned parts,
                      int64_t *ticket);
int tpm_stream_wait(tpm_ctx *ctx, int64_t ticket);

/* ---- Zel'dovich initial conditions (Cosmos/CosmosIC: PMSeedForce.c,
 * Zeldovich.c, MakeParticle.c). One particle per point of an n^3 lattice,
 * from the reference's random sequence (Numerical Recipes ran3/gasdev,
 * CosmosIC/nr.c:317-384) in the reference's mode order, so a seed gives the
 * reference's field. */
typedef struct tpm_ic_params {
  int32_t device;
  int32_t n;            /* lattice points (= mesh cells) per side, 8..1024, 2^a 3^b 5^c */
  int64_t iseed;        /* the reference's ISEED (PMSeedForce.c:219-223): >= 0 draws
                           unit-amplitude noise with seed -1; < 0 draws with this seed,
                           scaled by velpot */
  const float *velpot;  /* host, (n/2)^2 + 1 floats: the amplitude pamp*bpower(rk)/rk^2 of
                           PMSeedForce.c:326 at each integer k^2 = i^2 + ky^2 + kz^2
                           (k in units of the fundamental mode); needed when iseed < 0 */
  float fnl, gnl;       /* local non-Gaussianity (Zeldovich.c:44-61) */
  float vamp;           /* growing-mode velocity factor COS_VAMP1 (PMSeedForce.c:250-292) */
  float pfact;          /* offset per unit velocity, AI * NX (MakeParticle.c:205) */
  /* second order only (tpm_ic_2lpt): COS_VAMP2, COS_DAMP1, COS_DAMP2
     (PMSeedForce.c:250-305; damp1 = 1, damp2 = -3/7 in the reference) */
  float vamp2, damp1, damp2;
  /* second order with fnl or gnl (TwoLPT.c:284-335): COSBOXSIZE [Mpc/h],
     OMEP, AMAX and the growth factor COS_GROWTH = bini/bnow */
  float boxsize, omep, amax, growth;
} tpm_ic_params;

/* The noise spectrum of PMSeedForce.c:293-399 (one rank): spec receives
 * n*n*(n/2+1) complex values (re, im floats), [z][y][kx]. Replaces the mode
 * loop of PMSeedForce.c:293-334 and the conjugate completion of the kx = 0
 * plane (PMSeedForce.c:346-399). */
int tpm_ic_noise(const tpm_ic_params *p, float *spec, int mem);

/* Zel'dovich particles: n^3 records of the reference's dark-matter layout
 * (eunha.h:390-400, GOTPM with XYZDBL: 8-byte index i + n(j + n k), float
 * offsets x y z, float velocities vx vy vz; 32 bytes each), in lattice
 * order z, y, x. Velocity vamp * (vamp * psi) and offset pfact * velocity,
 * psi the displacement of Zeldovich.c:14-100. Replaces Zeldovichmain
 * (Zeldovichmain.c:28-84) for one rank with PORDER = 1. The records load
 * with tpm_load_lagrangian. */
int tpm_ic_zeldovich(const tpm_ic_params *p, void *records, int mem);

/* Second-order Lagrangian particles (PORDER = 2): TwoLPTmain
 * (Cosmos/CosmosIC/TwoLPTmain.c:157-240) for one rank. The second-order
 * potential of TwoLPT (TwoLPT.c:259-535) from the same noise, after its
 * non-Gaussian terms when fnl or gnl is set; velocity d/dx (vamp phi1 +
 * vamp2 phi2) and offset d/dx (pfact damp1 phi1 + pfact damp2 phi2) per
 * axis (TwoLPT_GetVR, cosmosic.h:141-163). Same records as
 * tpm_ic_zeldovich. */
int tpm_ic_2lpt(const tpm_ic_params *p, void *records, int mem);

/* Largest particle count tpm_morton_order_noalloc accepts: its scratch is a
 * fixed array of about 3.1 MB compiled into the library. */
#define TPM_NOALLOC_MAX_PARTICLES 262144

/* No counterpart in the reference. The engine's Morton ordering (the keys
 * and stable radix sort of tpm_compute_forces, bit-identical results) for
 * callers that cannot allocate device memory: codes that run all of the GPU's
 * memory through their own pool, where a library cudaMalloc would fail or
 * escape the pool's accounting, and latency-critical loops that cannot take
 * the device-wide synchronisation of cudaMalloc/cudaFree. It allocates
 * nothing: its scratch is a fixed device array of the library, reserved on
 * every GPU that loads it until the process exits.
 *   pos   device pointer, np x 3 uint32 fixed-point positions (AoS)
 *   keys  device pointer, np uint64: sorted 39-bit Morton keys (output)
 *   perm  device pointer, np uint32: sorted slot -> input index (output)
 *   stream  a cudaStream_t (NULL: the legacy default stream)
 * Work is queued on `stream`; the call does not wait for it. np above
 * TPM_NOALLOC_MAX_PARTICLES is rejected with TPM_E_ARG. The first call on a
 * device looks up the device address of its scratch (cudaGetSymbolAddress,
 * with that device current), so make that first call before any stream
 * capture. The address is kept for the life of the process, so a caller that
 * resets a device (cudaDeviceReset) must not call this entry point on that
 * device afterwards. All calls share the one scratch array: calls whose work
 * overlaps on the GPU race and must be serialised by the caller. */
int tpm_morton_order_noalloc(const uint32_t *pos, int64_t np, int32_t n_mesh, uint64_t *keys,
                             uint32_t *perm, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* TPM_ENGINE_H */
