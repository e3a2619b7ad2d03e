// Internal interfaces between the engine's CUDA translation units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace tpm {

// ---------------------------------------------------------------- errors
// Device-side error flags (bit mask) written by kernels with bounded waits
// or bounded work queues; read by the host after a stage.
enum DeviceError : uint32_t {
  kErrStackOverflow = 1u,    // tree-walk node stack full
  kErrNodeOverflow = 2u,     // tree node capacity exceeded
  kErrTmaTimeout = 4u,       // a TMA transaction did not complete in time
  kErrListOverflow = 8u,     // interaction list overflow
};

// ---------------------------------------------------------------- sort
struct SortScratch {
  uint32_t *hist = nullptr;  // [256][ntiles]
  uint32_t *dtotal = nullptr;  // [256]
  int64_t cap_tiles = 0;
};
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;

void launch_make_keys(const uint32_t *pos, int64_t np, uint32_t n, int sub_bits, uint64_t *key,
                      uint32_t *val, cudaStream_t st);
// Stable LSD radix sort of (key, val) pairs on bits [0, nbits). On return
// *key/*val point at whichever buffer holds the sorted result.
void radix_sort_pairs(uint64_t **key, uint32_t **val, uint64_t *key_alt, uint32_t *val_alt,
                      int64_t np, int nbits, SortScratch &scr, cudaStream_t st, int64_t *launches);
int64_t sort_tiles(int64_t np);
void launch_gather_pos(const uint32_t *pos, const uint32_t *perm, int64_t np, uint32_t *spos,
                       cudaStream_t st);
// start[t] = first sorted index whose key >> shift >= t, t in [0, ntable].
void launch_range_table(const uint64_t *key, int64_t np, int shift, uint32_t ntable, uint32_t *start,
                        cudaStream_t st);

// ---------------------------------------------------------------- PM
struct MeshGeom {
  int n;          // cells per side
  int cbits;      // ceil(log2 n)
  int sub_bits;   // kAxisBits - cbits
  int tiles_axis; // 2^(cbits-3): Morton tiles per side (tile = 8 cells)
  int hx;         // n/2 + 1
  int64_t spec_elems;  // n*n*hx complex
  int px, py, pz; // ghosted potential pitches (x padded to a multiple of 4)
};
constexpr int kTile = 8;     // PM tile: 8^3 cells
constexpr int kGhost = 8;    // ghost layers of the padded potential (8-point stencil + TSC)

MeshGeom make_geom(int n);

// With rho2 the particles also go onto the second grid of the interlaced pair,
// moved by half a cell along every axis (a second launch).
void launch_tsc_deposit(const MeshGeom &g, const uint32_t *spos, const uint32_t *tile_start,
                        float mass, float *rho, cudaStream_t st, float *rho2 = nullptr);
// Device memory arena (arena.cu): large blocks claimed from the driver once,
// sub-ranges handed out best fit and merged back on release. Thread-safe.
struct DeviceArena;
// step_bytes: the size of each block claimed when nothing free fits (<= 0: 1 GiB)
DeviceArena *arena_create(int device, int64_t step_bytes);
// frees every block; no range may be in use
void arena_destroy(DeviceArena *a);
// claims a block so that at least `bytes` are free
cudaError_t arena_reserve(DeviceArena *a, int64_t bytes);
void arena_usage(DeviceArena *a, int64_t *reserved, int64_t *in_use);
cudaError_t arena_alloc(DeviceArena *a, void **p, size_t bytes);
void arena_free(DeviceArena *a, void *p);
// From the arena when a is given, else cudaMalloc / cudaFree.
cudaError_t dmalloc(DeviceArena *a, void **p, size_t bytes);
void dfree(DeviceArena *a, void *p);
template <class T>
cudaError_t dmalloc(DeviceArena *a, T **p, size_t bytes) {
  return dmalloc(a, reinterpret_cast<void **>(p), bytes);
}

// FFT pipeline: rho (n^3 real) -> phi_pad (ghosted potential).
struct FftPlan {
  float2 *tw = nullptr;   // twiddles exp(-2 pi i k / L) for L = n and L = n/2
  float2 *tw_half = nullptr;
  int n = 0;
  DeviceArena *arena = nullptr;  // where the twiddles live (nullptr: cudaMalloc)
};
// twiddle tables are written on st
cudaError_t fft_plan_init(FftPlan &p, int n, cudaStream_t st, DeviceArena *arena = nullptr);
// plain unnormalised transforms: real [z][y][x] -> spec [z][y][hx] (e^{-i}),
// spec -> ghosted real (e^{+i}; spec is overwritten)
void fft_forward(const MeshGeom &g, const FftPlan &p, const float *real, float2 *spec, cudaStream_t st);
void fft_inverse(const MeshGeom &g, const FftPlan &p, float2 *spec, float *phi_pad, cudaStream_t st);
// exclusive scan of n u32 values: out[i] = local prefix within blocks of
// 4096, bsum[i / 4096] = the block's offset (bsum holds (n + 4095) / 4096
// entries), *total = the sum
void scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *bsum, uint32_t *total, cudaStream_t st);
void fft_plan_free(FftPlan &p);
// With rho2 (the half-cell-shifted deposit) the two grids are interlaced:
// their spectra are combined before the Green's function and phi2_pad gets
// the potential on the shifted grid.
void launch_poisson(const MeshGeom &g, const FftPlan &p, const float *rho, float2 *spec,
                    float *phi_pad, int law, float efold, float rs_split, cudaStream_t st,
                    int64_t *launches, const float *rho2 = nullptr, float2 *spec2 = nullptr,
                    float *phi2_pad = nullptr, const float *gt = nullptr, int want_px = 0, int want_tx = 0,
                    double *pk = nullptr);
// The optimal influence function of the interlaced pair with the 8-point
// gradient for split scale rs, [ky][kx][kz] with kx < n/2 + 1.
void launch_green_opt(float *gt, int n, double rs, cudaStream_t st);
// fda4: gradient and TSC interpolation per tile through TMA.
// half: positions moved by half a cell (the shifted grid); average: write the
// mean of the new force and the one already in fpm.
void launch_fda4(const MeshGeom &g, const CUtensorMap *tmap, int radius, const uint32_t *spos,
                 const uint32_t *tile_start, float *fpm, uint32_t *err, cudaStream_t st, int half = 0,
                 int average = 0);
// Both grids of the interlaced pair with the 8-point gradient in one pass:
// fpm = the mean of the two grids' forces.
void launch_fda4_pair(const MeshGeom &g, const CUtensorMap *tmap, const CUtensorMap *tmap2, const uint32_t *spos,
                      const uint32_t *tile_start, float *fpm, uint32_t *err, cudaStream_t st);
// Tensor maps of the potential for the 4-point (radius 2) and the 8-point
// (radius 4) gradient: their boxes differ.
int make_phi_tensor_map(const MeshGeom &g, float *phi_pad, int radius, CUtensorMap *out);

// ---------------------------------------------------------------- tree
// What the walk reads of one box (the ensemble walk holds an array of them).
struct WalkBox {
  const uint32_t *spos;
  const uint4 *walkA, *walkB;
  const float4 *mom0, *mom1, *mom2;
  const uint32_t *groups;
  const uint32_t *ngroups;  // device word: the box's group count
  float *ftree;
  uint32_t *err;
  // where each group's walk starts: the 4-cell cubes of the tree's level
  // cbits - 2 (2^start_bits per axis, Morton-indexed): the node of a cube, or
  // kNoNode, and the sorted particle range of every cube
  const uint32_t *cube_node, *start_cube;
  float cpu, mass, inv_ll;
  int n_cells, start_bits;
};
constexpr uint32_t kNoNode = 0xffffffffu;
struct TreeBuffers {
  int64_t cap_nodes = 0;
  uint32_t *start = nullptr, *count = nullptr, *child = nullptr, *nchild = nullptr;
  uint8_t *level = nullptr;
  uint4 *geo = nullptr;      // center u32 x3, half-size (float bits)
  float4 *mom0 = nullptr;    // com (u32 bits x3), mass
  float4 *mom1 = nullptr;    // Qxx Qyy Qzz Qxy
  float4 *mom2 = nullptr;    // Qxz Qyz trQ mass
  // walk records, written with the moments: walkA[2n] = cube centre u32 x3 +
  // half-size bits, walkA[2n+1] = com u32 x3 + size^2/theta^2 bits;
  // walkB[n] = start, count, first child, nchild | level << 16
  uint4 *walkA = nullptr;
  uint4 *walkB = nullptr;
  uint32_t *level_range = nullptr;  // [2*(kAxisBits+2)] begin/end per level
  uint32_t *tile_sum = nullptr;     // scan scratch
  int64_t cap_tiles = 0;
  uint32_t *groups = nullptr;       // walk groups: start | (count << 26) packed as 2 words
  int64_t cap_groups = 0;
  uint32_t *counters = nullptr;     // [8]: ngroups, next group, pp, pc, ...
  uint32_t *stack = nullptr;        // per-warp global stacks
  int64_t stack_words = 0;
  WalkBox *walkbox = nullptr;       // device copy of this box's walk record
  // the walk's start tables over the 4-cell cubes (mesh-sized, allocated
  // with the mesh): node of each cube at tree level cbits - 2 or kNoNode, and
  // the first sorted particle of each cube (ncubes4 + 1 entries)
  uint32_t *cube_node = nullptr;
  uint32_t *start_cube = nullptr;
  int64_t ncubes4 = 0;
};

struct TreeParams {
  uint32_t n;
  int sub_bits;
  float theta2;
  float rsphere;
  float cell_per_unit;  // n / 2^32
  float mass;
  int group_max = 32;   // targets per warp group (<= 32)
};

void tree_build(const TreeParams &tp, const uint64_t *key, const uint32_t *spos, int64_t np,
                TreeBuffers &tb, uint32_t *err, cudaStream_t st, int64_t *launches);
void tree_groups(const TreeParams &tp, const uint64_t *key, int64_t np, TreeBuffers &tb,
                 uint32_t *cube_start, int64_t ncubes, int cube_shift, cudaStream_t st,
                 int64_t *launches);
// The short-range law's columns on grids uniform in log r^2, indexed by the
// float bits of s = r^2 + kLogR2Floor (cells^2). Entry k covers
// [s_k, s_{k+1}), s_k the float whose top bits are (kLogBase + k) <<
// kLogShift: 2^kLogMantissa bins per octave from 2^-20 (= kLogR2Floor, so
// every s lands in the table without a lower clamp) to 2^6 cells^2. The
// particle-pair column is linear in s inside each bin, c.x + c.y * s:
// c.y = (v_{k+1} - v_k) / (s_{k+1} - s_k) and c.x = v_k - c.y s_k, v_k the
// value at r^2 = s_k - kLogR2Floor (one multiply-add on s itself, no
// extraction of the in-bin mantissa). The node columns (kPc*) are linear in
// m, the float of s's in-bin mantissa bits under exponent 0 (m in [1, 1 +
// 2^-kPcMantissa)): c.x + c.y m with c.y = (v_{k+1} - v_k) 2^kPcMantissa and
// c.x = v_k - c.y.
constexpr float kLogR2Floor = 9.5367431640625e-07f;  // 2^-20
constexpr int kLogMantissa = 7;
constexpr int kLogShift = 23 - kLogMantissa;
constexpr int kLogBase = (127 - 20) << kLogMantissa;
constexpr int kLogEntries = 26 << kLogMantissa;
// The node terms' derivative columns f2, f3 on a coarser log grid of r^2,
// 2^kPcMantissa bins per octave from 2^-8 to 2^6 cells^2 (closer nodes take
// the first bin), in the same c.x + c.y * m form: {f2 - df2, df2, f3 - df3,
// df3} with df = (f_{k+1} - f_k) * 2^kPcMantissa.
constexpr int kPcMantissa = 5;
constexpr int kPcShift = 23 - kPcMantissa;
constexpr int kPcBase = (127 - 8) << kPcMantissa;
constexpr int kPcEntries = 14 << kPcMantissa;
struct LawTable {
  float2 *tlog = nullptr;  // [kLogEntries + 1] {-f/r, slope per bin}
  float4 *tpc = nullptr;   // [kPcEntries + 1] the two node columns and slopes
  // 1: the walk tests r <= rsphere per pair (the reference's cut);
  // 0: tlog is zero from the cut on, so the pair test is not needed
  int hard_cut = 1;
  // without hard_cut: the float bits of s = r^2 + kLogR2Floor from which
  // every entry of tlog is zero ((kLogBase + k0) << kLogShift, k0 the first
  // zero entry)
  uint32_t cut_bits = 0xffffffffu;
};
WalkBox walk_box(const TreeParams &tp, const uint32_t *spos, const TreeBuffers &tb, float *ftree,
                 uint32_t *err);
// One launch over the groups of every box (boxes: device array); the boxes
// share law (same kind, softening, split and cut) and rsphere.
void tree_walk_multi(const WalkBox *boxes, int nbox, uint32_t *gprefix, uint32_t *gnext, uint32_t *stack,
                     int64_t stack_words, uint32_t *stats, const LawTable &law, float rsphere, cudaStream_t st);
void tree_walk(const TreeParams &tp, const uint32_t *spos, int64_t np, const TreeBuffers &tb,
               const LawTable &law, float *ftree, uint32_t *err, cudaStream_t st,
               int64_t *launches);

// ---------------------------------------------------------------- misc
// Sets the message tpm_last_error() returns on this thread.
void set_last_error(const char *msg);

void launch_finish_forces(const uint32_t *perm, int64_t np, const float *fpm, const float *ftree,
                          unsigned parts, float *force_out, cudaStream_t st);

}  // namespace tpm
