// Short-range tree correction (sm_100a).
//
// The reference builds, for every chaining-mesh bucket of 4^3 cells, an
// octree over the particles of the 27 surrounding buckets, split at the
// centre of mass with sub-octants of fewer than 10 particles left as bare
// particles (OST/ost.ver2.c:36-196), and walks it once per target with the
// opening test d^2 < size^2/theta^2 (ost.ver2.c:296-306), monopole +
// quadrupole node terms and particle terms from a tabulated law, both only
// inside rsphere (ost.ver2.c:247-293; OST/Model4TreeForce.c:34-46).
//
// Here one octree covers the whole periodic box. It is built level by level
// from the Morton-sorted keys (a node's children are the runs of its next
// octal key digit), keeps the reference's leaf rule (children with fewer than
// 10 particles stay bare), and carries the same moments: mass, centre of
// mass, second moments about it, trQ and size^2/theta^2. A warp walks the
// tree for a group of up to 32 spatially adjacent targets, opening a node if
// the test would open it for any target of the group, and evaluates the
// resulting particle and node lists per target with the reference's law and
// per-target rsphere cuts. Positions are uint32 fixed point; all relative
// coordinates are exact minimum-image differences converted to float.
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "engine_internal.cuh"

namespace tpm {

constexpr int kBuildThreads = 256;
constexpr int kBuildGrid = 148 * 8;
constexpr int kScanGrid = 148 * 2;

TPM_D float wrapf(uint32_t a, uint32_t b, float cpu) { return (float)(int32_t)(a - b) * cpu; }

// child boundary: first index in [lo, hi) whose digit at `shift` is >= d
TPM_D uint32_t lower_digit(const uint64_t *key, uint32_t lo, uint32_t hi, int shift, uint32_t d) {
  while (lo < hi) {
    uint32_t mid = lo + ((hi - lo) >> 1);
    uint32_t v = (uint32_t)(key[mid] >> shift) & 7u;
    if (v < d)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__global__ void k_tree_root(int64_t np, TreeBuffers tb, uint32_t n, int sub_bits) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    tb.start[0] = 0;
    tb.count[0] = (uint32_t)np;
    tb.child[0] = 0;
    tb.nchild[0] = 0;
    tb.level[0] = 0;
    // root cube: [0, 2^(13-sub_bits)) cells, centre at half of that
    double half = (double)(1u << (kAxisBits - 1)) / (double)(1u << sub_bits);
    double cu = half / (double)n;
    cu = cu - floor(cu);
    uint32_t c = (uint32_t)(unsigned long long)llrint(cu * 4294967296.0);
    tb.geo[0] = make_uint4(c, c, c, __float_as_uint((float)half));
    for (int l = 0; l < 2 * (kAxisBits + 2); l++) tb.level_range[l] = 0;
    tb.level_range[0] = 0;
    tb.level_range[1] = 1;
  }
}

// The level kernels give each node a segment of 8 lanes, lane d owning the
// node's d-th octant (its level-(l+1) digit): the eight child boundaries are
// found by eight independent binary searches instead of one chain of seven,
// and the children are written in parallel. Items are (node, digit) pairs;
// the loops over them are warp-uniform, so the segment shuffles stay
// converged.
constexpr int kScanChunk = 4096;  // nodes per block of the per-level scan

struct ChildRange {
  uint32_t node;  // absolute index of the segment's node
  bool valid;     // the node exists (item < 8 * nodes of the level)
  uint32_t lo, hi;  // this lane's child [lo, hi), empty when the node does not split
};

TPM_D ChildRange child_range(const uint64_t *__restrict__ key, const TreeBuffers &tb, uint32_t b,
                             uint32_t nn, uint64_t item, int l, int shift) {
  int d = threadIdx.x & 7;
  ChildRange r;
  r.valid = item < (uint64_t)nn * 8u;
  r.node = b + (uint32_t)(item >> 3);
  uint32_t s = 0, c = 0;
  if (r.valid) {
    s = tb.start[r.node];
    c = tb.count[r.node];
  }
  bool split = r.valid && c >= (uint32_t)kLeafMin && l < kAxisBits;
  uint32_t bnd = s;
  if (split && d > 0) bnd = lower_digit(key, s, s + c, shift, (uint32_t)d);
  uint32_t nxt = __shfl_down_sync(0xffffffffu, bnd, 1, 8);
  if (d == 7) nxt = s + c;
  r.lo = bnd;
  r.hi = split ? nxt : bnd;
  return r;
}

// Count the non-empty children of every level-l node that splits.
__global__ void __launch_bounds__(kBuildThreads) k_tree_count(const uint64_t *__restrict__ key,
                                                              TreeBuffers tb, int l) {
  uint32_t b = tb.level_range[2 * l], e = tb.level_range[2 * l + 1];
  uint32_t nn = e - b;
  int lane = threadIdx.x & 31;
  int shift = 3 * (kAxisBits - 1 - l);
  const unsigned seg = 0xffu << (lane & ~7);
  uint64_t total = (uint64_t)nn * 8u, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
    ChildRange cr = child_range(key, tb, b, nn, base + lane, l, shift);
    unsigned m = __ballot_sync(0xffffffffu, cr.hi > cr.lo) & seg;
    if (cr.valid && (lane & 7) == 0) tb.nchild[cr.node] = (uint32_t)__popc(m);
  }
}

// Per-level exclusive scan of nchild over chunks of kScanChunk nodes: the
// prefix within the chunk goes to child[node] (the write pass adds the
// chunk's offset and overwrites it), the chunk's total to tile_sum[chunk].
__global__ void __launch_bounds__(1024) k_tree_scan_chunks(TreeBuffers tb, int l) {
  __shared__ uint32_t wsum[32];
  uint32_t b = tb.level_range[2 * l], e = tb.level_range[2 * l + 1];
  uint32_t nn = e - b;
  uint32_t nchunks = (nn + kScanChunk - 1) / kScanChunk;
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    uint32_t base = ch * kScanChunk;
    uint32_t v[4], s = 0;
    for (int j = 0; j < 4; j++) {
      uint32_t i = base + 4 * tid + j;
      v[j] = i < nn ? tb.nchild[b + i] : 0u;
      s += v[j];
    }
    uint32_t x = s;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t t = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      wsum[lane] = t;
    }
    __syncthreads();
    uint32_t run = (warp ? wsum[warp - 1] : 0u) + x - s;
    for (int j = 0; j < 4; j++) {
      uint32_t i = base + 4 * tid + j;
      if (i < nn) tb.child[b + i] = run;
      run += v[j];
    }
    if (tid == 0) tb.tile_sum[ch] = wsum[31];
    __syncthreads();
  }
}

// Exclusive scan of the chunk sums of level l and the extent of level l+1.
__global__ void __launch_bounds__(1024) k_tree_scan(TreeBuffers tb, int l, uint32_t *err) {
  uint32_t b = tb.level_range[2 * l], e = tb.level_range[2 * l + 1];
  uint32_t ntiles = (e - b + kScanChunk - 1) / kScanChunk;
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t carry;
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < ntiles; base += 1024) {
    uint32_t i = base + tid;
    uint32_t v = i < ntiles ? tb.tile_sum[i] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t s = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s;
    }
    __syncthreads();
    if (i < ntiles) tb.tile_sum[i] = carry + (warp ? wsum[warp - 1] : 0u) + x - v;
    __syncthreads();
    if (tid == 0) carry += wsum[31];
    __syncthreads();
  }
  if (tid == 0) {
    uint64_t end = (uint64_t)e + carry;
    if (end > (uint64_t)tb.cap_nodes) {
      atomicOr(err, (uint32_t)kErrNodeOverflow);
      end = e;  // stop refining: the level's nodes stay leaves
    }
    tb.level_range[2 * (l + 1)] = e;
    tb.level_range[2 * (l + 1) + 1] = (uint32_t)end;
  }
}

// The three axis coordinates interleaved in a Morton key (bit 3i + a of the
// key is bit i of axis a).
TPM_D uint32_t morton_compact(uint64_t x) {
  x &= 0x1249249249249249ull;
  x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ull;
  x = (x ^ (x >> 4)) & 0x100f00f00f00f00full;
  x = (x ^ (x >> 8)) & 0x1f0000ff0000ffull;
  x = (x ^ (x >> 16)) & 0x1f00000000ffffull;
  x = (x ^ (x >> 32)) & 0x1fffffull;
  return (uint32_t)x;
}

// Write the children of level-l nodes: node records of level l+1 in the
// order of their parents, siblings contiguous in octant order.
// q_to_frac = 1 / (2^sub_bits n): axis units of the key to fractions of the
// box, so a cube centre is one FP64 multiply (no divisions per node).
__global__ void __launch_bounds__(kBuildThreads) k_tree_write(const uint64_t *__restrict__ key,
                                                              TreeBuffers tb, int l, uint32_t n,
                                                              int sub_bits, double q_to_frac) {
  uint32_t b = tb.level_range[2 * l], e = tb.level_range[2 * l + 1];
  uint32_t e1 = tb.level_range[2 * (l + 1) + 1];
  bool overflow = (e1 == e);  // capacity hit: nothing written below this level
  uint32_t nn = e - b;
  int lane = threadIdx.x & 31;
  int shift = 3 * (kAxisBits - 1 - l);
  const unsigned seg = 0xffu << (lane & ~7);
  int child_level = l + 1;
  // child cube: side 2^(13-child_level) q units
  uint32_t cside_q = 1u << (kAxisBits - child_level);
  float half_cells = (float)((double)cside_q * 0.5 / (double)(1u << sub_bits));
  uint64_t total = (uint64_t)nn * 8u, stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
    ChildRange cr = child_range(key, tb, b, nn, base + lane, l, shift);
    bool ne = !overflow && cr.hi > cr.lo;
    uint32_t first = 0;
    if (cr.valid) first = e + tb.child[cr.node] + tb.tile_sum[(cr.node - b) / kScanChunk];
    // every lane has read child[node] before the segment's lane 0 rewrites it
    unsigned m = __ballot_sync(0xffffffffu, ne) & seg;
    if (ne) {
      uint32_t slot = first + (uint32_t)__popc(m & ((1u << lane) - 1u));
      tb.start[slot] = cr.lo;
      tb.count[slot] = cr.hi - cr.lo;
      tb.child[slot] = 0;
      tb.nchild[slot] = 0;
      tb.level[slot] = (uint8_t)child_level;
      // cube of the child from its first key
      uint64_t k = key[cr.lo];
      uint32_t q[3] = {morton_compact(k), morton_compact(k >> 1), morton_compact(k >> 2)};
      uint32_t cu[3];
      for (int a = 0; a < 3; a++) {
        uint32_t qc = q[a] & ~(cside_q - 1u);
        double fr = ((double)qc + 0.5 * (double)cside_q) * q_to_frac;
        fr -= floor(fr);
        cu[a] = (uint32_t)(unsigned long long)llrint(fr * 4294967296.0);
      }
      tb.geo[slot] = make_uint4(cu[0], cu[1], cu[2], __float_as_uint(half_cells));
    }
    if (cr.valid && (lane & 7) == 0) {
      tb.child[cr.node] = m ? first : 0u;
      if (overflow) tb.nchild[cr.node] = 0;
    }
  }
}

// Moments of level-l nodes: leaves from their particles, inner nodes from
// their children (parallel-axis theorem). size is max |x - com| for leaves
// and the bound max_c(|com_c - com| + size_c) for inner nodes.
__global__ void __launch_bounds__(256) k_tree_moments(const uint32_t *__restrict__ spos, TreeBuffers tb,
                                                      int l, float cpu, float mass, float inv_theta2) {
  uint32_t b = tb.level_range[2 * l], e = tb.level_range[2 * l + 1];
  for (uint32_t node = b + blockIdx.x * blockDim.x + threadIdx.x; node < e;
       node += gridDim.x * blockDim.x) {
    uint4 geo = tb.geo[node];
    uint32_t nch = tb.nchild[node];
    float M = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    float qxx = 0, qyy = 0, qzz = 0, qxy = 0, qxz = 0, qyz = 0, size2 = 0.f;
    if (nch == 0) {
      uint32_t s = tb.start[node], c = tb.count[node];
      float sx = 0, sy = 0, sz = 0;
      for (uint32_t i = s; i < s + c; i++) {
        sx += wrapf(spos[3 * (int64_t)i + 0], geo.x, cpu);
        sy += wrapf(spos[3 * (int64_t)i + 1], geo.y, cpu);
        sz += wrapf(spos[3 * (int64_t)i + 2], geo.z, cpu);
      }
      float inv = 1.f / (float)c;
      cx = sx * inv;
      cy = sy * inv;
      cz = sz * inv;
      M = mass * (float)c;
      for (uint32_t i = s; i < s + c; i++) {
        float dx = wrapf(spos[3 * (int64_t)i + 0], geo.x, cpu) - cx;
        float dy = wrapf(spos[3 * (int64_t)i + 1], geo.y, cpu) - cy;
        float dz = wrapf(spos[3 * (int64_t)i + 2], geo.z, cpu) - cz;
        qxx += mass * dx * dx;
        qyy += mass * dy * dy;
        qzz += mass * dz * dz;
        qxy += mass * dx * dy;
        qxz += mass * dx * dz;
        qyz += mass * dy * dz;
        size2 = fmaxf(size2, dx * dx + dy * dy + dz * dz);
      }
    } else {
      uint32_t c0 = tb.child[node];
      for (uint32_t j = c0; j < c0 + nch; j++) {
        float4 m0 = tb.mom0[j];
        float m = m0.w;
        float dx = wrapf(__float_as_uint(m0.x), geo.x, cpu);
        float dy = wrapf(__float_as_uint(m0.y), geo.y, cpu);
        float dz = wrapf(__float_as_uint(m0.z), geo.z, cpu);
        M += m;
        cx += m * dx;
        cy += m * dy;
        cz += m * dz;
      }
      float inv = 1.f / M;
      cx *= inv;
      cy *= inv;
      cz *= inv;
      float size = 0.f;
      for (uint32_t j = c0; j < c0 + nch; j++) {
        float4 m0 = tb.mom0[j], m1 = tb.mom1[j], m2 = tb.mom2[j];
        float child_open2 = __uint_as_float(tb.walkA[2 * (int64_t)j + 1].w);
        float m = m0.w;
        float dx = wrapf(__float_as_uint(m0.x), geo.x, cpu) - cx;
        float dy = wrapf(__float_as_uint(m0.y), geo.y, cpu) - cy;
        float dz = wrapf(__float_as_uint(m0.z), geo.z, cpu) - cz;
        qxx += m1.x + m * dx * dx;
        qyy += m1.y + m * dy * dy;
        qzz += m1.z + m * dz * dz;
        qxy += m1.w + m * dx * dy;
        qxz += m2.x + m * dx * dz;
        qyz += m2.y + m * dy * dz;
        // child size from its open2 = size^2/theta^2
        float cs = sqrtf(child_open2 / inv_theta2);
        size = fmaxf(size, sqrtf(dx * dx + dy * dy + dz * dz) + cs);
      }
      size2 = size * size;
    }
    uint32_t comx = geo.x + (uint32_t)(int32_t)__float2int_rn(cx / cpu);
    uint32_t comy = geo.y + (uint32_t)(int32_t)__float2int_rn(cy / cpu);
    uint32_t comz = geo.z + (uint32_t)(int32_t)__float2int_rn(cz / cpu);
    tb.mom0[node] = make_float4(__uint_as_float(comx), __uint_as_float(comy), __uint_as_float(comz), M);
    tb.mom1[node] = make_float4(qxx, qyy, qzz, qxy);
    tb.mom2[node] = make_float4(qxz, qyz, qxx + qyy + qzz, M);
    tb.walkA[2 * (int64_t)node] = geo;
    tb.walkA[2 * (int64_t)node + 1] = make_uint4(comx, comy, comz, __float_as_uint(size2 * inv_theta2));
    tb.walkB[node] = make_uint4(tb.start[node], tb.count[node], tb.child[node],
                                nch | ((uint32_t)tb.level[node] << 16));
  }
}

// The walk's start table: the node of every 4-cell cube at tree level
// cbits - 2 (the table was cleared to kNoNode before).
__global__ void k_cube_nodes(const uint64_t *__restrict__ key, TreeBuffers tb, int lev, int shift) {
  uint32_t b = tb.level_range[2 * lev], e = tb.level_range[2 * lev + 1];
  for (uint32_t node = b + blockIdx.x * blockDim.x + threadIdx.x; node < e; node += gridDim.x * blockDim.x)
    tb.cube_node[key[tb.start[node]] >> shift] = node;
}

void tree_build(const TreeParams &tp, const uint64_t *key, const uint32_t *spos, int64_t np,
                TreeBuffers &tb, uint32_t *err, cudaStream_t st, int64_t *launches) {
  k_tree_root<<<1, 32, 0, st>>>(np, tb, tp.n, tp.sub_bits);
  int64_t nl = 1;
  for (int l = 0; l < kAxisBits; l++) {
    k_tree_count<<<kBuildGrid, kBuildThreads, 0, st>>>(key, tb, l);
    k_tree_scan_chunks<<<kScanGrid, 1024, 0, st>>>(tb, l);
    k_tree_scan<<<1, 1024, 0, st>>>(tb, l, err);
    k_tree_write<<<kBuildGrid, kBuildThreads, 0, st>>>(key, tb, l, tp.n, tp.sub_bits,
                                                       1.0 / ((double)(1u << tp.sub_bits) * (double)tp.n));
    nl += 4;
  }
  float inv_theta2 = 1.f / tp.theta2;
  for (int l = kAxisBits; l >= 0; l--) {
    k_tree_moments<<<kBuildGrid, 256, 0, st>>>(spos, tb, l, tp.cell_per_unit, tp.mass, inv_theta2);
    nl++;
  }
  // the walk's start tables over the 4-cell cubes
  const int cbits = kAxisBits - tp.sub_bits;
  const int shift = 3 * (tp.sub_bits + 2);
  launch_range_table(key, np, shift, (uint32_t)tb.ncubes4, tb.start_cube, st);
  cudaMemsetAsync(tb.cube_node, 0xff, sizeof(uint32_t) * tb.ncubes4, st);
  k_cube_nodes<<<kBuildGrid, 256, 0, st>>>(key, tb, cbits - 2, shift);
  nl += 3;
  if (launches) *launches += nl;
}

// ------------------------------------------------------------ walk groups
// Groups never cross a 4-cell cube and hold at most 32 particles.
__global__ void k_group_counts(const uint32_t *__restrict__ cube_start, int64_t ncubes,
                               uint32_t *__restrict__ gcount, uint32_t gmax) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncubes;
       c += (int64_t)gridDim.x * blockDim.x) {
    uint32_t cnt = cube_start[c + 1] - cube_start[c];
    gcount[c] = (cnt + gmax - 1) / gmax;
  }
}

// exclusive scan of n u32 values with one block per 4096 and a single-block
// pass over the block sums
__global__ void __launch_bounds__(1024) k_scan_block(const uint32_t *in, uint32_t *out, int64_t n,
                                                     uint32_t *bsum) {
  __shared__ uint32_t wsum[32];
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int64_t base = (int64_t)blockIdx.x * 4096;
  uint32_t v[4], s = 0;
  for (int j = 0; j < 4; j++) {
    int64_t i = base + 4 * tid + j;
    v[j] = i < n ? in[i] : 0u;
    s += v[j];
  }
  uint32_t x = s;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    wsum[lane] = t;
  }
  __syncthreads();
  uint32_t run = (warp ? wsum[warp - 1] : 0u) + x - s;
  for (int j = 0; j < 4; j++) {
    int64_t i = base + 4 * tid + j;
    if (i < n) out[i] = run;
    run += v[j];
  }
  if (tid == 0) bsum[blockIdx.x] = wsum[31];
}

__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t *bsum, int64_t nb, uint32_t *total) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t carry;
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nb; base += 1024) {
    int64_t i = base + tid;
    uint32_t v = i < nb ? bsum[i] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t s = wsum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s;
    }
    __syncthreads();
    if (i < nb) bsum[i] = carry + (warp ? wsum[warp - 1] : 0u) + x - v;
    __syncthreads();
    if (tid == 0) carry += wsum[31];
    __syncthreads();
  }
  if (tid == 0) *total = carry;
}

__global__ void k_write_groups(const uint32_t *__restrict__ cube_start, int64_t ncubes,
                               const uint32_t *__restrict__ goff, const uint32_t *__restrict__ bsum,
                               uint32_t *__restrict__ groups, uint32_t gmax) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncubes;
       c += (int64_t)gridDim.x * blockDim.x) {
    uint32_t s = cube_start[c], e = cube_start[c + 1];
    uint32_t g = goff[c] + bsum[c / 4096];
    for (uint32_t p = s; p < e; p += gmax, g++) {
      groups[2 * (int64_t)g] = p;
      groups[2 * (int64_t)g + 1] = min(gmax, e - p);
    }
  }
}

void scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *bsum, uint32_t *total, cudaStream_t st) {
  int64_t nb = (n + 4095) / 4096;
  k_scan_block<<<(unsigned)nb, 1024, 0, st>>>(in, out, n, bsum);
  k_scan_sums<<<1, 1024, 0, st>>>(bsum, nb, total);
}

void tree_groups(const TreeParams &tp, const uint64_t *key, int64_t np, TreeBuffers &tb,
                 uint32_t *cube_start, int64_t ncubes, int cube_shift, cudaStream_t st,
                 int64_t *launches) {
  uint32_t gmax = (uint32_t)std::max(1, std::min(32, tp.group_max));
  launch_range_table(key, np, cube_shift, (uint32_t)ncubes, cube_start, st);
  // gcount and offsets live in the tail of the group buffer's scratch
  uint32_t *gcount = tb.tile_sum;  // sized >= ncubes + blocks by the caller
  uint32_t *goff = gcount + ncubes;
  int64_t nb = (ncubes + 4095) / 4096;
  uint32_t *bsum = goff + ncubes;
  int blocks = (int)((ncubes + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_group_counts<<<blocks, 256, 0, st>>>(cube_start, ncubes, gcount, gmax);
  k_scan_block<<<(unsigned)nb, 1024, 0, st>>>(gcount, goff, ncubes, bsum);
  k_scan_sums<<<1, 1024, 0, st>>>(bsum, nb, &tb.counters[0]);
  k_write_groups<<<blocks, 256, 0, st>>>(cube_start, ncubes, goff, bsum, tb.groups, gmax);
  if (launches) *launches += 5;
}

// ------------------------------------------------------------------ walk
constexpr int kWalkWarps = 16;
constexpr int kWalkBlocksPerSm = 1;  // resident CTAs per SM the registers are sized for
constexpr int kWalkThreads = kWalkWarps * 32;
constexpr int kStackSmem = 640;    // per-warp stack entries in shared memory
constexpr int kStackCap = 8192;    // entries beyond kStackSmem live in global memory
constexpr int kPcCap = 64;
constexpr int kPpBatch = 128;       // particle sources evaluated per flush
constexpr int kLogSmemF4 = (kLogEntries + 2) / 2;  // the log-spaced table, in float4s

struct WarpLists {
  WalkBox box;                     // the box of the group this warp walks
  uint32_t pc[kPcCap];
  uint32_t pp[kPpBatch];
  float4 stage[kPpBatch];          // PP: x, y, z rows of the sources; PC: three float4 per node
  uint32_t stack[kStackSmem];
};

// the stage buffer holds the particle rows (x, y, z of kPpBatch sources, read
// four past the last) and the node rows (11 of 32)
static_assert(3 * kPpBatch + 4 <= 4 * kPpBatch && 11 * 32 <= 4 * kPpBatch, "stage buffer too small");

struct WalkCtx {
  float tx, ty, tz;       // this lane's target relative to u_ref (cells)
  float ax, ay, az;       // particle-particle sum (without the particle mass)
  float bx, by, bz;       // particle-node sum
  bool active;
  uint32_t rx, ry, rz;    // u_ref
};

// The law at s = r^2 + kLogR2Floor (cells^2) from the table indexed by the
// float bits of s: the exponent and the top kLogMantissa mantissa bits pick
// the bin, whose line in s gives the value, so neither a square root nor a
// conversion is needed, and s >= 2^-20 needs no lower clamp. tlb is the
// table's shared address with the base entry kLogBase folded in (s >= 2^-20
// keeps the entry >= 0; the clamp keeps it in range).
TPM_D float law_at(float s, uint32_t tlb) {
  uint32_t kk = min(__float_as_uint(s) >> kLogShift, (uint32_t)(kLogBase + kLogEntries));
  float2 c;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(c.x), "=f"(c.y) : "r"(tlb + (kk << 3)));
  return fmaf(c.y, s, c.x);
}

// The law at s with every pair beyond the cut reading one shared entry: the
// bin index is clamped at kcut (the first bin from which the Gaussian law's
// table is zero; for the reference law the bin of rsphere^2, whose value the
// per-pair test then discards), so the lanes with such pairs all load one
// address, a broadcast, and the warp's gather spreads over the banks of the
// pairs inside the cut only. Same value as law_at with the cut applied.
TPM_D float law_clamped(float s, uint32_t tlb, uint32_t kcut) {
  uint32_t kk = min(__float_as_uint(s) >> kLogShift, kcut);
  float2 c;
  asm("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(c.x), "=f"(c.y) : "r"(tlb + (kk << 3)));
  return fmaf(c.y, s, c.x);
}

// One source against this lane's target: the reference's AddPar
// (OST/ost.ver2.c:279-293) without the mass factor. The source comes negated
// (nsx = -x), so dx = tx + nsx is the IEEE difference tx - x. The target
// itself (r = 0) lands in bin 0 with a zero separation, adding nothing.
// kHardCut: the per-pair cut of the reference law, tested as s <= rsphere^2
// (a cut 2^-20 cells^2 inside r^2 <= rsphere^2); the Gaussian law's table is
// zero from the cut on and needs no test.
template <bool kHardCut>
TPM_D void pp_one(float nsx, float nsy, float nsz, const WalkCtx &w, float rs2, uint32_t kcut, uint32_t tlb,
                  float &ax, float &ay, float &az) {
  float dx = w.tx + nsx, dy = w.ty + nsy, dz = w.tz + nsz;
  float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, kLogR2Floor)));
  float f = law_clamped(r2, tlb, kcut);
  if (kHardCut) f = r2 <= rs2 ? f : 0.f;
  ax = fmaf(dx, f, ax);
  ay = fmaf(dy, f, ay);
  az = fmaf(dz, f, az);
}

// Two sources against this lane's target, the separations, r^2 and the
// accumulation as packed fp32x2 operations (sm_100 add/fma on register
// pairs): each half is the IEEE fp32 operation pp_one does, in the same
// order, so the sums are the same bits as two pp_one calls into the halves.
template <bool kHardCut>
TPM_D void pp_two(float2 nsx, float2 nsy, float2 nsz, float2 tx, float2 ty, float2 tz, float rs2, uint32_t kcut,
                  uint32_t tlb, float2 &ax, float2 &ay, float2 &az) {
  float2 dx = __fadd2_rn(tx, nsx), dy = __fadd2_rn(ty, nsy), dz = __fadd2_rn(tz, nsz);
  float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, make_float2(kLogR2Floor, kLogR2Floor))));
  float2 f = make_float2(law_clamped(r2.x, tlb, kcut), law_clamped(r2.y, tlb, kcut));
  if (kHardCut) {
    f.x = r2.x <= rs2 ? f.x : 0.f;
    f.y = r2.y <= rs2 ? f.y : 0.f;
  }
  ax = __ffma2_rn(dx, f, ax);
  ay = __ffma2_rn(dy, f, ay);
  az = __ffma2_rn(dz, f, az);
}

// The group's bounding box (cells, relative to u_ref) and the squared reach
// beyond it: a source farther than that from the box is outside rsphere of
// every target of the group.
struct GroupBox {
  float cx, cy, cz, hx, hy, hz;
  float reach2;
};

// Particle sources of the batch wl.pp[0..m): each lane loads one source,
// drops it if it lies beyond the group's reach (it would add nothing to any
// lane), and the kept ones are compacted, in order and negated, into the
// x, y and z rows of wl.stage; then every lane evaluates every kept source
// against its target, four at a time (one 16-byte broadcast load per row,
// two packed pairs), sources j, j+1, j+2, j+3 into accumulator sets 0-3.
template <bool kHardCut>
TPM_D void eval_pp(WarpLists &wl, int m, const uint32_t *__restrict__ spos, WalkCtx &w, float cpu,
                   const GroupBox &gb, float rs2, uint32_t kcut, const float2 *__restrict__ tl,
                   unsigned long long &npp) {
  int lane = threadIdx.x & 31;
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  float *nsx = reinterpret_cast<float *>(wl.stage);
  float *nsy = nsx + kPpBatch, *nsz = nsx + 2 * kPpBatch;
  // all loads of the batch are issued before any is used
  uint32_t u[kPpBatch / 32][3];
#pragma unroll
  for (int b = 0; b < kPpBatch / 32; b++) {
    int k = b * 32 + lane;
    if (k < m) {
      uint32_t idx = wl.pp[k];
      u[b][0] = spos[3 * (int64_t)idx + 0];
      u[b][1] = spos[3 * (int64_t)idx + 1];
      u[b][2] = spos[3 * (int64_t)idx + 2];
    }
  }
  int kept = 0;
#pragma unroll
  for (int b = 0; b < kPpBatch / 32; b++) {
    int k = b * 32 + lane;
    bool keep = false;
    float px = 0.f, py = 0.f, pz = 0.f;
    if (k < m) {
      px = wrapf(u[b][0], w.rx, cpu);
      py = wrapf(u[b][1], w.ry, cpu);
      pz = wrapf(u[b][2], w.rz, cpu);
      float dx = fmaxf(fabsf(px - gb.cx) - gb.hx, 0.f);
      float dy = fmaxf(fabsf(py - gb.cy) - gb.hy, 0.f);
      float dz = fmaxf(fabsf(pz - gb.cz) - gb.hz, 0.f);
      keep = dx * dx + dy * dy + dz * dz <= gb.reach2;
    }
    unsigned mk = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      int at = kept + __popc(mk & lanemask_lt);
      nsx[at] = -px;
      nsy[at] = -py;
      nsz[at] = -pz;
    }
    kept += __popc(mk);
  }
  __syncwarp();
  m = kept;
  const uint32_t tlb = (uint32_t)__cvta_generic_to_shared(tl) - (uint32_t)(kLogBase * 8);
  const float2 tx = make_float2(w.tx, w.tx), ty = make_float2(w.ty, w.ty), tz = make_float2(w.tz, w.tz);
  float2 a01x = make_float2(0.f, 0.f), a01y = a01x, a01z = a01x, a23x = a01x, a23y = a01x, a23z = a01x;
  // the rows of the next four sources are loaded before the arithmetic of
  // these four; past the last source that reads unused values still inside
  // wl.stage (the z row ends 128 floats before the buffer does)
  int j = 0;
  if (m >= 4) {
    float4 x = *reinterpret_cast<const float4 *>(nsx);
    float4 y = *reinterpret_cast<const float4 *>(nsy);
    float4 z = *reinterpret_cast<const float4 *>(nsz);
    for (; j + 4 <= m; j += 4) {
      float4 xn = *reinterpret_cast<const float4 *>(nsx + j + 4);
      float4 yn = *reinterpret_cast<const float4 *>(nsy + j + 4);
      float4 zn = *reinterpret_cast<const float4 *>(nsz + j + 4);
      pp_two<kHardCut>(make_float2(x.x, x.y), make_float2(y.x, y.y), make_float2(z.x, z.y), tx, ty, tz, rs2, kcut, tlb,
                       a01x, a01y, a01z);
      pp_two<kHardCut>(make_float2(x.z, x.w), make_float2(y.z, y.w), make_float2(z.z, z.w), tx, ty, tz, rs2, kcut, tlb,
                       a23x, a23y, a23z);
      x = xn;
      y = yn;
      z = zn;
    }
  }
  for (; j < m; j++) pp_one<kHardCut>(nsx[j], nsy[j], nsz[j], w, rs2, kcut, tlb, a01x.x, a01y.x, a01z.x);
  if (w.active) {
    w.ax += (a01x.x + a01x.y) + (a23x.x + a23x.y);
    w.ay += (a01y.x + a01y.y) + (a23y.x + a23y.y);
    w.az += (a01z.x + a01z.y) + (a23z.x + a23z.y);
    npp += (unsigned long long)m;
  }
  __syncwarp();
}

// Node terms: the reference's AddNode (OST/ost.ver2.c:247-277) with the y
// and z components on their own axes. Coordinates are in cells; the log-r^2
// tables in shared memory give the law and its derivatives. The batch's nodes
// are staged as eleven rows of 32 (negated x, y, z, mass, Qxx, Qyy, Qzz, Qxy,
// Qxz, Qyz, trQ; zero past the last node, which adds nothing) and evaluated
// two at a time in packed fp32x2 operations; the quadrupole contraction is
// d.(Qd) from the three rows of Qd.
TPM_D void eval_pc(WarpLists &wl, int m_all, const WalkBox &tb, WalkCtx &w, float cpu, float rs2,
                   const float2 *__restrict__ tl, const float4 *__restrict__ tq, unsigned long long &npc) {
  int lane = threadIdx.x & 31;
  float *row = reinterpret_cast<float *>(wl.stage);
  const uint32_t tlb = (uint32_t)__cvta_generic_to_shared(tl) - (uint32_t)(kLogBase * 8);
  const float2 tx = make_float2(w.tx, w.tx), ty = make_float2(w.ty, w.ty), tz = make_float2(w.tz, w.tz);
  const float2 floor2 = make_float2(kLogR2Floor, kLogR2Floor);
  for (int base = 0; base < m_all; base += 32) {
    int m = min(32, m_all - base);
    float v[11];
#pragma unroll
    for (int r = 0; r < 11; r++) v[r] = 0.f;
    if (lane < m) {
      uint32_t nd = wl.pc[base + lane];
      float4 m0 = tb.mom0[nd], m1 = tb.mom1[nd], m2 = tb.mom2[nd];
      v[0] = -wrapf(__float_as_uint(m0.x), w.rx, cpu);
      v[1] = -wrapf(__float_as_uint(m0.y), w.ry, cpu);
      v[2] = -wrapf(__float_as_uint(m0.z), w.rz, cpu);
      v[3] = m0.w;                                      // mass
      v[4] = m1.x, v[5] = m1.y, v[6] = m1.z, v[7] = m1.w;  // Qxx Qyy Qzz Qxy
      v[8] = m2.x, v[9] = m2.y, v[10] = m2.z;             // Qxz Qyz trQ
    }
#pragma unroll
    for (int r = 0; r < 11; r++) row[32 * r + lane] = v[r];
    __syncwarp();
    float2 ax = make_float2(0.f, 0.f), ay = ax, az = ax;
    for (int j = 0; j < m; j += 2) {
      auto at = [&](int r) { return *reinterpret_cast<const float2 *>(row + 32 * r + j); };
      float2 dx = __fadd2_rn(tx, at(0)), dy = __fadd2_rn(ty, at(1)), dz = __fadd2_rn(tz, at(2));
      float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, floor2)));
      // f1 from the particle-particle table, f2 and f3 from the coarse one,
      // both indexed by the bits of r^2 (shared memory)
      float2 f1, f2, f3;
      f1.x = law_at(r2.x, tlb);
      f1.y = law_at(r2.y, tlb);
      {
        uint32_t b0 = __float_as_uint(r2.x), b1 = __float_as_uint(r2.y);
        int k0 = min(max((int)(b0 >> kPcShift) - kPcBase, 0), kPcEntries);
        int k1 = min(max((int)(b1 >> kPcShift) - kPcBase, 0), kPcEntries);
        float m0 = __uint_as_float((b0 & ((1u << kPcShift) - 1u)) | 0x3f800000u);
        float m1 = __uint_as_float((b1 & ((1u << kPcShift) - 1u)) | 0x3f800000u);
        float4 d0 = tq[k0], d1 = tq[k1];
        f2 = make_float2(fmaf(d0.y, m0, d0.x), fmaf(d1.y, m1, d1.x));
        f3 = make_float2(fmaf(d0.w, m0, d0.z), fmaf(d1.w, m1, d1.z));
      }
      float2 qxx = at(4), qyy = at(5), qzz = at(6), qxy = at(7), qxz = at(8), qyz = at(9);
      float2 q1x = __ffma2_rn(qxz, dz, __ffma2_rn(qxy, dy, __fmul2_rn(qxx, dx)));
      float2 q2y = __ffma2_rn(qyz, dz, __ffma2_rn(qyy, dy, __fmul2_rn(qxy, dx)));
      float2 q3z = __ffma2_rn(qzz, dz, __ffma2_rn(qyz, dy, __fmul2_rn(qxz, dx)));
      float2 qq = __ffma2_rn(dz, q3z, __ffma2_rn(dy, q2y, __fmul2_rn(dx, q1x)));
      float2 in = make_float2(r2.x <= rs2 ? 1.f : 0.f, r2.y <= rs2 ? 1.f : 0.f);
      float2 tt = __fmul2_rn(__ffma2_rn(qq, f3, __ffma2_rn(at(10), f2, __fmul2_rn(at(3), f1))), in);
      float2 two2 = __fmul2_rn(__fadd2_rn(f2, f2), in);
      ax = __ffma2_rn(q1x, two2, __ffma2_rn(dx, tt, ax));
      ay = __ffma2_rn(q2y, two2, __ffma2_rn(dy, tt, ay));
      az = __ffma2_rn(q3z, two2, __ffma2_rn(dz, tt, az));
    }
    if (w.active) {
      w.bx += ax.x + ax.y;
      w.by += ay.x + ay.y;
      w.bz += az.x + az.y;
      npc += (unsigned long long)m;
    }
    __syncwarp();
  }
}

// The 4-cell cubes along one axis of an n-cell periodic box whose cells meet
// [lo, hi] (cells, unwrapped): run[0..1] = first cube and count of the first
// run, run[2..3] of the second (empty unless [lo, hi] wraps past n). Both
// runs together list each cube once; an interval of n cells or more lists
// every cube.
TPM_D void axis_runs(float lo, float hi, int n, int run[4]) {
  const int ncube = (n + 3) >> 2;
  const float fn = (float)n;
  run[0] = 0;
  run[1] = ncube;
  run[2] = 0;
  run[3] = 0;
  if (hi - lo >= fn) return;
  float lw = lo - fn * floorf(lo / fn);
  if (lw >= fn) lw = 0.f;
  if (lw < 0.f) lw = 0.f;
  float hw = lw + (hi - lo);
  int a = min((int)(lw * 0.25f), ncube - 1);
  if (hw < fn) {
    int b = min((int)(hw * 0.25f), ncube - 1);
    run[0] = a;
    run[1] = b - a + 1;
    return;
  }
  int b = min((int)((hw - fn) * 0.25f), ncube - 1);
  if (b >= a) return;  // the runs meet: every cube
  run[0] = a;
  run[1] = ncube - a;
  run[2] = 0;
  run[3] = b + 1;
}

// The walk stack: the first kStackSmem entries in shared memory, the rest in
// this warp's global region.
struct WarpStack {
  uint32_t *sm;
  uint32_t *gl;
  TPM_D uint32_t get(int i) const { return i < kStackSmem ? sm[i] : gl[i - kStackSmem]; }
  TPM_D void put(int i, uint32_t v) {
    if (i < kStackSmem)
      sm[i] = v;
    else
      gl[i - kStackSmem] = v;
  }
};

// One launch walks the groups of one box (nbox == 1) or of an ensemble
// (boxes[0..nbox), group g of the launch belonging to the box b with
// gprefix[b] <= g < gprefix[b+1]). The boxes share the law table, which is
// per unit LL: each box's forces are scaled by its 1/N^2 at the end.
template <bool kHardCut>
__global__ void __launch_bounds__(kWalkThreads, kWalkBlocksPerSm) k_tree_walk(
    const WalkBox *__restrict__ boxes, const uint32_t *__restrict__ gprefix, int nbox,
    uint32_t *__restrict__ gnext, uint32_t *__restrict__ stack_base, uint32_t *__restrict__ stats,
    const float2 *__restrict__ glog, const float4 *__restrict__ gpc, float rs2, uint32_t kcut) {
  extern __shared__ float4 smem4[];
  float2 *tl = reinterpret_cast<float2 *>(smem4);
  float4 *tq = smem4 + kLogSmemF4;
  WarpLists *lists = reinterpret_cast<WarpLists *>(smem4 + kLogSmemF4 + kPcEntries + 1);
  for (int i = threadIdx.x; i <= kLogEntries; i += kWalkThreads) tl[i] = glog[i];
  for (int i = threadIdx.x; i <= kPcEntries; i += kWalkThreads) tq[i] = gpc[i];
  __syncthreads();
  int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  WarpLists &wl = lists[wib];
  int64_t gwarp = (int64_t)blockIdx.x * kWalkWarps + wib;
  WarpStack stack{wl.stack, stack_base + gwarp * (kStackCap - kStackSmem)};
  const uint32_t ngroups = nbox == 1 ? *boxes[0].ngroups : gprefix[nbox];
  unsigned long long npp = 0, npc = 0, niter = 0, nvisit = 0;
  int max_top = 0;
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  int cur_box = -1;
  while (true) {
    uint32_t g = 0;
    if (lane == 0) g = atomicAdd(gnext, 1u);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= ngroups) break;
    int b = 0;
    if (nbox > 1) {
      int lo = 0, hi = nbox - 1;
      while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (gprefix[mid] <= g) lo = mid;
        else hi = mid - 1;
      }
      b = lo;
      g -= gprefix[b];
    }
    if (b != cur_box) {
      // the box record into this warp's shared memory, one word per lane
      const uint32_t *src = reinterpret_cast<const uint32_t *>(&boxes[b]);
      constexpr int kWords = (int)(sizeof(WalkBox) / 4);
      static_assert(kWords <= 32, "box record larger than a warp's load");
      uint32_t v = lane < kWords ? src[lane] : 0u;
      __syncwarp();
      if (lane < kWords) reinterpret_cast<uint32_t *>(&wl.box)[lane] = v;
      __syncwarp();
      cur_box = b;
    }
    // the box's fields are read from the warp's shared copy where they are
    // used, which keeps them out of the registers the inner loops need
    uint32_t gs = wl.box.groups[2 * (int64_t)g], gc = wl.box.groups[2 * (int64_t)g + 1];
    WalkCtx w;
    w.active = (uint32_t)lane < gc;
    uint32_t ux = 0, uy = 0, uz = 0;
    if (w.active) {
      ux = wl.box.spos[3 * (int64_t)(gs + lane) + 0];
      uy = wl.box.spos[3 * (int64_t)(gs + lane) + 1];
      uz = wl.box.spos[3 * (int64_t)(gs + lane) + 2];
    }
    w.rx = __shfl_sync(0xffffffffu, ux, 0);
    w.ry = __shfl_sync(0xffffffffu, uy, 0);
    w.rz = __shfl_sync(0xffffffffu, uz, 0);
    w.tx = w.active ? wrapf(ux, w.rx, wl.box.cpu) : 0.f;
    w.ty = w.active ? wrapf(uy, w.ry, wl.box.cpu) : 0.f;
    w.tz = w.active ? wrapf(uz, w.rz, wl.box.cpu) : 0.f;
    w.ax = w.ay = w.az = 0.f;
    w.bx = w.by = w.bz = 0.f;
    // group box in cells
    float lox = w.tx, hix = w.tx, loy = w.ty, hiy = w.ty, loz = w.tz, hiz = w.tz;
    for (int o = 16; o > 0; o >>= 1) {
      lox = fminf(lox, __shfl_xor_sync(0xffffffffu, lox, o));
      hix = fmaxf(hix, __shfl_xor_sync(0xffffffffu, hix, o));
      loy = fminf(loy, __shfl_xor_sync(0xffffffffu, loy, o));
      hiy = fmaxf(hiy, __shfl_xor_sync(0xffffffffu, hiy, o));
      loz = fminf(loz, __shfl_xor_sync(0xffffffffu, loz, o));
      hiz = fmaxf(hiz, __shfl_xor_sync(0xffffffffu, hiz, o));
    }
    float cx = 0.5f * (lox + hix), cy = 0.5f * (loy + hiy), cz = 0.5f * (loz + hiz);
    float hx = 0.5f * (hix - lox), hy = 0.5f * (hiy - loy), hz = 0.5f * (hiz - loz);
    // a little slack against float rounding of the relative coordinates
    float rs2_prune = rs2 * 1.0001f + 1e-4f;
    const GroupBox gbox{cx, cy, cz, hx, hy, hz, rs2_prune};
    int top = 0, npcl = 0, nppl = 0;
    // The walk starts at the 4-cell cubes (tree level cbits - 2) that meet
    // the group's reach, not at the root: per axis at most two runs of cube
    // coordinates (the reach wraps around the periodic box at most once),
    // one cube per lane per pass. A near cube pushes its node, or, when it
    // has none (its parent held fewer than kLeafMin particles), appends its
    // particles. Nodes above that level are larger than the reach and would
    // only be opened.
    const int ncell = wl.box.n_cells;
    const float inv_ncell = __frcp_rn((float)ncell);
    int srun[3][4];
    int stotal;
    {
      const float reach = sqrtf(rs2_prune) + 0.01f;
      const float gc[3] = {cx, cy, cz}, gh[3] = {hx, hy, hz};
      const uint32_t ur[3] = {w.rx, w.ry, w.rz};
      stotal = 1;
      for (int a = 0; a < 3; a++) {
        float ref = __uint2float_rn(ur[a]) * wl.box.cpu;
        axis_runs(ref + gc[a] - gh[a] - reach, ref + gc[a] + gh[a] + reach, ncell, srun[a]);
        stotal *= srun[a][1] + srun[a][3];
      }
    }
    int sj = 0;
    __syncwarp();
    bool failed = false;
    while (top > 0 || sj < stotal) {
      int kind = 0;  // 0 drop, 1 accept (PC), 2 open (push children), 3 particles (PP)
      uint32_t c0 = 0, nch = 0, ps = 0, pcnt = 0;
      uint32_t node = 0;
      niter++;
      if (sj < stotal) {
        int j = sj + lane;
        sj += 32;
        if (j < stotal) {
          int nx = srun[0][1] + srun[0][3], ny = srun[1][1] + srun[1][3];
          // j = jx + nx (jy + ny jz); below 2^20 the quotients come exact from
          // float reciprocals ((q + 0.5) / d lies 0.5 / d from an integer,
          // far above the float error), else from integer division
          int jj[3];
          if (stotal < (1 << 20)) {
            int qx = (int)(((float)j + 0.5f) * __frcp_rn((float)nx));
            int qy = (int)(((float)qx + 0.5f) * __frcp_rn((float)ny));
            jj[0] = j - qx * nx;
            jj[1] = qx - qy * ny;
            jj[2] = qy;
          } else {
            jj[0] = j % nx;
            jj[1] = (j / nx) % ny;
            jj[2] = j / (nx * ny);
          }
          const float gc[3] = {cx, cy, cz}, gh[3] = {hx, hy, hz};
          const uint32_t ur[3] = {w.rx, w.ry, w.rz};
          uint32_t cc[3];
          float d2 = 0.f;
          for (int a = 0; a < 3; a++) {
            int c = jj[a] < srun[a][1] ? srun[a][0] + jj[a] : srun[a][2] + (jj[a] - srun[a][1]);
            cc[a] = (uint32_t)c;
            // the cube's cells [4c, min(4c + 4, n)) against the group box,
            // minimum image
            float c_lo = (float)(4 * c), c_hi = (float)min(4 * c + 4, ncell);
            float ref = __uint2float_rn(ur[a]) * wl.box.cpu;
            float d = 0.5f * (c_lo + c_hi) - (ref + gc[a]);
            // minimum image (at exactly half a box both images are equally far)
            d -= (float)ncell * rintf(d * inv_ncell);
            float e = fmaxf(fabsf(d) - 0.5f * (c_hi - c_lo) - gh[a], 0.f);
            d2 += e * e;
          }
          nvisit++;
          if (d2 <= rs2_prune) {
            uint64_t cid = morton3(cc[0], cc[1], cc[2]);
            uint32_t nd = wl.box.cube_node[cid];
            if (nd != kNoNode) {
              kind = 2;
              c0 = nd;
              nch = 1;
            } else {
              uint32_t s0 = wl.box.start_cube[cid], s1 = wl.box.start_cube[cid + 1];
              if (s1 > s0) {
                kind = 3;
                ps = s0;
                pcnt = s1 - s0;
              }
            }
          }
        }
      } else {
      // narrower pops keep a deep frontier from growing further
      int take = min(top, top > kStackSmem / 2 ? 8 : 32);
      nvisit += (unsigned long long)take;
      bool has = lane < take;
      if (has) node = stack.get(top - take + lane);
      __syncwarp();
      top -= take;
      // classify: one 32-byte and one 16-byte record per node
      if (has) {
        uint4 geo = wl.box.walkA[2 * (int64_t)node];
        uint4 com = wl.box.walkA[2 * (int64_t)node + 1];
        uint4 rec = wl.box.walkB[node];
        int lev = (int)(rec.w >> 16);
        nch = rec.w & 0xffffu;
        float half = __uint_as_float(geo.w);
        float dx = fmaxf(fabsf(wrapf(geo.x, w.rx, wl.box.cpu) - cx) - half - hx, 0.f);
        float dy = fmaxf(fabsf(wrapf(geo.y, w.ry, wl.box.cpu) - cy) - half - hy, 0.f);
        float dz = fmaxf(fabsf(wrapf(geo.z, w.rz, wl.box.cpu) - cz) - half - hz, 0.f);
        bool near = lev < 2 || dx * dx + dy * dy + dz * dz <= rs2_prune;
        if (near) {
          if (lev > 0 && rec.y < (uint32_t)kLeafMin) {
            kind = 3;
            ps = rec.x;
            pcnt = rec.y;
          } else {
            float ex = fmaxf(fabsf(wrapf(com.x, w.rx, wl.box.cpu) - cx) - hx, 0.f);
            float ey = fmaxf(fabsf(wrapf(com.y, w.ry, wl.box.cpu) - cy) - hy, 0.f);
            float ez = fmaxf(fabsf(wrapf(com.z, w.rz, wl.box.cpu) - cz) - hz, 0.f);
            bool open = lev < 2 || ex * ex + ey * ey + ez * ez < __uint_as_float(com.w);
            if (!open)
              kind = 1;
            else if (nch > 0) {
              kind = 2;
              c0 = rec.z;
            } else {
              kind = 3;
              ps = rec.x;
              pcnt = rec.y;
            }
          }
        }
      }
      }
      // children to push (at most 8 per lane) and particles to append: one
      // inclusive scan of both, packed as push | cnt << 9 (the push sum is at
      // most 256 and the count sum below 2^23 while every count is below
      // 2^18), else two scans
      uint32_t push = kind == 2 ? nch : 0u;
      uint32_t cnt = kind == 3 ? pcnt : 0u;
      uint32_t incl, pincl, total, ptotal;
      if (__all_sync(0xffffffffu, cnt < (1u << 18))) {
        uint32_t pk = push | (cnt << 9);
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t y = __shfl_up_sync(0xffffffffu, pk, o);
          if (lane >= o) pk += y;
        }
        incl = pk & 511u;
        pincl = pk >> 9;
        uint32_t pkt = __shfl_sync(0xffffffffu, pk, 31);
        total = pkt & 511u;
        ptotal = pkt >> 9;
      } else {
        incl = push;
        pincl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
          uint32_t y2 = __shfl_up_sync(0xffffffffu, pincl, o);
          if (lane >= o) {
            incl += y;
            pincl += y2;
          }
        }
        total = __shfl_sync(0xffffffffu, incl, 31);
        ptotal = __shfl_sync(0xffffffffu, pincl, 31);
      }
      if (top + (int)total > kStackCap) {
        failed = true;
        break;
      }
      for (uint32_t j = 0; j < push; j++) stack.put(top + (int)(incl - push + j), c0 + j);
      top += (int)total;
      max_top = max(max_top, top);
      __syncwarp();
      // accepted nodes
      unsigned acc = __ballot_sync(0xffffffffu, kind == 1);
      if (acc) {
        int cntv = __popc(acc);
        if (kind == 1) wl.pc[npcl + __popc(acc & lanemask_lt)] = node;
        npcl += cntv;
        __syncwarp();
        if (npcl >= 32) {
          eval_pc(wl, npcl, wl.box, w, wl.box.cpu, rs2, tl, tq, npc);
          npcl = 0;
        }
      }
      // particle ranges of all lanes at once: an inclusive scan of the counts
      // gives each lane its slice of the source list (lane order, as a
      // one-lane-at-a-time append would), flushed through eval_pp whenever
      // the batch fills
      uint32_t pexcl = pincl - cnt;
      uint32_t done = 0;
      while (done < ptotal) {
        uint32_t chunk = min((uint32_t)(kPpBatch - nppl), ptotal - done);
        uint32_t lo = max(pexcl, done), hi = min(pincl, done + chunk);
        for (uint32_t g = lo; g < hi; g++) wl.pp[nppl + (int)(g - done)] = ps + (g - pexcl);
        nppl += (int)chunk;
        done += chunk;
        __syncwarp();
        if (nppl == kPpBatch) {
          eval_pp<kHardCut>(wl, nppl, wl.box.spos, w, wl.box.cpu, gbox, rs2, kcut, tl, npp);
          nppl = 0;
        }
      }
    }
    if (failed) {
      if (lane == 0) atomicOr(wl.box.err, (uint32_t)kErrStackOverflow);
      continue;
    }
    if (npcl > 0) eval_pc(wl, npcl, wl.box, w, wl.box.cpu, rs2, tl, tq, npc);
    if (nppl > 0) eval_pp<kHardCut>(wl, nppl, wl.box.spos, w, wl.box.cpu, gbox, rs2, kcut, tl, npp);
    if (w.active) {
      // the tables are per unit LL: this box's 1/N^2
      int64_t i = (int64_t)gs + lane;
      float md = wl.box.mass, il = wl.box.inv_ll;
      float *ftree = wl.box.ftree;
      ftree[3 * i + 0] = fmaf(w.ax, md, w.bx) * il;
      ftree[3 * i + 1] = fmaf(w.ay, md, w.by) * il;
      ftree[3 * i + 2] = fmaf(w.az, md, w.bz) * il;
    }
  }

  // interaction counters
  for (int o = 16; o > 0; o >>= 1) {
    npp += __shfl_down_sync(0xffffffffu, npp, o);
    npc += __shfl_down_sync(0xffffffffu, npc, o);
    niter += __shfl_down_sync(0xffffffffu, niter, o);
    nvisit += __shfl_down_sync(0xffffffffu, nvisit, o);
  }
  if (lane == 0) {
    atomicAdd(reinterpret_cast<unsigned long long *>(&stats[2]), npp);
    atomicAdd(reinterpret_cast<unsigned long long *>(&stats[4]), npc);
    atomicAdd(reinterpret_cast<unsigned long long *>(&stats[6]), niter / 32);
    atomicAdd(reinterpret_cast<unsigned long long *>(&stats[8]), nvisit / 32);
    atomicMax(&stats[10], (uint32_t)max_top);
  }
}

static int walk_grid(size_t smem) {
  // The dynamic shared-memory cap is an attribute of the function on the
  // current device: it is raised on every launch, so every device (and every
  // host thread) gets it.
  size_t max_smem = sizeof(float4) * (kLogSmemF4 + kPcEntries + 1) + sizeof(WarpLists) * kWalkWarps;
  cudaFuncSetAttribute(k_tree_walk<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
  cudaFuncSetAttribute(k_tree_walk<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tree_walk<true>, kWalkThreads, smem);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (per_sm < 1) per_sm = 1;
  return per_sm * sms;
}

int64_t walk_stack_words() {
  // enough for the largest grid the walk can use on this device
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (int64_t)sms * kWalkBlocksPerSm * kWalkWarps * (kStackCap - kStackSmem);
}

WalkBox walk_box(const TreeParams &tp, const uint32_t *spos, const TreeBuffers &tb, float *ftree,
                 uint32_t *err) {
  WalkBox b;
  b.spos = spos;
  b.walkA = tb.walkA;
  b.walkB = tb.walkB;
  b.mom0 = tb.mom0;
  b.mom1 = tb.mom1;
  b.mom2 = tb.mom2;
  b.groups = tb.groups;
  b.ngroups = tb.counters;  // counters[0] = the group count tree_groups wrote
  b.ftree = ftree;
  b.err = err;
  b.cube_node = tb.cube_node;
  b.start_cube = tb.start_cube;
  b.cpu = tp.cell_per_unit;
  b.mass = tp.mass;
  b.inv_ll = (float)(1.0 / ((double)tp.n * (double)tp.n));
  b.n_cells = (int)tp.n;
  b.start_bits = kAxisBits - tp.sub_bits - 2;
  return b;
}

static void launch_walk(const WalkBox *boxes, const uint32_t *gprefix, int nbox, uint32_t *gnext, uint32_t *stack,
                        int64_t stack_words, uint32_t *stats, const LawTable &law, float rsphere, cudaStream_t st) {
  size_t smem = sizeof(float4) * (kLogSmemF4 + kPcEntries + 1) + sizeof(WarpLists) * kWalkWarps;
  int grid = walk_grid(smem);
  int64_t max_grid = stack_words / ((int64_t)kWalkWarps * (kStackCap - kStackSmem));
  if (grid > max_grid) grid = (int)max_grid;
  const float rs2 = rsphere * rsphere;
  // the bin every pair beyond the cut reads: for the reference law the bin
  // of rsphere^2 (the per-pair test discards its value), for the Gaussian law
  // the first bin of the table's zero tail
  uint32_t kcut;
  if (law.hard_cut) {
    uint32_t b;
    memcpy(&b, &rs2, 4);
    kcut = b >> kLogShift;
  } else {
    kcut = law.cut_bits >> kLogShift;
  }
  if (law.hard_cut)
    k_tree_walk<true><<<grid, kWalkThreads, smem, st>>>(boxes, gprefix, nbox, gnext, stack, stats, law.tlog, law.tpc,
                                                        rs2, kcut);
  else
    k_tree_walk<false><<<grid, kWalkThreads, smem, st>>>(boxes, gprefix, nbox, gnext, stack, stats, law.tlog,
                                                         law.tpc, rs2, kcut);
}

__global__ void k_set_walkbox(WalkBox *dst, WalkBox v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = v;
}

void tree_walk(const TreeParams &tp, const uint32_t *spos, int64_t np, const TreeBuffers &tb,
               const LawTable &law, float *ftree, uint32_t *err, cudaStream_t st, int64_t *launches) {
  (void)np;
  // the box record goes to the device with the launch that precedes the walk
  k_set_walkbox<<<1, 32, 0, st>>>(tb.walkbox, walk_box(tp, spos, tb, ftree, err));
  // tb.counters[1] is the next-group counter (zeroed before tree_groups)
  launch_walk(tb.walkbox, nullptr, 1, &tb.counters[1], tb.stack, tb.stack_words, tb.counters, law, tp.rsphere, st);
  if (launches) *launches += 2;
}

// Prefix of the boxes' group counts and the launch's next-group counter.
__global__ void k_group_prefix(const WalkBox *__restrict__ boxes, int nbox, uint32_t *__restrict__ gprefix,
                               uint32_t *__restrict__ gnext) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    uint32_t run = 0;
    for (int b = 0; b < nbox; b++) {
      gprefix[b] = run;
      run += *boxes[b].ngroups;
    }
    gprefix[nbox] = run;
    *gnext = 0;
  }
}

void tree_walk_multi(const WalkBox *boxes, int nbox, uint32_t *gprefix, uint32_t *gnext, uint32_t *stack,
                     int64_t stack_words, uint32_t *stats, const LawTable &law, float rsphere, cudaStream_t st) {
  k_group_prefix<<<1, 32, 0, st>>>(boxes, nbox, gprefix, gnext);
  launch_walk(boxes, gprefix, nbox, gnext, stack, stack_words, stats, law, rsphere, st);
}

}  // namespace tpm
