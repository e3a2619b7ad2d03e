// Morton-key particle sort (sm_100a).
//
// The reference orders particles spatially with a chaining mesh of
// CellWidth = 4 cells and head-inserted linked lists (Cosmos/BasicCell.c:10-42,
// BasicCell.h:33-63) and then builds one octree per bucket
// (OST/ost.ver2.c:36-196). Here every particle gets a 39-bit Morton key of its
// quantised cell coordinate (13 bits per axis: ceil(log2 N) cell bits plus
// sub-cell bits) and the (key, index) pairs are sorted by a stable LSD radix
// sort with 8-bit digits. Ties keep the input order, so the permutation is
// the stable argsort of the keys and is bit-exact against a CPU recomputation.
#include "engine_internal.cuh"

namespace tpm {

__global__ void k_make_keys(const uint32_t *__restrict__ pos, int64_t np, uint32_t n, int sub_bits,
                            uint64_t *__restrict__ key, uint32_t *__restrict__ val) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t qx = quantize(pos[3 * i + 0], n, sub_bits);
    uint32_t qy = quantize(pos[3 * i + 1], n, sub_bits);
    uint32_t qz = quantize(pos[3 * i + 2], n, sub_bits);
    key[i] = morton3(qx, qy, qz);
    val[i] = (uint32_t)i;
  }
}

void launch_make_keys(const uint32_t *pos, int64_t np, uint32_t n, int sub_bits, uint64_t *key,
                      uint32_t *val, cudaStream_t st) {
  int blocks = (int)((np + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  k_make_keys<<<blocks, 256, 0, st>>>(pos, np, n, sub_bits, key, val);
}

int64_t sort_tiles(int64_t np) { return (np + kSortTile - 1) / kSortTile; }

// Per-tile digit histogram; hist is digit-major: hist[d * ntiles + tile].
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint64_t *__restrict__ key,
                                                             int64_t np, int shift,
                                                             uint32_t *__restrict__ hist,
                                                             int64_t ntiles) {
  __shared__ uint32_t cnt[8][256];
  int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < 8 * 256; i += kSortThreads) (&cnt[0][0])[i] = 0;
  __syncthreads();
  int64_t base = blockIdx.x * (int64_t)kSortTile;
#pragma unroll
  for (int r = 0; r < kSortItems; r++) {
    int64_t i = base + r * kSortThreads + tid;
    if (i < np) {
      uint32_t d = (uint32_t)(key[i] >> shift) & 0xffu;
      atomicAdd(&cnt[warp][d], 1u);
    }
  }
  __syncthreads();
  for (int d = tid; d < 256; d += kSortThreads) {
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) s += cnt[w][d];
    hist[(int64_t)d * ntiles + blockIdx.x] = s;
  }
}

// One block per digit: exclusive scan of hist[d][0..ntiles) in place and the
// digit total.
__global__ void __launch_bounds__(1024) k_radix_scan_digit(uint32_t *__restrict__ hist, int64_t ntiles,
                                                           uint32_t *__restrict__ dtotal) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t carry;
  uint32_t *h = hist + (int64_t)blockIdx.x * ntiles;
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < ntiles; base += 1024) {
    int64_t i = base + tid;
    uint32_t v = i < ntiles ? h[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t s = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s;  // inclusive
    }
    __syncthreads();
    uint32_t before = carry + (warp ? wsum[warp - 1] : 0u) + x - v;
    if (i < ntiles) h[i] = before;
    __syncthreads();
    if (tid == 0) carry += wsum[31];
    __syncthreads();
  }
  if (tid == 0) dtotal[blockIdx.x] = carry;
}

// Stable scatter. The tile is consumed in kSortItems rounds of 256 items in
// index order; inside a round an item's rank among equal digits is
// (items of that digit in earlier rounds) + (in earlier warps) + (in lower
// lanes of its warp), so the relative order of equal digits is kept.
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint64_t *__restrict__ kout,
    uint32_t *__restrict__ vout, int64_t np, int shift, const uint32_t *__restrict__ hist,
    const uint32_t *__restrict__ dtotal, int64_t ntiles) {
  __shared__ uint32_t base[256];   // global offset of each digit for this tile
  __shared__ uint32_t wcnt[8][256];
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  {
    // digit start = exclusive scan of dtotal (256 entries) + this tile's offset
    uint32_t v = dtotal[tid];
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    __shared__ uint32_t ws[8];
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    uint32_t pre = 0;
    for (int w = 0; w < warp; w++) pre += ws[w];
    base[tid] = pre + x - v + hist[(int64_t)tid * ntiles + blockIdx.x];
  }
  __syncthreads();
  int64_t tbase = blockIdx.x * (int64_t)kSortTile;
  uint32_t lanemask_lt = (1u << lane) - 1u;
  for (int r = 0; r < kSortItems; r++) {
    for (int i = tid; i < 8 * 256; i += kSortThreads) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    int64_t i = tbase + r * kSortThreads + tid;
    bool valid = i < np;
    uint64_t k = valid ? kin[i] : 0ull;
    uint32_t v = valid ? vin[i] : 0u;
    uint32_t d = valid ? (uint32_t)(k >> shift) & 0xffu : 0x100u;  // 0x100: no digit
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t rank = __popc(peers & lanemask_lt);
    bool leader = (peers & lanemask_lt) == 0;
    if (valid && leader) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    // per digit: prefix over warps, then advance the digit base
    {
      int dd = tid;
      uint32_t run = base[dd];
#pragma unroll
      for (int w = 0; w < 8; w++) {
        uint32_t c = wcnt[w][dd];
        wcnt[w][dd] = run;
        run += c;
      }
      base[dd] = run;
    }
    __syncthreads();
    if (valid) {
      uint32_t dst = wcnt[warp][d] + rank;
      kout[dst] = k;
      vout[dst] = v;
    }
    __syncthreads();
  }
}

void radix_sort_pairs(uint64_t **key, uint32_t **val, uint64_t *key_alt, uint32_t *val_alt,
                      int64_t np, int nbits, SortScratch &scr, cudaStream_t st, int64_t *launches) {
  int64_t ntiles = sort_tiles(np);
  if (np <= 1) return;
  uint64_t *kin = *key, *kout = key_alt;
  uint32_t *vin = *val, *vout = val_alt;
  for (int shift = 0; shift < nbits; shift += 8) {
    k_radix_hist<<<(unsigned)ntiles, kSortThreads, 0, st>>>(kin, np, shift, scr.hist, ntiles);
    k_radix_scan_digit<<<256, 1024, 0, st>>>(scr.hist, ntiles, scr.dtotal);
    k_radix_scatter<<<(unsigned)ntiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, np, shift,
                                                               scr.hist, scr.dtotal, ntiles);
    if (launches) *launches += 3;
    uint64_t *tk = kin;
    kin = kout;
    kout = tk;
    uint32_t *tv = vin;
    vin = vout;
    vout = tv;
  }
  *key = kin;
  *val = vin;
}

__global__ void k_gather_pos(const uint32_t *__restrict__ pos, const uint32_t *__restrict__ perm,
                             int64_t np, uint32_t *__restrict__ spos) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t p = perm[i];
    spos[3 * i + 0] = pos[3 * (int64_t)p + 0];
    spos[3 * i + 1] = pos[3 * (int64_t)p + 1];
    spos[3 * i + 2] = pos[3 * (int64_t)p + 2];
  }
}

void launch_gather_pos(const uint32_t *pos, const uint32_t *perm, int64_t np, uint32_t *spos,
                       cudaStream_t st) {
  int blocks = (int)((np + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  k_gather_pos<<<blocks, 256, 0, st>>>(pos, perm, np, spos);
}

__global__ void k_range_table(const uint64_t *__restrict__ key, int64_t np, int shift,
                              uint32_t ntable, uint32_t *__restrict__ start) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= np;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t t = i < np ? (int64_t)(key[i] >> shift) : (int64_t)ntable;
    int64_t tp = i > 0 ? (int64_t)(key[i - 1] >> shift) : -1;
    if (t > (int64_t)ntable) t = ntable;
    for (int64_t q = tp + 1; q <= t; q++) start[q] = (uint32_t)i;
  }
}

void launch_range_table(const uint64_t *key, int64_t np, int shift, uint32_t ntable, uint32_t *start,
                        cudaStream_t st) {
  int blocks = (int)((np + 256) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_range_table<<<blocks, 256, 0, st>>>(key, np, shift, ntable, start);
}

}  // namespace tpm
