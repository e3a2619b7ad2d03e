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

// Stable scatter of one tile of kSortTile items. Warp w owns the contiguous
// items [w*256, (w+1)*256) of the tile and ranks them in chunks of 32 against
// its own running digit counts (no block barrier per chunk); a prefix over the
// warps and over the digits then gives every item its place in the tile
// sorted by digit, which is written to shared memory. The tile is finally
// written out in that order, so each digit's run goes to consecutive global
// addresses. Items of equal digit keep their input order (chunks in order,
// lanes in order, warps in order), so the pass is a stable sort.
// Four blocks per SM: the ranking is a chain through each warp's digit
// counters (eight chunks), so the scatter is latency-bound and the tile is
// kept at 2048 items (39 KB of shared memory, each lane's 8 keys and values in
// 64 registers) for more resident warps; 4096-item tiles at three blocks per
// SM took 6% longer per sort.
constexpr int kScatterWarps = kSortThreads / 32;
constexpr int kWarpItems = kSortTile / kScatterWarps;
__global__ void __launch_bounds__(kSortThreads, 4) k_radix_scatter(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint64_t *__restrict__ kout,
    uint32_t *__restrict__ vout, int64_t np, int shift, const uint32_t *__restrict__ hist,
    const uint32_t *__restrict__ dtotal, int64_t ntiles) {
  extern __shared__ __align__(16) unsigned char sc_smem[];
  uint64_t *sk = reinterpret_cast<uint64_t *>(sc_smem);                 // [kSortTile] keys in digit order
  uint32_t *sv = reinterpret_cast<uint32_t *>(sk + kSortTile);          // [kSortTile] values
  uint16_t *rk = reinterpret_cast<uint16_t *>(sv + kSortTile);          // [kSortTile] rank in warp's digit
  uint32_t(*wc)[256] = reinterpret_cast<uint32_t(*)[256]>(rk + kSortTile);  // [warps][256]
  __shared__ uint32_t lstart[256];  // first slot of each digit in the tile
  __shared__ uint32_t gbase[256];   // global slot of each digit's first item of this tile
  __shared__ uint32_t ws[kScatterWarps];
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < kScatterWarps * 256; i += kSortThreads) (&wc[0][0])[i] = 0;
  __syncthreads();
  const int64_t tbase = blockIdx.x * (int64_t)kSortTile;
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  // this lane's items of the warp's segment, all loaded before any is ranked
  constexpr int kChunks = kWarpItems / 32;
  uint64_t kr[kChunks];
  uint32_t vr[kChunks];
#pragma unroll
  for (int c = 0; c < kChunks; c++) {
    int64_t i = tbase + warp * kWarpItems + c * 32 + lane;
    kr[c] = i < np ? kin[i] : 0ull;
    vr[c] = i < np ? vin[i] : 0u;
  }
  // ---- ranks inside each warp's segment
#pragma unroll
  for (int c = 0; c < kChunks; c++) {
    int j = warp * kWarpItems + c * 32 + lane;
    int64_t i = tbase + j;
    bool valid = i < np;
    uint32_t d = valid ? (uint32_t)(kr[c] >> shift) & 0xffu : 0x100u;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t prev = valid ? wc[warp][d] : 0u;
    __syncwarp();
    if (valid && (peers & lanemask_lt) == 0) wc[warp][d] = prev + __popc(peers);
    __syncwarp();
    rk[j] = (uint16_t)(prev + __popc(peers & lanemask_lt));
  }
  __syncthreads();
  // ---- per digit: prefix over the warps, the tile's count, and its global base
  uint32_t cnt;
  {
    int d = tid;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kScatterWarps; w++) {
      uint32_t t = wc[w][d];
      wc[w][d] = run;
      run += t;
    }
    cnt = run;
    // exclusive scans over the 256 digits: tile counts and global digit totals
    uint32_t x = cnt, g = dtotal[d];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      uint32_t h = __shfl_up_sync(0xffffffffu, g, o);
      if (lane >= o) {
        x += y;
        g += h;
      }
    }
    if (lane == 31) ws[warp] = x;
    __shared__ uint32_t wg[kScatterWarps];
    if (lane == 31) wg[warp] = g;
    __syncthreads();
    uint32_t px = 0, pg = 0;
    for (int w = 0; w < warp; w++) {
      px += ws[w];
      pg += wg[w];
    }
    lstart[d] = px + x - cnt;
    gbase[d] = pg + g - dtotal[d] + hist[(int64_t)d * ntiles + blockIdx.x];
  }
  __syncthreads();
  // ---- place every item at its slot of the tile sorted by digit
#pragma unroll
  for (int c = 0; c < kChunks; c++) {
    int j = warp * kWarpItems + c * 32 + lane;
    int64_t i = tbase + j;
    if (i < np) {
      uint64_t k = kr[c];
      uint32_t d = (uint32_t)(k >> shift) & 0xffu;
      uint32_t slot = lstart[d] + wc[warp][d] + rk[j];
      sk[slot] = k;
      sv[slot] = vr[c];
    }
  }
  __syncthreads();
  // ---- write out: consecutive slots of a digit go to consecutive addresses
  int64_t nt = np - tbase < kSortTile ? np - tbase : kSortTile;
  for (int j = tid; j < nt; j += kSortThreads) {
    uint64_t k = sk[j];
    uint32_t d = (uint32_t)(k >> shift) & 0xffu;
    uint32_t g = gbase[d] + ((uint32_t)j - lstart[d]);
    kout[g] = k;
    vout[g] = sv[j];
  }
}

constexpr size_t kScatterSmem = (size_t)kSortTile * (8 + 4 + 2) + sizeof(uint32_t) * kScatterWarps * 256;

void radix_sort_pairs(uint64_t **key, uint32_t **val, uint64_t *key_alt, uint32_t *val_alt,
                      int64_t np, int nbits, SortScratch &scr, cudaStream_t st, int64_t *launches) {
  int64_t ntiles = sort_tiles(np);
  if (np <= 1) return;
  uint64_t *kin = *key, *kout = key_alt;
  uint32_t *vin = *val, *vout = val_alt;
  // the cap is an attribute of the function on the current device: raised on
  // every call, so contexts and threads on any device get it
  cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kScatterSmem);
  for (int shift = 0; shift < nbits; shift += 8) {
    k_radix_hist<<<(unsigned)ntiles, kSortThreads, 0, st>>>(kin, np, shift, scr.hist, ntiles);
    k_radix_scan_digit<<<256, 1024, 0, st>>>(scr.hist, ntiles, scr.dtotal);
    k_radix_scatter<<<(unsigned)ntiles, kSortThreads, kScatterSmem, st>>>(kin, vin, kout, vout, np, shift,
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
