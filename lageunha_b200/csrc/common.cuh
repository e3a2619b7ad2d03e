// Shared device helpers of the TreePM engine (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define TPM_HD __host__ __device__ __forceinline__
#define TPM_D __device__ __forceinline__

// Bits per axis of the Morton key: cell bits + sub-cell bits = 13, so a key
// has 39 bits and sorts in 5 passes of 8 bits. With C = ceil(log2 N) cell
// bits the tree resolves 2^-(13-C) cells (1/16 cell at N = 512).
constexpr int kAxisBits = 13;
constexpr int kKeyBits = 3 * kAxisBits;

// Leaf rule of the reference octree: a sub-octant with fewer than 10
// particles is not a node (OST/ost.h:4, OST/ost.ver2.c:32,109-129).
constexpr int kLeafMin = 10;

TPM_HD uint64_t spread3_64(uint32_t v) {
  uint64_t x = v & 0x1fffffu;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// Morton key of per-axis quantised coordinates (x in the lowest bit).
TPM_HD uint64_t morton3(uint32_t qx, uint32_t qy, uint32_t qz) {
  return spread3_64(qx) | (spread3_64(qy) << 1) | (spread3_64(qz) << 2);
}

// Quantised coordinate: q = floor(x_cells * 2^sub_bits), x_cells = u*N/2^32.
TPM_HD uint32_t quantize(uint32_t u, uint32_t n, int sub_bits) {
  return (uint32_t)(((uint64_t)u * (uint64_t)n) >> (32 - sub_bits));
}

// Cell index floor(u*N/2^32) and fractional part in [0,1).
TPM_HD void cell_and_frac(uint32_t u, uint32_t n, int &cell, double &frac) {
  uint64_t p = (uint64_t)u * (uint64_t)n;
  cell = (int)(p >> 32);
  frac = (double)(uint32_t)(p & 0xffffffffu) * (1.0 / 4294967296.0);
}

// Position in cells (double) of a fixed-point coordinate.
TPM_HD double fixed_to_cells(uint32_t u, uint32_t n) {
  return (double)u * ((double)n / 4294967296.0);
}

// Minimum-image difference a - b in cells (exact wrap in fixed point).
TPM_HD float wrap_diff_cells(uint32_t a, uint32_t b, float cell_per_unit) {
  return (float)(int32_t)(a - b) * cell_per_unit;
}

TPM_HD int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
