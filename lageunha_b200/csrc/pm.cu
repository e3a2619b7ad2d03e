// Particle-mesh long-range force (sm_100a): TSC deposit, a shared-memory
// pencil FFT with the Green's function fused between the forward and the
// inverse z transform, and the 4-point gradient + TSC interpolation staged
// through TMA.
//
// Reference path (kjhan0606/LagEunha, GOTPM build):
//   TSC scatter            Cosmos/pmmain.h:81-159, pmmain.c:112-185
//   fold into FFT slab     Cosmos/pmmain.c:283-336, RkS/gmigrate.c:212-273
//   r2c / c2r              Cosmos/pmmain.c:475,492 (FFTW-MPI, unnormalised)
//   Green's function       Cosmos/psolver.c:13-86
//   ghosted potential      Cosmos/pmmain.c:337-388
//   gradient + interp.     Cosmos/fda4.h:11-103,276-384, fda4.c:45-46
#include <math.h>
#include <string.h>
#include <stdio.h>

#include <algorithm>

#include "engine_internal.cuh"

namespace tpm {

MeshGeom make_geom(int n) {
  MeshGeom g;
  g.n = n;
  int c = 0;
  while ((1 << c) < n) c++;
  if (c < 3) c = 3;
  g.cbits = c;
  g.sub_bits = kAxisBits - c;
  g.tiles_axis = 1 << (c - 3);
  g.hx = n / 2 + 1;
  g.spec_elems = (int64_t)n * n * g.hx;
  g.px = ((n + 2 * kGhost) + 3) / 4 * 4;
  g.py = n + 2 * kGhost;
  g.pz = n + 2 * kGhost;
  return g;
}

// ------------------------------------------------------------------ TSC
// Home node and the three per-axis TSC weights on offsets {-1, 0, +1}
// relative to it. The reference picks near = rint(x), xmin = x - near,
// sign = signbit(xmin) ? -1 : 1 and weights w1 = 0.75 - d^2 at near,
// w2 = 0.5 (0.5 + d)^2 at near + sign, w3 = 0.5 (0.5 - d)^2 at near - sign
// with d = |xmin| (pmmain.h:86-120). Here w[0], w[1], w[2] are the weights
// at near-1, near, near+1.
struct Axis {
  int near;     // nearest grid node (cells, absolute)
  float xmin;   // x - near in [-0.5, 0.5]
};

// half != 0: the position moved by exactly half a cell along the axis (the
// second grid of the interlaced deposit), without the periodic wrap, so a
// particle keeps the home-node range [8t, 8t+8] of its Morton tile t.
TPM_D Axis axis_of(uint32_t u, uint32_t n, uint32_t half = 0) {
  uint64_t p = (uint64_t)u * (uint64_t)n + (half ? 0x80000000ull : 0ull);
  int c = (int)(p >> 32);
  uint32_t fr = (uint32_t)p;
  // xmin is the FP64 value fr 2^-32 (or fr 2^-32 - 1) rounded to float:
  // both are a 32-bit integer times 2^-32, so rounding that integer to float
  // and scaling by the power of two gives the same bits without FP64
  Axis a;
  if (fr > 0x80000000u) {
    a.near = c + 1;
    a.xmin = -(__uint2float_rn(0u - fr) * 2.3283064365386963e-10f);
  } else {
    a.near = c;
    a.xmin = __uint2float_rn(fr) * 2.3283064365386963e-10f;
  }
  return a;
}

TPM_D void tsc_w(float xmin, float &w1, float &w2, float &w3, int &sign) {
  sign = signbit(xmin) ? -1 : 1;
  float d = fabsf(xmin);
  w1 = 0.75f - d * d;
  w3 = 0.5f * (0.25f + d * (d - 1.0f));
  w2 = w3 + d;
}

// The deposit tile's accumulator covers nodes [t-1, t+11) per axis (the
// stencils of particles in [t, t+8) reach [t-1, t+9]) with strides 1, 12,
// 144: a 4x4x2 block of home nodes, which 32 Morton-consecutive particles at
// one per cell occupy, falls on 32 distinct shared-memory banks, as do its 27
// shifted copies.
constexpr int kDepNx = 12;
constexpr int kDepNy = 12;
constexpr int kDepCells = kDepNx * kDepNy * kDepNy;
constexpr int kDepThreads = 256;

// Per-axis weights on offsets -1, 0, +1 around the home node of a particle,
// with or without the half-cell shift of the second interlaced grid.
TPM_D void tsc_axis3(uint32_t u, uint32_t n, uint32_t half, float scale, float w[3], int &near) {
  Axis a = axis_of(u, n, half);
  float w1, w2, w3;
  int s;
  tsc_w(a.xmin, w1, w2, w3, s);
  w[1] = w1 * scale;
  w[1 + s] = w2 * scale;
  w[1 - s] = w3 * scale;
  near = a.near;
}

// The tile accumulates in 32-bit fixed point (integer shared-memory atomics
// are single operations; float ones are not): weights carry the tile's scale
// 2^e, the largest power of two for which no node can exceed 2^32 - a node's
// mass is at most count * mass * 0.75^3 - and the flush multiplies by 2^-e,
// exactly. Integer sums do not depend on the order of the additions.
TPM_D void fix_add(uint32_t *acc, int i, float v) { atomicAdd(&acc[i], __float2uint_rn(v)); }

// Adds the 27 weights of every valid lane to acc. When at least half of the
// warp's lanes start a run of equal home nodes, every lane adds its own
// weights (integer atomics to one address serialise, but a few repeats cost
// less than merging); otherwise (dense clumps put many particles on one node)
// the runs are merged by a warp segmented sum first. Measured: the 512^3
// workload's deposit 5.53 -> 5.28 ms and the clustered 256^3 one 0.99 -> 0.93
// ms against merging whenever any two lanes share a node; always adding
// directly took 5.10 and 1.40 ms.
TPM_D void deposit_lanes(uint32_t *acc, bool valid, int home, const float wx[3], const float wy[3],
                         const float wz[3], int lane) {
  int key = valid ? home : -1 - lane;
  int prev = __shfl_up_sync(0xffffffffu, key, 1);
  bool head = lane == 0 || prev != key;
  unsigned heads = __ballot_sync(0xffffffffu, head);
  if (__popc(heads) >= 16) {
    if (valid) {
      for (int c = 0; c < 3; c++)
        for (int b = 0; b < 3; b++)
          for (int a = 0; a < 3; a++)
            fix_add(acc, home + (a - 1) + kDepNx * ((b - 1) + kDepNy * (c - 1)), wx[a] * wy[b] * wz[c]);
    }
    return;
  }
  // runs of equal home node: segmented sum onto the run's first lane, in
  // as many halving rounds as the warp's longest run needs
  unsigned le = heads & ((2u << lane) - 1u);
  int seg = 31 - __clz(le);
  unsigned above = heads & ~((2u << lane) - 1u);
  unsigned run = head ? (unsigned)((above ? __ffs(above) - 1 : 32) - lane) : 1u;
  unsigned maxrun = __reduce_max_sync(0xffffffffu, run);
  int rounds = 32 - __clz((int)maxrun - 1);
  float w[27];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
      for (int a = 0; a < 3; a++) w[a + 3 * b + 9 * c] = wx[a] * wy[b] * wz[c];
  for (int j = 0; j < rounds; j++) {
    int o = 1 << j;
    int s2 = __shfl_down_sync(0xffffffffu, seg, o);
    bool ok = (lane + o < 32) && s2 == seg;
#pragma unroll
    for (int q = 0; q < 27; q++) {
      float y = __shfl_down_sync(0xffffffffu, w[q], o);
      if (ok) w[q] += y;
    }
  }
  if (valid && head) {
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int b = 0; b < 3; b++)
#pragma unroll
        for (int a = 0; a < 3; a++)
          fix_add(acc, home + (a - 1) + kDepNx * ((b - 1) + kDepNy * (c - 1)), w[a + 3 * b + 9 * c]);
  }
}

// v in [-n, 2n) into [0, n): the flush's node coordinates lie within a few
// cells of the box (tile origin - 4 to + 12, n >= 16), so one conditional
// add or subtract replaces an integer remainder by the run-time n.
TPM_D int wrap_once(int v, int n) {
  v += v < 0 ? n : 0;
  return v >= n ? v - n : v;
}

// Adds a tile's shared-memory accumulator (origin ox = t-1 per axis) to the
// periodic mesh. vec4: the mesh's x rows are added as float4 groups aligned
// to 4 cells, [t-4, t), ..., [t+8, t+12), read from the accumulator with
// the cells outside it as zero.
TPM_D void flush_tile(const uint32_t *acc, float inv_scale, float *__restrict__ rho, int n, int ox, int oy, int oz,
                      int vec4, int tid) {
  constexpr int kUsed = kTile + 3;  // nodes [t-1, t+9] per axis
  if (vec4) {
    for (int i = tid; i < 4 * kUsed * kUsed; i += kDepThreads) {
      int q = i & 3, r = i >> 2;
      int y = r % kUsed, z = r / kUsed;
      const uint32_t *row = acc + kDepNx * (y + kDepNy * z);
      float v[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        int xi = 4 * q - 3 + j;
        v[j] = (xi >= 0 && xi < kUsed) ? (float)row[xi] * inv_scale : 0.f;
      }
      if (v[0] == 0.f && v[1] == 0.f && v[2] == 0.f && v[3] == 0.f) continue;
      int gx = wrap_once(ox - 3 + 4 * q, n), gy = wrap_once(oy + y, n), gz = wrap_once(oz + z, n);
      float4 *dst = reinterpret_cast<float4 *>(rho + gx + (int64_t)n * (gy + (int64_t)n * gz));
      atomicAdd(dst, make_float4(v[0], v[1], v[2], v[3]));
    }
  } else {
    for (int i = tid; i < kUsed * kUsed * kUsed; i += kDepThreads) {
      int x = i % kUsed, r = i / kUsed;
      int y = r % kUsed, z = r / kUsed;
      float v = (float)acc[x + kDepNx * (y + kDepNy * z)] * inv_scale;
      if (v == 0.f) continue;
      int gx = wrap_once(ox + x, n), gy = wrap_once(oy + y, n), gz = wrap_once(oz + z, n);
      atomicAdd(rho + gx + (int64_t)n * (gy + (int64_t)n * gz), v);
    }
  }
}

// TSC deposit of one 8^3 Morton tile; half != 0: the particles moved by half
// a cell (the second grid of the interlaced pair). One grid per launch: a
// kernel holding both grids' accumulators ran slower (fewer blocks per SM).
__global__ void __launch_bounds__(kDepThreads) k_tsc_deposit(
    const uint32_t *__restrict__ spos, const uint32_t *__restrict__ tile_start, int n, int cbits,
    float mass, float *__restrict__ rho, uint32_t half, int vec4) {
  __shared__ __align__(16) uint32_t acc[kDepCells];
  int tid = threadIdx.x, lane = tid & 31;
  // Morton tile index -> tile coordinates
  uint32_t t = blockIdx.x;
  uint32_t tx = 0, ty = 0, tz = 0;
  for (int b = 0; b < cbits - 3; b++) {
    tx |= ((t >> (3 * b)) & 1u) << b;
    ty |= ((t >> (3 * b + 1)) & 1u) << b;
    tz |= ((t >> (3 * b + 2)) & 1u) << b;
  }
  uint32_t p0 = tile_start[t], p1 = tile_start[t + 1];
  if (p0 == p1) return;
  int ox = (int)tx * kTile - 1, oy = (int)ty * kTile - 1, oz = (int)tz * kTile - 1;
  for (int i = tid; i < kDepCells; i += kDepThreads) acc[i] = 0u;
  // fixed-point scale 2^e: count * mass * 0.75^3 * 2^e < 2^31 (a factor two
  // below the 32-bit limit for the rounding of each contribution)
  int e;
  frexpf((float)(p1 - p0) * mass * 0.421875f, &e);
  e = min(31 - e, 40);
  const float scale = ldexpf(1.f, e), inv_scale = ldexpf(1.f, -e);
  __syncthreads();
  uint32_t nu = (uint32_t)n;
  int nwarp_items = (int)((p1 - p0 + 31) / 32) * 32;
  // each thread's next particle is loaded before this one's deposit
  uint32_t un[3] = {0u, 0u, 0u};
  if ((uint32_t)tid < p1 - p0) {
    int64_t i = (int64_t)p0 + tid;
    un[0] = spos[3 * i + 0];
    un[1] = spos[3 * i + 1];
    un[2] = spos[3 * i + 2];
  }
  for (int base = 0; base < nwarp_items; base += kDepThreads) {
    int k = base + tid;
    bool valid = (uint32_t)k < p1 - p0;
    uint32_t u[3] = {un[0], un[1], un[2]};
    if ((uint32_t)(k + kDepThreads) < p1 - p0) {
      int64_t i = (int64_t)p0 + k + kDepThreads;
      un[0] = spos[3 * i + 0];
      un[1] = spos[3 * i + 1];
      un[2] = spos[3 * i + 2];
    }
    float wx[3] = {0, 0, 0}, wy[3] = {0, 0, 0}, wz[3] = {0, 0, 0};
    int home = 0;
    if (valid) {
      int hx, hy, hz;
      tsc_axis3(u[0], nu, half, mass * scale, wx, hx);
      tsc_axis3(u[1], nu, half, 1.f, wy, hy);
      tsc_axis3(u[2], nu, half, 1.f, wz, hz);
      home = (hx - ox) + kDepNx * ((hy - oy) + kDepNy * (hz - oz));
    }
    deposit_lanes(acc, valid, home, wx, wy, wz, lane);
  }
  __syncthreads();
  flush_tile(acc, inv_scale, rho, n, ox, oy, oz, vec4, tid);
}

void launch_tsc_deposit(const MeshGeom &g, const uint32_t *spos, const uint32_t *tile_start,
                        float mass, float *rho, cudaStream_t st, float *rho2) {
  uint32_t ntiles = 1u << (3 * (g.cbits - 3));
  int vec4 = (g.n % 4) == 0;
  k_tsc_deposit<<<ntiles, kDepThreads, 0, st>>>(spos, tile_start, g.n, g.cbits, mass, rho, 0u, vec4);
  if (rho2) k_tsc_deposit<<<ntiles, kDepThreads, 0, st>>>(spos, tile_start, g.n, g.cbits, mass, rho2, 1u, vec4);
}

// ------------------------------------------------------------------ FFT
// Stockham autosort radix-16/8/4/2/3/5 transform of a batch of pencils held in
// shared memory (the formulation of Govindaraju et al., SC08): in stage s
// with radix R and Ns = product of the earlier radices, job j reads
// in[j + r L/R], twiddles by exp(dir 2 pi i r (j mod Ns) / (Ns R)), does a
// size-R DFT and writes out[(j / Ns) Ns R + (j mod Ns) + r Ns].

struct Factors {
  int nf;
  int r[16];
};

// global loads each thread issues before it stores them into shared memory
// (enough bytes in flight per SM for the transposing passes to stream)
constexpr int kLoadBatch = 8;

// radices of the x passes (packed rows) and of the column passes
constexpr int kXRadixMax = 16;
constexpr int kColRadixMax = 16;

static Factors factorize(int L, int rmax) {
  Factors f;
  f.nf = 0;
  while (rmax >= 16 && L % 16 == 0) {
    f.r[f.nf++] = 16;
    L /= 16;
  }
  if (rmax >= 8 && L % 8 == 0) {
    f.r[f.nf++] = 8;
    L /= 8;
  }
  while (L % 4 == 0) {
    f.r[f.nf++] = 4;
    L /= 4;
  }
  while (L % 2 == 0) {
    f.r[f.nf++] = 2;
    L /= 2;
  }
  while (L % 3 == 0) {
    f.r[f.nf++] = 3;
    L /= 3;
  }
  while (L % 5 == 0) {
    f.r[f.nf++] = 5;
    L /= 5;
  }
  if (L != 1) f.nf = -1;
  return f;
}

// Quotient by a divisor known only at run time, for 0 <= e < 2^24: a shift
// where the divisor is a power of two (the usual mesh and batch sizes), else
// the float reciprocal corrected by one step. The branch is uniform.
struct Div {
  int d, s;     // s >= 0: d == 1 << s
  float inv;
  TPM_D int q(int e) const {
    if (s >= 0) return e >> s;
    int p = (int)((float)e * inv);
    int r = e - p * d;
    return r < 0 ? p - 1 : (r >= d ? p + 1 : p);
  }
};
TPM_D Div make_div(int d) {
  Div r;
  r.d = d;
  r.s = (d & (d - 1)) == 0 ? __ffs(d) - 1 : -1;
  r.inv = r.s >= 0 ? 0.f : 1.f / (float)d;
  return r;
}

// Shared-memory slot of element m of a pencil: one spare slot after every 16
// elements. The first Stockham stage writes at stride R (up to 16 float2, so
// a half-warp's 16 lanes would hit one bank pair); with the spare slots those
// writes, and the column passes' transposing loads and stores, fall on
// distinct bank pairs.
TPM_HD int fslot(int m) { return m + (m >> 4); }
// slots a pencil of L elements spans
TPM_HD int fslots(int L) { return fslot(L - 1) + 1; }
// Pencil stride of the column passes for P pencils per block: at least
// fslots(n), and = 16/P (mod 16) for P < 16 (odd for P >= 16), so the P
// pencils of a transposing load's half-warp start on distinct bank pairs.
TPM_HD int col_stride(int n, int P) {
  int s = fslots(n);
  int r = P >= 16 ? 1 : (16 / P);
  return s + (((r - s) % 16) + 16) % 16;
}

TPM_D float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
TPM_D float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
TPM_D float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
TPM_D float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by dir * i
TPM_D float2 cmuli(float2 a, float dir) { return make_float2(-dir * a.y, dir * a.x); }

template <int R>
TPM_D void dft_small(float2 *v, float dir);

template <>
TPM_D void dft_small<2>(float2 *v, float) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}
template <>
TPM_D void dft_small<4>(float2 *v, float dir) {
  float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
  float2 s13 = cadd(v[1], v[3]), d13 = cmuli(csub(v[1], v[3]), dir);
  v[0] = cadd(s02, s13);
  v[2] = csub(s02, s13);
  v[1] = cadd(d02, d13);
  v[3] = csub(d02, d13);
}
template <>
TPM_D void dft_small<3>(float2 *v, float dir) {
  const float c = -0.5f, s = 0.86602540378443864676f;
  float2 t = cadd(v[1], v[2]);
  float2 m = make_float2(v[0].x + c * t.x, v[0].y + c * t.y);
  float2 d = cmuli(csub(v[1], v[2]), dir * s);
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, d);
  v[2] = csub(m, d);
}
template <>
TPM_D void dft_small<5>(float2 *v, float dir) {
  const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
  const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
  float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  float2 x0 = v[0];
  float2 m1 = make_float2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
  float2 m2 = make_float2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
  // i*dir*(s1 b1 + s2 b2) and i*dir*(s2 b1 - s1 b2)
  float2 n1 = cmuli(make_float2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), dir);
  float2 n2 = cmuli(make_float2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), dir);
  v[0] = make_float2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

// 8 points: even and odd halves by radix 4, combined with W8^k.
template <>
TPM_D void dft_small<8>(float2 *v, float dir) {
  const float h = 0.70710678118654752440f;  // cos(pi/4)
  float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  dft_small<4>(e, dir);
  dft_small<4>(o, dir);
  // W8^k = exp(dir 2 pi i k / 8)
  float2 t1 = make_float2(h * (o[1].x - dir * o[1].y), h * (o[1].y + dir * o[1].x));
  float2 t2 = cmuli(o[2], dir);
  float2 t3 = make_float2(-h * (o[3].x + dir * o[3].y), h * (dir * o[3].x - o[3].y));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], t1);
  v[5] = csub(e[1], t1);
  v[2] = cadd(e[2], t2);
  v[6] = csub(e[2], t2);
  v[3] = cadd(e[3], t3);
  v[7] = csub(e[3], t3);
}

// 16 points as 4 x 4: transforms over n1 of v[4 n1 + n2], twiddles
// W16^(n2 k1), transforms over n2; X[k1 + 4 k2].
template <>
TPM_D void dft_small<16>(float2 *v, float dir) {
  const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;  // cos, sin of pi/8
  const float h = 0.70710678118654752440f;
  float2 y[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) {
    float2 t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
    dft_small<4>(t, dir);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) y[n2][k1] = t[k1];
  }
  // W16^m = (cos(m pi/8), dir sin(m pi/8)) for m = n2 k1 in {1, 2, 3, 4, 6, 9}
  const float cw[10] = {1.f, c1, h, s1, 0.f, -s1, -h, -c1, -1.f, -c1};
  const float sw[10] = {0.f, s1, h, c1, 1.f, c1, h, s1, 0.f, -s1};
#pragma unroll
  for (int n2 = 1; n2 < 4; n2++)
#pragma unroll
    for (int k1 = 1; k1 < 4; k1++) {
      int m = n2 * k1;
      float2 w = make_float2(cw[m], dir * sw[m]);
      y[n2][k1] = cmul(y[n2][k1], w);
    }
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    float2 t[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
    dft_small<4>(t, dir);
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = t[k2];
  }
}

template <int R>
TPM_D void stockham_stage(const float2 *in, float2 *out, const float2 *tw, int L, int ld, int Ns, int P,
                          float dir, int tid, int nth) {
  int jobs_per = L / R;
  int step = L / (Ns * R);
  for (int job = tid; job < P * jobs_per; job += nth) {
    int p = job / jobs_per, j = job - p * jobs_per;
    const float2 *src = in + p * ld;
    float2 *dst = out + p * ld;
    int jn = j / Ns;
    int k = j - jn * Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      float2 x = src[fslot(j + r * jobs_per)];
      if (r) {
        float2 w = tw[r * k * step];  // r k step < L: r < R, k < Ns, step = L / (Ns R)
        if (dir > 0) w.y = -w.y;
        x = cmul(x, w);
      }
      v[r] = x;
    }
    dft_small<R>(v, dir);
    int d0 = jn * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) dst[fslot(d0 + r * Ns)] = v[r];
  }
}

// Transforms P pencils of length L (pencil p at p * ld, element m at slot
// fslot(m), ld >= fslots(L)) from a to scratch b
// and back as needed; returns the buffer holding the result. dir = -1
// forward, +1 backward (unnormalised, FFTW sign convention).
__device__ float2 *fft_pencils(float2 *a, float2 *b, const float2 *tw, int L, int ld, int P, float dir,
                               const int *radix, int nf) {
  int tid = threadIdx.x, nth = blockDim.x;
  int Ns = 1;
  float2 *in = a, *out = b;
  for (int s = 0; s < nf; s++) {
    int R = radix[s];
    if (R == 16)
      stockham_stage<16>(in, out, tw, L, ld, Ns, P, dir, tid, nth);
    else if (R == 8)
      stockham_stage<8>(in, out, tw, L, ld, Ns, P, dir, tid, nth);
    else if (R == 4)
      stockham_stage<4>(in, out, tw, L, ld, Ns, P, dir, tid, nth);
    else if (R == 2)
      stockham_stage<2>(in, out, tw, L, ld, Ns, P, dir, tid, nth);
    else if (R == 3)
      stockham_stage<3>(in, out, tw, L, ld, Ns, P, dir, tid, nth);
    else
      stockham_stage<5>(in, out, tw, L, ld, Ns, P, dir, tid, nth);
    __syncthreads();
    Ns *= R;
    float2 *t = in;
    in = out;
    out = t;
  }
  return in;
}

struct FftArgs {
  int n, hx, L;       // mesh size, n/2+1, pencil length of this pass
  int nf;
  int radix[16];
  int P;              // pencils per block
};

static FftArgs fft_args(int n, int L, int P, int rmax) {
  FftArgs a;
  a.n = n;
  a.hx = n / 2 + 1;
  a.L = L;
  Factors f = factorize(L, rmax);
  a.nf = f.nf;
  for (int i = 0; i < 16; i++) a.radix[i] = i < f.nf ? f.r[i] : 1;
  a.P = P;
  return a;
}

// twiddle table exp(-2 pi i k / L), k < L
__global__ void k_twiddles(float2 *tw, int L) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < L) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)L, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
}

__global__ void k_fft_x_r2c(const float *__restrict__ rho, float2 *__restrict__ spec, struct FftArgs a,
                            const float2 *__restrict__ tw_L, const float2 *__restrict__ tw_n, int64_t nrows);
__global__ void k_fft_x_c2r(const float2 *__restrict__ spec, float *__restrict__ phi, struct FftArgs a,
                            const float2 *__restrict__ tw_L, const float2 *__restrict__ tw_n, int64_t nrows,
                            int px, int py);
__global__ void k_fft_cols(float2 *__restrict__ spec, float2 *__restrict__ spec2, struct FftArgs a,
                           const float2 *__restrict__ tw_n, int axis, float dir, int with_green, struct GreenArgs ga,
                           int TX, int nspec);

cudaError_t fft_plan_init(FftPlan &p, int n, cudaStream_t st, DeviceArena *arena) {
  p.n = n;
  p.arena = arena;
  const int max_smem = 160 * 1024;
  cudaFuncSetAttribute(k_fft_x_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  cudaFuncSetAttribute(k_fft_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
  int h = n / 2 > 0 ? n / 2 : 1;
  cudaError_t e = dmalloc(arena, &p.tw, sizeof(float2) * n);
  if (e == cudaSuccess) e = dmalloc(arena, &p.tw_half, sizeof(float2) * h);
  if (e != cudaSuccess) return e;
  k_twiddles<<<(n + 255) / 256, 256, 0, st>>>(p.tw, n);
  k_twiddles<<<(h + 255) / 256, 256, 0, st>>>(p.tw_half, h);
  return cudaGetLastError();
}

void fft_plan_free(FftPlan &p) {
  dfree(p.arena, p.tw);
  dfree(p.arena, p.tw_half);
  p.tw = p.tw_half = nullptr;
}

// r2c along x. Even n: the row is packed as n/2 complex values z_m =
// x_2m + i x_2m+1, transformed, and split with
// X_k = (Z_k + conj Z_{L-k})/2 - i/2 W^k (Z_k - conj Z_{L-k}), W = e^{-2 pi i/n}.
// Odd n: a full complex transform of length n.
__global__ void k_fft_x_r2c(const float *__restrict__ rho, float2 *__restrict__ spec, FftArgs a,
                            const float2 *__restrict__ tw_L, const float2 *__restrict__ tw_n,
                            int64_t nrows) {
  extern __shared__ float2 sm[];
  int L = a.L, P = a.P, n = a.n, hx = a.hx, ld = fslots(L);
  float2 *twl = sm;
  float2 *A = sm + L;
  float2 *B = A + P * ld;
  int tid = threadIdx.x, nth = blockDim.x;
  for (int k = tid; k < L; k += nth) twl[k] = tw_L[k];
  int64_t row0 = (int64_t)blockIdx.x * P;
  bool packed = (L * 2 == n);
  const Div dL = make_div(L), dH = make_div(hx);
  for (int e0 = tid; e0 < P * L; e0 += kLoadBatch * nth) {
    float2 v[kLoadBatch];
#pragma unroll
    for (int u = 0; u < kLoadBatch; u++) {
      int e = e0 + u * nth;
      int p = dL.q(e), m = e - p * L;
      int64_t row = row0 + p;
      v[u] = make_float2(0.f, 0.f);
      if (e < P * L && row < nrows) {
        const float *r = rho + row * n;
        if (packed)
          v[u] = *reinterpret_cast<const float2 *>(r + 2 * m);
        else
          v[u] = make_float2(r[m], 0.f);
      }
    }
#pragma unroll
    for (int u = 0; u < kLoadBatch; u++) {
      int e = e0 + u * nth;
      if (e < P * L) {
        int p = dL.q(e);
        A[p * ld + fslot(e - p * L)] = v[u];
      }
    }
  }
  __syncthreads();
  float2 *res = fft_pencils(A, B, twl, L, ld, P, -1.f, a.radix, a.nf);
  for (int e = tid; e < P * hx; e += nth) {
    int p = dH.q(e), k = e - p * hx;
    int64_t row = row0 + p;
    if (row >= nrows) continue;
    float2 X;
    if (packed) {
      const float2 *Z = res + p * ld;
      float2 zk = Z[fslot(k == L ? 0 : k)], zc = cconj(Z[fslot(k == 0 ? 0 : L - k)]);  // k <= L
      float2 ev = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
      float2 od = make_float2(0.5f * (zk.x - zc.x), 0.5f * (zk.y - zc.y));  // times -i below
      float2 w = tw_n[k];  // k <= L < n
      float2 wo = cmul(w, make_float2(od.y, -od.x));
      X = cadd(ev, wo);
    } else {
      X = res[p * ld + fslot(k)];
    }
    spec[row * hx + k] = X;
  }
}

// Complex transform along y (stride hx) or z (stride n*hx) for a block of TX
// consecutive kx columns. For the z pass with green != 0 the block applies
// the Green's function between the forward and the inverse transform.
struct GreenArgs {
  int law;
  float sfact;   // reference law: -(pi efold / n)^2
  float irngc;   // 1 / n^3
  float rs2k;    // gaussian law: (2 pi rs / n)^2
  int n;
  const float *gt;  // tabulated influence function [ky][kx][kz] (interlaced grids), or null
  double *pk;       // power-spectrum bins [2][n+1] (sum of weights*|rho_k|^2, sum of weights), or null
};

// The reference's CorrMeasure (Cosmos/Correlation.c:13-79) on the forward
// spectrum of the first grid: for kx < n/2, |rho_k|^2 / n^6 divided by the
// squared TSC window, shared linearly between the bins floor(|m|) and its
// neighbour towards |m|. Bins are summed per block in shared memory (sbin,
// 2(n+1) floats) and added to the device totals in double.
TPM_D void pk_accumulate(float *sbin, int n, int kx, int wy, int wz, float2 v) {
  if (2 * kx >= n) return;
  float wave = sqrtf((float)(kx * kx + wy * wy + wz * wz));
  float conv = 1.f;
  int ks[3] = {kx, wy, wz};
  for (int d = 0; d < 3; d++) {
    if (ks[d] != 0) {
      float a = (float)ks[d] / (float)n;
      float sc = sinpif(a) / (3.14159265358979323846f * a);
      conv *= sc * sc * sc;
    }
  }
  float inv_n3 = 1.f / ((float)n * (float)n * (float)n);
  float re = v.x * inv_n3, im = v.y * inv_n3;
  float d = (re * re + im * im) / (conv * conv);
  int k1 = (int)wave;
  float w = wave - (float)k1;
  int k2 = k1 + (w > 0.f ? 1 : -1);
  if (k1 <= n) {
    atomicAdd(&sbin[k1], (1.f - w) * d);
    atomicAdd(&sbin[n + 1 + k1], 1.f - w);
  }
  if (k2 >= 0 && k2 <= n && w > 0.f) {
    atomicAdd(&sbin[k2], w * d);
    atomicAdd(&sbin[n + 1 + k2], w);
  }
}

TPM_D float green(const GreenArgs &g, int kx, int ky, int kz) {
  float wy = (float)ky, wz = (float)kz;
  if (wy > g.n / 2.f) wy -= (float)g.n;
  if (wz > g.n / 2.f) wz -= (float)g.n;
  float wave = (float)(kx * kx) + wy * wy + wz * wz;
  if (wave == 0.f) return 0.f;
  const float fact = -0.31830988618379067154f;  // -1/pi
  if (g.law == 0) return fact / wave * expf(wave * g.sfact) * g.irngc;
  // Gaussian split: filter exp(-k^2 rs^2), divided by the squared TSC window
  // of deposit and interpolation (sinc^3 per axis each).
  float s = 1.f;
  int ks[3] = {kx, (int)wy, (int)wz};
  for (int d = 0; d < 3; d++) {
    if (ks[d] != 0) {
      float arg = 3.14159265358979323846f * (float)ks[d] / (float)g.n;
      float sc = sinf(arg) / arg;
      float w = sc * sc * sc;
      s *= w * w;
    }
  }
  return fact / wave * expf(-wave * g.rs2k) * g.irngc / s;
}

// nspec == 2: the same columns of a second spectrum (the interlaced grid) go
// through the transform as TX more pencils; with the Green's function the two
// are combined, rho = (rho1 + e^{i k.s} rho2) / 2 with s = (1/2, 1/2, 1/2)
// cells, which cancels the odd alias images of the TSC assignment, and the
// potential goes back to both grids, phi1 = G rho and phi2 = e^{-i k.s} G rho.
// Nyquist planes of an even mesh, where the shift phase is ambiguous, are
// zeroed.
__global__ void k_fft_cols(float2 *__restrict__ spec, float2 *__restrict__ spec2, FftArgs a,
                           const float2 *__restrict__ tw_n, int axis, float dir, int with_green, GreenArgs ga,
                           int TX, int nspec) {
  extern __shared__ float2 sm[];
  // pencils one element apart beyond their length: the transposing loads
  // and stores (consecutive threads on consecutive pencils) hit distinct banks
  int n = a.n, hx = a.hx, L = n, P = TX * nspec, Lp = col_stride(n, P);
  float2 *twl = sm;
  float2 *A = sm + L;
  float2 *B = A + P * Lp;
  int tid = threadIdx.x, nth = blockDim.x;
  for (int k = tid; k < L; k += nth) twl[k] = tw_n[k];
  int ntx = (hx + TX - 1) / TX;
  int kx0 = (blockIdx.x % ntx) * TX;
  int outer = blockIdx.x / ntx;  // z for the y pass, y for the z pass
  int64_t stride = axis == 1 ? (int64_t)hx : (int64_t)n * hx;
  int64_t base = axis == 1 ? (int64_t)outer * n * hx : (int64_t)outer * hx;
  int tw_ = min(TX, hx - kx0);
  const Div dP = make_div(P), dL = make_div(L);
  for (int e0 = tid; e0 < P * L; e0 += kLoadBatch * nth) {
    float2 v[kLoadBatch];
#pragma unroll
    for (int u = 0; u < kLoadBatch; u++) {
      int e = e0 + u * nth;
      int m = dP.q(e), q = e - m * P;  // consecutive threads -> consecutive kx
      int qs = q < TX ? q : q - TX;
      const float2 *src = q < TX ? spec : spec2;
      v[u] = make_float2(0.f, 0.f);
      if (e < P * L && qs < tw_) v[u] = src[base + m * stride + kx0 + qs];
    }
#pragma unroll
    for (int u = 0; u < kLoadBatch; u++) {
      int e = e0 + u * nth;
      int m = dP.q(e);
      if (e < P * L) A[(e - m * P) * Lp + fslot(m)] = v[u];
    }
  }
  __syncthreads();
  float2 *res = fft_pencils(A, B, twl, L, Lp, P, dir, a.radix, a.nf);
  if (with_green && ga.pk) {
    float *sbin = reinterpret_cast<float *>(B + P * Lp);
    for (int e = tid; e < 2 * (n + 1); e += nth) sbin[e] = 0.f;
    __syncthreads();
    int wy = outer > n / 2 ? outer - n : outer;
    for (int e = tid; e < TX * L; e += nth) {
      int q = dL.q(e), m = e - q * L;
      if (kx0 + q < hx) pk_accumulate(sbin, n, kx0 + q, wy, m > n / 2 ? m - n : m, res[q * Lp + fslot(m)]);
    }
    __syncthreads();
    for (int e = tid; e < 2 * (n + 1); e += nth)
      if (sbin[e] != 0.f) atomicAdd(&ga.pk[e], (double)sbin[e]);
  }
  if (with_green) {
    if (nspec == 1) {
      for (int e = tid; e < P * L; e += nth) {
        int q = dL.q(e), m = e - q * L;
        float gk = green(ga, kx0 + q, outer, m);
        float2 v = res[q * Lp + fslot(m)];
        res[q * Lp + fslot(m)] = make_float2(v.x * gk, v.y * gk);
      }
    } else {
      int wy = outer > n / 2 ? outer - n : outer;
      for (int e0 = tid; e0 < TX * L; e0 += kLoadBatch * nth) {
        float gks[kLoadBatch];
        if (ga.gt) {
#pragma unroll
          for (int u = 0; u < kLoadBatch; u++) {
            int e = e0 + u * nth;
            int q = dL.q(e), m = e - q * L;
            gks[u] = e < TX * L && kx0 + q < hx ? ga.gt[((int64_t)outer * hx + kx0 + q) * n + m] : 0.f;
          }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; u++) {
        int e = e0 + u * nth;
        if (e >= TX * L) break;
        int q = dL.q(e), m = e - q * L;
        int kx = kx0 + q, wz = m > n / 2 ? m - n : m;
        float gk = ga.gt ? gks[u] : green(ga, kx, outer, m);
        if ((n & 1) == 0 && (2 * kx == n || 2 * wy == n || 2 * wz == n || -2 * wy == n || -2 * wz == n)) gk = 0.f;
        float s, c;
        sincospif((float)(kx + wy + wz) / (float)n, &s, &c);
        int i1 = q * Lp + fslot(m), i2 = (q + TX) * Lp + fslot(m);
        float2 r1 = res[i1], r2 = res[i2];
        // (rho1 + e^{i theta} rho2) / 2, then times G
        float2 rho = make_float2(0.5f * (r1.x + c * r2.x - s * r2.y), 0.5f * (r1.y + c * r2.y + s * r2.x));
        float2 ph = make_float2(rho.x * gk, rho.y * gk);
        res[i1] = ph;
        res[i2] = make_float2(c * ph.x + s * ph.y, c * ph.y - s * ph.x);  // e^{-i theta} phi
        }
      }
    }
    __syncthreads();
    float2 *other = res == A ? B : A;
    res = fft_pencils(res, other, twl, L, Lp, P, 1.f, a.radix, a.nf);
  }
  for (int e = tid; e < P * L; e += nth) {
    int m = dP.q(e), q = e - m * P;
    int qs = q < TX ? q : q - TX;
    float2 *dst = q < TX ? spec : spec2;
    if (qs < tw_) dst[base + m * stride + kx0 + qs] = res[q * Lp + fslot(m)];
  }
}

// c2r along x, written into the ghosted potential phi_pad with kGhost ghost
// layers on every side (x, y and z ghosts are periodic copies), the layout
// the fda4 tiles read (Cosmos/pmmain.c:365-382 builds the same ghosts).
__global__ void k_fft_x_c2r(const float2 *__restrict__ spec, float *__restrict__ phi, FftArgs a,
                            const float2 *__restrict__ tw_L, const float2 *__restrict__ tw_n,
                            int64_t nrows, int px, int py) {
  extern __shared__ float2 sm[];
  int L = a.L, P = a.P, n = a.n, hx = a.hx, ld = fslots(L);
  float2 *twl = sm;
  float2 *A = sm + L;
  float2 *B = A + P * ld;
  int tid = threadIdx.x, nth = blockDim.x;
  for (int k = tid; k < L; k += nth) twl[k] = tw_L[k];
  int64_t row0 = (int64_t)blockIdx.x * P;
  bool packed = (L * 2 == n);
  constexpr int kB = kLoadBatch / 2;  // two loads per element
  const Div dL = make_div(L);
  for (int e0 = tid; e0 < P * L; e0 += kB * nth) {
    float2 xa[kB], xb[kB];
#pragma unroll
    for (int u = 0; u < kB; u++) {
      int e = e0 + u * nth;
      int p = dL.q(e), k = e - p * L;
      int64_t row = row0 + p;
      xa[u] = xb[u] = make_float2(0.f, 0.f);
      if (e < P * L && row < nrows) {
        const float2 *X = spec + row * hx;
        if (packed) {
          xa[u] = X[k];
          xb[u] = X[L - k];
        } else {
          xa[u] = X[k < hx ? k : n - k];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kB; u++) {
      int e = e0 + u * nth;
      if (e >= P * L) break;
      int pk = dL.q(e), k = e - pk * L;
      float2 Zk;
      if (packed) {
        // Z_k = (X_k + conj X_{L-k}) + i conj(W^k) (X_k - conj X_{L-k})
        float2 xk = xa[u], xc = cconj(xb[u]);
        if (k == 0) {
          xk.y = 0.f;
          xc.y = 0.f;
        }
        float2 e2 = cadd(xk, xc), o2 = csub(xk, xc);
        float2 w = cconj(tw_n[k]);
        float2 t = cmul(w, o2);
        Zk = cadd(e2, make_float2(-t.y, t.x));
      } else {
        // full Hermitian row for odd n
        Zk = k < hx ? xa[u] : cconj(xa[u]);
        if (k == 0) Zk.y = 0.f;
      }
      A[pk * ld + fslot(k)] = Zk;
    }
  }
  __syncthreads();
  float2 *res = fft_pencils(A, B, twl, L, ld, P, 1.f, a.radix, a.nf);
  // threads run over (pencil, x) pairs of the block's rows, x in
  // [-kGhost, n + kGhost) (n >= 16 > kGhost, so one wrap maps x into [0, n))
  const int W = n + 2 * kGhost;
  const float inv_w = 1.f / (float)W;
  const int nrow = (int)min((int64_t)P, nrows - row0);
  const int y0 = (int)(row0 % n), z0 = (int)(row0 / n);
  for (int e = tid; e < nrow * W; e += nth) {
    // p = e / W from the float reciprocal, corrected by one step
    int p = (int)((float)e * inv_w);
    int r = e - p * W;
    if (r < 0) {
      p--;
      r += W;
    } else if (r >= W) {
      p++;
      r -= W;
    }
    int y = y0 + p, z = z0;
    while (y >= n) {
      y -= n;
      z++;
    }
    // rows to write: (y, z) and its ghost copies
    int ys[2] = {y, y < kGhost ? y + n : (y >= n - kGhost ? y - n : 0x7fffffff)};
    int zs[2] = {z, z < kGhost ? z + n : (z >= n - kGhost ? z - n : 0x7fffffff)};
    {
      int x = r - kGhost;
      int xs = x < 0 ? x + n : (x >= n ? x - n : x);
      float v;
      if (packed) {
        float2 c = res[p * ld + fslot(xs >> 1)];
        v = (xs & 1) ? c.y : c.x;
      } else {
        v = res[p * ld + fslot(xs)].x;
      }
      for (int iz = 0; iz < 2; iz++) {
        if (zs[iz] == 0x7fffffff) continue;
        for (int iy = 0; iy < 2; iy++) {
          if (ys[iy] == 0x7fffffff) continue;
          int64_t off = (int64_t)(x + kGhost) + (int64_t)px * ((ys[iy] + kGhost) + (int64_t)py * (zs[iz] + kGhost));
          phi[off] = v;
        }
      }
    }
  }
}

static int pencils_for(int L, int want = 0) {
  if (want > 0) {
    // a tuned count, kept within the 160 KB of shared memory
    int cap = (int)(((160 * 1024) / (int)sizeof(float2) - L) / (2 * fslots(L)));
    return std::max(1, std::min(want, cap));
  }
  int P = 4096 / L;
  if (P < 1) P = 1;
  if (P > 64) P = 64;
  return P;
}

// Columns per block of the y and z passes: 8 (16 below n = 256) consecutive
// kx, fewer where the block's shared memory (twiddles + two buffers of
// nspec * TX pencils) would exceed 160 KB.
static int cols_per_block(int n, int hx, int nspec, int want = 0) {
  int TX = want > 0 ? want : (n >= 256 ? 8 : 16);
  // room for the power-spectrum bins (2(n+1) floats) as well
  int tmax = (int)(((160 * 1024 - 8 * (n + 1)) / (int)sizeof(float2) - n) / (2 * nspec * (fslots(n) + 15)));
  if (TX > tmax) TX = tmax;
  if (TX > hx) TX = hx;
  if (TX < 1) TX = 1;
  return TX;
}

// The optimal influence function of the interlaced TSC pair with the 8-point
// gradient (Hockney & Eastwood, "Computer Simulation Using Particles", ch. 8;
// interlaced form after Neelov & Holm 2010): the Green's function that
// minimises the mean-square force error against the Gaussian-filtered
// reference force R(k) = -i k (-4 pi / k^2) exp(-k^2 rs^2), given the
// assignment window U and the difference operator D,
//   G(k) = sum_m U^2(k_m) R(k_m).D(k) / (|D(k)|^2 (sum_m U^2(k_m))^2),
// k_m = k + 2 pi m, over the alias images m in [-2, 2]^3 that survive
// interlacing (even m_x + m_y + m_z). In the reference's units (mode numbers,
// -1/(pi m^2), 1/n^3). Computed once per mesh and split scale, in FP64.
__global__ void k_green_opt(float *__restrict__ gt, int n, int hx, double rs, double irngc) {
  const double PI = 3.14159265358979323846;
  const double c[4] = {4.0 / 5.0, -1.0 / 5.0, 4.0 / 105.0, -1.0 / 280.0};
  int64_t total = (int64_t)n * hx * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int kz = (int)(i % n);
    int kx = (int)((i / n) % hx);
    int ky = (int)(i / ((int64_t)n * hx));
    int my = ky > n / 2 ? ky - n : ky, mz = kz > n / 2 ? kz - n : kz, mx = kx;
    float out = 0.f;
    bool nyq = (n % 2 == 0) && (2 * mx == n || 2 * my == n || 2 * mz == n || -2 * my == n || -2 * mz == n);
    if (!nyq && (mx | my | mz) != 0) {
      double k[3] = {2 * PI * mx / n, 2 * PI * my / n, 2 * PI * mz / n};
      double D[3];
      for (int a = 0; a < 3; a++) {
        D[a] = 0;
        for (int j = 0; j < 4; j++) D[a] += 2 * c[j] * sin((j + 1) * k[a]);
      }
      double D2 = D[0] * D[0] + D[1] * D[1] + D[2] * D[2];
      double num = 0, den = 0;
      for (int ax = -2; ax <= 2; ax++)
        for (int ay = -2; ay <= 2; ay++)
          for (int az = -2; az <= 2; az++) {
            if (((ax + ay + az) & 1) != 0) continue;
            double q[3] = {k[0] + 2 * PI * ax, k[1] + 2 * PI * ay, k[2] + 2 * PI * az};
            double U2 = 1;
            for (int a = 0; a < 3; a++) {
              double h = 0.5 * q[a];
              double s = h == 0 ? 1.0 : sin(h) / h;
              double s3 = s * s * s;
              U2 *= s3 * s3;
            }
            double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
            double m2 = q2 * (n / (2 * PI)) * (n / (2 * PI));
            double Rs = -1.0 / PI / m2 * exp(-q2 * rs * rs);
            num += U2 * Rs * (D[0] * q[0] + D[1] * q[1] + D[2] * q[2]);
            den += U2;
          }
      if (D2 > 0 && den > 0) out = (float)(num / (D2 * den * den) * irngc);
    }
    gt[i] = out;
  }
}

void launch_green_opt(float *gt, int n, double rs, cudaStream_t st) {
  int hx = n / 2 + 1;
  int64_t total = (int64_t)n * hx * n;
  int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  k_green_opt<<<blocks, 256, 0, st>>>(gt, n, hx, rs, 1.0 / ((double)n * n * n));
}

void launch_poisson(const MeshGeom &g, const FftPlan &p, const float *rho, float2 *spec,
                    float *phi_pad, int law, float efold, float rs_split, cudaStream_t st,
                    int64_t *launches, const float *rho2, float2 *spec2, float *phi2_pad, const float *gt,
                    int want_px, int want_tx, double *pk) {
  int n = g.n;
  int64_t nrows = (int64_t)n * n;
  bool packed = (n % 2) == 0;
  int Lx = packed ? n / 2 : n;
  int Px = pencils_for(Lx, want_px);
  FftArgs ax = fft_args(n, Lx, Px, kXRadixMax);
  const float2 *twL = packed ? p.tw_half : p.tw;
  size_t smx = sizeof(float2) * (Lx + 2 * Px * fslots(Lx));
  int thx = 256;
  int nspec = rho2 ? 2 : 1;
  k_fft_x_r2c<<<(unsigned)((nrows + Px - 1) / Px), thx, smx, st>>>(rho, spec, ax, twL, p.tw, nrows);
  if (rho2) k_fft_x_r2c<<<(unsigned)((nrows + Px - 1) / Px), thx, smx, st>>>(rho2, spec2, ax, twL, p.tw, nrows);
  // columns
  int TX = cols_per_block(n, g.hx, nspec, want_tx);
  FftArgs ac = fft_args(n, n, TX * nspec, kColRadixMax);
  size_t smc = sizeof(float2) * (n + 2 * TX * nspec * col_stride(n, TX * nspec)) +
               (pk ? sizeof(float) * 2 * (n + 1) : 0);
  int ntx = (g.hx + TX - 1) / TX;
  GreenArgs ga;
  ga.law = law;
  ga.n = n;
  ga.sfact = (float)(-pow(M_PI * (double)efold / (double)n, 2));
  ga.irngc = (float)(1.0 / ((double)n * n * n));
  ga.rs2k = (float)pow(2.0 * M_PI * (double)rs_split / (double)n, 2);
  ga.gt = rho2 ? gt : nullptr;
  ga.pk = pk;
  k_fft_cols<<<(unsigned)(n * ntx), 256, smc, st>>>(spec, spec2, ac, p.tw, 1, -1.f, 0, ga, TX, nspec);
  k_fft_cols<<<(unsigned)(n * ntx), 256, smc, st>>>(spec, spec2, ac, p.tw, 2, -1.f, 1, ga, TX, nspec);
  k_fft_cols<<<(unsigned)(n * ntx), 256, smc, st>>>(spec, spec2, ac, p.tw, 1, 1.f, 0, ga, TX, nspec);
  k_fft_x_c2r<<<(unsigned)((nrows + Px - 1) / Px), thx, smx, st>>>(spec, phi_pad, ax, twL, p.tw, nrows,
                                                                     g.px, g.py);
  if (rho2)
    k_fft_x_c2r<<<(unsigned)((nrows + Px - 1) / Px), thx, smx, st>>>(spec2, phi2_pad, ax, twL, p.tw, nrows,
                                                                       g.px, g.py);
  if (launches) *launches += rho2 ? 7 : 5;
}

// Plain transforms of an n^3 mesh with the same kernels (no Green's
// function, unnormalised): forward = x r2c, y and z passes with e^{-i};
// inverse = z and y passes with e^{+i}, x c2r into the ghosted layout.
void fft_forward(const MeshGeom &g, const FftPlan &p, const float *real, float2 *spec, cudaStream_t st) {
  int n = g.n;
  int64_t nrows = (int64_t)n * n;
  bool packed = (n % 2) == 0;
  int Lx = packed ? n / 2 : n;
  int Px = pencils_for(Lx);
  FftArgs ax = fft_args(n, Lx, Px, kXRadixMax);
  size_t smx = sizeof(float2) * (Lx + 2 * Px * fslots(Lx));
  k_fft_x_r2c<<<(unsigned)((nrows + Px - 1) / Px), 256, smx, st>>>(real, spec, ax, packed ? p.tw_half : p.tw,
                                                                   p.tw, nrows);
  int TX = cols_per_block(n, g.hx, 1);
  FftArgs ac = fft_args(n, n, TX, kColRadixMax);
  size_t smc = sizeof(float2) * (n + 2 * TX * col_stride(n, TX));
  int ntx = (g.hx + TX - 1) / TX;
  GreenArgs ga;
  memset(&ga, 0, sizeof(ga));
  k_fft_cols<<<(unsigned)(n * ntx), 256, smc, st>>>(spec, nullptr, ac, p.tw, 1, -1.f, 0, ga, TX, 1);
  k_fft_cols<<<(unsigned)(n * ntx), 256, smc, st>>>(spec, nullptr, ac, p.tw, 2, -1.f, 0, ga, TX, 1);
}

void fft_inverse(const MeshGeom &g, const FftPlan &p, float2 *spec, float *phi_pad, cudaStream_t st) {
  int n = g.n;
  int64_t nrows = (int64_t)n * n;
  bool packed = (n % 2) == 0;
  int Lx = packed ? n / 2 : n;
  int Px = pencils_for(Lx);
  FftArgs ax = fft_args(n, Lx, Px, kXRadixMax);
  size_t smx = sizeof(float2) * (Lx + 2 * Px * fslots(Lx));
  int TX = cols_per_block(n, g.hx, 1);
  FftArgs ac = fft_args(n, n, TX, kColRadixMax);
  size_t smc = sizeof(float2) * (n + 2 * TX * col_stride(n, TX));
  int ntx = (g.hx + TX - 1) / TX;
  GreenArgs ga;
  memset(&ga, 0, sizeof(ga));
  k_fft_cols<<<(unsigned)(n * ntx), 256, smc, st>>>(spec, nullptr, ac, p.tw, 2, 1.f, 0, ga, TX, 1);
  k_fft_cols<<<(unsigned)(n * ntx), 256, smc, st>>>(spec, nullptr, ac, p.tw, 1, 1.f, 0, ga, TX, 1);
  k_fft_x_c2r<<<(unsigned)((nrows + Px - 1) / Px), 256, smx, st>>>(spec, phi_pad, ax, packed ? p.tw_half : p.tw,
                                                                   p.tw, nrows, g.px, g.py);
}

// ------------------------------------------------------------------ fda4
// Per 8^3 tile: one TMA load of the potential around the tile, the gradient
// -dphi/dx at the (T+3)^3 TSC nodes in shared memory, then each particle sums
// its 27 nodes with the TSC weights in the reference's order.
//   radius 2: the reference's 4-point stencil, 2/3 and -1/12 (fda4.c:45-46)
//   radius 4: the 8-point stencil 4/5, -1/5, 4/105, -1/280 (the Gaussian law)
constexpr int kNodes = kTile + 3;  // gradient nodes per axis
// the gradient arrays' strides (1, 12, 144): the nodes of 32 Morton-
// consecutive particles fall on distinct shared-memory banks
constexpr int kGradSy = 12;
constexpr int kGradSz = kGradSy * 12;
constexpr int kGradSize = kGradSz * kNodes;
constexpr int kFdaThreads = 256;

template <int R>
struct FdaBox {
  static constexpr int H = R + 1;                   // node halo + stencil
  static constexpr int X0 = ((H + 3) / 4) * 4;      // x starts at t - X0 (16-byte aligned)
  static constexpr int BX = ((X0 + kTile + H + 3) / 4) * 4;
  static constexpr int BY = kTile + 2 * H + 1;
};

TPM_D uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Bounded wait on an mbarrier phase; returns false if it did not complete.
TPM_D bool mbar_wait_bounded(uint64_t *bar, uint32_t phase, int64_t limit) {
  uint32_t addr = smem_u32(bar);
  for (int64_t it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One TMA load of the potential box around the tile (x from x0 - X0, 16-byte
// aligned; y, z from -H) into box, completing the barrier's next phase; thread
// 0 issues it. The box may hold the previous grid's potential: every thread
// has passed a __syncthreads since its last read of it.
template <int R>
TPM_D void fda_load_box(const CUtensorMap *tmap, float *box, uint64_t *bar, int x0, int y0, int z0) {
  using B = FdaBox<R>;
  if (threadIdx.x == 0) {
    uint32_t a = smem_u32(bar);
    uint32_t bytes = sizeof(float) * B::BY * B::BY * B::BX;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
    int cx = x0 - B::X0 + kGhost, cy = y0 - B::H + kGhost, cz = z0 - B::H + kGhost;
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(box)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(cx), "r"(cy), "r"(cz), "r"(a)
        : "memory");
  }
}

// -dphi/dx, -dphi/dy, -dphi/dz at the tile's nodes [t-1, t+T+1]^3, one line
// of kNodes nodes per thread and axis: the line's kNodes + 2R potential
// values are read once and the differences taken in registers.
template <int R>
TPM_D void fda_node_gradients(const float *boxf, float *gx, float *gy, float *gz) {
  using B = FdaBox<R>;
  const float(*box)[B::BY][B::BX] = reinterpret_cast<const float(*)[B::BY][B::BX]>(boxf);
  constexpr int kLine = kNodes + 2 * R;
  for (int r = threadIdx.x; r < 3 * kNodes * kNodes; r += kFdaThreads) {
    int axis = r / (kNodes * kNodes), rr = r % (kNodes * kNodes);
    int p = rr % kNodes, q = rr / kNodes;
    // node (a, b, c) sits at box (a-1+X0, b-1+H, c-1+H); v[i] is the line's
    // value at node coordinate i - R
    float v[kLine];
    if (axis == 0) {
#pragma unroll
      for (int i = 0; i < kLine; i++) v[i] = box[q - 1 + B::H][p - 1 + B::H][B::X0 - 1 - R + i];
    } else if (axis == 1) {
#pragma unroll
      for (int i = 0; i < kLine; i++) v[i] = box[q - 1 + B::H][B::H - 1 - R + i][p - 1 + B::X0];
    } else {
#pragma unroll
      for (int i = 0; i < kLine; i++) v[i] = box[B::H - 1 - R + i][q - 1 + B::H][p - 1 + B::X0];
    }
#pragma unroll
    for (int a = 0; a < kNodes; a++) {
      const float *w = v + a + R;
      float f;
      if (R == 2) {
        const float f1 = (4.f / 3.f) / 2.f, f2 = (-1.f / 3.f) / 4.f;
        f = f1 * (w[-1] - w[1]) + f2 * (w[-2] - w[2]);
      } else {
        const float c1 = 4.f / 5.f, c2 = -1.f / 5.f, c3 = 4.f / 105.f, c4 = -1.f / 280.f;
        f = c1 * (w[-1] - w[1]) + c2 * (w[-2] - w[2]) + c3 * (w[-3] - w[3]) + c4 * (w[-4] - w[4]);
      }
      if (axis == 0)
        gx[a + kGradSy * p + kGradSz * q] = f;
      else if (axis == 1)
        gy[p + kGradSy * a + kGradSz * q] = f;
      else
        gz[p + kGradSy * q + kGradSz * a] = f;
    }
  }
}

// The force at one particle: its 27 nodes' gradients with the TSC weights,
// summed in the reference's order wt_n, n = a + 3b + 9c (fda4.h:67-102,
// 276-292); node indices i1 = near, i2 = near + sign, i3 = near - sign
// (fda4.h:46-54), relative to the tile's first node t - 1.
TPM_D float3 fda_interp(const float *gx, const float *gy, const float *gz, uint32_t ux, uint32_t uy, uint32_t uz,
                        uint32_t n, uint32_t half, int x0, int y0, int z0) {
  Axis ax = axis_of(ux, n, half), ay = axis_of(uy, n, half), az = axis_of(uz, n, half);
  float wx1, wx2, wx3, wy1, wy2, wy3, wz1, wz2, wz3;
  int sx, sy, sz;
  tsc_w(ax.xmin, wx1, wx2, wx3, sx);
  tsc_w(ay.xmin, wy1, wy2, wy3, sy);
  tsc_w(az.xmin, wz1, wz2, wz3, sz);
  int i1 = ax.near - (x0 - 1), j1 = ay.near - (y0 - 1), k1 = az.near - (z0 - 1);
  int ii[3] = {i1, i1 + sx, i1 - sx}, jj[3] = {j1, j1 + sy, j1 - sy}, kk[3] = {k1, k1 + sz, k1 - sz};
  float wxs[3] = {wx1, wx2, wx3}, wys[3] = {wy1, wy2, wy3}, wzs[3] = {wz1, wz2, wz3};
  float fx = 0.f, fy = 0.f, fz = 0.f;
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      float wab[3] = {wxs[0] * wys[b], wxs[1] * wys[b], wxs[2] * wys[b]};
#pragma unroll
      for (int a = 0; a < 3; a++) {
        float wt = wab[a] * wzs[c];
        int node = ii[a] + kGradSy * jj[b] + kGradSz * kk[c];
        fx += wt * gx[node];
        fy += wt * gy[node];
        fz += wt * gz[node];
      }
    }
  return make_float3(fx, fy, fz);
}

// kPair: both grids of the interlaced pair in one pass (tmap: the first grid,
// particles as they are; tmap2: the second, particles moved by half a cell),
// the force being the mean of the two; the box buffer is loaded twice and
// both gradient sets kept. Else one grid (half as given), averaged with the
// force already in fpm when average != 0.
template <int R, bool kPair>
__global__ void __launch_bounds__(kFdaThreads) k_fda4(const __grid_constant__ CUtensorMap tmap,
                                                      const __grid_constant__ CUtensorMap tmap2,
                                                      const uint32_t *__restrict__ spos,
                                                      const uint32_t *__restrict__ tile_start, int n,
                                                      int cbits, float *__restrict__ fpm,
                                                      uint32_t *__restrict__ err, uint32_t half, int average) {
  using B = FdaBox<R>;
  // dynamic shared memory: the potential box (128-byte aligned for TMA), then
  // the gradient at the nodes, -dphi/dx, -dphi/dy and -dphi/dz as three float
  // arrays (twice with kPair): with the strides 1, 12, 144 the 27 node reads
  // of 32 Morton-consecutive particles are each one wavefront
  extern __shared__ __align__(128) float fda_smem[];
  float *box = fda_smem;
  float *gx = fda_smem + B::BY * B::BY * B::BX;
  float *gy = gx + kGradSize;
  float *gz = gy + kGradSize;
  float *gx2 = gz + kGradSize;
  float *gy2 = gx2 + kGradSize;
  float *gz2 = gy2 + kGradSize;
  __shared__ __align__(8) uint64_t bar;
  int tid = threadIdx.x;
  uint32_t t = blockIdx.x;
  uint32_t tx = 0, ty = 0, tz = 0;
  for (int b = 0; b < cbits - 3; b++) {
    tx |= ((t >> (3 * b)) & 1u) << b;
    ty |= ((t >> (3 * b + 1)) & 1u) << b;
    tz |= ((t >> (3 * b + 2)) & 1u) << b;
  }
  uint32_t p0 = tile_start[t], p1 = tile_start[t + 1];
  if (p0 == p1) return;
  int x0 = (int)tx * kTile, y0 = (int)ty * kTile, z0 = (int)tz * kTile;
  if (tid == 0) {
    uint32_t a = smem_u32(&bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  constexpr int kGrids = kPair ? 2 : 1;
#pragma unroll
  for (int gi = 0; gi < kGrids; gi++) {
    fda_load_box<R>(gi == 0 ? &tmap : &tmap2, box, &bar, x0, y0, z0);
    if (!mbar_wait_bounded(&bar, (uint32_t)gi, 1ll << 20)) {
      if (tid == 0) atomicOr(err, (uint32_t)kErrTmaTimeout);
      mbar_wait_bounded(&bar, (uint32_t)gi, 1ll << 20);  // let an in-flight copy land before exit
      return;
    }
    fda_node_gradients<R>(box, gi == 0 ? gx : gx2, gi == 0 ? gy : gy2, gi == 0 ? gz : gz2);
    __syncthreads();
  }
  uint32_t nu = (uint32_t)n;
  // each thread's next particle is loaded before this one's interpolation
  uint32_t ux = 0, uy = 0, uz = 0;
  if (p0 + tid < p1) {
    ux = spos[3 * (int64_t)(p0 + tid) + 0];
    uy = spos[3 * (int64_t)(p0 + tid) + 1];
    uz = spos[3 * (int64_t)(p0 + tid) + 2];
  }
  for (uint32_t k = p0 + tid; k < p1; k += kFdaThreads) {
    uint32_t kn = k + kFdaThreads, nx = 0, ny = 0, nz = 0;
    if (kn < p1) {
      nx = spos[3 * (int64_t)kn + 0];
      ny = spos[3 * (int64_t)kn + 1];
      nz = spos[3 * (int64_t)kn + 2];
    }
    float3 f = fda_interp(gx, gy, gz, ux, uy, uz, nu, kPair ? 0u : half, x0, y0, z0);
    if (kPair) {
      // the mean of the two grids' forces
      float3 f2 = fda_interp(gx2, gy2, gz2, ux, uy, uz, nu, 1u, x0, y0, z0);
      f = make_float3(0.5f * (f.x + f2.x), 0.5f * (f.y + f2.y), 0.5f * (f.z + f2.z));
    } else if (average) {
      // the second grid of the interlaced pair: mean of the two grids' forces
      f = make_float3(0.5f * (fpm[3 * (int64_t)k + 0] + f.x), 0.5f * (fpm[3 * (int64_t)k + 1] + f.y),
                      0.5f * (fpm[3 * (int64_t)k + 2] + f.z));
    }
    fpm[3 * (int64_t)k + 0] = f.x;
    fpm[3 * (int64_t)k + 1] = f.y;
    fpm[3 * (int64_t)k + 2] = f.z;
    ux = nx;
    uy = ny;
    uz = nz;
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int make_phi_tensor_map(const MeshGeom &g, float *phi_pad, int radius, CUtensorMap *out) {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void *p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return -1;
    fn = (EncodeTiledFn)p;
  }
  cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.pz};
  cuuint64_t strides[2] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.px * g.py * 4};
  cuuint32_t box[3];
  if (radius == 2) {
    box[0] = FdaBox<2>::BX;
    box[1] = box[2] = FdaBox<2>::BY;
  } else {
    box[0] = FdaBox<4>::BX;
    box[1] = box[2] = FdaBox<4>::BY;
  }
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, phi_pad, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -2;
}

void launch_fda4(const MeshGeom &g, const CUtensorMap *tmap, int radius, const uint32_t *spos,
                 const uint32_t *tile_start, float *fpm, uint32_t *err, cudaStream_t st, int half, int average) {
  uint32_t ntiles = 1u << (3 * (g.cbits - 3));
  const size_t nodes = sizeof(float) * 3 * kGradSize;
  if (radius == 2) {
    size_t smem = sizeof(float) * FdaBox<2>::BY * FdaBox<2>::BY * FdaBox<2>::BX + nodes;
    cudaFuncSetAttribute(k_fda4<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_fda4<2, false><<<ntiles, kFdaThreads, smem, st>>>(*tmap, *tmap, spos, tile_start, g.n, g.cbits, fpm, err,
                                                        (uint32_t)half, average);
  } else {
    size_t smem = sizeof(float) * FdaBox<4>::BY * FdaBox<4>::BY * FdaBox<4>::BX + nodes;
    cudaFuncSetAttribute(k_fda4<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_fda4<4, false><<<ntiles, kFdaThreads, smem, st>>>(*tmap, *tmap, spos, tile_start, g.n, g.cbits, fpm, err,
                                                        (uint32_t)half, average);
  }
}

void launch_fda4_pair(const MeshGeom &g, const CUtensorMap *tmap, const CUtensorMap *tmap2, const uint32_t *spos,
                      const uint32_t *tile_start, float *fpm, uint32_t *err, cudaStream_t st) {
  uint32_t ntiles = 1u << (3 * (g.cbits - 3));
  size_t smem = sizeof(float) * FdaBox<4>::BY * FdaBox<4>::BY * FdaBox<4>::BX + 2 * sizeof(float) * 3 * kGradSize;
  cudaFuncSetAttribute(k_fda4<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_fda4<4, true><<<ntiles, kFdaThreads, smem, st>>>(*tmap, *tmap2, spos, tile_start, g.n, g.cbits, fpm, err, 0u, 0);
}

}  // namespace tpm
