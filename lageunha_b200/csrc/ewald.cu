// FP64 periodic Ewald force on a subsample of target particles: the
// accuracy check every force evaluation can report against (the reference
// has no such oracle). Box [0,N)^3 cells, G = m = 1, Plummer softening eps
// on the pairs inside the real-space cutoff, result divided by N^2 to the
// reference's code units.
//   F_i = sum_j d [erfc(a r)/r^3 + 2a/sqrt(pi) exp(-a^2 r^2)/r^2]  (r < rcut)
//       + sum_j d [1/(r^2+eps^2)^{3/2} - 1/r^3]                   (r < rcut)
//       - (8 pi / V) sum_{k in half space} exp(-k^2/4a^2)/k^2 k Im[e^{ik.x_i} conj S(k)]
// with d = x_j - x_i (minimum image) and S(k) = sum_j e^{ik.x_j}.
#include <math.h>

#include <vector>

#include "engine_internal.cuh"

namespace tpm {

__global__ void k_ewald_sk(const uint32_t *__restrict__ pos, int64_t np, double cell_per_unit,
                           const int *__restrict__ mv, int nk, double L, double *__restrict__ S) {
  // block: 256 particles x all k in chunks; per k a block reduction + atomic
  __shared__ double red[2][8];
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double tpi_L = 6.283185307179586476925286766559 / L;
  for (int64_t base = (int64_t)blockIdx.x * 256; base < np; base += (int64_t)gridDim.x * 256) {
    int64_t i = base + tid;
    double x = 0, y = 0, z = 0;
    bool ok = i < np;
    if (ok) {
      x = (double)pos[3 * i + 0] * cell_per_unit;
      y = (double)pos[3 * i + 1] * cell_per_unit;
      z = (double)pos[3 * i + 2] * cell_per_unit;
    }
    for (int k = 0; k < nk; k++) {
      double ph = tpi_L * (mv[3 * k] * x + mv[3 * k + 1] * y + mv[3 * k + 2] * z);
      double s = 0, c = 0;
      if (ok) sincos(ph, &s, &c);
      for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, o);
        s += __shfl_down_sync(0xffffffffu, s, o);
      }
      if (lane == 0) {
        red[0][warp] = c;
        red[1][warp] = s;
      }
      __syncthreads();
      if (tid == 0) {
        double cs = 0, ss = 0;
        for (int w = 0; w < 8; w++) {
          cs += red[0][w];
          ss += red[1][w];
        }
        atomicAdd(&S[2 * k], cs);
        atomicAdd(&S[2 * k + 1], ss);
      }
      __syncthreads();
    }
  }
}

// one block per target: real-space sum over all particles + k-space sum
__global__ void k_ewald_target(const uint32_t *__restrict__ pos, int64_t np, double cell_per_unit,
                               const int64_t *__restrict__ tg_sorted_idx, int nt, const int *__restrict__ mv,
                               int nk, const double *__restrict__ S, double L, double alpha, double rc2,
                               double eps2, double *__restrict__ out) {
  int t = blockIdx.x;
  if (t >= nt) return;
  int64_t ti = tg_sorted_idx[t];
  double px = (double)pos[3 * ti + 0] * cell_per_unit;
  double py = (double)pos[3 * ti + 1] * cell_per_unit;
  double pz = (double)pos[3 * ti + 2] * cell_per_unit;
  double fx = 0, fy = 0, fz = 0;
  const double spi = 1.7724538509055160272981674833411;
  for (int64_t j = threadIdx.x; j < np; j += blockDim.x) {
    if (j == ti) continue;
    double d[3] = {(double)pos[3 * j + 0] * cell_per_unit - px, (double)pos[3 * j + 1] * cell_per_unit - py,
                   (double)pos[3 * j + 2] * cell_per_unit - pz};
    for (int c = 0; c < 3; c++) d[c] -= L * floor(d[c] / L + 0.5);
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (r2 >= rc2 || r2 == 0.0) continue;
    double r = sqrt(r2);
    double g = erfc(alpha * r) / (r2 * r) + 2.0 * alpha / spi * exp(-alpha * alpha * r2) / r2;
    g += 1.0 / pow(r2 + eps2, 1.5) - 1.0 / (r2 * r);
    fx += d[0] * g;
    fy += d[1] * g;
    fz += d[2] * g;
  }
  const double tpi_L = 6.283185307179586476925286766559 / L;
  const double V = L * L * L;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) {
    double kx = tpi_L * mv[3 * k], ky = tpi_L * mv[3 * k + 1], kz = tpi_L * mv[3 * k + 2];
    double k2 = kx * kx + ky * ky + kz * kz;
    double ph = kx * px + ky * py + kz * pz;
    double s, c;
    sincos(ph, &s, &c);
    double im = s * S[2 * k] - c * S[2 * k + 1];
    double w = 8.0 * M_PI / V * exp(-k2 / (4 * alpha * alpha)) / k2 * im;
    fx -= w * kx;
    fy -= w * ky;
    fz -= w * kz;
  }
  __shared__ double red[3][32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_down_sync(0xffffffffu, fx, o);
    fy += __shfl_down_sync(0xffffffffu, fy, o);
    fz += __shfl_down_sync(0xffffffffu, fz, o);
  }
  if (lane == 0) {
    red[0][warp] = fx;
    red[1][warp] = fy;
    red[2][warp] = fz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) {
      a += red[0][w];
      b += red[1][w];
      c += red[2][w];
    }
    double inv = 1.0 / (L * L);
    out[3 * t + 0] = a * inv;
    out[3 * t + 1] = b * inv;
    out[3 * t + 2] = c * inv;
  }
}

// pos: caller-order fixed-point positions on the device.
int ewald_force(const uint32_t *pos, int64_t np, int n, float eps, int64_t nt, const int64_t *targets_host,
                double *out_host, cudaStream_t st) {
  double L = n;
  double rcut = 0.49 * L, alpha = 3.6 / rcut;
  int M = (int)ceil(2 * alpha * 3.6 * L / (2 * M_PI));
  std::vector<int> mv;
  for (int mz = 0; mz <= M; mz++)
    for (int my = -M; my <= M; my++)
      for (int mx = -M; mx <= M; mx++) {
        if (mz == 0 && (my < 0 || (my == 0 && mx <= 0))) continue;
        if (mx * mx + my * my + mz * mz > M * M) continue;
        mv.push_back(mx);
        mv.push_back(my);
        mv.push_back(mz);
      }
  int nk = (int)(mv.size() / 3);
  int *d_mv = nullptr;
  double *d_S = nullptr, *d_out = nullptr;
  int64_t *d_t = nullptr;
  if (cudaMalloc(&d_mv, sizeof(int) * mv.size()) != cudaSuccess) return -1;
  cudaMalloc(&d_S, sizeof(double) * 2 * nk);
  cudaMalloc(&d_out, sizeof(double) * 3 * nt);
  cudaMalloc(&d_t, sizeof(int64_t) * nt);
  cudaMemcpyAsync(d_mv, mv.data(), sizeof(int) * mv.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_t, targets_host, sizeof(int64_t) * nt, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d_S, 0, sizeof(double) * 2 * nk, st);
  double cpu = (double)n / 4294967296.0;
  int blocks = (int)((np + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_ewald_sk<<<blocks, 256, 0, st>>>(pos, np, cpu, d_mv, nk, L, d_S);
  k_ewald_target<<<(unsigned)nt, 512, 0, st>>>(pos, np, cpu, d_t, (int)nt, d_mv, nk, d_S, L, alpha,
                                              rcut * rcut, (double)eps * eps, d_out);
  cudaMemcpyAsync(out_host, d_out, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(d_mv);
  cudaFree(d_S);
  cudaFree(d_out);
  cudaFree(d_t);
  return e == cudaSuccess ? 0 : -3;
}

}  // namespace tpm
