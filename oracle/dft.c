/*
 * Double-precision mixed-radix DFT for the CPU oracle (test infrastructure).
 * A plain recursive decimation-in-time Cooley-Tukey over the smallest prime
 * factor, with twiddles taken from a per-length table of cos/sin evaluated in
 * double. It is written for clarity and accuracy, not speed; the 3D drivers
 * run independent 1D transforms under OpenMP. See dft.h for conventions.
 */
#include "dft.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static size_t smallest_factor(size_t n) {
  if (n % 2 == 0) return 2;
  for (size_t p = 3; p * p <= n; p += 2)
    if (n % p == 0) return p;
  return n;
}

/* out[k] = sum_j in[j*is] * exp(sign*2*pi*i*j*k/n); out is contiguous and
 * interleaved; tmp holds at least 2*n doubles; tw is the table of
 * exp(2*pi*i*j/ntw), j < ntw, with ntw a multiple of n. */
static void fft_rec(const double *in, size_t is, double *out, size_t n, int sign,
                    double *tmp, const double *tw, size_t ntw) {
  if (n == 1) {
    out[0] = in[0];
    out[1] = in[1];
    return;
  }
  size_t p = smallest_factor(n);
  size_t m = n / p;
  for (size_t r = 0; r < p; r++)
    fft_rec(in + 2 * r * is, is * p, out + 2 * r * m, m, sign, tmp, tw, ntw);
  /* Combine the p sub-transforms Y_r (stored at out[r*m .. r*m+m-1]):
   * X[k + q*m] = sum_r Y_r[k] * w^(r*(k+q*m)), w = exp(sign*2*pi*i/n).
   * For one k the inputs {r*m+k} and outputs {k+q*m} are the same slots, so
   * each k is combined through tmp and written back in place. */
  size_t step = ntw / n;
  for (size_t k = 0; k < m; k++) {
    for (size_t q = 0; q < p; q++) {
      double sr = 0.0, si = 0.0;
      size_t kk = k + q * m;
      for (size_t r = 0; r < p; r++) {
        double yr = out[2 * (r * m + k)], yi = out[2 * (r * m + k) + 1];
        size_t e = ((r * kk) % n) * step;
        double c = tw[2 * e], s = sign * tw[2 * e + 1];
        sr += yr * c - yi * s;
        si += yr * s + yi * c;
      }
      tmp[2 * q] = sr;
      tmp[2 * q + 1] = si;
    }
    for (size_t q = 0; q < p; q++) {
      out[2 * (k + q * m)] = tmp[2 * q];
      out[2 * (k + q * m) + 1] = tmp[2 * q + 1];
    }
  }
}

static double *make_twiddles(size_t n) {
  const double two_pi = 6.283185307179586476925286766559;
  double *tw = (double *)malloc(sizeof(double) * 2 * n);
  for (size_t j = 0; j < n; j++) {
    double ang = two_pi * (double)j / (double)n;
    tw[2 * j] = cos(ang);
    tw[2 * j + 1] = sin(ang);
  }
  return tw;
}

/* One strided 1D transform with a caller-provided table and scratch of 6*n
 * doubles. */
static void dft_1d_tw(double *data, size_t n, size_t stride, int sign, const double *tw,
                      double *scratch) {
  double *in = scratch, *out = scratch + 2 * n, *tmp = scratch + 4 * n;
  for (size_t j = 0; j < n; j++) {
    in[2 * j] = data[2 * j * stride];
    in[2 * j + 1] = data[2 * j * stride + 1];
  }
  fft_rec(in, 1, out, n, sign, tmp, tw, n);
  for (size_t j = 0; j < n; j++) {
    data[2 * j * stride] = out[2 * j];
    data[2 * j * stride + 1] = out[2 * j + 1];
  }
}

void odft_1d(double *data, size_t n, size_t stride, int sign) {
  double *tw = make_twiddles(n);
  double *scratch = (double *)malloc(sizeof(double) * 6 * n);
  dft_1d_tw(data, n, stride, sign, tw, scratch);
  free(scratch);
  free(tw);
}

void odft_r2c_3d(size_t nz, size_t ny, size_t nx, const double *in, double *out) {
  size_t hx = nx / 2 + 1;
  double *twx = make_twiddles(nx), *twy = make_twiddles(ny), *twz = make_twiddles(nz);
  size_t nmax = nx > ny ? nx : ny;
  nmax = nmax > nz ? nmax : nz;
#pragma omp parallel
  {
    double *scratch = (double *)malloc(sizeof(double) * 6 * nmax);
    double *row = (double *)malloc(sizeof(double) * 2 * nx);
#pragma omp for collapse(2)
    for (size_t z = 0; z < nz; z++)
      for (size_t y = 0; y < ny; y++) {
        const double *src = in + nx * (y + ny * z);
        for (size_t x = 0; x < nx; x++) {
          row[2 * x] = src[x];
          row[2 * x + 1] = 0.0;
        }
        dft_1d_tw(row, nx, 1, -1, twx, scratch);
        memcpy(out + 2 * hx * (y + ny * z), row, sizeof(double) * 2 * hx);
      }
#pragma omp for collapse(2)
    for (size_t z = 0; z < nz; z++)
      for (size_t x = 0; x < hx; x++)
        dft_1d_tw(out + 2 * (x + hx * ny * z), ny, hx, -1, twy, scratch);
#pragma omp for collapse(2)
    for (size_t y = 0; y < ny; y++)
      for (size_t x = 0; x < hx; x++)
        dft_1d_tw(out + 2 * (x + hx * y), nz, hx * ny, -1, twz, scratch);
    free(row);
    free(scratch);
  }
  free(twx);
  free(twy);
  free(twz);
}

void odft_c2r_3d(size_t nz, size_t ny, size_t nx, const double *in, double *out) {
  size_t hx = nx / 2 + 1;
  size_t nc = 2 * hx * ny * nz;
  double *work = (double *)malloc(sizeof(double) * nc);
  memcpy(work, in, sizeof(double) * nc);
  double *twx = make_twiddles(nx), *twy = make_twiddles(ny), *twz = make_twiddles(nz);
  size_t nmax = nx > ny ? nx : ny;
  nmax = nmax > nz ? nmax : nz;
#pragma omp parallel
  {
    double *scratch = (double *)malloc(sizeof(double) * 6 * nmax);
    double *row = (double *)malloc(sizeof(double) * 2 * nx);
#pragma omp for collapse(2)
    for (size_t y = 0; y < ny; y++)
      for (size_t x = 0; x < hx; x++)
        dft_1d_tw(work + 2 * (x + hx * y), nz, hx * ny, +1, twz, scratch);
#pragma omp for collapse(2)
    for (size_t z = 0; z < nz; z++)
      for (size_t x = 0; x < hx; x++)
        dft_1d_tw(work + 2 * (x + hx * ny * z), ny, hx, +1, twy, scratch);
#pragma omp for collapse(2)
    for (size_t z = 0; z < nz; z++)
      for (size_t y = 0; y < ny; y++) {
        const double *src = work + 2 * hx * (y + ny * z);
        /* rebuild the full Hermitian row; the imaginary parts of the DC and
         * Nyquist bins are ignored, as a c2r transform does */
        for (size_t x = 0; x < hx; x++) {
          row[2 * x] = src[2 * x];
          row[2 * x + 1] = src[2 * x + 1];
        }
        for (size_t x = hx; x < nx; x++) {
          row[2 * x] = src[2 * (nx - x)];
          row[2 * x + 1] = -src[2 * (nx - x) + 1];
        }
        row[1] = 0.0;
        if (nx % 2 == 0) row[2 * (nx / 2) + 1] = 0.0;
        dft_1d_tw(row, nx, 1, +1, twx, scratch);
        double *dst = out + nx * (y + ny * z);
        for (size_t x = 0; x < nx; x++) dst[x] = row[2 * x];
      }
    free(row);
    free(scratch);
  }
  free(twx);
  free(twy);
  free(twz);
  free(work);
}
