/*
 * Double-precision mixed-radix DFT used by the CPU oracle (test
 * infrastructure only; nothing in the engine links it).
 *
 * Conventions follow FFTW, which the reference calls for its PM solve
 * (Cosmos/pmmain.c:475,492; FFT/fft.c:130-146): forward transforms use
 * exp(-2*pi*i*j*k/n), backward use exp(+2*pi*i*j*k/n), and neither is
 * normalised.
 */
#ifndef ORACLE_DFT_H
#define ORACLE_DFT_H
#include <stddef.h>

/* In-place complex DFT of length n along a strided axis of interleaved
 * (re,im) doubles: element j lives at data[2*j*stride]. sign = -1 forward,
 * +1 backward. Any n >= 1 (radices 2,3,4,5 fast; other primes by direct sum). */
void odft_1d(double *data, size_t n, size_t stride, int sign);

/* 3D real-to-complex forward transform of an nz x ny x nx real array
 * (x fastest) into an nz x ny x (nx/2+1) complex array (interleaved). */
void odft_r2c_3d(size_t nz, size_t ny, size_t nx, const double *in, double *out);

/* 3D complex-to-real backward transform: nz x ny x (nx/2+1) complex in,
 * nz x ny x nx real out, unnormalised (FFTW c2r semantics; the input's
 * Hermitian redundancy is assumed). The input is not modified. */
void odft_c2r_3d(size_t nz, size_t ny, size_t nx, const double *in, double *out);

#endif
