/*
 * Test infrastructure (oracle), not the product: a plain FP64 complex FFT.
 *
 * It stands in for FFTW3 (the reference links libfftw3, unpinned nixpkgs:
 * default.nix:10-11, src/reference/default.nix:9-10) at the call sites
 * src/reference/grid.c:348-355,467,499 and src/reference/main.c:276-278.
 * FFTW computes the unnormalised DFT  X[k] = sum_j x[j] exp(sign*2*pi*i*j*k/n);
 * this file restates that definition with an iterative radix-2
 * decimation-in-time algorithm (Cooley & Tukey 1965) for power-of-two n and a
 * direct O(n^2) sum otherwise.  Twiddles come from cos/sin of the exact angle.
 */
#ifndef RG_ORACLE_FFT_H
#define RG_ORACLE_FFT_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

/* In-place 1-D transform of n points spaced `stride` elements apart. */
void rgo_fft1d(double complex *x, int n, int stride, int sign);

/* Out-of-place capable 2-D transform of an ny x nx row-major array
 * (in == out allowed).  sign = -1 (forward) or +1 (backward), unnormalised. */
void rgo_fft2d(const double complex *in, double complex *out, int ny, int nx, int sign);

#ifdef __cplusplus
}
#endif
#endif
