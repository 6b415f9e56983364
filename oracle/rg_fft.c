/*
 * Test infrastructure (oracle), not the product.  FP64 complex FFT used by the
 * CPU restatement and by the FFTW-API shim the reference grid.c is built
 * against.  Definition and method are stated in rg_fft.h.
 */
#include "rg_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* Direct sum for lengths that are not a power of two (small test sizes). */
static void dft_direct(double complex *x, int n, int stride, int sign)
{
    double complex *tmp = (double complex *)malloc(sizeof(double complex) * (size_t)n);
    for (int k = 0; k < n; k++) {
        double complex acc = 0;
        for (int j = 0; j < n; j++) {
            long long jk = ((long long)j * k) % n;
            double ang = sign * 2.0 * M_PI * (double)jk / (double)n;
            acc += x[(size_t)j * stride] * (cos(ang) + I * sin(ang));
        }
        tmp[k] = acc;
    }
    for (int k = 0; k < n; k++) x[(size_t)k * stride] = tmp[k];
    free(tmp);
}

void rgo_fft1d(double complex *x, int n, int stride, int sign)
{
    if (n <= 1) return;
    if (!is_pow2(n)) { dft_direct(x, n, stride, sign); return; }

    /* gather into a contiguous scratch buffer in bit-reversed order */
    double complex *a = (double complex *)malloc(sizeof(double complex) * (size_t)n);
    int bits = 0;
    while ((1 << bits) < n) bits++;
    for (int i = 0; i < n; i++) {
        unsigned r = 0, v = (unsigned)i;
        for (int b = 0; b < bits; b++) { r = (r << 1) | (v & 1u); v >>= 1; }
        a[r] = x[(size_t)i * stride];
    }
    /* twiddle table w[k] = exp(sign*2*pi*i*k/n), k < n/2: computed once per
     * thread, length and sign and kept (the same values every call, so the
     * results are unchanged; a plan's precomputed table, as FFTW keeps one) */
    static __thread double complex *tw_cache = NULL;
    static __thread int tw_n = 0, tw_sign = 0;
    if (tw_n != n || tw_sign != sign) {
        free(tw_cache);
        tw_cache = (double complex *)malloc(sizeof(double complex) * (size_t)(n / 2));
        for (int k = 0; k < n / 2; k++) {
            double ang = sign * 2.0 * M_PI * (double)k / (double)n;
            tw_cache[k] = cos(ang) + I * sin(ang);
        }
        tw_n = n;
        tw_sign = sign;
    }
    const double complex *w = tw_cache;
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (int s = 0; s < n; s += len) {
            for (int k = 0; k < half; k++) {
                double complex t = w[k * step] * a[s + k + half];
                double complex u = a[s + k];
                a[s + k] = u + t;
                a[s + k + half] = u - t;
            }
        }
    }
    for (int i = 0; i < n; i++) x[(size_t)i * stride] = a[i];
    free(a);
}

void rgo_fft2d(const double complex *in, double complex *out, int ny, int nx, int sign)
{
    size_t total = (size_t)ny * (size_t)nx;
    if (in != out) memmove(out, in, sizeof(double complex) * total);
    for (int y = 0; y < ny; y++) rgo_fft1d(out + (size_t)y * nx, nx, 1, sign);
    /* columns: copy out, transform contiguously, copy back (cache friendly) */
    double complex *col = (double complex *)malloc(sizeof(double complex) * (size_t)ny);
    for (int x = 0; x < nx; x++) {
        for (int y = 0; y < ny; y++) col[y] = out[(size_t)y * nx + x];
        rgo_fft1d(col, ny, 1, sign);
        for (int y = 0; y < ny; y++) out[(size_t)y * nx + x] = col[y];
    }
    free(col);
}
