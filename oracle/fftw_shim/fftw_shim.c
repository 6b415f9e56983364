/*
 * Test infrastructure (oracle), not the product: the FFTW-API shim declared in
 * fftw3.h, implemented on the FP64 FFT of rg_fft.c.
 */
#include "fftw3.h"
#include "../rg_fft.h"

#include <stdlib.h>

struct rgo_fftw_plan_s {
    int n0, n1, sign;
    fftw_complex *in, *out;
};

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags)
{
    (void)flags;
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->n0 = n0; p->n1 = n1; p->sign = sign; p->in = in; p->out = out;
    return p;
}

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out)
{
    rgo_fft2d(in, out, p->n0, p->n1, p->sign);
}

void fftw_execute(const fftw_plan p) { rgo_fft2d(p->in, p->out, p->n0, p->n1, p->sign); }

void fftw_destroy_plan(fftw_plan p) { free(p); }
