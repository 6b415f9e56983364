/*
 * Test infrastructure (oracle), not the product.
 *
 * Minimal FFTW3-compatible API so that the reference's src/reference/grid.c and
 * src/reference/main.c compile unmodified without libfftw3 (absent here).  Only
 * the calls those files make are provided: fftw_plan_dft_2d, fftw_execute_dft,
 * fftw_destroy_plan and the FFTW_MEASURE / FFTW_ESTIMATE planner flags.
 * Semantics follow FFTW's documented definition: unnormalised complex DFT,
 * sign -1 forward, +1 backward; a plan may be executed on other arrays of the
 * same shape (the new-array execute interface).  Execution is reentrant, so the
 * reference's OMP_TOWERS build may call it from several threads.
 */
#ifndef RG_FFTW3_SHIM_H
#define RG_FFTW3_SHIM_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex fftw_complex;
typedef struct rgo_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif
#endif
