/*
 * ORACLE — test infrastructure only.  Nothing in the product links this file:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * as the checker.
 *
 * A plain-C FP64 restatement of the reference CPU gridder
 * (KentJames/Radio-Gridders, src/reference/grid.c) on flat structure-of-arrays
 * visibilities (the layout of struct flat_vis_data, src/common/hdf5.cuh:31-37),
 * plus an FP64 direct-DFT image oracle written from the maths (the reference's
 * own DFTs are defective: src/dft/dft_cuda.cu:55-57, src/reference/dft.c:29-56).
 *
 * Parity is pinned by running the reference's own grid.c, compiled here from its
 * sources against an FFTW-API shim (oracle/Makefile -> oracle/_ref/), on the same
 * inputs: tests/test_oracle_pin.py requires bit-identical grids, and
 * tests/golden/ holds fixtures produced by that build.
 *
 * Conventions shared with the reference:
 *   - u, v, w are in wavelengths: uvw[m] * freq / c (grid.c:21-24).
 *   - complex grids are row-major N x N, v selects the row, u the column.
 *   - w-kernel table: data[((plane*ov + yf)*ov + xf)*size*size + y*size + x]
 *     (grid.c:53-56, hdf5.c:513-550), planes evenly spaced w_min + i*w_step.
 */
#ifndef RG_ORACLE_H
#define RG_ORACLE_H

#include <complex.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const double complex *data; /* [plane][ov][ov][size][size] */
    int plane_count;
    int size;                   /* support in cells (size_x == size_y) */
    int oversampling;
    double w_min, w_step;
} rgo_wkern;

/* grid.c:37-57 */
void rgo_frac_coord(int grid_size, int kernel_size, int oversample, double theta,
                    double u, double v, double d_u, double d_v,
                    int *grid_offset, int *sub_offset);

/* grid.c:187-202 (with w_project, grid.c:157-185).  Returns the flop count. */
uint64_t rgo_grid_wprojection(double complex *uvgrid, int grid_size, double theta,
                              int64_t nvis, const double *u, const double *v,
                              const double *w, const double complex *vis,
                              const rgo_wkern *wk);

/* grid.c:295-555 (serial build, i.e. without OMP_TOWERS).  If gridded_count is
 * non-NULL it receives, per visibility, how many times it was gridded (the
 * reference checks this is exactly once, grid.c:519-530).  If tower_sel is
 * non-NULL, only the towers t (row-major) with tower_sel[t] != 0 are gridded.
 * Returns flops. */
uint64_t rgo_grid_wtowers(double complex *uvgrid, int grid_size, double theta,
                          int64_t nvis, const double *u, const double *v,
                          const double *w, const double complex *vis,
                          const rgo_wkern *wk, int subgrid_size, int subgrid_margin,
                          double wincrement, int32_t *gridded_count,
                          const unsigned char *tower_sel);
/* Visibilities and active w-floors per tower under the same binning. */
void rgo_wtowers_census(int grid_size, double theta, int64_t nvis, const double *u, const double *v,
                        const double *w, int subgrid_size, int subgrid_margin, double wincrement,
                        int64_t *vis_per_tower, int32_t *floors_per_tower);

/* grid.c:83-99: nearest-cell gridding; 1 when a cell lies off the grid. */
int rgo_grid_simple(double complex *uvgrid, int grid_size, double theta, int64_t nvis, const double *u,
                    const double *v, const double complex *vis);

/* grid.c:59-81: uniform weighting, vis[i] /= count of visibilities in its cell. */
void rgo_weight(int grid_size, double theta, int64_t nvis, const double *u,
                const double *v, double complex *vis);

/* grid.c:639-662 and grid.c:665-680 */
void rgo_make_hermitian(double complex *uvgrid, int grid_size);
void rgo_fft_shift(double complex *uvgrid, int grid_size);

/* main.c:258-294: hermitian, shift, forward FFT (sign -1), shift; real part out.
 * Modifies uvgrid. */
void rgo_image_from_grid(double complex *uvgrid, int grid_size, double *image);

/* FP64 direct DFT in the imaging convention of the pipeline above:
 *   image[y][x] = factor * sum_k Re( V_k exp(-2 pi i (u_k l + v_k m + w_k (1 - n))) )
 *   l = theta (x - N/2) / N,  m = theta (y - N/2) / N,  n = sqrt(1 - l^2 - m^2)
 * factor = 2 reproduces the hermitian gridder pipeline, 1 the reference dft.out.
 * Summation is compensated (Neumaier) so the oracle's own error stays near
 * 1 ulp of the result.  Parallel over rows with OpenMP. */
void rgo_dft_image(double *image, int grid_size, double theta, int64_t nvis,
                   const double *u, const double *v, const double *w,
                   const double complex *vis, double factor);
/* The same DFT at the npix pixels (px[k], py[k]) only (column x, row y). */
void rgo_dft_pixels(double *out, int npix, const int *px, const int *py, int grid_size, double theta,
                    int64_t nvis, const double *u, const double *v, const double *w,
                    const double complex *vis, double factor);

/* W-stacking predict, src/wstack/predict.cpp:396-562: visibilities of unit
 * point sources at points[2k], points[2k+1] (l, m) from w-stacked planes of
 * the quantised, grid-corrected sky and a separable 3-D de-convolution with
 * the tables conv_uv / conv_w (data[ov_index * size + tap]) and the grid
 * correction tables corr_lm / corr_n.  Returns 0, or 1 (x0 gives no padded
 * grid), 2 (a source outside the grid or the correction tables), 3 (a
 * visibility's taps outside the planes). */
int rgo_wstack_planes(double theta, double lam, double dw, int support_w);
int rgo_wstack_predict(double theta, double lam, int npts, const double *points, int64_t nvis,
                       const double *u, const double *v, const double *w, double du, double dw, double x0,
                       const double *conv_uv, int uv_size, int uv_ov, const double *conv_w, int w_size,
                       int w_ov, const double *corr_lm, int lm_size, int lm_ov, const double *corr_n,
                       int n_size, int n_ov, double complex *vis_out);
/* predict_visibility_quantized_vec, src/wstack/predict.cpp:89-129. */
void rgo_predict_dft_quantized(double theta, double lam, int npts, const double *points, int64_t nvis,
                               const double *u, const double *v, const double *w, double complex *vis_out);

/* AW-projection, src/reference/grid.c:557-637 (convolve_aw_kernels +
 * grid_awprojection) on uniform hierarchical arrays; see rg_oracle.c. */
int rgo_grid_awprojection(double complex *uvgrid, int grid_size, double theta, int bl_min, int bl_max,
                          int nt, int nf, const int32_t *antenna1, const double *time, const double *freq,
                          const double *uvw, const double complex *vis, const rgo_wkern *wk, int ak_ant,
                          int ak_time, int ak_freq, double t_min, double t_step, double f_min, double f_step,
                          const double *akern_freq);

#ifdef __cplusplus
}
#endif
#endif
