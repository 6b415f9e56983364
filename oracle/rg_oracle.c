/*
 * ORACLE — test infrastructure only (see rg_oracle.h).  FP64 restatement of
 * the reference CPU gridder, src/reference/grid.c, on flat visibility arrays.
 * Each function names the reference lines it follows.  Arithmetic is written
 * in the same expression order as the reference so that, compiled with IEEE
 * semantics (no -ffast-math), results are bit-identical to grid.c itself.
 */
#include "rg_oracle.h"
#include "rg_fft.h"

#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* grid.c:37-57 */
void rgo_frac_coord(int grid_size, int kernel_size, int oversample, double theta,
                    double u, double v, double d_u, double d_v,
                    int *grid_offset, int *sub_offset)
{
    double x = theta * (u - d_u);
    double y = theta * (v - d_v);
    int cell_x = (int)floor(x + .5 / oversample);
    int cell_y = (int)floor(y + .5 / oversample);
    int frac_x = (int)floor((x - (double)cell_x) * oversample + .5);
    int frac_y = (int)floor((y - (double)cell_y) * oversample + .5);
    *grid_offset = (cell_y + grid_size / 2 - kernel_size / 2) * grid_size +
                   (cell_x + grid_size / 2 - kernel_size / 2);
    *sub_offset = kernel_size * kernel_size * (frac_y * oversample + frac_x);
}

/* grid.c:157-185: convolve one visibility onto the grid with the conjugated
 * nearest-w, nearest-sub-cell kernel.  No bounds check (as the reference). */
static uint64_t w_project_one(double complex *grid, int grid_size, double theta,
                              double u, double v, double w, double complex vis,
                              double d_u, double d_v, double d_w, const rgo_wkern *wk)
{
    int goff, soff;
    rgo_frac_coord(grid_size, wk->size, wk->oversampling, theta, u, v, d_u, d_v,
                   &goff, &soff);
    double wr = w - d_w;
    int plane = (int)floor((wr - wk->w_min) / wk->w_step + .5);
    assert(plane >= 0 && plane < wk->plane_count);
    const int ks = wk->size;
    const double complex *taps =
        wk->data + (size_t)plane * wk->oversampling * wk->oversampling * ks * ks;
    /* The reference has no bounds check (grid.c:177-182).  With a W-towers
     * margin equal to the kernel size, a visibility within 1/(2 ov) cell of a
     * tower's low edge puts its footprint one cell before the sub-grid: the
     * reference's linear index then lands on the previous row (kept here) or,
     * on row -1, before the buffer (undefined behaviour there, dropped here). */
    const long long limit = (long long)grid_size * grid_size;
    for (int y = 0; y < ks; y++)
        for (int x = 0; x < ks; x++) {
            long long idx = (long long)goff + (long long)y * grid_size + x;
            if (idx < 0 || idx >= limit) continue;
            grid[idx] += vis * conj(taps[soff + y * ks + x]);
        }
    return 8 * (uint64_t)ks * (uint64_t)ks;
}

/* grid.c:187-202 */
uint64_t rgo_grid_wprojection(double complex *uvgrid, int grid_size, double theta,
                              int64_t nvis, const double *u, const double *v,
                              const double *w, const double complex *vis,
                              const rgo_wkern *wk)
{
    uint64_t flops = 0;
    for (int64_t i = 0; i < nvis; i++)
        flops += w_project_one(uvgrid, grid_size, theta, u[i], v[i], w[i], vis[i],
                               0, 0, 0, wk);
    return flops;
}

/* Integer power by binary exponentiation, grid.c:280-293. */
static double complex int_power(double complex base, int e)
{
    if (e < 0) return 1 / int_power(base, -e);
    if (e == 1) return base;
    double complex acc = 1;
    while (e) {
        if (e & 1) acc *= base;
        e >>= 1;
        base *= base;
    }
    return acc;
}

/* Chunk bounds of tower (cx, cy), grid.c:425-442. */
static void tower_bounds(int c, int chunk_size, int grid_size, double theta,
                         int *x_min, double *lo, double *hi, double *mid)
{
    *x_min = chunk_size * c - grid_size / 2;
    *lo = ((double)*x_min - 0.5) / theta;
    *hi = *lo + chunk_size / theta;
    *mid = (double)(*x_min + chunk_size / 2) / theta;
}

/* grid.c:295-555 (its serial build).  The reference scans every baseline of a tower's bin
 * once per w-floor and grids the visibilities passing the half-open (u,v,w)
 * cut in baseline/time/frequency order.  Here the same cut is applied once per
 * visibility (testing the neighbouring towers/floors with the reference's exact
 * comparisons) and a stable counting sort keeps that order per (tower, floor),
 * which yields the same additions in the same order. */
uint64_t rgo_grid_wtowers(double complex *uvgrid, int grid_size, double theta,
                          int64_t nvis, const double *u, const double *v,
                          const double *w, const double complex *vis,
                          const rgo_wkern *wk, int subgrid_size, int subgrid_margin,
                          double wincrement, int32_t *gridded_count,
                          const unsigned char *tower_sel)
{
    const int S = subgrid_size, M = subgrid_margin;
    assert(M >= wk->size);
    assert(S % 2 == 0 && M % 2 == 0);

    /* Fresnel transfer pattern between neighbouring w-floors, grid.c:304-319 */
    double complex *wtransfer = (double complex *)malloc(sizeof(double complex) * S * S);
    for (int y = 0; y < S; y++)
        for (int x = 0; x < S; x++) {
            double l = theta * (double)(x - S / 2) / S;
            double m = theta * (double)(y - S / 2) / S;
            double ph = wincrement * (1 - sqrt(1 - l * l - m * m));
            wtransfer[y * S + x] = cexp(2 * M_PI * I * ph);
        }
    rgo_fft_shift(wtransfer, S);

    const int chunk = S - M;
    const int nchunk = grid_size / chunk + 1;

    /* w range, always including 0 (grid.c:357-367) */
    double wlo = 0, whi = 0;
    for (int64_t i = 0; i < nvis; i++) {
        if (w[i] < wlo) wlo = w[i];
        if (w[i] > whi) whi = w[i];
    }
    const int wp_min = (int)floor(wlo / wincrement + 0.5);
    const int wp_max = (int)floor(whi / wincrement + 0.5);
    const int nfloor = wp_max - wp_min + 1;
    const int64_t nbins = (int64_t)nchunk * nchunk * nfloor;

    /* assign visibilities to (tower, floor) bins with the reference's cuts */
    int64_t cap = nvis + 16, npairs = 0;
    int64_t *pair_bin = (int64_t *)malloc(sizeof(int64_t) * cap);
    int64_t *pair_vis = (int64_t *)malloc(sizeof(int64_t) * cap);
    for (int64_t i = 0; i < nvis; i++) {
        int cxc = (int)floor((u[i] * theta + 0.5 + grid_size / 2) / chunk);
        int cyc = (int)floor((v[i] * theta + 0.5 + grid_size / 2) / chunk);
        int wpc = (int)floor(w[i] / wincrement + 0.5);
        for (int cy = cyc - 1; cy <= cyc + 1; cy++) {
            if (cy < 0 || cy >= nchunk) continue;
            int y_min; double vlo, vhi, vmid;
            tower_bounds(cy, chunk, grid_size, theta, &y_min, &vlo, &vhi, &vmid);
            if (v[i] < vlo || v[i] >= vhi) continue;
            for (int cx = cxc - 1; cx <= cxc + 1; cx++) {
                if (cx < 0 || cx >= nchunk) continue;
                int x_min; double ulo, uhi, umid;
                tower_bounds(cx, chunk, grid_size, theta, &x_min, &ulo, &uhi, &umid);
                if (u[i] < ulo || u[i] >= uhi) continue;
                for (int wp = wpc - 1; wp <= wpc + 1; wp++) {
                    if (wp < wp_min || wp > wp_max) continue;
                    double wflo = ((double)wp - 0.5) * wincrement;
                    double wfhi = ((double)wp + 0.5) * wincrement;
                    if (w[i] < wflo || w[i] >= wfhi) continue;
                    if (npairs == cap) {
                        cap *= 2;
                        pair_bin = (int64_t *)realloc(pair_bin, sizeof(int64_t) * cap);
                        pair_vis = (int64_t *)realloc(pair_vis, sizeof(int64_t) * cap);
                    }
                    pair_bin[npairs] = ((int64_t)cy * nchunk + cx) * nfloor + (wp - wp_min);
                    pair_vis[npairs] = i;
                    npairs++;
                }
            }
        }
    }
    /* stable counting sort by bin */
    int64_t *start = (int64_t *)calloc((size_t)nbins + 1, sizeof(int64_t));
    for (int64_t p = 0; p < npairs; p++) start[pair_bin[p] + 1]++;
    for (int64_t b = 0; b < nbins; b++) start[b + 1] += start[b];
    int64_t *order = (int64_t *)malloc(sizeof(int64_t) * (npairs + 1));
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)nbins);
    memcpy(fill, start, sizeof(int64_t) * (size_t)nbins);
    for (int64_t p = 0; p < npairs; p++) order[fill[pair_bin[p]]++] = pair_vis[p];
    free(fill);
    if (gridded_count) memset(gridded_count, 0, sizeof(int32_t) * (size_t)nvis);

    uint64_t flops = 0;
    const int sg_norm = S * S;
    double complex *uvgrid_mid = uvgrid + (grid_size + 1) * grid_size / 2;
    /* Towers are independent until the add-back: each is computed on its own
     * thread into its own sub-image, and the sub-images are then added to the
     * grid one after another in tower order, so the result does not depend on
     * the thread count. */
    const int ntowers = nchunk * nchunk;
    double complex **finished = (double complex **)calloc((size_t)ntowers, sizeof(double complex *));

#pragma omp parallel reduction(+ : flops)
    {
    double complex *subgrid = (double complex *)calloc((size_t)S * S, sizeof(double complex));
    double complex *subimg = (double complex *)calloc((size_t)S * S, sizeof(double complex));
#pragma omp for schedule(dynamic, 1)
    for (int c = 0; c < ntowers; c++) {
        if (tower_sel && !tower_sel[c]) continue; /* another share's tower */
        int cx = c % nchunk, cy = c / nchunk;
        int x_min, y_min;
        double ulo, uhi, umid, vlo, vhi, vmid;
        tower_bounds(cx, chunk, grid_size, theta, &x_min, &ulo, &uhi, &umid);
        tower_bounds(cy, chunk, grid_size, theta, &y_min, &vlo, &vhi, &vmid);

        memset(subgrid, 0, sizeof(double complex) * S * S);
        memset(subimg, 0, sizeof(double complex) * S * S);
        int have_vis = 0, last_wp = wp_min;
        for (int wp = wp_min; wp <= wp_max; wp++) {
            int64_t b = (int64_t)c * nfloor + (wp - wp_min);
            if (start[b] == start[b + 1]) continue; /* grid.c:462 */
            double w_mid = (double)wp * wincrement;
            for (int64_t p = start[b]; p < start[b + 1]; p++) {
                int64_t i = order[p];
                flops += w_project_one(subgrid, S, theta, u[i], v[i], w[i], vis[i],
                                       umid, vmid, w_mid, wk);
                if (gridded_count) {
#pragma omp atomic
                    gridded_count[i]++;
                }
            }
            have_vis = 1;
            /* back to the image plane, step the accumulated sub-image to this
             * floor and add (grid.c:467-483) */
            rgo_fft2d(subgrid, subgrid, S, S, +1);
            for (int k = 0; k < S * S; k++) {
                double complex step = int_power(wtransfer[k], wp - last_wp);
                subimg[k] = step * subimg[k] + subgrid[k];
                subgrid[k] = 0;
            }
            last_wp = wp;
        }
        if (!have_vis) continue;
        /* to w = 0 (grid.c:490-496), back to the uv plane (grid.c:499) */
        if (last_wp != 0)
            for (int k = 0; k < S * S; k++) subimg[k] /= int_power(wtransfer[k], last_wp);
        rgo_fft2d(subimg, subimg, S, S, -1);
        finished[c] = subimg;
        subimg = (double complex *)calloc((size_t)S * S, sizeof(double complex));
    }
    free(subgrid);
    free(subimg);
    }

    for (int c = 0; c < ntowers; c++) {
        if (!finished[c]) continue;
        const double complex *subimg = finished[c];
        int cx = c % nchunk, cy = c / nchunk;
        int x_min, y_min;
        double ulo, uhi, umid, vlo, vhi, vmid;
        tower_bounds(cx, chunk, grid_size, theta, &x_min, &ulo, &uhi, &umid);
        tower_bounds(cy, chunk, grid_size, theta, &y_min, &vlo, &vhi, &vmid);
        /* add the sub-grid, margins included, clipped to the grid (grid.c:503-516) */
        int x0 = x_min - M / 2, x1 = x0 + S;
        int y0 = y_min - M / 2, y1 = y0 + S;
        if (x0 < -grid_size / 2) x0 = -grid_size / 2;
        if (y0 < -grid_size / 2) y0 = -grid_size / 2;
        if (x1 > grid_size / 2) x1 = grid_size / 2;
        if (y1 > grid_size / 2) y1 = grid_size / 2;
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++)
                uvgrid_mid[x + y * grid_size] +=
                    (subimg[(x - x_min + M / 2) + (y - y_min + M / 2) * S] / sg_norm);
        free(finished[c]);
    }

    free(finished); free(order); free(start);
    free(pair_bin); free(pair_vis); free(wtransfer);
    return flops;
}

/* Tower loads under the binning cuts of rgo_grid_wtowers (grid.c:357-367,
 * 425-458, 244-254): visibilities per tower and w-floors with data per tower
 * (towers row-major, cy * nchunk + cx). */
void rgo_wtowers_census(int grid_size, double theta, int64_t nvis, const double *u, const double *v,
                        const double *w, int subgrid_size, int subgrid_margin, double wincrement,
                        int64_t *vis_per_tower, int32_t *floors_per_tower)
{
    const int chunk = subgrid_size - subgrid_margin;
    const int nchunk = grid_size / chunk + 1;
    double wlo = 0, whi = 0;
    for (int64_t i = 0; i < nvis; i++) {
        if (w[i] < wlo) wlo = w[i];
        if (w[i] > whi) whi = w[i];
    }
    const int wp_min = (int)floor(wlo / wincrement + 0.5);
    const int wp_max = (int)floor(whi / wincrement + 0.5);
    const int nfloor = wp_max - wp_min + 1;
    unsigned char *active = (unsigned char *)calloc((size_t)nchunk * nchunk * nfloor, 1);
    memset(vis_per_tower, 0, sizeof(int64_t) * (size_t)nchunk * nchunk);
    for (int64_t i = 0; i < nvis; i++) {
        int cxc = (int)floor((u[i] * theta + 0.5 + grid_size / 2) / chunk);
        int cyc = (int)floor((v[i] * theta + 0.5 + grid_size / 2) / chunk);
        int wpc = (int)floor(w[i] / wincrement + 0.5);
        for (int cy = cyc - 1; cy <= cyc + 1; cy++) {
            if (cy < 0 || cy >= nchunk) continue;
            int y_min; double vlo, vhi, vmid;
            tower_bounds(cy, chunk, grid_size, theta, &y_min, &vlo, &vhi, &vmid);
            if (v[i] < vlo || v[i] >= vhi) continue;
            for (int cx = cxc - 1; cx <= cxc + 1; cx++) {
                if (cx < 0 || cx >= nchunk) continue;
                int x_min; double ulo, uhi, umid;
                tower_bounds(cx, chunk, grid_size, theta, &x_min, &ulo, &uhi, &umid);
                if (u[i] < ulo || u[i] >= uhi) continue;
                for (int wp = wpc - 1; wp <= wpc + 1; wp++) {
                    if (wp < wp_min || wp > wp_max) continue;
                    if (w[i] < ((double)wp - 0.5) * wincrement || w[i] >= ((double)wp + 0.5) * wincrement) continue;
                    vis_per_tower[cy * nchunk + cx]++;
                    active[((size_t)cy * nchunk + cx) * nfloor + (wp - wp_min)] = 1;
                }
            }
        }
    }
    for (int t = 0; t < nchunk * nchunk; t++) {
        int c = 0;
        for (int f = 0; f < nfloor; f++) c += active[(size_t)t * nfloor + f];
        floors_per_tower[t] = c;
    }
    free(active);
}

/* grid.c:27-35 */
static int nearest_cell(int grid_size, double theta, double u, double v)
{
    int x = (int)floor(theta * u + .5);
    int y = (int)floor(theta * v + .5);
    return (y + grid_size / 2) * grid_size + (x + grid_size / 2);
}

/* grid.c:83-99: each visibility added to its nearest cell (grid.c:27-35).
 * Returns 1 (nothing written past the grid) when a cell lies off the grid. */
int rgo_grid_simple(double complex *uvgrid, int grid_size, double theta, int64_t nvis, const double *u,
                    const double *v, const double complex *vis)
{
    int bad = 0;
    for (int64_t i = 0; i < nvis; i++) {
        int x = (int)floor(theta * u[i] + .5), y = (int)floor(theta * v[i] + .5);
        if (x + grid_size / 2 < 0 || x + grid_size / 2 >= grid_size || y + grid_size / 2 < 0 ||
            y + grid_size / 2 >= grid_size) {
            bad = 1;
            continue;
        }
        uvgrid[nearest_cell(grid_size, theta, u[i], v[i])] += vis[i];
    }
    return bad;
}

/* grid.c:59-81 */
void rgo_weight(int grid_size, double theta, int64_t nvis, const double *u,
                const double *v, double complex *vis)
{
    unsigned int *count = (unsigned int *)calloc((size_t)grid_size * grid_size,
                                                 sizeof(unsigned int));
    for (int64_t i = 0; i < nvis; i++) count[nearest_cell(grid_size, theta, u[i], v[i])]++;
    for (int64_t i = 0; i < nvis; i++) vis[i] /= count[nearest_cell(grid_size, theta, u[i], v[i])];
    free(count);
}

/* grid.c:639-662: G(k) += conj(G(-k)) pairwise; the zero frequency of an
 * even-sized grid sits at (N/2, N/2), so row 0 and column 0 are skipped. */
void rgo_make_hermitian(double complex *uvgrid, int grid_size)
{
    double complex *lo = (grid_size % 2 == 0) ? uvgrid + grid_size + 1 : uvgrid;
    double complex *hi = uvgrid + (size_t)grid_size * grid_size - 1;
    while (lo < hi) {
        double complex keep = *lo;
        *lo++ += conj(*hi);
        *hi-- += conj(keep);
    }
    assert(lo == hi && lo == uvgrid + (grid_size + 1) * (grid_size / 2));
    *lo += conj(*lo);
}

/* grid.c:665-680: exchange quadrants (both axes shift by N/2). */
void rgo_fft_shift(double complex *uvgrid, int grid_size)
{
    assert(grid_size % 2 == 0);
    const long long n2 = (long long)grid_size * grid_size;
    const long long jump = (long long)(grid_size + 1) * (grid_size / 2);
    for (int y = 0; y < grid_size; y++)
        for (int x = 0; x < grid_size / 2; x++) {
            long long a = (long long)y * grid_size + x;
            long long b = (a + jump) % n2;
            double complex t = uvgrid[a];
            uvgrid[a] = uvgrid[b];
            uvgrid[b] = t;
        }
}

/* main.c:258-294 */
void rgo_image_from_grid(double complex *uvgrid, int grid_size, double *image)
{
    rgo_make_hermitian(uvgrid, grid_size);
    rgo_fft_shift(uvgrid, grid_size);
    rgo_fft2d(uvgrid, uvgrid, grid_size, grid_size, -1);
    rgo_fft_shift(uvgrid, grid_size);
    for (long long k = 0; k < (long long)grid_size * grid_size; k++) image[k] = creal(uvgrid[k]);
}

/* One pixel of the FP64 DFT oracle: factor * sum_k Re(V_k exp(2 pi i ph_k)),
 * ph = u l + v m + w (1 - n) reduced to [-1/2, 1/2] turns in FP64 before the
 * FP64 sin/cos, summed with Neumaier compensation. */
static double dft_pixel(int x, int y, int N, double theta, int64_t nvis, const double *u,
                        const double *v, const double *w, const double complex *vis, double factor)
{
    double m = theta * (double)(y - N / 2) / N;
    double l = theta * (double)(x - N / 2) / N;
    double one_minus_n = 1.0 - sqrt(1.0 - l * l - m * m);
    double sum = 0.0, comp = 0.0;
    for (int64_t k = 0; k < nvis; k++) {
        double ph = u[k] * l + v[k] * m + w[k] * one_minus_n;
        ph -= nearbyint(ph);
        double a = 2.0 * M_PI * ph;
        double term = creal(vis[k]) * cos(a) + cimag(vis[k]) * sin(a);
        double t = sum + term; /* Neumaier compensated sum */
        if (fabs(sum) >= fabs(term)) comp += (sum - t) + term;
        else comp += (term - t) + sum;
        sum = t;
    }
    return factor * (sum + comp);
}

void rgo_dft_image(double *image, int grid_size, double theta, int64_t nvis,
                   const double *u, const double *v, const double *w,
                   const double complex *vis, double factor)
{
    const int N = grid_size;
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < N; y++)
        for (int x = 0; x < N; x++)
            image[(size_t)y * N + x] = dft_pixel(x, y, N, theta, nvis, u, v, w, vis, factor);
}

void rgo_dft_pixels(double *out, int npix, const int *px, const int *py, int grid_size, double theta,
                    int64_t nvis, const double *u, const double *v, const double *w,
                    const double complex *vis, double factor)
{
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < npix; k++)
        out[k] = dft_pixel(px[k], py[k], grid_size, theta, nvis, u, v, w, vis, factor);
}

/* ------------------------------------------------------------------------
 * W-stacking predict (degridding), src/wstack/predict.cpp:396-562 with the
 * sky (:187-245), the Fresnel pattern (:152-183), the plane stepping
 * (:248-273), the quadrant swap (:295-320) and the separable 3-D
 * de-convolution of one visibility (src/wstack/wstack_common.h:423-484).
 * Arrays are row-major [row][column]; the reference's (i, j) element access
 * is column i of row j.  Separable tables: data[ov_index * size + tap].
 * ------------------------------------------------------------------------ */

/* fft_shift_2Darray, predict.cpp:295-320 (even sizes) */
static void swap_quadrants(double complex *a, int n)
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n / 2; i++) {
            int i1 = i + n / 2;
            int j1 = j < n / 2 ? j + n / 2 : j - n / 2;
            double complex t = a[(size_t)j * n + i];
            a[(size_t)j * n + i] = a[(size_t)j1 * n + i1];
            a[(size_t)j1 * n + i1] = t;
        }
}

int rgo_wstack_planes(double theta, double lam, double dw, int support_w)
{
    int grid_size = (int)floor(theta * lam);
    double max_w = sin(theta / 2) * sqrt(2 * (grid_size * grid_size));
    return (int)ceil(max_w / dw) + support_w + 1;
}

int rgo_wstack_predict(double theta, double lam, int npts, const double *points, int64_t nvis,
                       const double *u, const double *v, const double *w, double du, double dw, double x0,
                       const double *conv_uv, int uv_size, int uv_ov, const double *conv_w, int w_size,
                       int w_ov, const double *corr_lm, int lm_size, int lm_ov, const double *corr_n,
                       int n_size, int n_ov, double complex *vis_out)
{
    const int N = (int)floor(theta * lam);
    const double x0ih = round(0.5 / x0);
    const int G = (int)(x0ih * N);
    if (G <= N || G % 2) return 1;
    const int gd = (G - N) / 2;
    const int w_planes = rgo_wstack_planes(theta, lam, dw, w_size);
    const size_t g2 = (size_t)G * G;

    /* Fresnel pattern (predict.cpp:152-183) */
    double complex *wtransfer = (double complex *)calloc(g2, sizeof(double complex));
    for (int y = 0; y < N; y++)
        for (int x = 0; x < N; x++) {
            double l = theta * ((double)x - N / 2) / N;
            double m = theta * ((double)y - N / 2) / N;
            double ph = dw * (1.0 - sqrt(1.0 - l * l - m * m));
            wtransfer[(size_t)(y + gd) * G + (x + gd)] = cexp(I * 2 * M_PI * ph);
        }
    /* the quantised sky over the grid correction (predict.cpp:187-245) */
    double complex *sky = (double complex *)calloc(g2, sizeof(double complex));
    const int lm_t = lm_size * lm_ov, n_t = n_size * n_ov;
    const double lm_step = 1.0 / (double)lm_t, n_step = 1.0 / (double)n_t;
    for (int i = 0; i < npts; i++) {
        double l = points[2 * i], m = points[2 * i + 1];
        int lc = (int)floor((l / theta + 0.5) * (double)N);
        int mc = (int)floor((m / theta + 0.5) * (double)N);
        double lq = (double)lc / lam - theta / 2;
        double mq = (double)mc / lam - theta / 2;
        double n = sqrt(1.0 - lq * lq - mq * mq) - 1.0;
        int aau = (int)floor((du * lq) / lm_step) + lm_t / 2;
        int aav = (int)floor((du * mq) / lm_step) + lm_t / 2;
        int aaw = (int)floor((dw * n) / n_step) + n_t / 2;
        if (aau < 0 || aau >= lm_t || aav < 0 || aav >= lm_t || aaw < 0 || aaw >= n_t) return 2;
        if (gd + lc < 0 || gd + lc >= G || gd + mc < 0 || gd + mc >= G) return 2;
        double a = 1.0;
        a *= corr_lm[aau];
        a *= corr_lm[aav];
        a *= corr_n[aaw];
        sky[(size_t)(gd + mc) * G + (gd + lc)] += 1.0 / a;
    }
    swap_quadrants(sky, G);
    swap_quadrants(wtransfer, G);
    /* to the first plane (predict.cpp:472: the pattern to the power
     * floor(-w_planes / 2), skipping the zeros of the pattern) */
    const int t0 = -w_planes / 2;
    for (size_t k = 0; k < g2; k++) {
        if (t0 == 1) sky[k] *= wtransfer[k];
        else if (wtransfer[k] != 0) sky[k] *= cpow(wtransfer[k], (double)t0);
    }
    /* the planes (predict.cpp:480-491) */
    double complex *stack = (double complex *)malloc(sizeof(double complex) * g2 * (size_t)w_planes);
    for (int p = 0; p < w_planes; p++) {
        double complex *plane = stack + g2 * (size_t)p;
        rgo_fft2d(sky, plane, G, G, -1);
        swap_quadrants(plane, G);
        for (size_t k = 0; k < g2; k++) sky[k] *= wtransfer[k];
    }
    /* de-convolve each visibility (wstack_common.h:423-484) */
    const int aa_h = uv_size / 2, aaw_h = w_size / 2;
    int bad = 0;
#pragma omp parallel for schedule(static, 1000) reduction(| : bad)
    for (int64_t i = 0; i < nvis; i++) {
        double complex acc = 0;
        double flu = u[i] - ceil(u[i] / du) * du;
        double flv = v[i] - ceil(v[i] / du) * du;
        double flw = w[i] - ceil(w[i] / dw) * dw;
        int ovu = (int)floor(fabs(flu) / du * uv_ov);
        int ovv = (int)floor(fabs(flv) / du * uv_ov);
        int ovw = (int)floor(fabs(flw) / dw * w_ov);
        for (int dwi = -aaw_h; dwi < aaw_h; dwi++) {
            int dws = (int)ceil(w[i] / dw) + w_planes / 2 + dwi;
            double gw = conv_w[w_size * ovw + (dwi + aaw_h)];
            for (int dvi = -aa_h; dvi < aa_h; dvi++) {
                int dvs = (int)ceil(v[i] / du) + N + dvi;
                double guv = gw * conv_uv[uv_size * ovv + (dvi + aa_h)];
                for (int dui = -aa_h; dui < aa_h; dui++) {
                    int dus = (int)ceil(u[i] / du) + N + dui;
                    double g = guv * conv_uv[uv_size * ovu + (dui + aa_h)];
                    if (dus < 0 || dus >= G || dvs < 0 || dvs >= G || dws < 0 || dws >= w_planes) {
                        bad = 1;
                        continue;
                    }
                    acc += stack[g2 * (size_t)dws + (size_t)dvs * G + dus] * g;
                }
            }
        }
        vis_out[i] = acc;
    }
    free(stack);
    free(sky);
    free(wtransfer);
    return bad ? 3 : 0;
}

/* predict_visibility_quantized_vec, src/wstack/predict.cpp:89-129: the direct
 * sum over the sources snapped to the image grid, unit amplitude. */
void rgo_predict_dft_quantized(double theta, double lam, int npts, const double *points, int64_t nvis,
                               const double *u, const double *v, const double *w, double complex *vis_out)
{
    const double grid_size = floor(theta * lam);
#pragma omp parallel for schedule(static, 256)
    for (int64_t k = 0; k < nvis; k++) {
        double complex acc = 0;
        for (int i = 0; i < npts; i++) {
            double lc = floor((points[2 * i] / theta + 0.5) * grid_size);
            double mc = floor((points[2 * i + 1] / theta + 0.5) * grid_size);
            double lq = lc / lam - theta / 2;
            double mq = mc / lam - theta / 2;
            double n = sqrt(1.0 - lq * lq - mq * mq) - 1.0;
            acc += cexp(-2 * M_PI * I * (u[k] * lq + v[k] * mq + w[k] * n));
        }
        vis_out[k] = acc;
    }
}

/* ------------------------------------------------------------------------
 * AW-projection, src/reference/grid.c:557-637: convolve_aw_kernels picks, per
 * baseline, time and A-kernel frequency channel, the w-plane nearest to
 * w = uvw_w * f_A / c with f_A the frequency of antenna 1's A-kernel for that
 * time and channel (and copies that w-kernel: the A-kernel convolution is a
 * placeholder there, :583-590); grid_awprojection grids each visibility with
 * the kernel of its nearest A-kernel channel.  Baselines [bl_min, bl_max) of
 * arrays with uniform time and frequency counts: antenna1 [bl], time
 * [bl][nt], freq [bl][nf], uvw [bl][nt][3] metres, vis [bl][nt][nf];
 * akern_freq [ant][at][af].  Returns 0, or 1 when an index leaves its table.
 * ------------------------------------------------------------------------ */
int rgo_grid_awprojection(double complex *uvgrid, int grid_size, double theta, int bl_min, int bl_max,
                          int nt, int nf, const int32_t *antenna1, const double *time, const double *freq,
                          const double *uvw, const double complex *vis, const rgo_wkern *wk, int ak_ant,
                          int ak_time, int ak_freq, double t_min, double t_step, double f_min, double f_step,
                          const double *akern_freq)
{
    const double c = 299792458.0; /* grid.c:19 */
    const int ks = wk->size, ov = wk->oversampling;
    int *plane_of = (int *)malloc(sizeof(int) * (size_t)nt * ak_freq);
    for (int bl = bl_min; bl < bl_max; bl++) {
        const double *bt = time + (size_t)bl * nt, *bf = freq + (size_t)bl * nf;
        const double *bu = uvw + (size_t)bl * nt * 3;
        for (int t = 0; t < nt; t++)
            for (int af = 0; af < ak_freq; af++) {
                int atime = (int)floor((bt[t] - t_min) / t_step + .5);
                if (antenna1[bl] < 0 || antenna1[bl] >= ak_ant || atime < 0 || atime >= ak_time) {
                    free(plane_of);
                    return 1;
                }
                int a1i = antenna1[bl] * ak_time * ak_freq + atime * ak_freq + af;
                double w = bu[t * 3 + 2] * akern_freq[a1i] / c;
                int w_plane = (int)floor((w - wk->w_min) / wk->w_step + .5);
                if (w_plane < 0 || w_plane >= wk->plane_count) {
                    free(plane_of);
                    return 1;
                }
                plane_of[t * ak_freq + af] = w_plane;
            }
        for (int t = 0; t < nt; t++)
            for (int f = 0; f < nf; f++) {
                double u = bu[t * 3 + 0] * bf[f] / c; /* uvw_lambda, grid.c:21-24 */
                double v = bu[t * 3 + 1] * bf[f] / c;
                int goff, soff;
                rgo_frac_coord(grid_size, ks, ov, theta, u, v, 0, 0, &goff, &soff);
                int afreq = (int)floor((bf[f] - f_min) / f_step + .5);
                if (afreq < 0 || afreq >= ak_freq) {
                    free(plane_of);
                    return 1;
                }
                const double complex *awk =
                    wk->data + (size_t)plane_of[t * ak_freq + afreq] * ov * ov * ks * ks;
                double complex vv = vis[((size_t)bl * nt + t) * nf + f];
                const long long limit = (long long)grid_size * grid_size;
                for (int y = 0; y < ks; y++)
                    for (int x = 0; x < ks; x++) {
                        long long idx = (long long)goff + (long long)y * grid_size + x;
                        if (idx < 0 || idx >= limit) continue;
                        uvgrid[idx] += vv * conj(awk[soff + y * ks + x]);
                    }
            }
    }
    free(plane_of);
    return 0;
}
