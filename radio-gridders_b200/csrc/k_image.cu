// Element-wise and image-formation kernels: kernel-table conversion, uniform
// weighting, make_hermitian, fft_shift, real part / grid correction, and the
// FP32 -> FP64 grid accumulation of the W-projection path.
#include "rg_internal.h"

namespace rg {

static inline int blocks_for(int64_t n, int threads = 256, int cap = 148 * 32)
{
    int64_t b = (n + threads - 1) / threads;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

__global__ void convert_table_kernel(const double2 *__restrict__ src, float2 *__restrict__ dst, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 z = src[i];
        dst[i] = make_float2((float)z.x, (float)z.y);
    }
}

void launch_convert_table(cudaStream_t s, const double2 *src, float2 *dst, int64_t n)
{
    convert_table_kernel<<<blocks_for(n), 256, 0, s>>>(src, dst, n);
}

// Each kk-tap slice written twice in a row: dst[s][0..2kk) = src[s][t mod kk].
__global__ void convert_table_dup_kernel(const double2 *__restrict__ src, float2 *__restrict__ dst, int64_t n_out,
                                         int kk)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_out;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t slice = i / (2 * kk);
        const double2 z = src[slice * kk + (int)(i % (2 * kk)) % kk];
        dst[i] = make_float2((float)z.x, (float)z.y);
    }
}

// The same for a power-of-two slice length (every supported kernel size): one
// thread per two source taps (two 16-byte loads), each converted pair stored
// twice as one 16-byte store; shifts instead of 64-bit divisions.
__global__ void convert_table_dup_pow2_kernel(const double2 *__restrict__ src, float4 *__restrict__ dst,
                                              int64_t n_pairs, int kk_lg)
{
    const int64_t half = (int64_t)1 << (kk_lg - 1);  // pairs per slice
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pairs;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = src[2 * i], b = src[2 * i + 1];
        const float4 f = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
        const int64_t slice = i >> (kk_lg - 1), t = i & (half - 1);
        float4 *d = dst + (slice << kk_lg) + t;
        d[0] = f;
        d[half] = f;
    }
}

void launch_convert_table_dup(cudaStream_t s, const double2 *src, float2 *dst, int64_t n, int kk)
{
    int lg = 0;
    while ((1 << lg) < kk) lg++;
    if ((1 << lg) == kk && lg >= 1)
        convert_table_dup_pow2_kernel<<<blocks_for(n / 2), 256, 0, s>>>(src, (float4 *)dst, n / 2, lg);
    else
        convert_table_dup_kernel<<<blocks_for(2 * n), 256, 0, s>>>(src, dst, 2 * n, kk);
}

// make_hermitian, src/reference/grid.c:639-662: the pointer walk pairs linear
// index base + t with N^2 - 1 - t (base = N + 1 for even N, 0 for odd) until
// they meet at the zero frequency (N + 1) * (N / 2).  Pairs are disjoint, so
// one thread per pair reproduces it.
__global__ void make_hermitian_kernel(double2 *__restrict__ g, int64_t base, int64_t last,
                                      int64_t pairs, int64_t centre)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < pairs;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + t, j = last - t;
        const double2 a = g[i], b = g[j];
        g[i] = make_double2(a.x + b.x, a.y - b.y);
        g[j] = make_double2(b.x + a.x, b.y - a.y);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const double2 c = g[centre];
        g[centre] = make_double2(c.x + c.x, c.y - c.y);
    }
}

void launch_make_hermitian(cudaStream_t s, double2 *grid, int n)
{
    const int64_t base = (n % 2 == 0) ? (int64_t)n + 1 : 0;
    const int64_t last = (int64_t)n * n - 1;
    const int64_t pairs = (last - base) / 2;
    const int64_t centre = (int64_t)(n + 1) * (n / 2);
    make_hermitian_kernel<<<blocks_for(pairs), 256, 0, s>>>(grid, base, last, pairs, centre);
}

// fft_shift, src/reference/grid.c:665-680: swap (y, x) with
// ((y*N + x + (N+1)*(N/2)) mod N^2) for x < N/2; the pairs are disjoint.
__global__ void fft_shift_kernel(double2 *__restrict__ g, int n)
{
    const int64_t half = n / 2;
    const int64_t total = (int64_t)n * half;
    const int64_t n2 = (int64_t)n * n, jump = (int64_t)(n + 1) * half;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t y = t / half, x = t % half;
        const int64_t a = y * n + x, b = (a + jump) % n2;
        const double2 tmp = g[a];
        g[a] = g[b];
        g[b] = tmp;
    }
}

void launch_fft_shift(cudaStream_t s, double2 *grid, int n)
{
    fft_shift_kernel<<<blocks_for((int64_t)n * (n / 2)), 256, 0, s>>>(grid, n);
}

__global__ void real_part_kernel(const double2 *__restrict__ g, double *__restrict__ img, int n,
                                 const double *__restrict__ taper)
{
    const int64_t total = (int64_t)n * n;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        double v = g[k].x;
        if (taper) v /= taper[k / n] * taper[k % n];
        img[k] = v;
    }
}

void launch_real_part(cudaStream_t s, const double2 *grid, double *img, int n, const double *taper)
{
    real_part_kernel<<<blocks_for((int64_t)n * n), 256, 0, s>>>(grid, img, n, taper);
}

// nearest cell, src/reference/grid.c:27-35 (index checked here; the
// reference writes out of bounds for data outside the grid)
__device__ __forceinline__ int64_t nearest_cell(double u, double v, int n, double theta)
{
    const int x = (int)floor(__dadd_rn(__dmul_rn(theta, u), .5));
    const int y = (int)floor(__dadd_rn(__dmul_rn(theta, v), .5));
    const int cx = x + n / 2, cy = y + n / 2;
    if (cx < 0 || cx >= n || cy < 0 || cy >= n) return -1;
    return (int64_t)cy * n + cx;
}

__global__ void weight_count_kernel(const double *__restrict__ u, const double *__restrict__ v,
                                    int64_t nvis, int n, double theta, unsigned *__restrict__ count)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nvis;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = nearest_cell(u[i], v[i], n, theta);
        if (c >= 0) atomicAdd(count + c, 1u);
    }
}

__global__ void weight_apply_kernel(const double *__restrict__ u, const double *__restrict__ v,
                                    const double2 *__restrict__ vis, double2 *__restrict__ out,
                                    int64_t nvis, int n, double theta,
                                    const unsigned *__restrict__ count)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nvis;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = nearest_cell(u[i], v[i], n, theta);
        const double2 z = vis[i];
        if (c < 0) {
            out[i] = z;
            continue;
        }
        const double d = (double)count[c];
        out[i] = make_double2(__ddiv_rn(z.x, d), __ddiv_rn(z.y, d));
    }
}

void launch_weight_count(cudaStream_t s, const double *u, const double *v, int64_t nvis, int n,
                         double theta, unsigned *count)
{
    weight_count_kernel<<<blocks_for(nvis), 256, 0, s>>>(u, v, nvis, n, theta, count);
}

void launch_weight_apply(cudaStream_t s, const double *u, const double *v, const double2 *vis,
                         double2 *out, int64_t nvis, int n, double theta, const unsigned *count)
{
    weight_apply_kernel<<<blocks_for(nvis), 256, 0, s>>>(u, v, vis, out, nvis, n, theta, count);
}

// grid_simple (src/reference/grid.c:83-99): each visibility added to its
// nearest cell, FP64 atomics on the master grid; a cell off the grid sets
// DERR_GRID_RANGE (the reference writes out of bounds).
__global__ void simple_grid_kernel(const double *__restrict__ u, const double *__restrict__ v,
                                   const double2 *__restrict__ vis, int64_t nvis, int n, double theta,
                                   double2 *__restrict__ grid, unsigned *err)
{
    bool bad = false;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nvis;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double uu = u[i], vv = v[i];
        if (!isfinite(uu) || !isfinite(vv) || fabs(theta * uu) > 1e9 || fabs(theta * vv) > 1e9) {
            bad = true;
            continue;
        }
        const int64_t c = nearest_cell(uu, vv, n, theta);
        if (c < 0) {
            bad = true;
            continue;
        }
        const double2 z = vis[i];
        atomicAdd(&grid[c].x, z.x);
        atomicAdd(&grid[c].y, z.y);
    }
    if (bad) atomicOr(err, DERR_GRID_RANGE);
}

__global__ void add_f64_kernel(const double2 *__restrict__ src, double2 *__restrict__ dst, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = src[i], b = dst[i];
        dst[i] = make_double2(b.x + a.x, b.y + a.y);
    }
}

void launch_add_f64(cudaStream_t s, const double2 *src, double2 *dst, int64_t n)
{
    add_f64_kernel<<<blocks_for(n), 256, 0, s>>>(src, dst, n);
}

void launch_simple_grid(cudaStream_t s, const double *u, const double *v, const double2 *vis, int64_t nvis, int n,
                        double theta, double2 *grid, unsigned *err)
{
    simple_grid_kernel<<<blocks_for(nvis), 256, 0, s>>>(u, v, vis, nvis, n, theta, grid, err);
}

__global__ void add_f32_to_f64_kernel(const float2 *__restrict__ src, double2 *__restrict__ dst,
                                      int64_t n, int overwrite)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float2 a = src[i];
        if (overwrite) {
            dst[i] = make_double2((double)a.x, (double)a.y);
        } else {
            const double2 b = dst[i];
            dst[i] = make_double2(b.x + (double)a.x, b.y + (double)a.y);
        }
    }
}

void launch_add_f32_to_f64(cudaStream_t s, const float2 *src, double2 *dst, int64_t n, int overwrite)
{
    add_f32_to_f64_kernel<<<blocks_for(n), 256, 0, s>>>(src, dst, n, overwrite);
}

}  // namespace rg
