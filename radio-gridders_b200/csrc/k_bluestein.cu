// FP64 transforms of any length up to 4096 for image formation: lengths that
// are not powers of two go through Bluestein's chirp-z algorithm (Bluestein
// 1970; Rabiner, Schafer & Rader 1969), i.e. with c[m] = exp(s pi i m^2 / n)
//
//   X[k] = c[k] * sum_j (x[j] c[j]) conj(c[k - j]),
//
// a cyclic convolution of length L = the power of two >= 2n - 1 done with
// power-of-two FFTs (L <= 8192, one row per CTA, in place in shared memory).
// The reference transforms any even grid size with FFTW
// (src/reference/main.c:269-294), and grid.out's grid size is
// floor(lambda * theta), rarely a power of two.
#include <algorithm>
#include <cmath>
#include <vector>

#include "rg_internal.h"

namespace rg {

bool fft64_any_supported(int n) { return n >= 2 && n <= 4096; }

static int pow2_at_least(int m)
{
    int l = 1;
    while (l < m) l <<= 1;
    return l;
}

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// One row of length L (a power of two, <= 8192) per CTA: bit-reversed load
// into shared memory, then log2 L in-place radix-2 butterfly passes
// (decimation in time); tw[k] = exp(-2 pi i k / L), k < L/2, conjugated for
// sign +1.
__global__ void fft64_inplace_rows_kernel(double2 *__restrict__ data, int L, int lg, int sign,
                                          const double2 *__restrict__ tw)
{
    extern __shared__ double2 a64[];
    double2 *row = data + (int64_t)blockIdx.x * L;
    for (int i = threadIdx.x; i < L; i += blockDim.x) a64[__brev((unsigned)i) >> (32 - lg)] = row[i];
    __syncthreads();
    for (int half = 1, lh = 0; half < L; half <<= 1, lh++) {
        for (int t = threadIdx.x; t < L / 2; t += blockDim.x) {
            const int k = t & (half - 1);
            const int base = ((t >> lh) << (lh + 1)) + k;
            double2 w = tw[(int64_t)k * (L >> (lh + 1))];
            if (sign > 0) w.y = -w.y;
            const double2 x = a64[base], y = a64[base + half];
            const double2 ty = make_double2(w.x * y.x - w.y * y.y, w.x * y.y + w.y * y.x);
            a64[base] = make_double2(x.x + ty.x, x.y + ty.y);
            a64[base + half] = make_double2(x.x - ty.x, x.y - ty.y);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < L; i += blockDim.x) row[i] = a64[i];
}

// c[m] = exp(s pi i m^2 / n), the phase reduced exactly: m^2 mod 2n in
// integers, then sincospi.
__global__ void chirp_kernel(double2 *__restrict__ c, int n, int sign)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    const long long q = ((long long)m * m) % (2LL * n);
    double sn, cs;
    sincospi((double)sign * (double)q / (double)n, &sn, &cs);
    c[m] = make_double2(cs, sn);
}

// The convolution filter: bb[m] = conj(c[m]) for m < n, conj(c[L - m]) for
// L - m < n, else 0 (b is even in m).
__global__ void chirp_filter_kernel(const double2 *__restrict__ c, int n, int L, double2 *__restrict__ bb)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= L) return;
    double2 v = make_double2(0.0, 0.0);
    if (m < n) v = make_double2(c[m].x, -c[m].y);
    else if (L - m < n) v = make_double2(c[L - m].x, -c[L - m].y);
    bb[m] = v;
}

// work[r][m] = x[r][m] c[m] (m < n), 0 up to L
__global__ void chirp_pre_kernel(const double2 *__restrict__ x, int n, int L, int rows,
                                 const double2 *__restrict__ c, double2 *__restrict__ work)
{
    const int64_t total = (int64_t)rows * L;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int m = (int)(k % L);
        const int64_t r = k / L;
        double2 v = make_double2(0.0, 0.0);
        if (m < n) {
            const double2 a = x[r * n + m], b = c[m];
            v = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
        }
        work[k] = v;
    }
}

__global__ void chirp_mul_kernel(double2 *__restrict__ work, const double2 *__restrict__ B, int L, int rows)
{
    const int64_t total = (int64_t)rows * L;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = work[k], b = B[k % L];
        work[k] = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    }
}

// x[r][k] = c[k] work[r][k] / L
__global__ void chirp_post_kernel(double2 *__restrict__ x, int n, int L, int rows, const double2 *__restrict__ c,
                                  const double2 *__restrict__ work)
{
    const int64_t total = (int64_t)rows * n;
    const double inv = 1.0 / (double)L;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int m = (int)(k % n);
        const int64_t r = k / n;
        const double2 a = work[r * L + m], b = c[m];
        x[k] = make_double2((a.x * b.x - a.y * b.y) * inv, (a.x * b.y + a.y * b.x) * inv);
    }
}

static unsigned grid_for(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16); }

static void inplace_rows(cudaStream_t s, double2 *data, int64_t rows, int L, int sign, const double2 *tw)
{
    const size_t smem = sizeof(double2) * (size_t)L;
    cudaFuncSetAttribute(fft64_inplace_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int lg = 0;
    while ((1 << lg) < L) lg++;
    const int threads = L / 2 < 512 ? (L / 2 > 32 ? L / 2 : 32) : 512;
    fft64_inplace_rows_kernel<<<(unsigned)rows, threads, smem, s>>>(data, L, lg, sign, tw);
}

// Rows of length n, any n in [2, 4096]: the power-of-two kernel when it
// applies, otherwise Bluestein over chunks of rows through `work`.
// Work space: (fft64_any_work_elems) double2.
int64_t fft64_any_work_elems(int n)
{
    if (is_pow2(n)) return 0;
    const int L = pow2_at_least(2 * n - 1);
    return (int64_t)n + 2 * (int64_t)L + (int64_t)kBluesteinRows * L;
}

static void bluestein_rows(cudaStream_t s, double2 *data, int64_t rows, int n, int sign, double2 *work,
                           const double2 *(*twiddles)(cudaStream_t, int))
{
    const int L = pow2_at_least(2 * n - 1);
    double2 *c = work, *bb = work + n, *B = bb + L, *buf = B + L;
    const double2 *tw = twiddles(s, L);
    chirp_kernel<<<(n + 255) / 256, 256, 0, s>>>(c, n, sign);
    chirp_filter_kernel<<<(L + 255) / 256, 256, 0, s>>>(c, n, L, bb);
    cudaMemcpyAsync(B, bb, sizeof(double2) * L, cudaMemcpyDeviceToDevice, s);
    inplace_rows(s, B, 1, L, -1, tw);
    for (int64_t r0 = 0; r0 < rows; r0 += kBluesteinRows) {
        const int cnt = (int)std::min<int64_t>(kBluesteinRows, rows - r0);
        double2 *x = data + r0 * n;
        chirp_pre_kernel<<<grid_for((int64_t)cnt * L), 256, 0, s>>>(x, n, L, cnt, c, buf);
        inplace_rows(s, buf, cnt, L, -1, tw);
        chirp_mul_kernel<<<grid_for((int64_t)cnt * L), 256, 0, s>>>(buf, B, L, cnt);
        inplace_rows(s, buf, cnt, L, +1, tw);
        chirp_post_kernel<<<grid_for((int64_t)cnt * n), 256, 0, s>>>(x, n, L, cnt, c, buf);
    }
}

void launch_fft64_any_rows(cudaStream_t s, double2 *data, int64_t rows, int n, int sign, double2 *work)
{
    if (is_pow2(n)) {
        launch_fft64_pow2_rows(s, data, rows, n, sign);
        return;
    }
    bluestein_rows(s, data, rows, n, sign, work, fft64_twiddles);
}

}  // namespace rg
