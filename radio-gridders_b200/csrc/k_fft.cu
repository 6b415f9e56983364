// The project's own FFT kernels.
//
// FP32 (sub-grids, power-of-two n in [64, 1024]): four-step row and column
// transforms (rg_fft_device.cuh) and the fused W-towers column stage, which for
// one tower and a strip of columns runs, per active w-floor, the backward column
// transform, multiplies by the floor's Fresnel factor and accumulates, then
// applies the forward column transform to the sum — the per-floor
// fftw_execute_dft(ifft_plan) / cipow step / w=0 transfer / fft_plan sequence of
// src/reference/grid.c:467-499 with the per-floor row transforms done by the
// row kernel beforehand.
//
// FP64 (image formation, power-of-two n <= 4096): radix-2 Stockham rows in
// shared memory plus tiled transposes; not on the timed path.
#include <cmath>
#include <vector>

#include "rg_fft_device.cuh"
#include "rg_internal.h"

namespace rg {

constexpr int kPad = 33;  // padded k2 stride (float2 units) of the exchange buffer

bool fft32_supported(int n) { return n >= 64 && n <= 1024 && (n & (n - 1)) == 0; }

void fft32_init_twiddles(cudaStream_t s, float2 *tw, int n)
{
    std::vector<float2> h(n);
    for (int k = 0; k < n; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        h[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    cudaMemcpyAsync(tw, h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
}

template <int SIGN>
__device__ __forceinline__ float2 twiddle(const float2 *W, int k)
{
    float2 t = W[k];
    if (SIGN > 0) t.y = -t.y;
    return t;
}

// ---------------------------------------------------------------------------
// rows: R rows of length N = N1*32 per CTA, 256 threads
// ---------------------------------------------------------------------------
// rows: the row count, or, when count_dev is given, min(rows, *count_dev * N)
// (the number of active sub-grids lives on the device; the grid is sized for
// the capacity and CTAs past the live rows return at once).
template <int N1, int SIGN>
__global__ void __launch_bounds__(256) fft32_rows_kernel(float2 *__restrict__ data, int64_t rows,
                                                         const float2 *__restrict__ tw,
                                                         const int *__restrict__ count_dev)
{
    constexpr int N = N1 * 32, R = 16, LB = ilog2c(N1);
    extern __shared__ float2 smem[];
    float2 *T = smem;                 // [R][N1][kPad]
    float2 *W = smem + R * N1 * kPad;  // [N]
    const int64_t row0 = (int64_t)blockIdx.x * R;
    if (count_dev) {
        const int64_t live = (int64_t)(*count_dev) * N;
        if (live < rows) rows = live;
    }
    if (row0 >= rows) return;
    for (int i = threadIdx.x; i < N; i += blockDim.x) W[i] = tw[i];
    __syncthreads();

    for (int it = threadIdx.x; it < R * N1; it += blockDim.x) {
        const int n1 = it % N1, r = it / N1;
        const int64_t row = row0 + r;
        float2 a[32];
        if (row < rows) {
            const float2 *src = data + row * N + n1;
#pragma unroll
            for (int n2 = 0; n2 < 32; n2++) a[n2] = src[n2 * N1];
        } else {
#pragma unroll
            for (int n2 = 0; n2 < 32; n2++) a[n2] = make_float2(0.f, 0.f);
        }
        reg_fft<32, SIGN>(a);
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const int k2 = bitrevc(j, 5);
            T[(r * N1 + n1) * kPad + k2] = cmulf(a[j], twiddle<SIGN>(W, n1 * k2));
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < R * 32; it += blockDim.x) {
        const int k2 = it % 32, r = it / 32;
        const int64_t row = row0 + r;
        float2 b[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) b[n1] = T[(r * N1 + n1) * kPad + k2];
        reg_fft<N1, SIGN>(b);
        if (row < rows) {
            float2 *dst = data + row * N + k2;
#pragma unroll
            for (int j = 0; j < N1; j++) dst[32 * bitrevc(j, LB)] = b[j];
        }
    }
}

// ---------------------------------------------------------------------------
// columns: a strip of C columns of one N x N array per CTA, 256 threads
// ---------------------------------------------------------------------------
template <int N1, int CW = (N1 >= 32 ? 8 : 16)>
struct ColGeom {
    static constexpr int N = N1 * 32;
    static constexpr int C = CW;                            // strip width
    // per-column stride in T: N1*kPad + 16/C makes the 64-bit exchange accesses
    // of a half-warp (C columns x 16/C rows) hit distinct banks
    static constexpr int CS = N1 * kPad + 16 / CW;
    static constexpr int T_ELEMS = C * CS;
    static constexpr int LB = ilog2c(N1);
};

// Step 1 of a column transform: load from `src` (row stride `ld`, column c of
// the strip at src[row*ld + c]), 32-point transforms, twiddle, into T.
template <int N1, int SIGN, int CW = ColGeom<N1>::C, bool CLEAR = false>
__device__ __forceinline__ void col_step1(const float2 *__restrict__ src, int ld, float2 *T,
                                          const float2 *W)
{
    using G = ColGeom<N1, CW>;
    for (int it = threadIdx.x; it < G::C * N1; it += blockDim.x) {
        const int c = it % G::C, n1 = it / G::C;
        float2 a[32];
#pragma unroll
        for (int n2 = 0; n2 < 32; n2++) a[n2] = src[(int64_t)(n1 + n2 * N1) * ld + c];
        if (CLEAR) {  // leave the sub-grid zeroed for the next gridding pass
            float2 *dst = const_cast<float2 *>(src);
#pragma unroll
            for (int n2 = 0; n2 < 32; n2++) dst[(int64_t)(n1 + n2 * N1) * ld + c] = make_float2(0.f, 0.f);
        }
        reg_fft<32, SIGN>(a);
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const int k2 = bitrevc(j, 5);
            T[c * G::CS + n1 * kPad + k2] = cmulf(a[j], twiddle<SIGN>(W, n1 * k2));
        }
    }
}

template <int N1, int SIGN>
__global__ void __launch_bounds__(256) fft32_cols_kernel(float2 *__restrict__ data,
                                                         const float2 *__restrict__ tw)
{
    using G = ColGeom<N1>;
    constexpr int N = G::N;
    extern __shared__ float2 smem[];
    float2 *T = smem;
    float2 *W = smem + G::T_ELEMS;
    for (int i = threadIdx.x; i < N; i += blockDim.x) W[i] = tw[i];
    const int strip = blockIdx.x % (N / G::C);
    const int64_t arr = blockIdx.x / (N / G::C);
    float2 *base = data + arr * N * N + strip * G::C;
    __syncthreads();
    col_step1<N1, SIGN>(base, N, T, W);
    __syncthreads();
    for (int it = threadIdx.x; it < G::C * 32; it += blockDim.x) {
        const int c = it % G::C, k2 = it / G::C;
        float2 b[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) b[n1] = T[c * G::CS + n1 * kPad + k2];
        reg_fft<N1, SIGN>(b);
#pragma unroll
        for (int j = 0; j < N1; j++) base[(int64_t)(k2 + 32 * bitrevc(j, G::LB)) * N + c] = b[j];
    }
}

// ---------------------------------------------------------------------------
// W-towers column stage, in two kernels so uneven towers balance.
//
// tower_partial_kernel: CTA = (floor group, strip of C columns).  A group is up
// to G consecutive active floors of one tower.  For each floor: backward column
// transform of the row-transformed sub-grid, times exp(-2 pi i wp ph(l, m)) with
// ph = winc (1 - sqrt(1 - l^2 - m^2)) — the reference's wtransfer^(-wp),
// grid.c:304-319 and :473-496, which also covers the w = 0 transfer —
// accumulated in registers; the strip sum is written to the group's partial
// buffer.  Phase products are formed and reduced modulo 1 in FP64; sin/cos of
// the reduced phase in FP32.
//
// tower_finish_kernel: CTA = (tower, strip).  Sums the tower's group partials in
// group order (deterministic) and applies the forward column transform into the
// tower's sub-image (grid.c:499, with the row half done by the row kernel).
// ---------------------------------------------------------------------------
constexpr int kPartialThreads = 128;
template <int N1>
using PartialGeom = ColGeom<N1, 8>;

template <int N1>
__global__ void __launch_bounds__(kPartialThreads) tower_partial_kernel(
    float2 *__restrict__ slots, const int *__restrict__ bin_of_slot,
    const int *__restrict__ group_begin, const int *__restrict__ group_end,
    const int *__restrict__ range, const int *__restrict__ counts, int slot_cap,
    const double *__restrict__ ph, float2 *__restrict__ partial, const float2 *__restrict__ tw)
{
    using G = PartialGeom<N1>;
    constexpr int N = G::N, C = G::C;
    constexpr int ITEMS = C * 32;
    constexpr int PER = (ITEMS + kPartialThreads - 1) / kPartialThreads;
    extern __shared__ float2 smem[];
    float2 *T = smem;
    float2 *W = smem + G::T_ELEMS;
    double *P = reinterpret_cast<double *>(W + N);  // [N][C] Fresnel phase of the strip
    const int strips = N / C;
    const int group = blockIdx.x / strips, strip = blockIdx.x % strips;
    if (group >= counts[1]) return;  // groups live on the device; grid sized for capacity
    const int wp_min = range[0], nfloor = range[1];
    const int begin = group_begin[group];
    const int end = group_end[group] < slot_cap ? group_end[group] : slot_cap;
    for (int i = threadIdx.x; i < N; i += blockDim.x) W[i] = tw[i];
    for (int e = threadIdx.x; e < N * C; e += blockDim.x)
        P[e] = ph[(int64_t)(e / C) * N + strip * C + e % C];

    float2 acc[PER][N1];
#pragma unroll
    for (int q = 0; q < PER; q++)
#pragma unroll
        for (int j = 0; j < N1; j++) acc[q][j] = make_float2(0.f, 0.f);
    __syncthreads();

    for (int slot = begin; slot < end; slot++) {
        const double mwp = -(double)(wp_min + bin_of_slot[slot] % nfloor);
        const float2 *base = slots + (int64_t)slot * N * N + strip * C;
        col_step1<N1, +1, C, true>(base, N, T, W);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int it = threadIdx.x + q * kPartialThreads;
            if (it < ITEMS) {
                const int c = it % C, k2 = it / C;
                float2 b[N1];
#pragma unroll
                for (int n1 = 0; n1 < N1; n1++) b[n1] = T[c * G::CS + n1 * kPad + k2];
                reg_fft<N1, +1>(b);
#pragma unroll
                for (int j = 0; j < N1; j++) {
                    const int row = k2 + 32 * bitrevc(j, G::LB);
                    double phase = mwp * P[row * C + c];
                    phase -= rint(phase);  // |phase| <= 1/2 after the FP64 reduction
                    float sn, cs;
                    __sincosf(6.28318530717958647f * (float)phase, &sn, &cs);
                    acc[q][j] = caddf(acc[q][j], cmulf(b[j], make_float2(cs, sn)));
                }
            }
        }
        __syncthreads();
    }
    float2 *out = partial + (int64_t)group * N * N + strip * C;
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int it = threadIdx.x + q * kPartialThreads;
        if (it < ITEMS) {
            const int c = it % C, k2 = it / C;
#pragma unroll
            for (int j = 0; j < N1; j++) out[(int64_t)(k2 + 32 * bitrevc(j, G::LB)) * N + c] = acc[q][j];
        }
    }
}

template <int N1>
__global__ void __launch_bounds__(256) tower_finish_kernel(
    const float2 *__restrict__ partial, const int *__restrict__ tower_group_first,
    const int *__restrict__ tower_group_count, int group_cap, float2 *__restrict__ subimg,
    const float2 *__restrict__ tw)
{
    using G = ColGeom<N1>;
    constexpr int N = G::N, C = G::C;
    extern __shared__ float2 smem[];
    float2 *T = smem;
    float2 *W = smem + G::T_ELEMS;
    float2 *U = W + N;  // [N][C]
    const int strips = N / C;
    const int tower = blockIdx.x / strips, strip = blockIdx.x % strips;
    const int gfirst = tower_group_first[tower];
    int gcount = tower_group_count[tower];
    if (gfirst + gcount > group_cap) gcount = group_cap - gfirst;  // capacity overflow: rerun
    if (gcount <= 0) return;
    for (int i = threadIdx.x; i < N; i += blockDim.x) W[i] = tw[i];
    for (int e = threadIdx.x; e < N * C; e += blockDim.x) {
        const int row = e / C, c = e % C;
        float2 sum = make_float2(0.f, 0.f);
        for (int g = 0; g < gcount; g++)
            sum = caddf(sum, partial[(int64_t)(gfirst + g) * N * N + (int64_t)row * N + strip * C + c]);
        U[e] = sum;
    }
    __syncthreads();
    col_step1<N1, -1>(U, C, T, W);
    __syncthreads();
    float2 *out = subimg + (int64_t)tower * N * N + strip * C;
    for (int it = threadIdx.x; it < C * 32; it += blockDim.x) {
        const int c = it % C, k2 = it / C;
        float2 b[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) b[n1] = T[c * G::CS + n1 * kPad + k2];
        reg_fft<N1, -1>(b);
#pragma unroll
        for (int j = 0; j < N1; j++) out[(int64_t)(k2 + 32 * bitrevc(j, G::LB)) * N + c] = b[j];
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int N1>
static size_t rows_smem() { return sizeof(float2) * (16 * N1 * kPad + N1 * 32); }
template <int N1>
static size_t cols_smem() { return sizeof(float2) * (ColGeom<N1>::T_ELEMS + N1 * 32); }
template <int N1>
static size_t partial_smem()
{
    return sizeof(float2) * (PartialGeom<N1>::T_ELEMS + N1 * 32) +
           sizeof(double) * N1 * 32 * PartialGeom<N1>::C;
}
template <int N1>
static size_t finish_smem()
{
    return sizeof(float2) * (ColGeom<N1>::T_ELEMS + N1 * 32 + N1 * 32 * ColGeom<N1>::C);
}

template <int N1>
static void rows_impl(cudaStream_t s, float2 *data, int64_t rows, int sign, const float2 *tw,
                      const int *count_dev)
{
    const size_t sm = rows_smem<N1>();
    const unsigned blocks = (unsigned)((rows + 15) / 16);
    if (blocks == 0) return;
    if (sign < 0) {
        cudaFuncSetAttribute(fft32_rows_kernel<N1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        fft32_rows_kernel<N1, -1><<<blocks, 256, sm, s>>>(data, rows, tw, count_dev);
    } else {
        cudaFuncSetAttribute(fft32_rows_kernel<N1, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        fft32_rows_kernel<N1, +1><<<blocks, 256, sm, s>>>(data, rows, tw, count_dev);
    }
}

template <int N1>
static void cols_impl(cudaStream_t s, float2 *data, int batch, int sign, const float2 *tw)
{
    const size_t sm = cols_smem<N1>();
    const unsigned blocks = (unsigned)batch * (N1 * 32 / ColGeom<N1>::C);
    if (sign < 0) {
        cudaFuncSetAttribute(fft32_cols_kernel<N1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        fft32_cols_kernel<N1, -1><<<blocks, 256, sm, s>>>(data, tw);
    } else {
        cudaFuncSetAttribute(fft32_cols_kernel<N1, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        fft32_cols_kernel<N1, +1><<<blocks, 256, sm, s>>>(data, tw);
    }
}

template <int N1>
static void tower_impl(cudaStream_t s, float2 *slots, const int *bin_of_slot,
                       const int *group_begin, const int *group_end, const int *range,
                       const int *counts, int slot_cap, int group_cap,
                       const int *tower_group_first, const int *tower_group_count, int ntowers,
                       const double *ph, float2 *partial, float2 *subimg, const float2 *tw)
{
    const int pstrips = N1 * 32 / PartialGeom<N1>::C;
    const int strips = N1 * 32 / ColGeom<N1>::C;
    const size_t sm1 = partial_smem<N1>();
    cudaFuncSetAttribute(tower_partial_kernel<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
    if (group_cap > 0)
        tower_partial_kernel<N1><<<(unsigned)group_cap * pstrips, kPartialThreads, sm1, s>>>(
            slots, bin_of_slot, group_begin, group_end, range, counts, slot_cap, ph, partial, tw);
    const size_t sm2 = finish_smem<N1>();
    cudaFuncSetAttribute(tower_finish_kernel<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
    tower_finish_kernel<N1><<<(unsigned)ntowers * strips, 256, sm2, s>>>(
        partial, tower_group_first, tower_group_count, group_cap, subimg, tw);
}

#define RG_DISPATCH_N1(n, CALL) \
    switch ((n) / 32) {         \
        case 2: CALL(2); break;  \
        case 4: CALL(4); break;  \
        case 8: CALL(8); break;  \
        case 16: CALL(16); break; \
        case 32: CALL(32); break; \
        default: break;          \
    }

void launch_fft32_rows(cudaStream_t s, float2 *data, int64_t rows, int n, int sign, const float2 *tw,
                       const int *count_dev)
{
#define CALL(N1) rows_impl<N1>(s, data, rows, sign, tw, count_dev)
    RG_DISPATCH_N1(n, CALL)
#undef CALL
}

void launch_fft32_cols(cudaStream_t s, float2 *data, int batch, int n, int sign, const float2 *tw)
{
#define CALL(N1) cols_impl<N1>(s, data, batch, sign, tw)
    RG_DISPATCH_N1(n, CALL)
#undef CALL
}

void launch_tower_columns(cudaStream_t s, float2 *slots, const int *bin_of_slot,
                          const int *group_begin, const int *group_end, const int *range,
                          const int *counts, int slot_cap, int group_cap,
                          const int *tower_group_first, const int *tower_group_count, int ntowers,
                          const double *ph, float2 *partial, float2 *subimg, int subgrid,
                          const float2 *tw)
{
#define CALL(N1) tower_impl<N1>(s, slots, bin_of_slot, group_begin, group_end, range, counts, slot_cap, \
                                group_cap, tower_group_first, tower_group_count, ntowers, ph, partial,  \
                                subimg, tw)
    RG_DISPATCH_N1(subgrid, CALL)
#undef CALL
}

int fft32_strips(int n) { return n / 8; }  // strips of the partial (column) stage

// ---------------------------------------------------------------------------
// FP64 transforms (image formation)
// ---------------------------------------------------------------------------
bool fft64_supported(int n) { return n >= 2 && n <= 4096 && (n & (n - 1)) == 0; }

// One row per CTA: radix-2 Stockham autosort in shared memory (ping-pong),
// twiddles from an FP64 table exp(-2 pi i k / n), k < n/2.
__global__ void fft64_rows_kernel(double2 *__restrict__ data, int n, int sign,
                                  const double2 *__restrict__ tw)
{
    extern __shared__ double2 sm64[];
    double2 *a = sm64, *b = sm64 + n;
    double2 *row = data + (int64_t)blockIdx.x * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = row[i];
    __syncthreads();
    const int half = n / 2;
    // Stockham radix-2 autosort: sub-transforms of length Ns double each pass
    for (int Ns = 1; Ns < n; Ns <<= 1) {
        for (int t = threadIdx.x; t < half; t += blockDim.x) {
            const int k = t % Ns;
            double2 w = tw[k * (n / (2 * Ns))];
            if (sign > 0) w.y = -w.y;
            const double2 x = a[t];
            const double2 y = a[t + half];
            const double2 ty = make_double2(w.x * y.x - w.y * y.y, w.x * y.y + w.y * y.x);
            const int d = (t / Ns) * Ns * 2 + k;
            b[d] = make_double2(x.x + ty.x, x.y + ty.y);
            b[d + Ns] = make_double2(x.x - ty.x, x.y - ty.y);
        }
        __syncthreads();
        double2 *t2 = a; a = b; b = t2;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) row[i] = a[i];
}

__global__ void transpose64_kernel(const double2 *__restrict__ in, double2 *__restrict__ out,
                                   int ny, int nx)
{
    __shared__ double2 tile[32][33];
    const int64_t off = (int64_t)blockIdx.z * ny * nx;
    int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 32 + threadIdx.y;
    for (int k = 0; k < 32; k += 8)
        if (x < nx && y + k < ny) tile[threadIdx.y + k][threadIdx.x] = in[off + (int64_t)(y + k) * nx + x];
    __syncthreads();
    x = blockIdx.y * 32 + threadIdx.x;
    y = blockIdx.x * 32 + threadIdx.y;
    for (int k = 0; k < 32; k += 8)
        if (x < ny && y + k < nx) out[off + (int64_t)(y + k) * ny + x] = tile[threadIdx.x][threadIdx.y + k];
}

static double2 *twiddles64(cudaStream_t s, int n)
{
    // one table per size per process (small; kept for reuse)
    static std::map<int, double2 *> cache;
    auto it = cache.find(n);
    if (it != cache.end()) return it->second;
    std::vector<double2> h(n / 2 > 0 ? n / 2 : 1);
    for (int k = 0; k < n / 2; k++) {
        double a = -2.0 * M_PI * (double)k / (double)n;
        h[k] = make_double2(std::cos(a), std::sin(a));
    }
    double2 *d = nullptr;
    cudaMalloc(&d, sizeof(double2) * h.size());
    cudaMemcpyAsync(d, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    cache[n] = d;
    return d;
}

static void rows64(cudaStream_t s, double2 *data, int64_t rows, int n, int sign)
{
    const size_t sm = sizeof(double2) * 2 * n;
    cudaFuncSetAttribute(fft64_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const int threads = n / 2 < 512 ? (n / 2 > 32 ? n / 2 : 32) : 512;
    fft64_rows_kernel<<<(unsigned)rows, threads, sm, s>>>(data, n, sign, twiddles64(s, n));
}

void launch_fft64_2d(cudaStream_t s, double2 *data, double2 *tmp, int batch, int ny, int nx, int sign)
{
    rows64(s, data, (int64_t)batch * ny, nx, sign);
    dim3 blk(32, 8);
    dim3 g1((nx + 31) / 32, (ny + 31) / 32, batch);
    transpose64_kernel<<<g1, blk, 0, s>>>(data, tmp, ny, nx);
    rows64(s, tmp, (int64_t)batch * nx, ny, sign);
    dim3 g2((ny + 31) / 32, (nx + 31) / 32, batch);
    transpose64_kernel<<<g2, blk, 0, s>>>(tmp, data, nx, ny);
}

}  // namespace rg
