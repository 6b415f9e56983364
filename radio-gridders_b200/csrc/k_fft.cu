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
// FP64 (image formation, any n <= 4096): radix-2 Stockham rows in shared
// memory for powers of two, Bluestein's algorithm (k_bluestein.cu) for other
// lengths, plus tiled transposes; not on the timed path.
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

// The four-step twiddles W_N^(n1 k2) in shared memory, laid out [k2][n1]: the
// lanes of a warp (consecutive n1 for one k2) read consecutive entries, free of
// bank conflicts.  tw is the length-N table exp(-2 pi i k / N).
template <int N1>
__device__ __forceinline__ void load_twiddles(float2 *W, const float2 *__restrict__ tw)
{
    for (int i = threadIdx.x; i < N1 * 32; i += blockDim.x) W[i] = tw[(i % N1) * (i / N1)];
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
    load_twiddles<N1>(W, tw);
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
        reg_fft_dif<32, SIGN>(a);
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const int k2 = bitrevc(j, 5);
            T[(r * N1 + n1) * kPad + k2] = cmulf(a[j], twiddle<SIGN>(W, k2 * N1 + n1));
        }
    }
    __syncthreads();
    for (int it = threadIdx.x; it < R * 32; it += blockDim.x) {
        const int k2 = it % 32, r = it / 32;
        const int64_t row = row0 + r;
        float2 b[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) b[n1] = T[(r * N1 + n1) * kPad + k2];
        reg_fft_dif<N1, SIGN>(b);
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
        reg_fft_dif<32, SIGN>(a);
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const int k2 = bitrevc(j, 5);
            T[c * G::CS + n1 * kPad + k2] = cmulf(a[j], twiddle<SIGN>(W, k2 * N1 + n1));
        }
    }
}

template <int N1, int SIGN>
__global__ void __launch_bounds__(256) fft32_cols_kernel(float2 *__restrict__ data,
                                                         const float2 *__restrict__ tw,
                                                         const int *__restrict__ live)
{
    using G = ColGeom<N1>;
    constexpr int N = G::N;
    extern __shared__ float2 smem[];
    float2 *T = smem;
    float2 *W = smem + G::T_ELEMS;
    const int strip = blockIdx.x % (N / G::C);
    const int64_t arr = blockIdx.x / (N / G::C);
    if (live && live[arr] == 0) return;  // an array nobody reads (a tower without data)
    load_twiddles<N1>(W, tw);
    float2 *base = data + arr * N * N + strip * G::C;
    __syncthreads();
    col_step1<N1, SIGN>(base, N, T, W);
    __syncthreads();
    for (int it = threadIdx.x; it < G::C * 32; it += blockDim.x) {
        const int c = it % G::C, k2 = it / G::C;
        float2 b[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) b[n1] = T[c * G::CS + n1 * kPad + k2];
        reg_fft_dif<N1, SIGN>(b);
#pragma unroll
        for (int j = 0; j < N1; j++) base[(int64_t)(k2 + 32 * bitrevc(j, G::LB)) * N + c] = b[j];
    }
}

// ---------------------------------------------------------------------------
// Sparse W-towers transforms.
//
// A sub-grid is non-zero only in the column strips its bin's visibilities
// marked (kStripCols columns each; typically a quarter of them), so the 2-D
// backward transform runs columns first: sparse_cols_kernel transforms only the
// marked strips, in place.  A row of the result is then non-zero only in those
// strips, which is all the row stage reads (and clears).
// ---------------------------------------------------------------------------
int mask_words(int subgrid) { return (subgrid / kStripCols + 31) / 32; }

// One warp per mask word: lane s of warp (slot, word) tests strip 32*word + s.
__global__ void slot_masks_kernel(const unsigned char *__restrict__ marks, const int *__restrict__ bin_of_slot,
                                  const int *counts, int slot_cap, int strips, int words,
                                  unsigned *__restrict__ masks)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t wi = i / 32;  // (slot, word)
    const int slot = (int)(wi / words), s = (int)(wi % words) * 32 + (int)(i % 32);
    const int live = counts[0] < slot_cap ? counts[0] : slot_cap;
    bool f = false;
    if (slot < live && s < strips) f = marks[(int64_t)bin_of_slot[slot] * strips + s] != 0;
    const unsigned b = __ballot_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && slot < slot_cap) {
        masks[wi] = b;
        if (b) atomicAdd((int *)counts + 3, __popc(b));  // marked strips, for the statistics
    }
}

void launch_slot_masks(cudaStream_t s, const unsigned char *marks, const int *bin_of_slot, const int *counts,
                       int slot_cap, int subgrid, unsigned *masks)
{
    const int words = mask_words(subgrid);
    const int64_t threads = (int64_t)slot_cap * words * 32;
    if (threads <= 0) return;
    slot_masks_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(marks, bin_of_slot, counts, slot_cap,
                                                                      subgrid / kStripCols, words, masks);
}

constexpr int kSparseColThreads = 128;
template <int N1>
using StripGeom = ColGeom<N1, kStripCols>;

// Persistent: the (slot, strip) pairs of the live slots are dealt round-robin
// to the CTAs; each CTA gathers its marked pairs into a shared list, then
// transforms them one after another, loading the next strip while the
// current one finishes.
template <int N1>
__global__ void __launch_bounds__(kSparseColThreads) sparse_cols_kernel(
    float2 *__restrict__ slots, const unsigned *__restrict__ masks, const int *__restrict__ counts, int slot_cap,
    const float2 *__restrict__ tw)
{
    using G = StripGeom<N1>;
    constexpr int N = G::N, C = G::C, STRIPS = N / C, WORDS = (STRIPS + 31) / 32;
    constexpr int NW = kSparseColThreads / 32;
    extern __shared__ float2 smem[];
    float2 *T = smem;
    float2 *W = smem + G::T_ELEMS;
    __shared__ int list[kSparseColThreads];
    __shared__ int warp_base[NW + 1];
    load_twiddles<N1>(W, tw);
    const int live = counts[0] < slot_cap ? counts[0] : slot_cap;
    const int64_t total = (int64_t)live * STRIPS;
    const int64_t stride = (int64_t)gridDim.x * kSparseColThreads;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t base = 0; base < total; base += stride) {
        const int64_t i = base + (int64_t)threadIdx.x * gridDim.x + blockIdx.x;
        bool f = false;
        if (i < total) {
            const int slot = (int)(i / STRIPS), st = (int)(i % STRIPS);
            f = (masks[(int64_t)slot * WORDS + st / 32] >> (st & 31)) & 1u;
        }
        const unsigned b = __ballot_sync(0xffffffffu, f);
        __syncthreads();  // the previous round's list is consumed
        if (lane == 0) warp_base[warp + 1] = __popc(b);
        __syncthreads();
        if (threadIdx.x == 0) {
            warp_base[0] = 0;
            for (int k = 1; k <= NW; k++) warp_base[k] += warp_base[k - 1];
        }
        __syncthreads();
        if (f) list[warp_base[warp] + __popc(b & ((1u << lane) - 1u))] = (int)(i - base);
        __syncthreads();
        const int n = warp_base[NW];
        // strips are contiguous N x C blocks (strip-major sub-grids): row stride C
        auto strip_of = [&](int k) -> float2 * {
            const int64_t item = base + list[k];
            return slots + (item / STRIPS) * N * N + (item % STRIPS) * (int64_t)(C * N);
        };
        auto step2 = [&](float2 *col) {
            for (int it = threadIdx.x; it < C * 32; it += blockDim.x) {
                const int c = it % C, k2 = it / C;
                float2 v[N1];
#pragma unroll
                for (int n1 = 0; n1 < N1; n1++) v[n1] = T[c * G::CS + n1 * kPad + k2];
                reg_fft<N1, +1>(v);
#pragma unroll
                for (int j = 0; j < N1; j++) col[(k2 + 32 * bitrevc(j, G::LB)) * C + c] = v[j];
            }
        };
        if constexpr (C * N1 <= kSparseColThreads) {
            // one step-1 item per thread: the next strip's loads are issued
            // before this strip's step 2, so they are in flight meanwhile
            const bool act = threadIdx.x < C * N1;
            const int c = threadIdx.x % C, n1 = threadIdx.x / C;
            float2 a[32];
            if (n > 0 && act) {
                const float2 *src = strip_of(0);
#pragma unroll
                for (int n2 = 0; n2 < 32; n2++) a[n2] = src[(n1 + n2 * N1) * C + c];
            }
            for (int k = 0; k < n; k++) {
                if (act) {
                    reg_fft<32, +1>(a);
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        const int k2 = bitrevc(j, 5);
                        T[c * G::CS + n1 * kPad + k2] = cmulf(a[j], twiddle<+1>(W, k2 * N1 + n1));
                    }
                }
                __syncthreads();
                if (k + 1 < n && act) {
                    const float2 *src = strip_of(k + 1);
#pragma unroll
                    for (int n2 = 0; n2 < 32; n2++) a[n2] = src[(n1 + n2 * N1) * C + c];
                }
                step2(strip_of(k));
                __syncthreads();
            }
        } else {
            for (int k = 0; k < n; k++) {
                float2 *col = strip_of(k);
                col_step1<N1, +1, C>(col, C, T, W);
                __syncthreads();
                step2(col);
                __syncthreads();
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Row stage, in two kernels so uneven towers balance.
//
// tower_rows_kernel: CTA = (floor group, R rows: four mirror pairs (y, N - y)
// when R = 8, so each Fresnel factor serves two rows; else a strip).  For each floor of
// the group: backward row transform of the column-transformed sub-grid (only
// the slot's marked strips are read, then zeroed), times exp(-2 pi i wp
// ph(l, m)) with ph = winc (1 - sqrt(1 - l^2 - m^2)) — the reference's
// wtransfer^(-wp), grid.c:304-319 and :473-496, which also covers the w = 0
// transfer — accumulated in registers; the strip sum goes to the group's
// partial buffer.  The phase -wp * ph is formed modulo one turn as an integer
// product with the 32-bit fixed-point table (fresnel_table_kernel), converted
// to FP32 (24 significant bits) for sin/cos.
//
// tower_rows_finish_kernel: CTA = (tower, strip of R rows).  Sums the tower's
// group partials in group order (deterministic) and applies the forward row
// transform into the tower's sub-image (the row half of grid.c:499).
// ---------------------------------------------------------------------------
constexpr int kRowThreads = 128;
template <int N1>
struct RowGeom {
    static constexpr int N = N1 * 32;
    static constexpr int R = N1 >= 32 ? 4 : 8;  // rows per CTA
    static constexpr int LB = ilog2c(N1);
    static constexpr int STRIPS = N / kStripCols;
    static constexpr int WORDS = (STRIPS + 31) / 32;
    static constexpr int ITEMS1 = R * N1;  // step-1 items (n1, row)
    static constexpr int ITEMS2 = R * 32;  // step-2 items (k2, row)
    static constexpr int PER = (ITEMS2 + kRowThreads - 1) / kRowThreads;
    static constexpr int T_ELEMS = R * N1 * kPad;
};

int tower_row_strips(int subgrid) { return subgrid / (subgrid >= 1024 ? 4 : 8); }

// Bit n2 (n2 < 32) of the result = strip (n1 + n2*N1)/kStripCols of the
// 128-bit strip mask (lo, hi) is marked: the element n1 + n2*N1 of a row that
// the step-1 item n1 loads.  Strided bit gathers by mask-and-fold.
__device__ __forceinline__ unsigned long long keep_every2(unsigned long long x)
{
    x &= 0x5555555555555555ull;
    x = (x | (x >> 1)) & 0x3333333333333333ull;
    x = (x | (x >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x >> 4)) & 0x00FF00FF00FF00FFull;
    x = (x | (x >> 8)) & 0x0000FFFF0000FFFFull;
    return (x | (x >> 16)) & 0x00000000FFFFFFFFull;
}
__device__ __forceinline__ unsigned long long keep_every4(unsigned long long x)
{
    x &= 0x1111111111111111ull;
    x = (x | (x >> 3)) & 0x0303030303030303ull;
    x = (x | (x >> 6)) & 0x000F000F000F000Full;
    x = (x | (x >> 12)) & 0x000000FF000000FFull;
    return (x | (x >> 24)) & 0xFFFFull;
}
template <int N1>
__device__ __forceinline__ unsigned element_bits(unsigned long long lo, unsigned long long hi, int n1)
{
    static_assert(kStripCols == 8, "strip gathers assume 8-column strips");
    if (N1 == 8) return (unsigned)lo;                              // strip = n2
    if (N1 == 16) return (unsigned)keep_every2(lo >> (n1 >> 3));   // strip = 2 n2 + n1/8
    if (N1 == 32)                                                  // strip = 4 n2 + n1/8
        return (unsigned)(keep_every4(lo >> (n1 >> 3)) | keep_every4(hi >> (n1 >> 3)) << 16);
    unsigned b = 0;  // N1 < 8: several n2 share a strip
#pragma unroll
    for (int n2 = 0; n2 < 32; n2++) b |= (unsigned)((lo >> ((n1 + n2 * N1) / kStripCols)) & 1ull) << n2;
    return b;
}

// a = *p when on, else a is left as it is.  A predicated load: the register is
// written only by the load, so no select waits on the load's result and all of
// a thread's loads stay in flight together.  The memory clobber keeps later
// stores (the clearing) after it.
__device__ __forceinline__ void ld_if(float2 &a, const float2 *p, bool on)
{
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t@q ld.global.v2.f32 {%0, %1}, [%2];\n\t}"
        : "+f"(a.x), "+f"(a.y)
        : "l"(p), "r"((unsigned)on)
        : "memory");
}

template <int N1>
__global__ void __launch_bounds__(kRowThreads) tower_rows_kernel(
    float2 *__restrict__ slots, const unsigned *__restrict__ masks, const int *__restrict__ bin_of_slot,
    const int *__restrict__ group_begin, const int *__restrict__ group_end, const int *__restrict__ range,
    const int *__restrict__ counts, int slot_cap, const uint32_t *__restrict__ phq, float2 *__restrict__ partial,
    const float2 *__restrict__ tw)
{
    using G = RowGeom<N1>;
    constexpr int N = G::N, R = G::R;
    extern __shared__ float2 smem[];
    float2 *T = smem;                                // [R][N1][kPad]
    float2 *W = smem + G::T_ELEMS;                   // [N]
    uint32_t *P = reinterpret_cast<uint32_t *>(W + N);  // [R][N] Fresnel phase of the strip (turns, 2^-32)
    __shared__ unsigned smask[G::WORDS];
    const int rstrips = N / R;
    const int group = blockIdx.x / rstrips, blk = blockIdx.x % rstrips;
    if (group >= counts[1]) return;  // groups live on the device; grid sized for capacity
    // MIRROR: the CTA's rows are four mirror pairs (y, N - y) — pair p is
    // (p, N - p), pair 0 is (0, N/2) — local rows 0-3 the first rows and 4-7
    // their mirrors.  ph(l, m) depends on m^2 only and the table's rows y and
    // N - y hold the same values, so a thread's two step-2 items (the same
    // column, rows r and r + 4) share each Fresnel factor, except in pair 0.
    constexpr bool MIRROR = R == 8 && G::PER == 2 && G::ITEMS2 == 2 * kRowThreads;
    auto row_of = [&](int r) -> int {
        if constexpr (!MIRROR) {
            return blk * R + r;
        } else {
            const int p = 4 * blk + (r & 3);
            return r < 4 ? p : (p == 0 ? N / 2 : N - p);
        }
    };
    const int wp_min = range[0], nfloor = range[1];
    const int begin = group_begin[group];
    const int end = group_end[group] < slot_cap ? group_end[group] : slot_cap;
    load_twiddles<N1>(W, tw);
    for (int e = threadIdx.x; e < R * N; e += blockDim.x) P[e] = phq[(int64_t)row_of(e / N) * N + e % N];

    float2 acc[G::PER][N1];
#pragma unroll
    for (int q = 0; q < G::PER; q++)
#pragma unroll
        for (int j = 0; j < N1; j++) acc[q][j] = make_float2(0.f, 0.f);

    // the next floor's strip mask is loaded a floor ahead, so only the strip
    // loads wait on memory at the top of a floor
    unsigned mnext = (threadIdx.x < G::WORDS && begin < end) ? masks[(int64_t)begin * G::WORDS + threadIdx.x] : 0u;
    for (int slot = begin; slot < end; slot++) {
        const uint32_t mwp = (uint32_t)(-(wp_min + bin_of_slot[slot] % nfloor));  // two's complement
        if (threadIdx.x < G::WORDS) {
            smask[threadIdx.x] = mnext;
            if (slot + 1 < end) mnext = masks[(int64_t)(slot + 1) * G::WORDS + threadIdx.x];
        }
        __syncthreads();  // masks visible; the previous floor's step 2 is done with T
        // the slot's strip mask in two 64-bit registers (at most 128 strips)
        const unsigned long long m_lo = smask[0] | (G::WORDS > 1 ? (unsigned long long)smask[1] << 32 : 0ull);
        const unsigned long long m_hi =
            G::WORDS > 2 ? (smask[2] | (G::WORDS > 3 ? (unsigned long long)smask[3] << 32 : 0ull)) : 0ull;
        for (int it = threadIdx.x; it < G::ITEMS1; it += blockDim.x) {
            const int n1 = it % N1, r = it / N1;
            // strip-major sub-grid: column col of row (row0 + r) at (col/8)*8N + row*8 + col%8;
            // for N1 >= 8 element n2 lies n2 * (N1/8) strips after the thread's first,
            // a compile-time offset from one per-thread base
            float2 *row_base = slots + (int64_t)slot * N * N + row_of(r) * kStripCols;
            float2 *src = row_base + (n1 / kStripCols) * (kStripCols * N) + n1 % kStripCols;
            auto elem = [&](int n2) -> float2 * {
                if constexpr (N1 >= kStripCols) {
                    return src + n2 * (N1 / kStripCols) * (kStripCols * N);
                } else {
                    const int col = n1 + n2 * N1;
                    return row_base + (col / kStripCols) * (kStripCols * N) + col % kStripCols;
                }
            };
            const unsigned on = element_bits<N1>(m_lo, m_hi, n1);
            float2 a[32];
            // all 32 loads issue before any clearing store
#pragma unroll
            for (int n2 = 0; n2 < 32; n2++) {
                a[n2] = make_float2(0.f, 0.f);
                ld_if(a[n2], elem(n2), (on >> n2) & 1u);
            }
#pragma unroll
            for (int n2 = 0; n2 < 32; n2++)
                if ((on >> n2) & 1u) *elem(n2) = make_float2(0.f, 0.f);  // leave the sub-grid zeroed
            reg_fft<32, +1>(a);
#pragma unroll
            for (int j = 0; j < 32; j++) {
                const int k2 = bitrevc(j, 5);
                T[(r * N1 + n1) * kPad + k2] = cmulf(a[j], twiddle<+1>(W, k2 * N1 + n1));
            }
        }
        __syncthreads();
        // -wp ph modulo one turn as a signed 32-bit fraction of a turn, rounded
        // to 24 significant bits by the conversion (at most 64 units of 2^-32,
        // 2^-26 turns, off); acc += b * (cs + i sn) as two packed-pair fused
        // multiply-adds, (acc + b.x (cs, sn)) + b.y (-sn, cs)
        auto fresnel = [&](uint32_t phase, float &sn, float &cs) {
            const int k = (int)(mwp * phase);
            __sincosf(__int2float_rn(k) * (6.28318530717958647f / 4294967296.f), &sn, &cs);
        };
        auto accumulate = [&](float2 &a, float2 v, float sn, float cs) {
            a = __ffma2_rn(make_float2(v.x, v.x), make_float2(cs, sn), a);
            a = __ffma2_rn(make_float2(v.y, v.y), make_float2(-sn, cs), a);
        };
        if constexpr (MIRROR) {
            const int k2 = threadIdx.x % 32, r = threadIdx.x / 32;  // items (k2, r) and (k2, r + 4)
            float2 b0[N1], b1[N1];
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++) {
                b0[n1] = T[(r * N1 + n1) * kPad + k2];
                b1[n1] = T[((r + 4) * N1 + n1) * kPad + k2];
            }
            reg_fft<N1, +1>(b0);
            reg_fft<N1, +1>(b1);
            if (blk != 0 || r != 0) {  // a mirror pair: one factor for both rows
#pragma unroll
                for (int j = 0; j < N1; j++) {
                    const int col = k2 + 32 * bitrevc(j, G::LB);
                    float sn, cs;
                    fresnel(P[r * N + col], sn, cs);
                    accumulate(acc[0][j], b0[j], sn, cs);
                    accumulate(acc[1][j], b1[j], sn, cs);
                }
            } else {  // pair 0: rows 0 and N/2
#pragma unroll
                for (int j = 0; j < N1; j++) {
                    const int col = k2 + 32 * bitrevc(j, G::LB);
                    float sn, cs;
                    fresnel(P[r * N + col], sn, cs);
                    accumulate(acc[0][j], b0[j], sn, cs);
                    fresnel(P[(r + 4) * N + col], sn, cs);
                    accumulate(acc[1][j], b1[j], sn, cs);
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < G::PER; q++) {
                const int it = threadIdx.x + q * kRowThreads;
                if (it < G::ITEMS2) {
                    const int k2 = it % 32, r = it / 32;
                    float2 b[N1];
#pragma unroll
                    for (int n1 = 0; n1 < N1; n1++) b[n1] = T[(r * N1 + n1) * kPad + k2];
                    reg_fft<N1, +1>(b);
#pragma unroll
                    for (int j = 0; j < N1; j++) {
                        float sn, cs;
                        fresnel(P[r * N + k2 + 32 * bitrevc(j, G::LB)], sn, cs);
                        accumulate(acc[q][j], b[j], sn, cs);
                    }
                }
            }
        }
    }
    float2 *out = partial + (int64_t)group * N * N;
#pragma unroll
    for (int q = 0; q < G::PER; q++) {
        const int it = threadIdx.x + q * kRowThreads;
        if (it < G::ITEMS2) {
            const int k2 = it % 32, r = it / 32;
            float2 *o = out + (int64_t)row_of(r) * N + k2;
#pragma unroll
            for (int j = 0; j < N1; j++) o[32 * bitrevc(j, G::LB)] = acc[q][j];
        }
    }
}

template <int N1>
__global__ void __launch_bounds__(kRowThreads) tower_rows_finish_kernel(
    const float2 *__restrict__ partial, const int *__restrict__ tower_group_first,
    const int *__restrict__ tower_group_count, int group_cap, float2 *__restrict__ subimg,
    const float2 *__restrict__ tw)
{
    using G = RowGeom<N1>;
    constexpr int N = G::N, R = G::R;
    extern __shared__ float2 smem[];
    float2 *T = smem;
    float2 *W = smem + G::T_ELEMS;
    const int rstrips = N / R;
    const int tower = blockIdx.x / rstrips, row0 = (blockIdx.x % rstrips) * R;
    const int gfirst = tower_group_first[tower];
    int gcount = tower_group_count[tower];
    if (gfirst + gcount > group_cap) gcount = group_cap - gfirst;  // capacity overflow: rerun
    if (gcount <= 0) return;
    load_twiddles<N1>(W, tw);
    __syncthreads();
    for (int it = threadIdx.x; it < G::ITEMS1; it += blockDim.x) {
        const int n1 = it % N1, r = it / N1;
        float2 a[32];
#pragma unroll
        for (int n2 = 0; n2 < 32; n2++) a[n2] = make_float2(0.f, 0.f);
        for (int g = 0; g < gcount; g++) {
            const float2 *src = partial + ((int64_t)(gfirst + g) * N + row0 + r) * N + n1;
#pragma unroll
            for (int n2 = 0; n2 < 32; n2++) a[n2] = caddf(a[n2], src[n2 * N1]);
        }
        reg_fft<32, -1>(a);
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const int k2 = bitrevc(j, 5);
            T[(r * N1 + n1) * kPad + k2] = cmulf(a[j], twiddle<-1>(W, k2 * N1 + n1));
        }
    }
    __syncthreads();
    float2 *out = subimg + ((int64_t)tower * N + row0) * N;
    for (int it = threadIdx.x; it < G::ITEMS2; it += blockDim.x) {
        const int k2 = it % 32, r = it / 32;
        float2 b[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) b[n1] = T[(r * N1 + n1) * kPad + k2];
        reg_fft<N1, -1>(b);
#pragma unroll
        for (int j = 0; j < N1; j++) out[(int64_t)r * N + k2 + 32 * bitrevc(j, G::LB)] = b[j];
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
static size_t sparse_cols_smem() { return sizeof(float2) * (StripGeom<N1>::T_ELEMS + N1 * 32); }
template <int N1>
static size_t tower_rows_smem()
{
    return sizeof(float2) * (RowGeom<N1>::T_ELEMS + N1 * 32) + sizeof(uint32_t) * RowGeom<N1>::R * N1 * 32;
}
template <int N1>
static size_t tower_finish_smem() { return sizeof(float2) * (RowGeom<N1>::T_ELEMS + N1 * 32); }

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
static void cols_impl(cudaStream_t s, float2 *data, int batch, int sign, const float2 *tw, const int *live)
{
    const size_t sm = cols_smem<N1>();
    const unsigned blocks = (unsigned)batch * (N1 * 32 / ColGeom<N1>::C);
    if (sign < 0) {
        cudaFuncSetAttribute(fft32_cols_kernel<N1, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        fft32_cols_kernel<N1, -1><<<blocks, 256, sm, s>>>(data, tw, live);
    } else {
        cudaFuncSetAttribute(fft32_cols_kernel<N1, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        fft32_cols_kernel<N1, +1><<<blocks, 256, sm, s>>>(data, tw, live);
    }
}

template <int N1>
static void sparse_cols_impl(cudaStream_t s, float2 *slots, const unsigned *masks, const int *counts, int slot_cap,
                             const float2 *tw, int sm_count)
{
    const size_t sm = sparse_cols_smem<N1>();
    cudaFuncSetAttribute(sparse_cols_kernel<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sparse_cols_kernel<N1>, kSparseColThreads, sm);
    if (per_sm < 1) per_sm = 1;
    sparse_cols_kernel<N1><<<(unsigned)(per_sm * sm_count), kSparseColThreads, sm, s>>>(slots, masks, counts,
                                                                                        slot_cap, tw);
}

template <int N1>
static void tower_rows_impl(cudaStream_t s, float2 *slots, const unsigned *masks, const int *bin_of_slot,
                            const int *group_begin, const int *group_end, const int *range, const int *counts,
                            int slot_cap, int group_cap, const uint32_t *ph, float2 *partial, const float2 *tw)
{
    const int rstrips = RowGeom<N1>::N / RowGeom<N1>::R;
    const size_t sm1 = tower_rows_smem<N1>();
    cudaFuncSetAttribute(tower_rows_kernel<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1);
    if (group_cap > 0)
        tower_rows_kernel<N1><<<(unsigned)group_cap * rstrips, kRowThreads, sm1, s>>>(
            slots, masks, bin_of_slot, group_begin, group_end, range, counts, slot_cap, ph, partial, tw);
}

template <int N1>
static void tower_finish_impl(cudaStream_t s, int group_cap, const int *tower_group_first,
                              const int *tower_group_count, int ntowers, const float2 *partial, float2 *subimg,
                              const float2 *tw)
{
    const int rstrips = RowGeom<N1>::N / RowGeom<N1>::R;
    const size_t sm2 = tower_finish_smem<N1>();
    cudaFuncSetAttribute(tower_rows_finish_kernel<N1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
    tower_rows_finish_kernel<N1><<<(unsigned)ntowers * rstrips, kRowThreads, sm2, s>>>(
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

void launch_fft32_cols(cudaStream_t s, float2 *data, int batch, int n, int sign, const float2 *tw, const int *live)
{
#define CALL(N1) cols_impl<N1>(s, data, batch, sign, tw, live)
    RG_DISPATCH_N1(n, CALL)
#undef CALL
}

void launch_sparse_cols(cudaStream_t s, float2 *slots, const unsigned *masks, const int *counts, int slot_cap,
                        int subgrid, const float2 *tw, int sm_count)
{
#define CALL(N1) sparse_cols_impl<N1>(s, slots, masks, counts, slot_cap, tw, sm_count)
    RG_DISPATCH_N1(subgrid, CALL)
#undef CALL
}

void launch_tower_rows(cudaStream_t s, float2 *slots, const unsigned *masks, const int *bin_of_slot,
                       const int *group_begin, const int *group_end, const int *range, const int *counts,
                       int slot_cap, int group_cap, const uint32_t *ph, float2 *partial, int subgrid,
                       const float2 *tw)
{
#define CALL(N1) tower_rows_impl<N1>(s, slots, masks, bin_of_slot, group_begin, group_end, range, counts, \
                                     slot_cap, group_cap, ph, partial, tw)
    RG_DISPATCH_N1(subgrid, CALL)
#undef CALL
}

void launch_tower_finish(cudaStream_t s, int group_cap, const int *tower_group_first, const int *tower_group_count,
                         int ntowers, const float2 *partial, float2 *subimg, int subgrid, const float2 *tw)
{
#define CALL(N1) tower_finish_impl<N1>(s, group_cap, tower_group_first, tower_group_count, ntowers, partial, \
                                       subimg, tw)
    RG_DISPATCH_N1(subgrid, CALL)
#undef CALL
}

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

const double2 *fft64_twiddles(cudaStream_t s, int n) { return twiddles64(s, n); }

static void rows64(cudaStream_t s, double2 *data, int64_t rows, int n, int sign)
{
    const size_t sm = sizeof(double2) * 2 * n;
    cudaFuncSetAttribute(fft64_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const int threads = n / 2 < 512 ? (n / 2 > 32 ? n / 2 : 32) : 512;
    fft64_rows_kernel<<<(unsigned)rows, threads, sm, s>>>(data, n, sign, twiddles64(s, n));
}

void launch_fft64_pow2_rows(cudaStream_t s, double2 *data, int64_t rows, int n, int sign)
{
    rows64(s, data, rows, n, sign);
}

void launch_fft64_2d(cudaStream_t s, double2 *data, double2 *tmp, int batch, int ny, int nx, int sign,
                     double2 *work)
{
    launch_fft64_any_rows(s, data, (int64_t)batch * ny, nx, sign, work);
    dim3 blk(32, 8);
    dim3 g1((nx + 31) / 32, (ny + 31) / 32, batch);
    transpose64_kernel<<<g1, blk, 0, s>>>(data, tmp, ny, nx);
    launch_fft64_any_rows(s, tmp, (int64_t)batch * nx, ny, sign, work);
    dim3 g2((ny + 31) / 32, (nx + 31) / 32, batch);
    transpose64_kernel<<<g2, blk, 0, s>>>(tmp, data, nx, ny);
}

}  // namespace rg
