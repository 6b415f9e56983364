// W-towers helpers: the Fresnel phase table and the owner-computes add-back of
// the towers' sub-grids into the FP64 master grid.
#include "rg_internal.h"

namespace rg {

// ph = winc (1 - sqrt(1 - l^2 - m^2)) for the fft-shifted pixel (y, x), i.e.
// the reference's transfer pattern phase before cexp, at centred coordinates
// ((x + S/2) mod S, (y + S/2) mod S) (src/reference/grid.c:304-319 followed by
// fft_shift), computed in FP64 with round-to-nearest intrinsics (no
// contraction) and stored as its fraction of a turn in 32-bit fixed point:
// phq[y*S + x] = round(frac(ph) 2^32) mod 2^32.  The row stage raises
// exp(2 pi i ph) to the power -wp as the integer product -wp * phq mod 2^32,
// exact to |wp| 2^-33 turns.
__global__ void fresnel_table_kernel(uint32_t *__restrict__ phq, int S, double theta, double winc)
{
    const int64_t total = (int64_t)S * S;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(k / S), x = (int)(k % S);
        const int xc = (x + S / 2) % S, yc = (y + S / 2) % S;
        const double l = __ddiv_rn(__dmul_rn(theta, (double)(xc - S / 2)), (double)S);
        const double m = __ddiv_rn(__dmul_rn(theta, (double)(yc - S / 2)), (double)S);
        const double r = __dsqrt_rn(__dsub_rn(__dsub_rn(1.0, __dmul_rn(l, l)), __dmul_rn(m, m)));
        const double ph = __dmul_rn(winc, __dsub_rn(1.0, r));
        const double frac = __dsub_rn(ph, floor(ph));  // [0, 1), exact
        phq[k] = (uint32_t)__double2ull_rn(ldexp(frac, 32));  // 2^32 wraps to 0
    }
}

void launch_fresnel_table(cudaStream_t s, uint32_t *phq, int subgrid, double theta, double winc)
{
    const int64_t total = (int64_t)subgrid * subgrid;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    fresnel_table_kernel<<<blocks, 256, 0, s>>>(phq, subgrid, theta, winc);
}

// a / d for 0 <= a < 2^24, d > 0: float reciprocal estimate, corrected to the
// exact quotient (saves the integer division sequence).
__device__ __forceinline__ int div_nonneg(int a, int d, float inv)
{
    int q = __float2int_rz((float)a * inv);
    if (q * d > a) q--;
    else if ((q + 1) * d <= a) q++;
    return q;
}

// Owner-computes add-back (src/reference/grid.c:503-516): every master pixel
// sums, in tower order (cy, then cx), the overlapping towers' forward-
// transformed sub-images divided by S^2, in FP64.  Deterministic.
// When a capacity overflowed (range[2] == 0 or a live count above its
// capacity) nothing is written, so the caller can rerun on the same grid.  In
// a batch (poison != nullptr) an overflow also stops the later passes' writes
// until the batch reruns them.
constexpr int kAddBackRows = 4;

__global__ void add_back_kernel(const float2 *__restrict__ subimg, const int *__restrict__ tower_count,
                                double2 *__restrict__ master, int N, int S, int M, int chunk,
                                int nchunk, int overwrite, const int *__restrict__ range,
                                const int *__restrict__ counts, int slot_cap, int group_cap, int *poison)
{
    const int gx = blockIdx.x * blockDim.x + threadIdx.x;
    if (gx >= N) return;
    if (range && (!range[2] || counts[0] > slot_cap || counts[1] > group_cap)) {
        if (poison) *poison = 1;  // later passes of a batch may see unconsumed sub-grids
        return;
    }
    if (poison && *poison) return;
    const int ax = gx + M / 2;  // x + N/2 + M/2 with x = gx - N/2
    const float inv = 1.0f / (float)chunk;
    int cx_hi = div_nonneg(ax, chunk, inv);
    const int cx_lo = (ax - S) >= 0 ? div_nonneg(ax - S, chunk, inv) + 1 : 0;
    if (cx_hi >= nchunk) cx_hi = nchunk - 1;
    // S is a power of two, so 1 / S^2 is exact and multiplying by it gives
    // the quotient the division would, bit for bit
    const double inv_norm = 1.0 / (double)(S * S);
    // kAddBackRows rows per thread, blockDim.y apart (the column's tower range
    // is found once)
    const int gy_end = min(N, (int)(blockIdx.y + 1) * (int)blockDim.y * kAddBackRows);
#pragma unroll 1
    for (int gy = blockIdx.y * blockDim.y * kAddBackRows + threadIdx.y; gy < gy_end; gy += blockDim.y) {
        const int ay = gy + M / 2;
        int cy_hi = div_nonneg(ay, chunk, inv);
        const int cy_lo = (ay - S) >= 0 ? div_nonneg(ay - S, chunk, inv) + 1 : 0;
        if (cy_hi >= nchunk) cy_hi = nchunk - 1;
        const int64_t at = (int64_t)gy * N + gx;
        double2 acc = overwrite ? make_double2(0.0, 0.0) : master[at];
        for (int cy = cy_lo; cy <= cy_hi; cy++) {
            const int sy = ay - chunk * cy;
            if (sy < 0 || sy >= S) continue;
            for (int cx = cx_lo; cx <= cx_hi; cx++) {
                const int sx = ax - chunk * cx;
                if (sx < 0 || sx >= S) continue;
                const int t = cy * nchunk + cx;
                if (tower_count[t] == 0) continue;
                const float2 z = subimg[(int64_t)t * S * S + (int64_t)sy * S + sx];
                acc.x += (double)z.x * inv_norm;
                acc.y += (double)z.y * inv_norm;
            }
        }
        master[at] = acc;
    }
}

void launch_add_back(cudaStream_t s, const float2 *subimg, const int *tower_count, double2 *master,
                     int grid_size, int subgrid, int margin, int chunk, int nchunk, int overwrite,
                     const int *range, const int *counts, int slot_cap, int group_cap, int *poison)
{
    dim3 blk(32, 8);
    dim3 grd((grid_size + 31) / 32, (grid_size + 8 * kAddBackRows - 1) / (8 * kAddBackRows));
    add_back_kernel<<<grd, blk, 0, s>>>(subimg, tower_count, master, grid_size, subgrid, margin,
                                        chunk, nchunk, overwrite, range, counts, slot_cap, group_cap, poison);
}

}  // namespace rg
