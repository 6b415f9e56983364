// Romein scatter gridder (Romein 2012, "An efficient work-distribution
// strategy for gridding radio-telescope data on GPUs"), FP32.
//
// A CTA has K*K threads; thread (myU, myV) owns the grid points whose column is
// congruent to myU and row to myV modulo K.  For each visibility with footprint
// origin (col0, row0) exactly one tap of the K x K footprint falls on a point
// the thread owns: column col0 + ((myU - col0) mod K), likewise for rows.  The
// thread keeps a register sum for its current point and only flushes it (one
// 8-byte vector atomic) when the point or the (tower, floor) sub-grid changes,
// so visibilities that move slowly along a baseline track coalesce in
// registers.  Per tap: sum += vis * conj(tap), the reference's
// grid += v * conj(wk) (src/reference/grid.c:177-182), as two packed-pair
// fused multiply-adds: sum + tap.y (vis.y, -vis.x) + tap.x (vis.x, vis.y),
// the same roundings as the scalar form.
//
// Sub-grids of the W-towers pass (STRIP): the linear index grid_offset + cv *
// side + cu is the reference's grid_offset + y*size + x (grid.c:177-182),
// mapped to the strip-major layout (whose kernel table holds every slice
// twice); points outside [0, side^2) are dropped.  The record carries
// grid_offset and the footprint origin's residues modulo 64.
// The W-projection grid (not STRIP): each tap's column and row are checked
// separately and taps outside [0, side) on either axis are dropped, as the
// reference GPU gridder does (src/grid/grid_cuda.cu:25-41; the CPU grid.c
// checks nothing, so a footprint crossing the left or right edge would wrap
// into the neighbouring row).  The record carries the origin itself,
// r.w = (row0 + 64) << 16 | (col0 + 64).  Either way a thread's tap (cu, cv)
// is two subtractions and masks (K divides 64).
//
// Visibilities are staged through shared memory in batches (coalesced 16-byte
// record and 8-byte visibility loads); taps are read through the read-only
// cache, one oversampled K x K slice per visibility.
#include "rg_internal.h"

namespace rg {

// P grid points per thread: thread (myU, myV0) owns the points of column
// residue myU and row residues myV0 + j*K/P, j < P, so a visibility's record is
// decoded once for P taps.  A visibility whose sub-grid, linear origin and
// origin residues equal the previous one's (about half of them along a track)
// skips the per-point change tests: all of the thread's points are unchanged.
// Occupancy floor for the register allocator: 48 resident warps per SM (24
// with eight points per thread), at most 32 CTAs.
template <int K, int P>
struct RomeinBounds {
    static constexpr int NT = K * K / P;
    static constexpr int want = (P >= 8 ? 768 : 1536) / NT;
    static constexpr int min_ctas = want > 32 ? 32 : (want < 1 ? 1 : want);
};

// F64 (row-major grids only): taps are read from the caller's FP64 table and
// rounded to FP32 as they are loaded, exactly as the table conversion rounds
// them, for calls whose taps are fewer than the table's entries.
template <int K, int P, bool STRIP, bool F64 = false>
__global__ void __launch_bounds__(K *K / P, (RomeinBounds<K, P>::min_ctas)) romein_kernel(
    const int4 *__restrict__ rec, const float2 *__restrict__ visf, int64_t n,
    const float2 *__restrict__ taps, const double2 *__restrict__ taps64, float2 *__restrict__ grids,
    const int *__restrict__ slot_of_bin, int64_t grid_stride, int side, int64_t chunk, int slot_cap, int strip_lg)
{
    constexpr int NT = K * K / P;     // threads
    constexpr int BATCH = 256;        // visibilities staged per round
    constexpr int RS = K / P;         // row stride between a thread's points
    __shared__ int4 srec[BATCH];
    __shared__ float2 svis[BATCH];
    const int myU = threadIdx.x % K, myV0 = threadIdx.x / K;
    // Each point is tracked by its key: its element offset in the grid (the
    // strip-major address for sub-grids), or -1 when it lies off the grid.
    // Keys are equal exactly when the points are.

    for (int64_t c0 = (int64_t)blockIdx.x * chunk; c0 < n; c0 += (int64_t)gridDim.x * chunk) {
        const int64_t c1 = c0 + chunk < n ? c0 + chunk : n;
        int cur_bin = -1, cur_goff = 0, cur_res = 0;
        float2 *cur_grid = nullptr;  // the current bin's sub-grid (null: past the slot capacity)
        int cur_key[P];
        float2 sum[P];
#pragma unroll
        for (int p = 0; p < P; p++) {
            cur_key[p] = -1;
            sum[p] = make_float2(0.f, 0.f);
        }
        for (int64_t b0 = c0; b0 < c1; b0 += BATCH) {
            const int cnt = (int)(c1 - b0 < BATCH ? c1 - b0 : BATCH);
            __syncthreads();
            for (int j = threadIdx.x; j < cnt; j += NT) {
                srec[j] = rec[b0 + j];
                svis[j] = visf[b0 + j];
            }
            __syncthreads();
            for (int j = 0; j < cnt; j++) {
                const int4 r = srec[j];
                if (r.x < 0) continue;
                const int cu = (myU - (r.w & 0xff)) & (K - 1);
                // slice row of the thread's first point
                const int cv0 = (myV0 - (STRIP ? (r.w >> 8) : (r.w >> 16))) & (K - 1);
                float2 t[P];
                if (STRIP) {
                    // duplicated slices (2K rows): rows cv0 + p*RS need no wrap, so the
                    // loads are one base plus compile-time offsets
                    const float2 *tp = taps + 2 * (int64_t)r.z + cv0 * K + cu;
#pragma unroll
                    for (int p = 0; p < P; p++) t[p] = __ldg(tp + p * RS * K);
                } else if (F64) {
#pragma unroll
                    for (int p = 0; p < P; p++) {
                        const double2 d = __ldg(taps64 + r.z + ((cv0 + p * RS) & (K - 1)) * K + cu);
                        t[p] = make_float2((float)d.x, (float)d.y);
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < P; p++) t[p] = __ldg(taps + r.z + ((cv0 + p * RS) & (K - 1)) * K + cu);
                }
                const float2 vz = svis[j];
                const float2 vzr = make_float2(vz.y, -vz.x);
                // in a sub-grid goff alone fixes the origin (its columns span
                // chunk + 1 < S values), hence the residues
                if (r.x == cur_bin && r.y == cur_goff && (STRIP || r.w == cur_res)) {
                    // same sub-grid and footprint origin: every point unchanged
#pragma unroll
                    for (int p = 0; p < P; p++) {
                        sum[p] = __ffma2_rn(make_float2(t[p].y, t[p].y), vzr, sum[p]);
                        sum[p] = __ffma2_rn(make_float2(t[p].x, t[p].x), vz, sum[p]);
                    }
                    continue;
                }
                cur_goff = r.y;
                cur_res = r.w;
                int key[P];
                if (STRIP) {
                    // the thread's points share one linear column: L = base + cv*S has
                    // column base mod S and row floor(base / S) + cv, so the strip-major
                    // address is a column part plus 8 per row (strip_addr, unrolled)
                    const int base = r.y + cu;
                    const int col = base & (side - 1);
                    const int colpart = ((col >> 3) << (strip_lg + 3)) + (col & 7);
                    const int rowb = base >> strip_lg;
                    if (rowb >= 0 && rowb + K <= side) {
                        // every footprint row inside: the thread's row offsets cv0 + p RS
                        // (mod K) rise by RS and wrap once, at p = pw
                        const int key0 = colpart + ((rowb + cv0) << 3);
                        const int pw = (K - cv0 + RS - 1) / RS;
#pragma unroll
                        for (int p = 0; p < P; p++) key[p] = key0 + ((p * RS) << 3) - (p >= pw ? (K << 3) : 0);
                    } else {
#pragma unroll
                        for (int p = 0; p < P; p++) {
                            const int row = rowb + ((cv0 + p * RS) & (K - 1));
                            key[p] = (unsigned)row < (unsigned)side ? colpart + (row << 3) : -1;
                        }
                    }
                } else {
                    // per-axis check; -1 (never flushed) for a tap off the grid
                    const int col = (r.w & 0xffff) - 64 + cu;
                    const int row0 = (r.w >> 16) - 64;
#pragma unroll
                    for (int p = 0; p < P; p++) {
                        const int row = row0 + ((cv0 + p * RS) & (K - 1));
                        key[p] = ((unsigned)col < (unsigned)side && (unsigned)row < (unsigned)side) ? row * side + col
                                                                                                  : -1;
                    }
                }
                if (r.x != cur_bin) {
#pragma unroll
                    for (int p = 0; p < P; p++) {
                        if (cur_grid && cur_key[p] >= 0) atomicAdd(cur_grid + cur_key[p], sum[p]);
                        cur_key[p] = key[p];
                        sum[p] = make_float2(0.f, 0.f);
                    }
                    cur_bin = r.x;
                    const int slot = slot_of_bin[cur_bin];
                    cur_grid = slot < slot_cap ? grids + (int64_t)slot * grid_stride : nullptr;
                }
#pragma unroll
                for (int p = 0; p < P; p++) {
                    if (key[p] != cur_key[p]) {
                        if (cur_grid && cur_key[p] >= 0) atomicAdd(cur_grid + cur_key[p], sum[p]);
                        cur_key[p] = key[p];
                        sum[p] = make_float2(0.f, 0.f);
                    }
                    sum[p] = __ffma2_rn(make_float2(t[p].y, t[p].y), vzr, sum[p]);
                    sum[p] = __ffma2_rn(make_float2(t[p].x, t[p].x), vz, sum[p]);
                }
            }
        }
        if (cur_grid) {
#pragma unroll
            for (int p = 0; p < P; p++)
                if (cur_key[p] >= 0) atomicAdd(cur_grid + cur_key[p], sum[p]);
        }
    }
}

template <int K, int P>
static void romein_launch(cudaStream_t s, const int4 *rec, const float2 *visf, int64_t n, const float2 *taps,
                          const double2 *taps64, float2 *grids, const int *slot_of_bin, int64_t grid_stride,
                          int grid_side, int sm_count, int slot_cap, int strip_lg)
{
    // Every CTA resident at once, each with an equal contiguous run of
    // visibilities: occupancy, not the chunk size, decides the grid.
    constexpr int NT = K * K / P;
    int per_sm = 0;  // of the instantiation that runs (the register counts can differ)
    if (strip_lg)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, romein_kernel<K, P, true>, NT, 0);
    else if (taps64)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, romein_kernel<K, P, false, true>, NT, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, romein_kernel<K, P, false>, NT, 0);
    if (per_sm < 1) per_sm = 1;
    int64_t blocks = (int64_t)sm_count * per_sm;
    int64_t chunk = (n + blocks - 1) / blocks;
    if (chunk < 8) chunk = 8;
    blocks = (n + chunk - 1) / chunk;
    if (blocks < 1) blocks = 1;
    if (strip_lg)
        romein_kernel<K, P, true><<<(unsigned)blocks, NT, 0, s>>>(rec, visf, n, taps, nullptr, grids, slot_of_bin,
                                                                  grid_stride, grid_side, chunk, slot_cap, strip_lg);
    else if (taps64)
        romein_kernel<K, P, false, true><<<(unsigned)blocks, NT, 0, s>>>(rec, visf, n, nullptr, taps64, grids,
                                                                         slot_of_bin, grid_stride, grid_side, chunk,
                                                                         slot_cap, 0);
    else
        romein_kernel<K, P, false><<<(unsigned)blocks, NT, 0, s>>>(rec, visf, n, taps, nullptr, grids, slot_of_bin,
                                                                   grid_stride, grid_side, chunk, slot_cap, 0);
}

void launch_romein(cudaStream_t s, const int4 *rec, const float2 *visf, int64_t n,
                   const float2 *taps, float2 *grids, const int *slot_of_bin, int64_t grid_stride,
                   int grid_side, int ksize, int sm_count, int slot_cap, int points, int strip_lg,
                   const double2 *taps64)
{
    if (strip_lg) taps64 = nullptr;  // sub-grids always read the converted, duplicated table
#define RG_ROMEIN(K, P) \
    romein_launch<K, P>(s, rec, visf, n, taps, taps64, grids, slot_of_bin, grid_stride, grid_side, sm_count, \
                        slot_cap, strip_lg)
    switch (ksize) {
        case 4: RG_ROMEIN(4, 1); break;
        case 8:
            if (points == 1) RG_ROMEIN(8, 1);
            else if (points == 4) RG_ROMEIN(8, 4);
            else RG_ROMEIN(8, 2);
            break;
        case 16:
            if (points == 2) RG_ROMEIN(16, 2);
            else if (points == 8) RG_ROMEIN(16, 8);
            else RG_ROMEIN(16, 4);
            break;
        case 32:
            if (points == 8) RG_ROMEIN(32, 8);
            else RG_ROMEIN(32, 4);
            break;
        default: break;
    }
#undef RG_ROMEIN
}

}  // namespace rg
