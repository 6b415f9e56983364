// Visibility preparation: per-visibility FP64 coordinate work done once, so the
// gridder reads a 16-byte record and an FP32 visibility.
//
// Coordinates follow the reference's arithmetic operation for operation, with
// explicit round-to-nearest intrinsics so nothing is contracted into an FMA:
//   frac_coord          src/reference/grid.c:37-57
//   w-plane selection   src/reference/grid.c:168-170
//   tower/floor cuts    src/reference/grid.c:357-367, 425-458, 244-254
// Record layout (int4): x = bin (tower*nfloor + floor, -1 = not gridded),
// y = row0 * side + col0, the linear index of the footprint origin (the
// reference's grid_offset; may be slightly negative at a tower's low edge),
// z = tap base index into the FP32 kernel table,
// w = ((row0 mod 64) << 8) | (col0 mod 64), the residues the Romein threads need.
#include <cfloat>

#include "rg_internal.h"

namespace rg {

__device__ __forceinline__ bool finite3(double a, double b, double c)
{
    return isfinite(a) && isfinite(b) && isfinite(c);
}

// block-wide min/max of w (min starts at 0, max at 0: grid.c:357-367)
__global__ void minmax_w_kernel(const double *__restrict__ u, const double *__restrict__ v,
                                const double *__restrict__ w, int64_t n,
                                unsigned long long *out_bits, unsigned *err)
{
    double lo = 0.0, hi = 0.0;
    bool bad = false;
    // four independent loads in flight per thread per round
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
        double ww[4];
#pragma unroll
        for (int k = 0; k < 4; k++) ww[k] = i0 + k * stride < n ? w[i0 + k * stride] : 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!isfinite(ww[k])) {  // u and v are checked by the binning kernel
                bad = true;
                continue;
            }
            lo = fmin(lo, ww[k]);
            hi = fmax(hi, ww[k]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    __shared__ double slo[32], shi[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        slo[wid] = lo;
        shi[wid] = hi;
    }
    if (bad) atomicOr(err, DERR_NONFINITE);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            lo = fmin(lo, slo[k]);
            hi = fmax(hi, shi[k]);
        }
        // min <= 0 and max >= 0: IEEE bit patterns order monotonically in
        // magnitude within one sign, so unsigned max works for both.
        if (lo < 0.0) atomicMax(out_bits + 0, (unsigned long long)__double_as_longlong(lo));
        if (hi > 0.0) atomicMax(out_bits + 1, (unsigned long long)__double_as_longlong(hi));
    }
}

void launch_minmax_w(cudaStream_t s, const double *u, const double *v, const double *w, int64_t n,
                     double *out2, unsigned *err)
{
    // out2 as bit patterns, both starting at +0.0 (all-zero bits): the range
    // always contains 0, and a negative minimum's pattern (sign bit set)
    // compares above zero as an unsigned integer.  A device memset keeps the
    // sequence free of host copies (it is replayed from a captured graph).
    cudaMemsetAsync(out2, 0, 2 * sizeof(double), s);
    // few CTAs: each ends with two atomics on the same two words, which
    // serialise in L2
    int blocks = (int)((n + 1023) / 1024);
    if (blocks > 512) blocks = 512;
    if (blocks < 1) blocks = 1;
    minmax_w_kernel<<<blocks, 256, 0, s>>>(u, v, w, n, (unsigned long long *)out2, err);
}

// Floors spanned by the w range (grid.c:357-367): wp = floor(w / winc + 0.5)
// for the range's ends (which include 0).
__global__ void w_floors_kernel(const double *__restrict__ wrange, double winc, int floors_cap,
                                int *__restrict__ range, unsigned *err)
{
    const int wp_min = (int)floor(wrange[0] / winc + 0.5);
    const int wp_max = (int)floor(wrange[1] / winc + 0.5);
    const long long nfloor = (long long)wp_max - wp_min + 1;
    range[0] = wp_min;
    range[1] = (int)(nfloor < (1 << 30) ? nfloor : (1 << 30));
    range[2] = nfloor <= floors_cap ? 1 : 0;
    if (nfloor > floors_cap) atomicOr(err, DERR_CAPACITY);
}

void launch_w_floors(cudaStream_t s, const double *wrange, double winc, int floors_cap, int *range,
                     unsigned *err)
{
    w_floors_kernel<<<1, 1, 0, s>>>(wrange, winc, floors_cap, range, err);
}

struct Bounds {
    double lo, hi, mid;
    int origin;
};

// tower bounds along one axis, grid.c:425-442
__device__ __forceinline__ Bounds tower_axis(int c, int chunk, int grid_size, double theta)
{
    Bounds b;
    b.origin = chunk * c - grid_size / 2;
    b.lo = __ddiv_rn(__dsub_rn((double)b.origin, 0.5), theta);
    b.hi = __dadd_rn(b.lo, __ddiv_rn((double)chunk, theta));
    b.mid = __ddiv_rn((double)(b.origin + chunk / 2), theta);
    return b;
}

// frac_coord along one axis: cell and sub-cell index
__device__ __forceinline__ void frac_axis(double coord, double mid, double theta, int ov,
                                          double half_over_ov, int &cell, int &frac)
{
    const double x = __dmul_rn(theta, __dsub_rn(coord, mid));
    cell = (int)floor(__dadd_rn(x, half_over_ov));
    frac = (int)floor(__dadd_rn(__dmul_rn(__dsub_rn(x, (double)cell), (double)ov), 0.5));
}

// cp.async (shared <- global) of 8 or 16 bytes, its commit and bounded-depth wait
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The (tower, w-floor) bin of a visibility with the reference's half-open
// cuts (grid.c:425-458 for the towers, :244-254 for the floors): the nearest
// chunk and floor are first guesses, the exact comparisons decide among their
// neighbours.  sb caches the per-chunk bounds when `cached`.
struct BinHit {
    int cx, cy, wp;
    Bounds bx, by;
};
__device__ __forceinline__ bool locate_bin(double uu, double vv, double ww, const TowerGeom &g, const Bounds *sb,
                                           bool cached, int wp_min, int wp_max, double inv_chunk, double inv_winc,
                                           BinHit &h)
{
    const double half_n = (double)(g.grid_size / 2);
    const int cxc = (int)floor((uu * g.theta + 0.5 + half_n) * inv_chunk);
    const int cyc = (int)floor((vv * g.theta + 0.5 + half_n) * inv_chunk);
    const int wpc = (int)floor(ww * inv_winc + 0.5);
    int found_cx = -1, found_cy = -1;
    for (int cy = cyc - 1; cy <= cyc + 1 && found_cy < 0; cy++) {
        if (cy < 0 || cy >= g.nchunk) continue;
        const Bounds t = cached ? sb[cy] : tower_axis(cy, g.chunk, g.grid_size, g.theta);
        if (vv < t.lo || vv >= t.hi) continue;
        found_cy = cy;
        h.by = t;
    }
    for (int cx = cxc - 1; cx <= cxc + 1 && found_cx < 0; cx++) {
        if (cx < 0 || cx >= g.nchunk) continue;
        const Bounds t = cached ? sb[cx] : tower_axis(cx, g.chunk, g.grid_size, g.theta);
        if (uu < t.lo || uu >= t.hi) continue;
        found_cx = cx;
        h.bx = t;
    }
    bool have_wp = false;
    for (int wp = wpc - 1; wp <= wpc + 1 && !have_wp; wp++) {
        if (wp < wp_min || wp > wp_max) continue;
        const double wlo = __dmul_rn(__dsub_rn((double)wp, 0.5), g.winc);
        const double whi = __dmul_rn(__dadd_rn((double)wp, 0.5), g.winc);
        if (ww < wlo || ww >= whi) continue;
        have_wp = true;
        h.wp = wp;
    }
    h.cx = found_cx;
    h.cy = found_cy;
    return found_cx >= 0 && found_cy >= 0 && have_wp;
}

constexpr int kPrepTile = 256;  // = the kernel's block size
constexpr int kPrepStages = 4;

__global__ void prepare_towers_kernel(const double *__restrict__ u, const double *__restrict__ v,
                                      const double *__restrict__ w, const double2 *__restrict__ vis,
                                      int64_t n, TowerGeom g, const int *__restrict__ range,
                                      int4 *__restrict__ rec, float2 *__restrict__ visf,
                                      int *__restrict__ active, unsigned char *__restrict__ marks,
                                      unsigned *err, unsigned long long *counters, float4 *__restrict__ feat)
{
    if (!range[2]) {
        // more floors than the bin capacity: the caller reruns.  Every record is
        // marked dropped so the gridding kernels of this pass read none of the
        // buffer's earlier contents.
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            rec[i] = make_int4(-1, 0, 0, 0);
        return;
    }
    const int wp_min = range[0], nfloor = range[1];
    const double half_over_ov = 0.5 / (double)g.ov;
    const int wp_max = wp_min + nfloor - 1;
    const int taps_total = g.planes * g.ov * g.ov * g.ksize * g.ksize;
    unsigned local_err = 0, gridded = 0, dropped = 0;
    // tower bounds per chunk index, computed once per CTA (three FP64
    // divisions each) when they fit; the per-visibility search reads them
    constexpr int kBoundsCache = 256;
    __shared__ Bounds sb[kBoundsCache];
    __shared__ __align__(16) double s_u[kPrepStages][kPrepTile], s_v[kPrepStages][kPrepTile],
        s_w[kPrepStages][kPrepTile];
    __shared__ __align__(16) double2 s_vz[kPrepStages][kPrepTile];
    const bool cached = g.nchunk <= kBoundsCache;
    if (cached)
        for (int c = threadIdx.x; c < g.nchunk; c += blockDim.x) sb[c] = tower_axis(c, g.chunk, g.grid_size, g.theta);
    __syncthreads();
    // first guesses only (the exact half-open tests below decide)
    const double inv_chunk = 1.0 / (double)g.chunk, inv_winc = 1.0 / g.winc;
    // one visibility: the binning, coordinates and marks below
    auto one = [&](int64_t i, double uu, double vv, double ww, double2 vz) {
        visf[i] = make_float2((float)vz.x, (float)vz.y);
        int4 r = make_int4(-1, 0, 0, 0);
        if (!finite3(uu, vv, ww)) {
            local_err |= DERR_NONFINITE;
            rec[i] = r;
            return;
        }
        BinHit h;
        if (!locate_bin(uu, vv, ww, g, sb, cached, wp_min, wp_max, inv_chunk, inv_winc, h)) {
            dropped++;
            rec[i] = r;
            return;
        }
        const int tower = h.cy * g.nchunk + h.cx;
        if (g.tower_sel && !g.tower_sel[tower]) {  // another share's tower
            rec[i] = r;
            return;
        }
        const int found_wp = h.wp;
        const Bounds &bx = h.bx, &by = h.by;
        int cell_x, frac_x, cell_y, frac_y;
        const double wmid = __dmul_rn((double)found_wp, g.winc);
        const double wr = __dsub_rn(ww, wmid);
        long long tap = 0;
        if (feat) {  // learned taps: continuous offsets, no table
            const double x = __dmul_rn(g.theta, __dsub_rn(uu, bx.mid));
            const double y = __dmul_rn(g.theta, __dsub_rn(vv, by.mid));
            const double fx = floor(x), fy = floor(y);
            cell_x = (int)fx;
            cell_y = (int)fy;
            feat[i] = make_float4((float)wr, (float)(x - fx), (float)(y - fy), 0.f);
        } else {
            frac_axis(uu, bx.mid, g.theta, g.ov, half_over_ov, cell_x, frac_x);
            frac_axis(vv, by.mid, g.theta, g.ov, half_over_ov, cell_y, frac_y);
            const int plane = (int)floor(__dadd_rn(__ddiv_rn(__dsub_rn(wr, g.wk_wmin), g.wk_wstep), 0.5));
            const int ks2 = g.ksize * g.ksize;
            tap = (long long)plane * g.ov * g.ov * ks2 + (long long)ks2 * (frac_y * g.ov + frac_x);
            if (plane < 0 || plane >= g.planes || tap < 0 || tap + ks2 > taps_total) {
                local_err |= DERR_PLANE_RANGE;
                rec[i] = r;
                return;
            }
        }
        const int col0 = cell_x + g.subgrid / 2 - g.ksize / 2;
        const int row0 = cell_y + g.subgrid / 2 - g.ksize / 2;
        const int bin = tower * nfloor + (found_wp - wp_min);
        r.x = bin;
        r.y = row0 * g.subgrid + col0;
        r.z = (int)tap;
        r.w = ((row0 & 63) << 8) | (col0 & 63);
        rec[i] = r;
        active[bin] = 1;
        // column strips (kStripCols wide) the footprint's taps land in; the
        // linear sub-grid index wraps a column past either edge into the
        // neighbouring row, i.e. to column (col mod S)
        unsigned char *mk = marks + (int64_t)bin * (g.subgrid / kStripCols);
        for (int c = col0; c < col0 + g.ksize; c += kStripCols) mk[(c & (g.subgrid - 1)) / kStripCols] = 1;
        mk[((col0 + g.ksize - 1) & (g.subgrid - 1)) / kStripCols] = 1;
        gridded++;
    };
    // Inputs in tiles of kPrepTile visibilities staged through shared memory by
    // cp.async, kPrepStages deep: each thread copies and then reads only its
    // own elements, so the wait on its copy groups is the only ordering needed
    // and kPrepStages - 1 tiles stay in flight while one is processed.
    const int tid = threadIdx.x;
    const int64_t ntiles = (n + kPrepTile - 1) / kPrepTile;
    auto fetch = [&](int64_t tile, int stage) {
        const int64_t i = tile * kPrepTile + tid;
        if (tile < ntiles && i < n) {
            cp_async8(&s_u[stage][tid], u + i);
            cp_async8(&s_v[stage][tid], v + i);
            cp_async8(&s_w[stage][tid], w + i);
            cp_async16(&s_vz[stage][tid], vis + i);
        }
        cp_async_commit();  // possibly empty: keeps the group count per tile
    };
    for (int s = 0; s < kPrepStages - 1; s++) fetch(blockIdx.x + (int64_t)s * gridDim.x, s);
    int k = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, k++) {
        fetch(tile + (int64_t)(kPrepStages - 1) * gridDim.x, (k + kPrepStages - 1) % kPrepStages);
        cp_async_wait<kPrepStages - 1>();
        const int stage = k % kPrepStages;
        const int64_t i = tile * kPrepTile + tid;
        if (i < n) one(i, s_u[stage][tid], s_v[stage][tid], s_w[stage][tid], s_vz[stage][tid]);
    }
    cp_async_wait<0>();
    if (local_err) atomicOr(err, local_err);
    // warp-aggregated counters
    for (int o = 16; o > 0; o >>= 1) {
        gridded += __shfl_xor_sync(0xffffffffu, gridded, o);
        dropped += __shfl_xor_sync(0xffffffffu, dropped, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (gridded) atomicAdd(counters + 0, (unsigned long long)gridded);
        if (dropped) atomicAdd(counters + 1, (unsigned long long)dropped);
    }
}

void launch_prepare_towers(cudaStream_t s, const double *u, const double *v, const double *w,
                           const double2 *vis, int64_t n, TowerGeom g, const int *range,
                           int4 *rec, float2 *visf, int *active, unsigned char *marks, unsigned *err,
                           unsigned long long *counters, float4 *feat)
{
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    prepare_towers_kernel<<<blocks, 256, 0, s>>>(u, v, w, vis, n, g, range, rec, visf, active, marks, err,
                                                 counters, feat);
}

// Tower census: visibilities per tower (shared-memory histogram when the
// towers fit, else global atomics) and the active (tower, floor) bins.
__global__ void tower_census_kernel(const double *__restrict__ u, const double *__restrict__ v,
                                    const double *__restrict__ w, int64_t n, TowerGeom g,
                                    const int *__restrict__ range, unsigned long long *__restrict__ vis_count,
                                    int *__restrict__ active, int ntowers, unsigned *err)
{
    if (!range[2]) return;  // more floors than the capacity: reported by the w-floors kernel
    const int wp_min = range[0], nfloor = range[1];
    const int wp_max = wp_min + nfloor - 1;
    constexpr int kBoundsCache = 256, kHist = 2048;
    __shared__ Bounds sb[kBoundsCache];
    __shared__ unsigned hist[kHist];
    const bool cached = g.nchunk <= kBoundsCache;
    const bool local = ntowers <= kHist;
    if (cached)
        for (int c = threadIdx.x; c < g.nchunk; c += blockDim.x) sb[c] = tower_axis(c, g.chunk, g.grid_size, g.theta);
    if (local)
        for (int t = threadIdx.x; t < ntowers; t += blockDim.x) hist[t] = 0;
    __syncthreads();
    const double inv_chunk = 1.0 / (double)g.chunk, inv_winc = 1.0 / g.winc;
    bool bad = false;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double uu = u[i], vv = v[i], ww = w[i];
        if (!finite3(uu, vv, ww)) {
            bad = true;
            continue;
        }
        BinHit h;
        if (!locate_bin(uu, vv, ww, g, sb, cached, wp_min, wp_max, inv_chunk, inv_winc, h)) continue;
        const int tower = h.cy * g.nchunk + h.cx;
        active[(int64_t)tower * nfloor + (h.wp - wp_min)] = 1;
        if (local) atomicAdd(&hist[tower], 1u);
        else atomicAdd(vis_count + tower, 1ull);
    }
    if (bad) atomicOr(err, DERR_NONFINITE);
    __syncthreads();
    if (local)
        for (int t = threadIdx.x; t < ntowers; t += blockDim.x)
            if (hist[t]) atomicAdd(vis_count + t, (unsigned long long)hist[t]);
}

__global__ void tower_floors_kernel(const int *__restrict__ active, const int *__restrict__ range, int ntowers,
                                    int *__restrict__ floors)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntowers) return;
    int c = 0;
    if (range[2])
        for (int f = 0; f < range[1]; f++) c += active[(int64_t)t * range[1] + f] != 0;
    floors[t] = c;
}

void launch_tower_census(cudaStream_t s, const double *u, const double *v, const double *w, int64_t n,
                         TowerGeom g, const int *range, unsigned long long *vis_count, int *active, int *floors,
                         int ntowers, int floors_cap, unsigned *err)
{
    (void)floors_cap;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    if (n > 0) tower_census_kernel<<<blocks, 256, 0, s>>>(u, v, w, n, g, range, vis_count, active, ntowers, err);
    tower_floors_kernel<<<(ntowers + 127) / 128, 128, 0, s>>>(active, range, ntowers, floors);
}

__global__ void prepare_wproj_kernel(const double *__restrict__ u, const double *__restrict__ v,
                                     const double *__restrict__ w, const double2 *__restrict__ vis,
                                     int64_t n, int grid_size, double theta, int ksize, int ov,
                                     int planes, double wk_wmin, double wk_wstep,
                                     int4 *__restrict__ rec, float2 *__restrict__ visf,
                                     unsigned *err)
{
    const double half_over_ov = 0.5 / (double)ov;
    const int ks2 = ksize * ksize;
    const long long taps_total = (long long)planes * ov * ov * ks2;
    unsigned local_err = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double uu = u[i], vv = v[i], ww = w[i];
        const double2 vz = vis[i];
        visf[i] = make_float2((float)vz.x, (float)vz.y);
        int4 r = make_int4(-1, 0, 0, 0);
        if (!finite3(uu, vv, ww)) {
            local_err |= DERR_NONFINITE;
            rec[i] = r;
            continue;
        }
        int cell_x, frac_x, cell_y, frac_y;
        frac_axis(uu, 0.0, theta, ov, half_over_ov, cell_x, frac_x);
        frac_axis(vv, 0.0, theta, ov, half_over_ov, cell_y, frac_y);
        const int plane = (int)floor(__dadd_rn(__ddiv_rn(__dsub_rn(__dsub_rn(ww, 0.0), wk_wmin), wk_wstep), 0.5));
        const long long tap = (long long)plane * ov * ov * ks2 + (long long)ks2 * (frac_y * ov + frac_x);
        if (plane < 0 || plane >= planes || tap < 0 || tap + ks2 > taps_total) {
            local_err |= DERR_PLANE_RANGE;
            rec[i] = r;
            continue;
        }
        const int col0 = cell_x + grid_size / 2 - ksize / 2;
        const int row0 = cell_y + grid_size / 2 - ksize / 2;
        if (col0 < -ksize || col0 > grid_size || row0 < -ksize || row0 > grid_size) {
            local_err |= DERR_GRID_RANGE;
            rec[i] = r;
            continue;
        }
        r.x = 0;
        r.y = row0 * grid_size + col0;
        r.z = (int)tap;
        r.w = ((row0 + 64) << 16) | (col0 + 64);  // the origin itself: Romein checks each axis
        rec[i] = r;
    }
    if (local_err) atomicOr(err, local_err);
}

void launch_prepare_wproj(cudaStream_t s, const double *u, const double *v, const double *w,
                          const double2 *vis, int64_t n, int grid_size, double theta, int ksize,
                          int ov, int planes, double wk_wmin, double wk_wstep, int4 *rec,
                          float2 *visf, unsigned *err)
{
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    prepare_wproj_kernel<<<blocks, 256, 0, s>>>(u, v, w, vis, n, grid_size, theta, ksize, ov,
                                                planes, wk_wmin, wk_wstep, rec, visf, err);
}

// Block-wide exclusive scan (blockDim a multiple of 32, <= 1024).  Returns the
// exclusive prefix of x; *total receives the block sum.  warp_sums: 32 ints of
// shared memory.  Must be called by every thread of the block.
__device__ int block_exclusive_scan(int x, int *warp_sums, int *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int incl = x;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int y = lane < nw ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += t;
        }
        if (lane < nw) warp_sums[lane] = y;
    }
    __syncthreads();
    const int excl = (wid > 0 ? warp_sums[wid - 1] : 0) + incl - x;
    *total = warp_sums[nw - 1];
    __syncthreads();
    return excl;
}

// Single-CTA compaction of active (tower, floor) bins into slots, in bin order,
// so each tower's slots are contiguous and ordered by floor; then the floor
// groups of the column stage (up to G consecutive slots of one tower, G chosen
// so the stage has about target_items (group, strip) work items).
__global__ void compact_bins_kernel(const int *__restrict__ active, const int *__restrict__ range,
                                    int *__restrict__ slot_of_bin, int *__restrict__ bin_of_slot,
                                    int *__restrict__ counts, int *__restrict__ tower_first,
                                    int *__restrict__ tower_count, int ntowers, int strips,
                                    int target_items, int *__restrict__ group_begin,
                                    int *__restrict__ group_end, int *__restrict__ tower_group_first,
                                    int *__restrict__ tower_group_count)
{
    __shared__ int warp_sums[32];
    const int nfloor = range[2] ? range[1] : 0;
    const int nbins = ntowers * nfloor;
    int carry = 0;
    for (int base = 0; base < nbins; base += blockDim.x) {
        const int b = base + threadIdx.x;
        const int a = (b < nbins && active[b]) ? 1 : 0;
        int total;
        const int excl = carry + block_exclusive_scan(a, warp_sums, &total);
        if (b < nbins) slot_of_bin[b] = excl;  // exclusive prefix for now
        if (a) bin_of_slot[excl] = b;
        carry += total;
    }
    const int n_active = carry;
    __syncthreads();
    for (int t = threadIdx.x; t < ntowers; t += blockDim.x) {
        const int first = nfloor ? slot_of_bin[t * nfloor] : 0;
        const int next = (t + 1 < ntowers && nfloor) ? slot_of_bin[(t + 1) * nfloor] : n_active;
        tower_first[t] = first;
        tower_count[t] = next - first;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        if (!active[b]) slot_of_bin[b] = -1;
    long long want = ((long long)n_active * strips + target_items - 1) / (target_items > 0 ? target_items : 1);
    int G = (int)(want < 4 ? 4 : (want > 64 ? 64 : want));
    carry = 0;
    int with_data = 0;
    for (int base = 0; base < ntowers; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const int cnt = t < ntowers ? tower_count[t] : 0;
        const int ng = (cnt + G - 1) / G;
        int total;
        const int gfirst = carry + block_exclusive_scan(ng, warp_sums, &total);
        if (t < ntowers) {
            with_data += cnt > 0;
            tower_group_first[t] = gfirst;
            tower_group_count[t] = ng;
            const int sfirst = tower_first[t];
            for (int j = 0; j < ng; j++) {
                const int b0 = sfirst + j * G;
                const int b1 = b0 + G < sfirst + cnt ? b0 + G : sfirst + cnt;
                group_begin[gfirst + j] = b0;
                group_end[gfirst + j] = b1;
            }
        }
        carry += total;
    }
    int total_with_data;
    const int unused = block_exclusive_scan(with_data, warp_sums, &total_with_data);
    (void)unused;
    if (threadIdx.x == 0) {
        counts[0] = n_active;
        counts[1] = carry;
        counts[2] = total_with_data;
        counts[3] = 0;  // marked column strips, counted by the mask kernel
    }
}

void launch_compact_bins(cudaStream_t s, const int *active, const int *range, int *slot_of_bin,
                         int *bin_of_slot, int *counts, int *tower_first, int *tower_count,
                         int ntowers, int strips, int target_items, int *group_begin,
                         int *group_end, int *tower_group_first, int *tower_group_count)
{
    compact_bins_kernel<<<1, 1024, 0, s>>>(active, range, slot_of_bin, bin_of_slot, counts,
                                           tower_first, tower_count, ntowers, strips, target_items,
                                           group_begin, group_end, tower_group_first,
                                           tower_group_count);
}

}  // namespace rg
