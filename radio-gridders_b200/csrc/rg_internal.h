// Internal declarations shared by the C-ABI layer (rg_api.cu) and the kernel
// files.  Not installed; the public interface is include/radio_gridders.h.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <vector>
#include <string>

#include "../../include/radio_gridders.h"

namespace rg {

// ---------------------------------------------------------------------------
// status / errors
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
rg_status fail(rg_status st, const std::string &msg);
rg_status cuda_fail(cudaError_t e, const char *what);

#define RG_CUDA(call)                                                  \
    do {                                                               \
        cudaError_t rg_e_ = (call);                                    \
        if (rg_e_ != cudaSuccess) return ::rg::cuda_fail(rg_e_, #call); \
    } while (0)

#define RG_CHECK(call)                     \
    do {                                   \
        rg_status rg_s_ = (call);          \
        if (rg_s_ != RG_OK) return rg_s_;  \
    } while (0)

// ---------------------------------------------------------------------------
// device error word written by kernels (bit flags)
// ---------------------------------------------------------------------------
enum DeviceError : unsigned {
    DERR_NONFINITE = 1u << 0,     // NaN/Inf in u, v, w
    DERR_PLANE_RANGE = 1u << 1,   // w outside the kernel table
    DERR_GRID_RANGE = 1u << 2,    // footprint leaves the grid (W-projection)
    DERR_CAPACITY = 1u << 3,      // internal capacity exceeded
    DERR_TIMEOUT = 1u << 4,       // a bounded wait for tensor-core work gave up
};

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct Buffer {
    void *ptr = nullptr;
    size_t bytes = 0;
};

// Learned taps for the W-towers gridder (the network of an rg_mlp).
struct LearnedTaps {
    const float *P;
    const void *PB;
    int ksize;
    float inv_wmax, scale;
    double wmax;
};
// part_of_tower (ntowers entries) with part: grid only the towers t with
// part_of_tower[t] == part (one share of a tower-partitioned observation).
rg_status grid_wtowers_impl(rg_context *ctx, double *uvgrid, int grid_size, double theta, const rg_vis *vis,
                            const rg_wkern *wkern, const LearnedTaps *lt, int subgrid_size, int subgrid_margin,
                            double wincrement, int flags, const int32_t *part_of_tower = nullptr, int part = 0);

}  // namespace rg

// Schedule knobs of a W-towers pass (picked by the autotuner).
struct TowerTuning {
    int romein_points = 8;  // grid points per Romein thread (threads per CTA = K^2 / points)
    int group_items = 8;    // row-stage work items per SM (sets the floor-group size)
};

struct TowerPlan {
    bool valid = false;
    int floors_cap = 0, slots_cap = 0, groups_cap = 0;
    int seen_floors = 0, seen_slots = 0, seen_groups = 0;
    size_t zeroed_slots = 0;  // sub-grids known to be zero (cleared on consumption)
    TowerTuning tune;
    bool tuned = false;
    cudaGraphExec_t graph_exec = nullptr;  // captured pass for graph_key's buffers
    std::string graph_key;
    int graph_launches = 0;
    uint64_t graph_scratch_gen = 0;  // scratch generation the graph's pointers belong to
    const unsigned char *tower_sel = nullptr;  // device: the towers this plan grids (nullptr: all)
};

struct rg_stage_event {
    std::string name;
    cudaEvent_t start = nullptr, stop = nullptr;
};

struct rg_context {
    int device = 0;
    bool profiling = false;
    std::vector<rg_stage_event> events;  // pool, reused across calls
    int n_events = 0;                    // used by the current call
    std::vector<std::pair<std::string, float>> timings;  // last call
    std::map<std::string, TowerPlan> tower_plans;         // capacities per W-towers shape
    const TowerPlan *slots_owner = nullptr;               // plan whose pass last used "slots"
    int sm_count = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::map<std::string, rg::Buffer> scratch;
    uint64_t scratch_gen = 0;  // bumped on every scratch (re)allocation: captured graphs go stale
    // batched W-towers calls: copy streams, their events, per-step diagnostics
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    static constexpr int kBatchSets = 3;  // staging sets of a batch call
    cudaEvent_t ev_in[kBatchSets] = {}, ev_used[kBatchSets] = {};
    cudaEvent_t ev_done[kBatchSets] = {}, ev_out[kBatchSets] = {};
    void *pinned_steps = nullptr;
    size_t pinned_steps_bytes = 0;
    void *pinned = nullptr;  // small pinned host buffer (diagnostics read-back)
    bool autotune = true;    // tune W-towers schedules once per shape
    bool use_graphs = true;  // replay W-towers passes as CUDA graphs
    int64_t stats[11] = {0};
    int launches = 0;
};

namespace rg {

// Stage timing: begin_stage/end_stage bracket launches with events when the
// context is profiling; collect_timings (after a stream sync) fills timings.
void begin_call(rg_context *ctx);
void begin_stage(rg_context *ctx, const char *name);
void end_stage(rg_context *ctx);
void collect_timings(rg_context *ctx);

// Argument checks shared by the entry points: the visibility arrays (NULL
// pointers, negative or > 2^31 counts) and the w-kernel table description
// (support, oversampling, plane count, finite w_min and positive w_step).
rg_status check_vis(const rg_vis *vis);
rg_status check_wkern(const rg_wkern *wk);

// Device scratch that persists in the context and grows on demand.
rg_status scratch(rg_context *ctx, const char *name, size_t bytes, void **out);

// Device view of a caller buffer: the pointer itself when device-accessible,
// else a scratch copy (host -> device on the context stream).
rg_status stage_in(rg_context *ctx, const void *ptr, size_t bytes, const char *name,
                   const void **dev);
bool is_device_pointer(const void *p);

// Output view of a caller buffer: the device pointer itself, or a scratch
// buffer (loaded from the host buffer when `load`) that finish_out copies
// back on the context stream.
struct OutView {
    void *user = nullptr;
    void *dev = nullptr;
    size_t bytes = 0;
    bool host = false;
};
rg_status out_view(rg_context *ctx, void *ptr, size_t bytes, const char *name, bool load, OutView *ov);

// Device error word + counters in one small scratch area: diag_begin zeroes
// it on the context stream; diag_end reads it back (synchronising) and turns
// the error bits into a status.
struct Diag {
    unsigned *err;
    unsigned long long *counters;  // [0] gridded, [1] dropped
};
rg_status diag_begin(rg_context *ctx, Diag *d);
rg_status diag_end(rg_context *ctx, const Diag &d, unsigned long long *counters_out);
rg_status finish_out(rg_context *ctx, const OutView &ov);

// One baseline of a crocodile visibility file (rg_io.cu): antenna ids (-1
// when the file has none), times, frequencies (Hz), uvw [time][3] metres,
// visibilities [time][freq] complex interleaved.
struct BaselineRecord {
    int a1 = -1, a2 = -1;
    std::vector<double> time, freq, uvw, vis;
};
// Calls fn for every baseline of the file (hierarchical or legacy flat
// layout) whose first uvw sample's length lies in [bl_min, bl_max) metres.
rg_status visit_vis_hdf5(const char *path, double bl_min, double bl_max,
                         const std::function<void(const BaselineRecord &)> &fn);

// ---------------------------------------------------------------------------
// kernel launchers (defined in k_*.cu)
// ---------------------------------------------------------------------------

// k_image.cu
void launch_convert_table(cudaStream_t s, const double2 *src, float2 *dst, int64_t n);
// The W-towers gridder's copy: every K x K slice stored twice (2 K^2 taps), so
// a thread's rows (r0 + j) mod K are read as r0 + j without wrapping.
void launch_convert_table_dup(cudaStream_t s, const double2 *src, float2 *dst, int64_t n, int kk);
void launch_make_hermitian(cudaStream_t s, double2 *grid, int n);
void launch_fft_shift(cudaStream_t s, double2 *grid, int n);
void launch_real_part(cudaStream_t s, const double2 *grid, double *img, int n,
                      const double *taper);
void launch_weight_count(cudaStream_t s, const double *u, const double *v, int64_t nvis,
                         int n, double theta, unsigned *count);
void launch_weight_apply(cudaStream_t s, const double *u, const double *v,
                         const double2 *vis, double2 *out, int64_t nvis, int n, double theta,
                         const unsigned *count);
void launch_add_f32_to_f64(cudaStream_t s, const float2 *src, double2 *dst, int64_t n,
                           int overwrite);
void launch_add_f64(cudaStream_t s, const double2 *src, double2 *dst, int64_t n);
void launch_simple_grid(cudaStream_t s, const double *u, const double *v, const double2 *vis, int64_t nvis, int n,
                        double theta, double2 *grid, unsigned *err);

// k_fft.cu — FP32 four-step FFTs for power-of-two n in [64, 1024]
bool fft32_supported(int n);
void fft32_init_twiddles(cudaStream_t s, float2 *tw, int n);  // tw: n entries
// batched row transforms: rows = count of rows of length n (contiguous)
void launch_fft32_rows(cudaStream_t s, float2 *data, int64_t rows, int n, int sign,
                       const float2 *tw, const int *count_dev = nullptr);
// column transforms of `batch` n x n arrays; arrays b with live[b] == 0 are
// left as they are (live may be NULL: all)
void launch_fft32_cols(cudaStream_t s, float2 *data, int batch, int n, int sign,
                       const float2 *tw, const int *live = nullptr);
// FP64 transforms for image formation: power-of-two n <= 4096 directly,
// any other n <= 4096 by Bluestein's algorithm (k_bluestein.cu), which needs
// fft64_any_work_elems(n) double2 of work space (0 for powers of two).
bool fft64_supported(int n);
bool fft64_any_supported(int n);
constexpr int kBluesteinRows = 512;  // rows per Bluestein chunk (work space)
int64_t fft64_any_work_elems(int n);
const double2 *fft64_twiddles(cudaStream_t s, int n);  // exp(-2 pi i k / n), k < n/2 (cached)
void launch_fft64_pow2_rows(cudaStream_t s, double2 *data, int64_t rows, int n, int sign);
void launch_fft64_any_rows(cudaStream_t s, double2 *data, int64_t rows, int n, int sign, double2 *work);
void launch_fft64_2d(cudaStream_t s, double2 *data, double2 *tmp, int batch, int ny, int nx,
                     int sign, double2 *work = nullptr);

// k_prepare.cu
struct TowerGeom {
    int grid_size, subgrid, margin, chunk, nchunk, ksize, ov, planes;
    double theta, winc, wk_wmin, wk_wstep;
    // towers this call grids (one byte per tower, nonzero = grid it), or
    // nullptr for all: the visibilities of the other towers are skipped (not
    // counted as dropped) — one share of a tower-partitioned observation
    const unsigned char *tower_sel = nullptr;
};
// Per-tower load of a W-towers observation: visibilities and active w-floors
// of each tower (vis_count: ntowers int64, active: ntowers*nfloor ints zeroed
// by the caller, floors: ntowers ints), with the binning cuts of the gridder.
void launch_tower_census(cudaStream_t s, const double *u, const double *v, const double *w, int64_t n,
                         TowerGeom g, const int *range, unsigned long long *vis_count, int *active,
                         int *floors, int ntowers, int floors_cap, unsigned *err);
void launch_minmax_w(cudaStream_t s, const double *u, const double *v, const double *w,
                     int64_t n, double *out4, unsigned *err);
// range[0] = wp_min, range[1] = nfloor, range[2] = 1 if nfloor <= floors_cap
// (grid.c:357-367 from the reduced w range)
void launch_w_floors(cudaStream_t s, const double *wrange, double winc, int floors_cap, int *range,
                     unsigned *err);
// Column strips: sub-grid columns in groups of kStripCols; a (bin, strip) mark
// byte is set when any visibility of the bin has a tap in the strip.  Only
// marked strips are ever non-zero, so the column transforms and the row stage
// touch only them.
constexpr int kStripCols = 8;
// Sub-grids of the W-towers pass are stored strip-major: element (row, col)
// of an S x S sub-grid (S = 2^lg) at (col / 8) * 8S + row * 8 + col % 8, so a
// column strip is one contiguous 8S-element block.  L is the row-major linear
// index row * S + col, 0 <= L < S^2.
__host__ __device__ __forceinline__ int strip_addr(int L, int lg)
{
    return ((L & ((1 << lg) - 1)) >> 3) * (8 << lg) + (L >> lg) * 8 + (L & 7);
}
// feat == nullptr: table taps (frac_coord cells and oversampled sub-cell
// indices, the reference's).  feat != nullptr: learned taps — cell = floor(x)
// with the continuous offsets feat[i] = {w - w_mid, du, dv, 0}; no table.
void launch_prepare_towers(cudaStream_t s, const double *u, const double *v, const double *w,
                           const double2 *vis, int64_t n, TowerGeom g, const int *range,
                           int4 *rec, float2 *visf, int *active, unsigned char *marks, unsigned *err,
                           unsigned long long *counters, float4 *feat = nullptr);
void launch_prepare_wproj(cudaStream_t s, const double *u, const double *v, const double *w,
                          const double2 *vis, int64_t n, int grid_size, double theta,
                          int ksize, int ov, int planes, double wk_wmin, double wk_wstep,
                          int4 *rec, float2 *visf, unsigned *err);
// counts[0] = active slots, counts[1] = floor groups (target_items: aim for
// about this many (group, strip) work items in the column stage)
void launch_compact_bins(cudaStream_t s, const int *active, const int *range, int *slot_of_bin,
                         int *bin_of_slot, int *counts, int *tower_first, int *tower_count,
                         int ntowers, int strips, int target_items, int *group_begin,
                         int *group_end, int *tower_group_first, int *tower_group_count);

// k_romein.cu
// Sub-grids with slot index >= slot_cap are skipped (capacity overflow: the
// caller detects it from the slot count and reruns).
// points: grid points per thread (0: the default for ksize).  strip_lg = 0:
// row-major grids; otherwise log2(grid_side) and strip-major sub-grids.
// taps64 (row-major grids only; taps unused then): the FP64 table itself, each
// tap rounded to FP32 as it is loaded.
void launch_romein(cudaStream_t s, const int4 *rec, const float2 *visf, int64_t n,
                   const float2 *taps, float2 *grids, const int *slot_of_bin,
                   int64_t grid_stride, int grid_side, int ksize, int sm_count, int slot_cap = 1,
                   int points = 0, int strip_lg = 0, const double2 *taps64 = nullptr);

// k_towers.cu
void launch_fresnel_table(cudaStream_t s, uint32_t *phq, int subgrid, double theta, double winc);
// Sparse sub-grid transforms and the W-towers row stage.  Group g covers
// active slots [group_begin[g], group_end[g]) of one tower; partial holds one
// sub-grid per group; tower t's groups are [tower_group_first[t],
// +tower_group_count[t]).  range = {wp_min, nfloor, ok} and counts = {slots,
// groups, towers} live on the device; launches are sized by the capacities.
//
// slot_masks: bit s of word masks[slot*mask_words(S) + s/32] = strip s of the
// slot's bin is marked.
int mask_words(int subgrid);
void launch_slot_masks(cudaStream_t s, const unsigned char *marks, const int *bin_of_slot,
                       const int *counts, int slot_cap, int subgrid, unsigned *masks);
// Backward column transform, in place, of the marked strips of the live slots.
void launch_sparse_cols(cudaStream_t s, float2 *slots, const unsigned *masks, const int *counts,
                        int slot_cap, int subgrid, const float2 *tw, int sm_count);
// Row stage: per group and strip of rows, for each floor the backward row
// transform (reading only marked strips and leaving them zeroed: the reference
// clears its sub-grid after each floor, grid.c:473-481), times the floor's
// Fresnel factor, accumulated into the group's partial sub-grid.
void launch_tower_rows(cudaStream_t s, float2 *slots, const unsigned *masks, const int *bin_of_slot,
                       const int *group_begin, const int *group_end, const int *range,
                       const int *counts, int slot_cap, int group_cap, const uint32_t *phq,
                       float2 *partial, int subgrid, const float2 *tw);
// Per tower: the sum of its groups' partials (in group order) and the forward
// row transform into subimg.  The forward column transform of subimg follows
// (launch_fft32_cols).
void launch_tower_finish(cudaStream_t s, int group_cap, const int *tower_group_first,
                         const int *tower_group_count, int ntowers, const float2 *partial,
                         float2 *subimg, int subgrid, const float2 *tw);
int tower_row_strips(int subgrid);  // row strips per sub-grid in the row stage
void launch_add_back(cudaStream_t s, const float2 *subimg, const int *tower_count,
                     double2 *master, int grid_size, int subgrid, int margin, int chunk,
                     int nchunk, int overwrite, const int *range, const int *counts, int slot_cap,
                     int group_cap, int *poison = nullptr);

// k_dft.cu
// rows [row0, row0 + nrows) of the image into image (nrows x grid_size);
// nrows < 0: the whole image
void launch_dft(cudaStream_t s, const double *u, const double *v, const double *w,
                const double2 *vis, int64_t n, double *image, int grid_size, double theta,
                int precision, double factor, int sm_count, int row0 = 0, int nrows = -1);

// k_mlp.cu — learned w-kernel
int mlp_param_count();
int mlp_bf16_count();
void launch_mlp_grad(cudaStream_t s, const float *P, const void *PB, const float *in, const float2 *target,
                     int n, int ksize, float inv_wmax, float inv_scale, float *grad, float *loss);
void launch_mlp_adam(cudaStream_t s, float *P, void *PB, float *grad, float *m, float *v, float lr, int step);
void launch_mlp_to_bf16(cudaStream_t s, const float *P, void *PB);
void launch_mlp_eval(cudaStream_t s, const float *P, const void *PB, const float *in, int n, int ksize,
                     float inv_wmax, float scale, float2 *out, int sm_count, unsigned *err);
void launch_mbar_timeout_probe(cudaStream_t s, unsigned *err, long long limit);
void launch_learned_wproj(cudaStream_t s, const double *u, const double *v, const double *w,
                          const double2 *vis, int64_t n, int N, double theta, const float *P, const void *PB,
                          int ksize, float inv_wmax, float scale, float2 *grid, int sm_count, unsigned *err);
// W-towers with learned taps: per record, taps from the network at the
// visibility's continuous (w - w_mid, du, dv) (feat), scattered into its slot's
// sub-grid with the linear index rule of the table gridder.
void launch_learned_towers(cudaStream_t s, const int4 *rec, const float2 *visf, const float4 *feat, int64_t n,
                           const int *slot_of_bin, int slot_cap, float2 *slots, int subgrid, const float *P,
                           const void *PB, int ksize, float inv_wmax, float scale, int sm_count, unsigned *err);

}  // namespace rg
