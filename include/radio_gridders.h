/*
 * radio_gridders.h — C ABI of the B200-native radio imager.
 *
 * Plain C: pointers, sizes and status codes only.  Every buffer argument may be
 * a host pointer (pageable or pinned) or a CUDA device pointer; the library
 * detects which (cudaPointerGetAttributes) and stages host buffers through the
 * context's device memory.  Results are identical either way.
 *
 * The reference (KentJames/Radio-Gridders) has no library API: its paths sit
 * behind CLI binaries and the host wrappers declared in
 * src/grid/grid_common.cuh:45-64 and src/dft/dft_common.cuh:12-18, plus the CPU
 * functions of src/reference/grid.h:113-137.  Each entry point below names the
 * reference interface it replaces.  Differences from those interfaces:
 *   - inputs are in-memory arrays, not file names (the crocodile HDF5 readers
 *     are separate entry points: rg_hdf5_*);
 *   - errors are returned as rg_status (never exit(), unlike
 *     src/common/radio.cuh:27-43), with a thread-local message in
 *     rg_last_error();
 *   - nothing is leaked: device scratch lives in the context and is reused.
 *
 * Threading: a context belongs to one host thread at a time; calls on one
 * context are serialised on its CUDA stream.  Different contexts are
 * independent.
 */
#ifndef RADIO_GRIDDERS_H
#define RADIO_GRIDDERS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rg_status {
    RG_OK = 0,
    RG_ERR_INVALID_ARGUMENT = 1, /* bad sizes, NULL pointers, data outside the grid/kernel */
    RG_ERR_CUDA = 2,             /* a CUDA runtime call failed */
    RG_ERR_OUT_OF_MEMORY = 3,
    RG_ERR_UNSUPPORTED = 4,      /* valid request outside this build's limits */
    RG_ERR_IO = 5,               /* file missing or not in the expected format */
    RG_ERR_NO_DEVICE = 6
} rg_status;

typedef struct rg_context rg_context;

/* Flat visibilities: the reference's struct flat_vis_data
 * (src/common/hdf5.cuh:31-37), produced by flatten_visibilities_CUDA
 * (src/common/hdf5.c:827-872).  u, v, w in wavelengths; vis interleaved
 * (re, im) float64, 2*n doubles. */
typedef struct rg_vis {
    const double *u;
    const double *v;
    const double *w;
    const double *vis;
    int64_t n;
} rg_vis;

/* Oversampled w-kernel table: struct w_kernel_data (src/reference/grid.h:34-49)
 * with kern_by_w flattened.  data holds plane_count*ov*ov*size*size complex
 * float64 taps (interleaved), index
 * ((plane*ov + yf)*ov + xf)*size*size + y*size + x  (src/reference/grid.c:53-56);
 * plane p is used for w nearest w_min + p*w_step (grid.c:168-170). */
typedef struct rg_wkern {
    const double *data;
    int plane_count;
    int size;
    int oversampling;
    double w_min;
    double w_step;
} rg_wkern;

/* rg_grid_* flags */
#define RG_GRID_ACCUMULATE 0 /* uvgrid += gridded visibilities (grid.c semantics) */
#define RG_GRID_OVERWRITE 1  /* uvgrid  = gridded visibilities (prior contents ignored) */

/* rg_dft_image precision modes (the precision study) */
#define RG_DFT_FP32_NAIVE 0  /* phase argument and sincos in FP32 */
#define RG_DFT_FP64_REDUCED 1 /* per-tile phase reduced in FP64, FP32 increments */
#define RG_DFT_FP64 2        /* all FP64 */

/* ---- context ----------------------------------------------------------- */

/* Replaces the device selection and setup of src/grid/grid.cpp:161-165
 * (-device) and src/dft/dft.cpp.  Creates a context on `device`. */
rg_status rg_context_create(int device, rg_context **ctx);
rg_status rg_context_destroy(rg_context *ctx);
/* Use the caller's cudaStream_t (passed as void*) for subsequent calls; NULL
 * restores the context's own stream. */
rg_status rg_context_set_stream(rg_context *ctx, void *cuda_stream);
/* Message describing the last failed call on this host thread. */
const char *rg_last_error(void);
/* Statistics of the last gridding call on this context: element 0 number of
 * visibilities gridded, 1 active (tower, floor) sub-grids, 2 towers with data,
 * 3 w-floors spanned, 4 visibilities dropped for lying outside every tower
 * (cf. the per-baseline check at src/reference/grid.c:519-530), 5 kernel
 * launches issued by the call; W-towers only: 6 sub-grid column strips of 8
 * columns holding data (the strips the transforms touch), 7 floor groups of
 * the row stage, 8 Romein grid points per thread and 9 row-stage work items
 * per SM in use (the tuned schedule), 10 one when the pass ran as a captured
 * graph.
 * Returns the count written (<= n). */
int rg_last_stats(rg_context *ctx, int64_t *out, int n);

/* Per-stage timing (the reference's cudaEvent timing around gridding,
 * src/grid/grid_cuda.cu:677-734).  When enabled, every stage of a call is
 * bracketed by CUDA events on the context stream; rg_last_timings then returns
 * the stage names and milliseconds of the last call (count written). */
rg_status rg_context_set_profiling(rg_context *ctx, int enabled);
int rg_last_timings(rg_context *ctx, const char **names, float *ms, int n);

/* W-towers schedules (no counterpart in the reference, whose launch shapes are
 * fixed, src/grid/grid_cuda.cu:241-280 and :665-666).
 * Autotuning (default on): the first call of a shape (grid size, sub-grid,
 * margin, w increment, visibility count, table or learned taps) times whole
 * passes into a scratch grid over the Romein points-per-thread and row-stage
 * group-size choices and keeps the fastest for that shape; the caller's grid
 * is written by an ordinary pass before tuning.
 * Graph replay (default on): when the visibilities and the output grid are
 * the caller's device buffers and profiling is off, the second and later calls
 * of a tuned shape with the same buffers launch the whole pass as one captured
 * CUDA graph; new buffer addresses or data that outgrow the sized capacities
 * fall back to ordinary launches and capture again. */
rg_status rg_context_set_autotune(rg_context *ctx, int enabled);
rg_status rg_context_set_graphs(rg_context *ctx, int enabled);

/* ---- gridders ---------------------------------------------------------- */

/* W-projection, Romein scatter.  Replaces grid_wprojection
 * (src/reference/grid.h:121-122, grid.c:187-202) and the GPU wrapper
 * wproj_CUDA_flat (src/grid/grid_common.cuh:59-62, grid_cuda.cu:826-921) up to
 * the FFT.  uvgrid: grid_size*grid_size complex float64 (interleaved). */
rg_status rg_grid_wprojection(rg_context *ctx, double *uvgrid, int grid_size, double theta,
                              const rg_vis *vis, const rg_wkern *wkern, int flags);

/* Nearest-cell gridding without a kernel: each visibility added to the grid
 * cell nearest its (u, v).  Replaces grid_simple (src/reference/grid.h:115-116,
 * grid.c:83-99), grid_CPU.out's gridder when no w-kernel file is given
 * (src/reference/main.c:200-206).  FP64 atomics (the order of additions to a
 * cell varies from call to call: grids agree to FP64 rounding).  A
 * visibility whose cell lies off the grid returns RG_ERR_INVALID_ARGUMENT
 * (the reference writes out of bounds) and leaves uvgrid unchanged. */
rg_status rg_grid_simple(rg_context *ctx, double *uvgrid, int grid_size, double theta, const rg_vis *vis,
                         int flags);

/* W-projection that allocates nothing.  No counterpart in the reference.
 * For callers that cannot allocate device memory or let a library do it:
 * code running while another framework owns the device memory pool and its
 * budget, real-time pipelines that forbid allocation after start-up, embedders
 * with a fixed memory plan.  No context, stream, event or allocation is
 * created; the caller passes device pointers for every input and the output
 * (host pointers are rejected) and the stream to run on (NULL = default).
 * Intermediates live in one file-scope device array (about 13.5 MiB, held by
 * every GPU that loads the library until exit), which limits grid_size to
 * 1024 and the w-kernel table to 524288 taps; larger requests fail with
 * RG_ERR_UNSUPPORTED.  Any number of visibilities.  The first call on each
 * device resolves the array's address (cudaGetSymbolAddress).  Calls share
 * the array: calls that overlap on the GPU (other streams, other host
 * threads) race.  Runs on the calling thread's current device.  The call synchronises with `cuda_stream` twice:
 * it reads the error word back before it touches uvgrid (a call rejected for
 * its data, e.g. w outside the table, leaves uvgrid as it was), and it returns
 * after the grid is written.  A CUDA error already pending when the call
 * starts is returned as RG_ERR_CUDA with a message that says so. */
rg_status rg_grid_wprojection_noalloc(double *uvgrid, int grid_size, double theta,
                                      const rg_vis *vis, const rg_wkern *wkern, int flags,
                                      void *cuda_stream);

/* W-towers.  Replaces grid_wtowers (src/reference/grid.h:123-126,
 * grid.c:295-555) and the GPU wrapper wtowers_CUDA_flat
 * (src/grid/grid_common.cuh:52-55, grid_cuda.cu:522-744) up to the final FFT:
 * the master uv grid after add-back, FP64. */
rg_status rg_grid_wtowers(rg_context *ctx, double *uvgrid, int grid_size, double theta,
                          const rg_vis *vis, const rg_wkern *wkern, int subgrid_size,
                          int subgrid_margin, double wincrement, int flags);

/* ---- one observation's towers over several GPUs ------------------------
 * No counterpart in the reference, which grids every tower on one device
 * (src/grid/grid.cpp:161-165, src/grid/grid_cuda.cu:644-655); its work unit
 * is the tower (src/reference/grid.c:413-416).  Towers are independent until
 * the add-back, so rank r of R grids the towers of part r into its own FP64
 * master grid (rg_grid_wtowers_part) and one sum of the R master grids (an
 * NCCL reduce or reduce-scatter) gives rg_grid_wtowers' grid, up to the order
 * of the FP64 additions of overlapping towers.  Every rank needs the
 * visibilities of its own towers only; a rank given all of them skips the
 * others' after binning. */

/* Towers of a W-towers shape: (grid_size / (subgrid - margin) + 1)^2, ordered
 * row-major (cy * n + cx). */
int rg_wtowers_tower_count(int grid_size, int subgrid_size, int subgrid_margin);
/* Load of each tower: visibilities (vis_per_tower) and active w-floors
 * (floors_per_tower) under the gridder's binning cuts.  ntowers must equal
 * rg_wtowers_tower_count. */
rg_status rg_wtowers_tower_loads(rg_context *ctx, int grid_size, double theta, const rg_vis *vis,
                                 int subgrid_size, int subgrid_margin, double wincrement, int64_t *vis_per_tower,
                                 int32_t *floors_per_tower, int ntowers);
/* Host only: towers into nparts parts balanced by vis + vis_per_floor *
 * floors (0: the default 2400, the measured cost ratio of a sub-grid's
 * transforms to one visibility's gridding on B200), largest first to the
 * least loaded part.  Deterministic: every rank computes the same parts. */
rg_status rg_wtowers_partition(const int64_t *vis_per_tower, const int32_t *floors_per_tower, int ntowers,
                               int nparts, double vis_per_floor, int32_t *part_of_tower);
/* rg_grid_wtowers restricted to the towers t with part_of_tower[t] == part;
 * other towers' visibilities are skipped (last_stats counts only this
 * part's gridded visibilities). */
rg_status rg_grid_wtowers_part(rg_context *ctx, double *uvgrid, int grid_size, double theta, const rg_vis *vis,
                               const rg_wkern *wkern, int subgrid_size, int subgrid_margin, double wincrement,
                               int flags, const int32_t *part_of_tower, int part);

/* count observations of one shape (same visibility count) with one kernel
 * table: the same result as count rg_grid_wtowers calls in order (grid i from
 * vis[i] into uvgrids[i]), with the host-to-device copies of later
 * observations and the device-to-host copies of earlier grids overlapping each
 * pass (three staging sets of inputs and grid in device memory, three
 * streams).  For streams of snapshots imaged
 * with one set of kernels; no counterpart in the reference.  Inputs and grids
 * in pinned host memory overlap fully; device buffers are used in place.
 * Returns the first error; the grids of the steps before it are complete. */
rg_status rg_grid_wtowers_batch(rg_context *ctx, int count, double *const *uvgrids, int grid_size, double theta,
                                const rg_vis *vis, const rg_wkern *wkern, int subgrid_size, int subgrid_margin,
                                double wincrement, int flags);

/* Uniform weighting: vis_out[i] = vis[i] / (visibilities in its nearest cell).
 * Replaces weight() (src/reference/grid.h:116-117, grid.c:59-81) as called by
 * src/reference/main.c:153.  vis_out: 2*n doubles (may alias vis->vis). */
rg_status rg_weight(rg_context *ctx, int grid_size, double theta, const rg_vis *vis,
                    double *vis_out);

/* ---- image formation --------------------------------------------------- */

/* make_hermitian (src/reference/grid.h:135, grid.c:639-662), in place. */
rg_status rg_make_hermitian(rg_context *ctx, double *uvgrid, int grid_size);
/* fft_shift (src/reference/grid.h:136, grid.c:665-680), in place. */
rg_status rg_fft_shift(rg_context *ctx, double *uvgrid, int grid_size);
/* Dirty image from a uv grid: make_hermitian, fft_shift, 2-D FFT (sign -1),
 * fft_shift, real part (src/reference/main.c:258-294).  uvgrid is consumed
 * (overwritten); image_out: grid_size*grid_size float64.  If
 * taper_1d != NULL the image is divided by taper_1d[x]*taper_1d[y] (grid
 * correction; the reference applies none). */
rg_status rg_image_from_grid(rg_context *ctx, double *uvgrid, int grid_size,
                             double *image_out, const double *taper_1d);
/* Batched 2-D complex FFT (unnormalised, sign -1 or +1), the project's own
 * kernels; exposed so they can be checked against cuFFT.  data: batch*ny*nx
 * complex, float32 (complex_bytes 8) or float64 (complex_bytes 16). */
rg_status rg_fft2d(rg_context *ctx, void *data, int batch, int ny, int nx, int sign,
                   int complex_bytes);

/* ---- direct DFT -------------------------------------------------------- */

/* Direct Fourier transform image.  Replaces image_dft_host_flat
 * (src/dft/dft_common.cuh:16-18, dft_cuda.cu:170-223) with the defects of
 * src/dft/dft_cuda.cu:55-57 and :98-112 removed:
 *   image[y][x] = factor * sum_k Re(V_k exp(-2 pi i (u_k l + v_k m + w_k (1 - n))))
 *   l = theta (x - N/2)/N, m = theta (y - N/2)/N, n = sqrt(1 - l^2 - m^2).
 * factor 2 matches the hermitian gridder pipeline, 1 the reference dft.out. */
rg_status rg_dft_image(rg_context *ctx, double *image_out, int grid_size, double theta,
                       const rg_vis *vis, int precision, double factor);
/* Rows [row0, row0 + nrows) of the same image into image_out (nrows rows of
 * grid_size), e.g. one GPU's share of an image whose rows are split over
 * several GPUs (the shares are then gathered; no counterpart in the
 * reference, whose DFT runs on one GPU).  A share starting on a row that is a
 * multiple of 32 equals those rows of rg_dft_image bit for bit; other starts
 * differ within the precision mode's rounding. */
rg_status rg_dft_image_rows(rg_context *ctx, double *image_out, int grid_size, double theta,
                            const rg_vis *vis, int precision, double factor, int row0, int nrows);

/* ---- file-level drop-ins for the reference's host wrappers --------------- */

/* Same arguments as the reference's wrappers, so grid.cpp / dft.cpp change
 * only the function name: read the crocodile HDF5 files (the rg_read_*_hdf5
 * readers below: visibilities to wavelengths, baselines with first-sample
 * length in [bl_min, bl_max) metres, w-kernels of group wkern/<theta %g>),
 * grid or transform, and leave the dirty image in the caller's grid_size^2
 * complex-double buffers as real part (imaginary part 0): the device buffer
 * (which also holds the uv grid on the way) and, when non-NULL, the host
 * one.  The image is the reference CPU pipeline's (src/reference/main.c:
 * 258-294, hermitian then FFT); the reference's GPU wrappers leave half of it
 * mirrored (no hermitian step, inverse FFT).  lambda, threads_per_block,
 * blocks and threads_block are accepted and unused (the caller derives
 * grid_size from lambda; launch shapes are the library's own).  Runs on the
 * calling thread's current device with a context of its own; returns a status
 * instead of exiting.
 *
 * Replaces wtowers_CUDA_flat (src/grid/grid_common.cuh:49-52,
 * src/grid/grid_cuda.cu:522-744). */
rg_status rg_wtowers_cuda_flat(const char *visfile, const char *wkernfile, double *grid, double *gridh,
                               int grid_size, double theta, double lambda, double bl_min, double bl_max,
                               int subgrid_size, int subgrid_margin, double winc);
/* Replaces wproj_CUDA_flat (src/grid/grid_common.cuh:59-62). */
rg_status rg_wproj_cuda_flat(const char *visfile, const char *wkernfile, double *grid, double *gridh,
                             int grid_size, double theta, double lambda, double bl_min, double bl_max,
                             int threads_per_block);
/* Replaces image_dft_host_flat (src/dft/dft_common.cuh:16-18): the direct DFT
 * image (FP64-reduced phase, the reference dft.out's scale) into grid_host
 * and/or grid_dev. */
rg_status rg_image_dft_host_flat(const char *visfile, double *grid_host, double *grid_dev, int grid_size,
                                 double theta, double lambda, double bl_min, double bl_max, int blocks,
                                 int threads_block);

/* ---- crocodile HDF5 files ------------------------------------------------- */

/* Flat visibilities read from a file; arrays owned by the struct, released
 * with rg_free_vis_data. */
typedef struct rg_vis_data {
    double *u, *v, *w, *vis; /* vis: 2*n doubles */
    int64_t n;
    int64_t bl_count;
} rg_vis_data;

/* Replaces load_vis + flatten_visibilities_CUDA (src/reference/hdf5.c:173-318,
 * src/common/hdf5.c:827-872): reads the hierarchical /vis/<a1>/<a2>/... or the
 * legacy flat /vis layout, keeps baselines whose first uvw sample has length
 * in [bl_min, bl_max) metres, and flattens to u, v, w in wavelengths in
 * baseline/time/frequency order.  Project-written HDF5 reader (superblock
 * 0/1, symbol-table groups, contiguous datasets); RG_ERR_IO otherwise. */
rg_status rg_read_vis_hdf5(const char *path, double bl_min, double bl_max, rg_vis_data *out);
void rg_free_vis_data(rg_vis_data *d);

/* An oversampled w-kernel table read from a file (rg_wkern layout). */
typedef struct rg_wkern_data {
    double *data;
    int plane_count, size, oversampling;
    double w_min, w_step;
} rg_wkern_data;

/* Replaces load_wkern (src/reference/hdf5.c:321-413): group wkern/<theta %g>,
 * one child per w plane, planes re-indexed nearest to w_min + i*w_step. */
rg_status rg_read_wkern_hdf5(const char *path, double theta, rg_wkern_data *out);
void rg_free_wkern_data(rg_wkern_data *d);

/* Writers of the same layouts (hierarchical visibilities: time [bl][time],
 * uvw [bl][time][3] metres, freq [bl][nf] Hz, vis [bl][time][nf] complex
 * interleaved; one /vis/<ant1>/<ant2> group per baseline). */
rg_status rg_write_vis_hdf5(const char *path, int n_bl, int n_time, int n_freq, const int *ant1,
                            const int *ant2, const double *time, const double *freq,
                            const double *uvw, const double *vis);
rg_status rg_write_wkern_hdf5(const char *path, double theta, const rg_wkern *wk);
/* The legacy flat layout (src/common/hdf5.c:199-300): /vis with attribute
 * type = "Visibility" and rows of one time sample each — antenna1/antenna2
 * [rows] int64, time [rows], uvw [rows][3] metres, frequency [nf] Hz (shared by
 * all rows), vis [rows][nf][1] complex. */
rg_status rg_write_vis_flat_hdf5(const char *path, int n_rows, int n_freq, const int *ant1, const int *ant2,
                                 const double *time, const double *freq, const double *uvw, const double *vis);
/* Generic access used for other crocodile files (e.g. the separable kernels
 * of src/common/hdf5.c:372-500): a float64 / int64 / {r, i} dataset by path
 * (out may be NULL to query dims; up to 8 dims; a compound element adds a
 * trailing axis of its member count), and a numeric attribute. */
rg_status rg_hdf5_read_f64(const char *path, const char *dataset, double *out, int64_t capacity,
                           int64_t *dims, int *ndims);
rg_status rg_hdf5_attr_f64(const char *path, const char *object, const char *name, double *out);

/* ---- AW-projection ------------------------------------------------------ */

/* Hierarchical visibilities (the reference's struct vis_data,
 * src/reference/grid.h:7-30, with every baseline holding time_count times and
 * freq_count channels): antenna1/antenna2 [bl], time [bl][time] (the file's
 * time unit), freq [bl][freq] Hz, uvw [bl][time][3] metres, vis
 * [bl][time][freq] complex interleaved. */
typedef struct rg_vis_bl {
    int bl_count, time_count, freq_count;
    const int32_t *antenna1, *antenna2;
    const double *time, *freq, *uvw, *vis;
} rg_vis_bl;

/* A-kernels per (antenna, time slot, channel) on evenly spaced axes
 * t_min + i t_step, f_min + j f_step (struct a_kernel_data,
 * src/reference/grid.h:69-85, as load_akern indexes it: kern_by_atf,
 * src/common/hdf5.c:775-818): freq and time [ant][t][f] are each slot's own
 * kernel frequency (Hz) and time, data [ant][t][f][size_y][size_x] complex. */
typedef struct rg_akern {
    int antenna_count, time_count, freq_count, size_x, size_y;
    double t_min, t_step, f_min, f_step;
    const double *freq, *time, *data;
} rg_akern;

/* AW-projection: grid_awprojection after convolve_aw_kernels
 * (src/reference/grid.c:557-637) for baselines [bl_min, bl_max).  Each
 * visibility is gridded like W-projection (rg_grid_wprojection) with the
 * w-kernel plane nearest to uvw_w * f_A / c, f_A the frequency of antenna 1's
 * A-kernel for the visibility's time slot and nearest channel; the A x W
 * convolution is the reference's placeholder (it copies the w-kernel,
 * grid.c:583-590), so the A-kernel values are not used.  Sizes of both
 * kernel tables must agree (grid.c:562-563).  Every array of vis except
 * vis->vis, and akern->freq, must be host memory; a time or channel outside
 * the A-kernel axes or an antenna without kernels returns
 * RG_ERR_INVALID_ARGUMENT (the reference indexes past its tables). */
rg_status rg_grid_awprojection(rg_context *ctx, double *uvgrid, int grid_size, double theta, const rg_vis_bl *vis,
                               const rg_wkern *wkern, const rg_akern *akern, int bl_min, int bl_max, int flags);

/* Owned forms read from files (released with the matching free). */
typedef struct rg_vis_bl_data {
    int bl_count, time_count, freq_count;
    int32_t *antenna1, *antenna2;
    double *time, *freq, *uvw, *vis;
} rg_vis_bl_data;
typedef struct rg_akern_data {
    int antenna_count, time_count, freq_count, size_x, size_y;
    double t_min, t_step, f_min, f_step;
    double *freq, *time, *data;
} rg_akern_data;
/* Hierarchical visibilities of a crocodile file (either layout), baselines
 * whose first uvw sample has length in [bl_min, bl_max) metres; every
 * baseline must have the same time and channel counts (else
 * RG_ERR_UNSUPPORTED).  Replaces load_vis (src/reference/hdf5.c:173-318). */
rg_status rg_read_vis_bl_hdf5(const char *path, double bl_min, double bl_max, rg_vis_bl_data *out);
void rg_free_vis_bl_data(rg_vis_bl_data *d);
/* Replaces load_akern (src/common/hdf5.c:652-820): group akern/<theta %g>,
 * children <antenna>/<time>/<freq>/kern [size_y][size_x] complex; evenly
 * spaced axes from the extremes, each slot the antenna's nearest kernel. */
rg_status rg_read_akern_hdf5(const char *path, double theta, rg_akern_data *out);
void rg_free_akern_data(rg_akern_data *d);
rg_status rg_write_akern_hdf5(const char *path, double theta, const rg_akern *ak);

/* ---- W-stacking predict (degridding) ------------------------------------ */

/* A separable kernel table: real values data[ov_index * size + tap] (the
 * layout the reference's de-convolution indexes,
 * src/wstack/wstack_common.h:460-478, from load_sep_kern /
 * load_sep_kern_T, src/common/hdf5.c:372-497).  For a grid correction the
 * size * oversampling entries sample one function on [-1/2, 1/2). */
typedef struct rg_sepkern {
    const double *data;
    int size;
    int oversampling;
} rg_sepkern;

/* Model visibilities of npoints unit point sources (points: l, m pairs) at
 * (u, v, w) (wavelengths) by W-stacking: the quantised sky divided by the
 * grid correction corr_lm(du l) corr_lm(du m) corr_n(dw n), padded to
 * round(0.5 / x0) times floor(theta lambda) pixels, one FP64 FFT per w plane
 * (planes every dw; ceil(sin(theta/2) sqrt(2) N / dw) + conv_w.size + 1 of
 * them), then per visibility the separable conv_w x conv_uv^2 sum over the
 * stack (du: the uv cell of the padded grid).  Replaces wstack_predict
 * (src/wstack/predict.cpp:396-562) and wstack_predict_cu_3D
 * (src/wstack/predict.cu:808-1081).  vis_out: 2*nvis doubles.  FP64.
 * RG_ERR_INVALID_ARGUMENT for a source outside the image or a visibility
 * whose taps leave the stack (the reference reads past its arrays). */
rg_status rg_wstack_predict(rg_context *ctx, double theta, double lambda, const double *points, int npoints,
                            const double *u, const double *v, const double *w, int64_t nvis, double du, double dw,
                            double x0, const rg_sepkern *conv_uv, const rg_sepkern *conv_w,
                            const rg_sepkern *corr_lm, const rg_sepkern *corr_n, double *vis_out);

/* ---- w-kernel generator --------------------------------------------------- */

/* An oversampled w-kernel table (rg_wkern layout: plane_count * ov * ov * size
 * * size complex float64, interleaved) for the given w planes:
 *   tap[plane][yf][xf][ty][tx] = K_w(tx - size/2 - xf/ov, ty - size/2 - yf/ov),
 *   K_w(p, q) = 1/M^2 sum_ij A(l_i) A(m_j) exp(2 pi i w (1 - n_ij))
 *               exp(-2 pi i (p l_i + q m_j) / theta),
 * on an M x M screen (screen_pixels; <= 0: 128), l_i = theta (i - M/2) / M,
 * A(l) = psi_0(c, 2 l / theta) (c <= 0: pi (size - 2) / 2).  The reference
 * has no generator (its kernels come from the crocodile scripts as files,
 * README.md:25-26, loaded by src/common/hdf5.c:1362-1509); this produces the
 * tables its load_wkern would return (src/reference/hdf5.c:321-413), for
 * rg_grid_* or rg_write_wkern_hdf5.  data_out: host or device pointer.  FP64
 * throughout; the screen and the sums run on the device. */
rg_status rg_wkern_generate(rg_context *ctx, double theta, const double *w_planes, int plane_count, int size,
                            int oversampling, double c, int screen_pixels, double *data_out);
/* Host only: the zeroth prolate spheroidal wave function psi_0(c, x),
 * normalised to psi_0(c, 0) = 1, at n points x in [-1, 1] (the generator's
 * taper and the image-plane grid correction). */
rg_status rg_pswf0(double c, const double *x, int64_t n, double *out);

/* ---- learned w-kernel ---------------------------------------------------- */

/* A small MLP that returns the tap of the w-kernel for a continuous (w, du, dv)
 * and tap (tx, ty), in place of the quantised oversampled table.  No
 * counterpart in the reference (whose kernels come from crocodile table files,
 * src/common/hdf5.c:1362-1509).  Network: 21 features -> 128 -> 128 -> 128
 * (SiLU) -> complex tap / out_scale; tensor-core layers with FP32
 * accumulation (FP16 tcgen05 MMAs with TMEM accumulators in evaluation and
 * gridding, BF16 in training); trained by the library's own forward/backward
 * kernels with Adam.  Samples are [5][n] float arrays (w, du, dv, tx, ty),
 * taps complex float interleaved.  A network belongs to the context's device.
 * The tensor-core waits are bounded: a wait that runs out returns RG_ERR_CUDA
 * ("timed out") with the context still usable. */
typedef struct rg_mlp rg_mlp;
int rg_mlp_param_count(void);
rg_status rg_mlp_create(rg_context *ctx, int ksize, double wmax, double out_scale, uint64_t seed,
                        rg_mlp **mlp);
rg_status rg_mlp_destroy(rg_mlp *mlp);
rg_status rg_mlp_set_params(rg_context *ctx, rg_mlp *mlp, const float *params);
rg_status rg_mlp_get_params(rg_context *ctx, rg_mlp *mlp, float *params);
/* Loss and gradient of one batch without updating (checked against the CPU oracle). */
rg_status rg_mlp_gradient(rg_context *ctx, rg_mlp *mlp, const float *samples, const float *targets,
                          int n, float *grad_out, float *loss_out);
/* `steps` Adam steps over consecutive batches of the training set. */
rg_status rg_mlp_train(rg_context *ctx, rg_mlp *mlp, const float *samples, const float *targets,
                       int64_t n, int batch, int steps, float lr, float *loss_out);
rg_status rg_mlp_eval(rg_context *ctx, rg_mlp *mlp, const float *samples, int64_t n, float *taps_out);
/* W-projection with taps evaluated by the network at each visibility's exact
 * sub-cell offset and w (no oversampling quantisation).  Replaces the table
 * lookup of grid_wprojection (src/reference/grid.c:157-202). */
rg_status rg_grid_wprojection_learned(rg_context *ctx, rg_mlp *mlp, double *uvgrid, int grid_size,
                                      double theta, const rg_vis *vis, int flags);

/* W-towers with the learned kernel: the rg_grid_wtowers pass (tower and floor
 * binning, sub-grid transforms, Fresnel steps, FP64 add-back) with every
 * visibility's taps evaluated by the network at its continuous residual
 * w - w_mid and sub-cell offsets (footprint origin floor(x) - K/2) instead of
 * the oversampled table.  The network's w range must cover wincrement / 2.
 * No counterpart in the reference. */
rg_status rg_grid_wtowers_learned(rg_context *ctx, rg_mlp *mlp, double *uvgrid, int grid_size, double theta,
                                  const rg_vis *vis, int subgrid_size, int subgrid_margin, double wincrement,
                                  int flags);

/* Self-test of the bounded tensor-core wait: one CTA waits ~2 ms on an
 * mbarrier that nothing arrives on.  Returns RG_ERR_CUDA with a "timed out"
 * message when the timeout path works (RG_OK would mean it does not). */
rg_status rg_selftest_wait_timeout(rg_context *ctx);

#ifdef __cplusplus
}
#endif
#endif /* RADIO_GRIDDERS_H */
