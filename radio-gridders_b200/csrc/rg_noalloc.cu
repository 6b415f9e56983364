// W-projection gridding for callers that cannot allocate device memory.
//
// Some callers may not call cudaMalloc (or have a library do it for them):
// code that runs while another framework owns the device memory pool and its
// budget, real-time pipelines that forbid allocation after start-up, and
// embedders whose memory is fixed up front.  rg_grid_wprojection_noalloc
// serves them: the caller passes device buffers for inputs and output, and
// every intermediate the W-projection gridder needs (the FP32 kernel table,
// the per-visibility records, the FP32 accumulation grid and the error word)
// lives in one file-scope __device__ array below.  The call creates no
// context, stream, event or allocation.
//
// Limits, fixed by the array's layout: grid_size <= 1024, kernel table <= 2^19
// taps (e.g. 16x16 taps x 8x8 oversampling x 32 planes); any number of
// visibilities (they are processed in batches of 65,536).  Every GPU that loads
// the library holds the array (about 13.5 MiB) until the process exits.
#include <cmath>
#include <cstring>
#include <mutex>

#include "rg_internal.h"

namespace rg {
namespace {

constexpr int kMaxGrid = 1024;
constexpr int64_t kMaxTaps = int64_t(1) << 19;
constexpr int64_t kBatch = int64_t(1) << 16;

constexpr size_t kGridBytes = sizeof(float2) * kMaxGrid * kMaxGrid;  // 8 MiB
constexpr size_t kTapBytes = sizeof(float2) * kMaxTaps;             // 4 MiB
constexpr size_t kRecBytes = sizeof(int4) * kBatch;                 // 1 MiB
constexpr size_t kVisBytes = sizeof(float2) * kBatch;               // 512 KiB
constexpr size_t kMiscBytes = 512;                                  // error word + slot index
constexpr size_t kOffGrid = 0;
constexpr size_t kOffTaps = kOffGrid + kGridBytes;
constexpr size_t kOffRec = kOffTaps + kTapBytes;
constexpr size_t kOffVis = kOffRec + kRecBytes;
constexpr size_t kOffMisc = kOffVis + kVisBytes;
constexpr size_t kScratchBytes = kOffMisc + kMiscBytes;

}  // namespace

// The shared scratch.  Host code must not use this name as an address (it is a
// host-side stand-in); the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_addr[kMaxDevices] = {nullptr};
int g_sm_count[kMaxDevices] = {0};

// Once per device, with that device current: resolve the array's device
// address (and the SM count).  Runs on the first call on each device.
rg_status scratch_for_current_device(unsigned char **base, int *sms)
{
    int dev = 0;
    RG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(RG_ERR_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return fail(RG_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                         cudaGetErrorString(e));
        }
        int n = 0;
        RG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        g_sm_count[dev] = n;
        g_scratch_addr[dev] = (unsigned char *)p;
    }
    *base = g_scratch_addr[dev];
    *sms = g_sm_count[dev];
    return RG_OK;
}

bool on_device(const void *p)
{
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace rg

using namespace rg;

extern "C" rg_status rg_grid_wprojection_noalloc(double *uvgrid, int grid_size, double theta,
                                                 const rg_vis *vis, const rg_wkern *wkern,
                                                 int flags, void *cuda_stream)
{
    if (!uvgrid) return fail(RG_ERR_INVALID_ARGUMENT, "uvgrid must be non-NULL");
    if (grid_size < 2 || grid_size > kMaxGrid)
        return fail(RG_ERR_UNSUPPORTED, "rg_grid_wprojection_noalloc: grid_size must be in [2, 1024] "
                                        "(its fixed scratch holds a 1024 x 1024 FP32 grid)");
    if (!(theta > 0.0) || !std::isfinite(theta)) return fail(RG_ERR_INVALID_ARGUMENT, "theta must be > 0");
    // the checks rg_grid_wprojection makes (finite w_min, positive w_step, ...)
    RG_CHECK(check_vis(vis));
    RG_CHECK(check_wkern(wkern));
    const int K = wkern->size;
    const int64_t ntaps = (int64_t)wkern->plane_count * wkern->oversampling * wkern->oversampling * K * K;
    if (ntaps > kMaxTaps)
        return fail(RG_ERR_UNSUPPORTED, "rg_grid_wprojection_noalloc: the w-kernel table must hold at "
                                        "most 524288 taps (its fixed scratch)");
    // every buffer must already be on the device: staging host data would need memory
    if (!on_device(uvgrid) || !on_device(wkern->data) ||
        (vis->n > 0 && (!on_device(vis->u) || !on_device(vis->v) || !on_device(vis->w) ||
                        !on_device(vis->vis))))
        return fail(RG_ERR_INVALID_ARGUMENT,
                    "rg_grid_wprojection_noalloc takes device pointers only (no staging memory)");

    // an error left pending by the caller's earlier work is reported as such,
    // not as a failure of the launches below
    const cudaError_t pending = cudaGetLastError();
    if (pending != cudaSuccess)
        return cuda_fail(pending, "a CUDA error was already pending before rg_grid_wprojection_noalloc");
    unsigned char *base = nullptr;
    int sms = 148;
    RG_CHECK(scratch_for_current_device(&base, &sms));
    cudaStream_t st = (cudaStream_t)cuda_stream;
    float2 *grid32 = (float2 *)(base + kOffGrid);
    float2 *taps32 = (float2 *)(base + kOffTaps);
    int4 *rec = (int4 *)(base + kOffRec);
    float2 *visf = (float2 *)(base + kOffVis);
    unsigned *err = (unsigned *)(base + kOffMisc);
    int *slot = (int *)(base + kOffMisc + 256);
    const int N = grid_size;
    const int64_t cells = (int64_t)N * N;

    // the array keeps the previous call's contents: clear what must start at zero
    RG_CUDA(cudaMemsetAsync(grid32, 0, sizeof(float2) * cells, st));
    RG_CUDA(cudaMemsetAsync(base + kOffMisc, 0, kMiscBytes, st));
    launch_convert_table(st, (const double2 *)wkern->data, taps32, ntaps);
    for (int64_t off = 0; off < vis->n; off += kBatch) {
        const int64_t cnt = vis->n - off < kBatch ? vis->n - off : kBatch;
        launch_prepare_wproj(st, vis->u + off, vis->v + off, vis->w + off,
                             (const double2 *)vis->vis + off, cnt, N, theta, K, wkern->oversampling,
                             wkern->plane_count, wkern->w_min, wkern->w_step, rec, visf, err);
        launch_romein(st, rec, visf, cnt, taps32, grid32, slot, 0, N, K, sms);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "rg_grid_wprojection_noalloc launch");
    // the error word is read before the caller's grid is touched: a rejected
    // call leaves it as it was
    unsigned herr = 0;
    RG_CUDA(cudaMemcpyAsync(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost, st));
    RG_CUDA(cudaStreamSynchronize(st));
    if (herr & DERR_NONFINITE) return fail(RG_ERR_INVALID_ARGUMENT, "non-finite u, v or w in the visibilities");
    if (herr & DERR_PLANE_RANGE)
        return fail(RG_ERR_INVALID_ARGUMENT, "a visibility's w (or sub-cell index) falls outside the w-kernel table");
    if (herr & DERR_GRID_RANGE)
        return fail(RG_ERR_INVALID_ARGUMENT, "a visibility's kernel footprint lies outside the grid");
    launch_add_f32_to_f64(st, grid32, (double2 *)uvgrid, cells, (flags & RG_GRID_OVERWRITE) ? 1 : 0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "rg_grid_wprojection_noalloc launch");
    RG_CUDA(cudaStreamSynchronize(st));
    return RG_OK;
}
