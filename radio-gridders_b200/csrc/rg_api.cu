// C-ABI layer: argument checks, host/device staging, scratch management and
// the launch sequences of each entry point (include/radio_gridders.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rg_internal.h"

namespace rg {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

rg_status fail(rg_status st, const std::string &msg)
{
    set_error(msg);
    return st;
}

rg_status cuda_fail(cudaError_t e, const char *what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(e == cudaErrorMemoryAllocation ? RG_ERR_OUT_OF_MEMORY : RG_ERR_CUDA, m);
}

bool is_device_pointer(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

rg_status scratch(rg_context *ctx, const char *name, size_t bytes, void **out)
{
    Buffer &b = ctx->scratch[name];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
        if (b.ptr) {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(b.ptr);
            b.ptr = nullptr;
            b.bytes = 0;
        }
        size_t want = bytes + bytes / 8;  // some headroom against regrowth
        if (cudaMalloc(&b.ptr, want) != cudaSuccess) {
            cudaGetLastError();
            b.ptr = nullptr;
            if (cudaMalloc(&b.ptr, bytes) != cudaSuccess) {
                cudaGetLastError();
                b.ptr = nullptr;
                return fail(RG_ERR_OUT_OF_MEMORY,
                            std::string("device allocation failed for scratch '") + name + "' (" +
                                std::to_string(bytes) + " bytes)");
            }
            want = bytes;
        }
        b.bytes = want;
        ctx->scratch_gen++;
    }
    *out = b.ptr;
    return RG_OK;
}

rg_status stage_in(rg_context *ctx, const void *ptr, size_t bytes, const char *name, const void **dev)
{
    if (bytes == 0) {
        *dev = ptr;
        return RG_OK;
    }
    if (is_device_pointer(ptr)) {
        *dev = ptr;
        return RG_OK;
    }
    void *d = nullptr;
    RG_CHECK(scratch(ctx, name, bytes, &d));
    RG_CUDA(cudaMemcpyAsync(d, ptr, bytes, cudaMemcpyHostToDevice, ctx->stream));
    *dev = d;
    return RG_OK;
}

rg_status out_view(rg_context *ctx, void *ptr, size_t bytes, const char *name, bool load,
                          OutView *ov)
{
    ov->user = ptr;
    ov->bytes = bytes;
    if (is_device_pointer(ptr)) {
        ov->dev = ptr;
        ov->host = false;
        return RG_OK;
    }
    ov->host = true;
    RG_CHECK(scratch(ctx, name, bytes, &ov->dev));
    if (load) RG_CUDA(cudaMemcpyAsync(ov->dev, ptr, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return RG_OK;
}

rg_status finish_out(rg_context *ctx, const OutView &ov)
{
    if (ov.host) RG_CUDA(cudaMemcpyAsync(ov.user, ov.dev, ov.bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return RG_OK;
}

static rg_status check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what);
    return RG_OK;
}

rg_status diag_begin(rg_context *ctx, Diag *d)
{
    void *p = nullptr;
    RG_CHECK(scratch(ctx, "diag", 64, &p));
    RG_CUDA(cudaMemsetAsync(p, 0, 64, ctx->stream));
    d->err = (unsigned *)p;
    d->counters = (unsigned long long *)((char *)p + 16);
    return RG_OK;
}

rg_status diag_end(rg_context *ctx, const Diag &d, unsigned long long *counters_out)
{
    unsigned char host[64];
    RG_CUDA(cudaMemcpyAsync(host, d.err, 64, cudaMemcpyDeviceToHost, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    unsigned err;
    std::memcpy(&err, host, sizeof(err));
    if (counters_out) std::memcpy(counters_out, host + 16, 2 * sizeof(unsigned long long));
    if (err & DERR_NONFINITE) return fail(RG_ERR_INVALID_ARGUMENT, "non-finite u, v or w in the visibilities");
    if (err & DERR_PLANE_RANGE)
        return fail(RG_ERR_INVALID_ARGUMENT, "a visibility's w (or sub-cell index) falls outside the w-kernel table");
    if (err & DERR_GRID_RANGE)
        return fail(RG_ERR_INVALID_ARGUMENT, "a visibility's kernel footprint lies outside the grid");
    if (err & DERR_CAPACITY) return fail(RG_ERR_UNSUPPORTED, "internal capacity exceeded");
    return RG_OK;
}

rg_status check_vis(const rg_vis *vis)
{
    if (!vis) return fail(RG_ERR_INVALID_ARGUMENT, "vis is NULL");
    if (vis->n < 0) return fail(RG_ERR_INVALID_ARGUMENT, "vis->n is negative");
    if (vis->n > 0 && (!vis->u || !vis->v || !vis->w || !vis->vis))
        return fail(RG_ERR_INVALID_ARGUMENT, "vis arrays must be non-NULL when n > 0");
    if (vis->n > (int64_t)1 << 31) return fail(RG_ERR_UNSUPPORTED, "more than 2^31 visibilities in one call");
    return RG_OK;
}

rg_status check_wkern(const rg_wkern *wk)
{
    if (!wk || !wk->data) return fail(RG_ERR_INVALID_ARGUMENT, "w-kernel table is NULL");
    if (wk->size != 4 && wk->size != 8 && wk->size != 16 && wk->size != 32)
        return fail(RG_ERR_UNSUPPORTED, "kernel support must be 4, 8, 16 or 32 cells");
    if (wk->oversampling < 1 || wk->oversampling > 64)
        return fail(RG_ERR_INVALID_ARGUMENT, "oversampling must be in [1, 64]");
    if (wk->plane_count < 1) return fail(RG_ERR_INVALID_ARGUMENT, "plane_count must be >= 1");
    if (!(wk->w_step > 0.0) || !std::isfinite(wk->w_min))
        return fail(RG_ERR_INVALID_ARGUMENT, "w_step must be > 0 and w_min finite");
    const double taps = (double)wk->plane_count * wk->oversampling * wk->oversampling * wk->size * wk->size;
    if (taps > 2.0e9) return fail(RG_ERR_UNSUPPORTED, "w-kernel table too large");
    return RG_OK;
}

struct DevVis {
    const double *u, *v, *w;
    const double2 *vis;
    int64_t n;
    bool device = false;  // every array is the caller's own device buffer (nothing staged)
};

static rg_status stage_vis(rg_context *ctx, const rg_vis *vis, DevVis *dv)
{
    const size_t b = sizeof(double) * (size_t)vis->n;
    const void *p;
    RG_CHECK(stage_in(ctx, vis->u, b, "in_u", &p));
    dv->u = (const double *)p;
    RG_CHECK(stage_in(ctx, vis->v, b, "in_v", &p));
    dv->v = (const double *)p;
    RG_CHECK(stage_in(ctx, vis->w, b, "in_w", &p));
    dv->w = (const double *)p;
    RG_CHECK(stage_in(ctx, vis->vis, 2 * b, "in_vis", &p));
    dv->vis = (const double2 *)p;
    dv->n = vis->n;
    dv->device = dv->u == vis->u && dv->v == vis->v && dv->w == vis->w && (const void *)dv->vis == vis->vis;
    return RG_OK;
}

// dup: the W-towers layout with each slice stored twice (launch_convert_table_dup)
static rg_status stage_taps(rg_context *ctx, const rg_wkern *wk, float2 **taps, bool dup = false)
{
    const int64_t ntaps = (int64_t)wk->plane_count * wk->oversampling * wk->oversampling * wk->size * wk->size;
    const void *src;
    RG_CHECK(stage_in(ctx, wk->data, sizeof(double2) * ntaps, "in_wkern", &src));
    void *dst;
    RG_CHECK(scratch(ctx, dup ? "taps32_dup" : "taps32", sizeof(float2) * ntaps * (dup ? 2 : 1), &dst));
    if (dup)
        launch_convert_table_dup(ctx->stream, (const double2 *)src, (float2 *)dst, ntaps, wk->size * wk->size);
    else
        launch_convert_table(ctx->stream, (const double2 *)src, (float2 *)dst, ntaps);
    ctx->launches++;
    *taps = (float2 *)dst;
    return check_launch("convert w-kernel table");
}

void begin_call(rg_context *ctx)
{
    ctx->n_events = 0;
    ctx->timings.clear();
    ctx->launches = 0;
    for (int64_t &v : ctx->stats) v = 0;
}

void begin_stage(rg_context *ctx, const char *name)
{
    if (!ctx->profiling) return;
    if (ctx->n_events == (int)ctx->events.size()) {
        rg_stage_event e;
        cudaEventCreate(&e.start);
        cudaEventCreate(&e.stop);
        ctx->events.push_back(e);
    }
    rg_stage_event &e = ctx->events[ctx->n_events];
    e.name = name;
    cudaEventRecord(e.start, ctx->stream);
}

void end_stage(rg_context *ctx)
{
    if (!ctx->profiling) return;
    cudaEventRecord(ctx->events[ctx->n_events].stop, ctx->stream);
    ctx->n_events++;
}

void collect_timings(rg_context *ctx)
{
    ctx->timings.clear();
    if (!ctx->profiling) return;
    for (int i = 0; i < ctx->n_events; i++) {
        float ms = 0.f;
        cudaEventSynchronize(ctx->events[i].stop);
        cudaEventElapsedTime(&ms, ctx->events[i].start, ctx->events[i].stop);
        ctx->timings.emplace_back(ctx->events[i].name, ms);
    }
}

static int ilog2_int(int n)
{
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}

static rg_status get_twiddles32(rg_context *ctx, int n, float2 **tw)
{
    std::string name = "tw32_" + std::to_string(n);
    auto it = ctx->scratch.find(name);
    bool fresh = it == ctx->scratch.end();
    void *p;
    RG_CHECK(scratch(ctx, name.c_str(), sizeof(float2) * n, &p));
    if (fresh) fft32_init_twiddles(ctx->stream, (float2 *)p, n);
    *tw = (float2 *)p;
    return RG_OK;
}

}  // namespace rg

using namespace rg;

extern "C" {

const char *rg_last_error(void) { return g_last_error.c_str(); }

rg_status rg_context_create(int device, rg_context **out)
{
    if (!out) return fail(RG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(RG_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) return fail(RG_ERR_INVALID_ARGUMENT, "device index out of range");
    RG_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    RG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return fail(RG_ERR_UNSUPPORTED, std::string("this build targets sm_100a (B200); device is ") + prop.name);
    rg_context *ctx = new rg_context();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return fail(RG_ERR_CUDA, "cudaStreamCreate failed");
    }
    ctx->stream = ctx->own_stream;
    if (cudaMallocHost(&ctx->pinned, 256) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamDestroy(ctx->own_stream);
        delete ctx;
        return fail(RG_ERR_OUT_OF_MEMORY, "pinned host allocation failed");
    }
    *out = ctx;
    return RG_OK;
}

rg_status rg_context_destroy(rg_context *ctx)
{
    if (!ctx) return RG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto &kv : ctx->tower_plans)
        if (kv.second.graph_exec) cudaGraphExecDestroy(kv.second.graph_exec);
    for (int b = 0; b < rg_context::kBatchSets; b++)
        for (cudaEvent_t e : {ctx->ev_in[b], ctx->ev_used[b], ctx->ev_done[b], ctx->ev_out[b]})
            if (e) cudaEventDestroy(e);
    if (ctx->copy_in) {
        cudaStreamSynchronize(ctx->copy_in);
        cudaStreamDestroy(ctx->copy_in);
    }
    if (ctx->copy_out) {
        cudaStreamSynchronize(ctx->copy_out);
        cudaStreamDestroy(ctx->copy_out);
    }
    if (ctx->pinned_steps) cudaFreeHost(ctx->pinned_steps);
    for (auto &kv : ctx->scratch)
        if (kv.second.ptr) cudaFree(kv.second.ptr);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    for (auto &e : ctx->events) {
        cudaEventDestroy(e.start);
        cudaEventDestroy(e.stop);
    }
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return RG_OK;
}

rg_status rg_context_set_stream(rg_context *ctx, void *stream)
{
    if (!ctx) return fail(RG_ERR_INVALID_ARGUMENT, "ctx is NULL");
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return RG_OK;
}

rg_status rg_context_set_autotune(rg_context *ctx, int enabled)
{
    if (!ctx) return fail(RG_ERR_INVALID_ARGUMENT, "ctx is NULL");
    ctx->autotune = enabled != 0;
    return RG_OK;
}

rg_status rg_context_set_graphs(rg_context *ctx, int enabled)
{
    if (!ctx) return fail(RG_ERR_INVALID_ARGUMENT, "ctx is NULL");
    ctx->use_graphs = enabled != 0;
    return RG_OK;
}

rg_status rg_context_set_profiling(rg_context *ctx, int enabled)
{
    if (!ctx) return fail(RG_ERR_INVALID_ARGUMENT, "ctx is NULL");
    ctx->profiling = enabled != 0;
    return RG_OK;
}

int rg_last_timings(rg_context *ctx, const char **names, float *ms, int n)
{
    if (!ctx) return 0;
    int k = 0;
    for (auto &t : ctx->timings) {
        if (k >= n) break;
        if (names) names[k] = t.first.c_str();
        if (ms) ms[k] = t.second;
        k++;
    }
    return k;
}

int rg_last_stats(rg_context *ctx, int64_t *out, int n)
{
    if (!ctx || !out) return 0;
    int k = n < 11 ? n : 11;
    for (int i = 0; i < k; i++) out[i] = ctx->stats[i];
    return k;
}

rg_status rg_grid_wprojection(rg_context *ctx, double *uvgrid, int grid_size, double theta,
                              const rg_vis *vis, const rg_wkern *wkern, int flags)
{
    if (!ctx || !uvgrid) return fail(RG_ERR_INVALID_ARGUMENT, "ctx and uvgrid must be non-NULL");
    if (grid_size < 2 || grid_size > 16384) return fail(RG_ERR_UNSUPPORTED, "grid_size must be in [2, 16384]");
    if (!(theta > 0.0) || !std::isfinite(theta)) return fail(RG_ERR_INVALID_ARGUMENT, "theta must be > 0");
    RG_CHECK(check_vis(vis));
    RG_CHECK(check_wkern(wkern));
    RG_CUDA(cudaSetDevice(ctx->device));
    begin_call(ctx);
    const int N = grid_size;
    const int64_t cells = (int64_t)N * N;
    DevVis dv;
    begin_stage(ctx, "stage_in");
    RG_CHECK(stage_vis(ctx, vis, &dv));
    // Gridding reads K^2 taps per visibility.  When those are fewer bytes
    // (16 per FP64 tap) than converting the whole table moves (its FP64 read
    // and FP32 write, 24 per entry), the gridder reads the FP64 table itself
    // and rounds each tap as the conversion would.
    float2 *taps = nullptr;
    const double2 *taps64 = nullptr;
    const int64_t ntaps =
        (int64_t)wkern->plane_count * wkern->oversampling * wkern->oversampling * wkern->size * wkern->size;
    if ((double)vis->n * wkern->size * wkern->size * 16.0 < 24.0 * (double)ntaps) {
        const void *src;
        RG_CHECK(stage_in(ctx, wkern->data, sizeof(double2) * ntaps, "in_wkern", &src));
        taps64 = (const double2 *)src;
    } else {
        RG_CHECK(stage_taps(ctx, wkern, &taps));
    }
    end_stage(ctx);
    Diag d;
    RG_CHECK(diag_begin(ctx, &d));
    void *rec, *visf, *grid32, *zero_slot;
    RG_CHECK(scratch(ctx, "rec", sizeof(int4) * (size_t)dv.n, &rec));
    RG_CHECK(scratch(ctx, "visf", sizeof(float2) * (size_t)dv.n, &visf));
    RG_CHECK(scratch(ctx, "grid32", sizeof(float2) * (size_t)cells, &grid32));
    RG_CHECK(scratch(ctx, "zero_slot", 16, &zero_slot));
    RG_CUDA(cudaMemsetAsync(zero_slot, 0, 16, ctx->stream));
    RG_CUDA(cudaMemsetAsync(grid32, 0, sizeof(float2) * (size_t)cells, ctx->stream));
    if (dv.n > 0) {
        begin_stage(ctx, "prepare");
        launch_prepare_wproj(ctx->stream, dv.u, dv.v, dv.w, dv.vis, dv.n, N, theta, wkern->size,
                             wkern->oversampling, wkern->plane_count, wkern->w_min, wkern->w_step,
                             (int4 *)rec, (float2 *)visf, d.err);
        end_stage(ctx);
        begin_stage(ctx, "romein");
        launch_romein(ctx->stream, (const int4 *)rec, (const float2 *)visf, dv.n, taps,
                      (float2 *)grid32, (const int *)zero_slot, 0, N, wkern->size, ctx->sm_count, 1, 0, 0, taps64);
        end_stage(ctx);
        ctx->launches += 2;
        RG_CHECK(check_launch("W-projection gridding"));
    }
    OutView ov;
    RG_CHECK(out_view(ctx, uvgrid, sizeof(double2) * (size_t)cells, "out_grid",
                      !(flags & RG_GRID_OVERWRITE), &ov));
    begin_stage(ctx, "to_fp64");
    launch_add_f32_to_f64(ctx->stream, (const float2 *)grid32, (double2 *)ov.dev, cells,
                          (flags & RG_GRID_OVERWRITE) ? 1 : 0);
    end_stage(ctx);
    ctx->launches++;
    RG_CHECK(check_launch("grid accumulation"));
    begin_stage(ctx, "stage_out");
    RG_CHECK(finish_out(ctx, ov));
    end_stage(ctx);
    RG_CHECK(diag_end(ctx, d, nullptr));
    collect_timings(ctx);
    ctx->stats[0] = dv.n;
    ctx->stats[1] = 1;
    ctx->stats[2] = 1;
    ctx->stats[3] = 0;
    ctx->stats[4] = 0;
    ctx->stats[5] = ctx->launches;
    return RG_OK;
}

}  // extern "C"

namespace rg {

// One W-towers pass with fixed capacities: every launch is sized by the plan's
// capacities and reads the live counts (w floors, active sub-grids, floor
// groups) from device memory, so the host enqueues the whole pass without
// waiting; one read-back at the end returns the error word, the counters and
// the live counts.  *overflow is set when a capacity was too small (the caller
// grows the plan and runs again).
// Enqueues one W-towers pass on ctx->stream, ending with the copy of the
// diagnostics block (error word, counters, counts, floor range) into the
// context's pinned host buffer; wtowers_check reads it after a sync.  Nothing
// here synchronises, so the sequence can also be captured into a CUDA graph.
static rg_status wtowers_enqueue(rg_context *ctx, const DevVis &dv, const float2 *taps, const rg_wkern *wkern,
                                 const LearnedTaps *lt, double *out_dev, int N, double theta, int S, int M,
                                 double winc, int flags, TowerPlan &pl, void *diag_host = nullptr,
                                 int *poison = nullptr)
{
    cudaStream_t st = ctx->stream;
    const int K = lt ? lt->ksize : wkern->size;
    const int chunk = S - M;
    const int nchunk = N / chunk + 1;
    const int ntowers = nchunk * nchunk;
    const int64_t sub_cells = (int64_t)S * S;
    const int nbins_cap = ntowers * pl.floors_cap;

    Diag d;
    RG_CHECK(diag_begin(ctx, &d));
    int *range = (int *)((char *)d.err + 48);    // {wp_min, nfloor, ok}
    int *counts = (int *)((char *)d.err + 32);   // {slots, groups, towers with data, marked strips}

    void *mm, *active, *marks, *masks, *rec, *visf, *slot_of_bin, *bin_of_slot, *tfirst, *tcount, *gbegin, *gend,
        *tgfirst, *tgcount, *slots, *partial, *subimg, *ph;
    const int strips = S / kStripCols;
    RG_CHECK(scratch(ctx, "wminmax", 16, &mm));
    RG_CHECK(scratch(ctx, "active", sizeof(int) * (size_t)nbins_cap, &active));
    RG_CHECK(scratch(ctx, "strip_marks", (size_t)nbins_cap * strips, &marks));
    RG_CHECK(scratch(ctx, "slot_masks", sizeof(unsigned) * (size_t)pl.slots_cap * mask_words(S), &masks));
    RG_CHECK(scratch(ctx, "rec", sizeof(int4) * (size_t)dv.n, &rec));
    RG_CHECK(scratch(ctx, "visf", sizeof(float2) * (size_t)dv.n, &visf));
    void *feat = nullptr;
    if (lt) RG_CHECK(scratch(ctx, "learned_feat", sizeof(float4) * (size_t)dv.n, &feat));
    RG_CHECK(scratch(ctx, "slot_of_bin", sizeof(int) * (size_t)nbins_cap, &slot_of_bin));
    RG_CHECK(scratch(ctx, "bin_of_slot", sizeof(int) * (size_t)nbins_cap, &bin_of_slot));
    RG_CHECK(scratch(ctx, "tower_first", sizeof(int) * (size_t)ntowers, &tfirst));
    RG_CHECK(scratch(ctx, "tower_count", sizeof(int) * (size_t)ntowers, &tcount));
    RG_CHECK(scratch(ctx, "group_begin", sizeof(int) * (size_t)nbins_cap, &gbegin));
    RG_CHECK(scratch(ctx, "group_end", sizeof(int) * (size_t)nbins_cap, &gend));
    RG_CHECK(scratch(ctx, "tower_group_first", sizeof(int) * (size_t)ntowers, &tgfirst));
    RG_CHECK(scratch(ctx, "tower_group_count", sizeof(int) * (size_t)ntowers, &tgcount));
    RG_CHECK(scratch(ctx, "slots", sizeof(float2) * (size_t)(sub_cells * pl.slots_cap), &slots));
    RG_CHECK(scratch(ctx, "partial", sizeof(float2) * (size_t)(sub_cells * pl.groups_cap), &partial));
    RG_CHECK(scratch(ctx, "subimg", sizeof(float2) * (size_t)(sub_cells * ntowers), &subimg));
    float2 *tw;
    RG_CHECK(get_twiddles32(ctx, S, &tw));
    {
        char key[160];
        std::snprintf(key, sizeof(key), "phq_%d_%.17g_%.17g", S, theta, winc);
        bool fresh = ctx->scratch.find(key) == ctx->scratch.end();
        RG_CHECK(scratch(ctx, key, sizeof(uint32_t) * (size_t)sub_cells, &ph));
        if (fresh) {
            launch_fresnel_table(st, (uint32_t *)ph, S, theta, winc);
            ctx->launches++;
        }
    }
    RG_CUDA(cudaMemsetAsync(active, 0, sizeof(int) * (size_t)nbins_cap, st));
    RG_CUDA(cudaMemsetAsync(marks, 0, (size_t)nbins_cap * strips, st));
    if (ctx->slots_owner != &pl) {  // the slot buffer was last used by another shape
        pl.zeroed_slots = 0;
        ctx->slots_owner = &pl;
    }

    TowerGeom g;
    g.grid_size = N;
    g.subgrid = S;
    g.margin = M;
    g.chunk = chunk;
    g.nchunk = nchunk;
    g.ksize = K;
    g.ov = lt ? 1 : wkern->oversampling;
    g.planes = lt ? 1 : wkern->plane_count;
    g.theta = theta;
    g.winc = winc;
    g.wk_wmin = lt ? 0.0 : wkern->w_min;
    g.wk_wstep = lt ? 1.0 : wkern->w_step;
    g.tower_sel = pl.tower_sel;

    begin_stage(ctx, "w_range");
    launch_minmax_w(st, dv.u, dv.v, dv.w, dv.n, (double *)mm, d.err);
    launch_w_floors(st, (const double *)mm, winc, pl.floors_cap, range, d.err);
    end_stage(ctx);
    begin_stage(ctx, "prepare");
    if (dv.n > 0)
        launch_prepare_towers(st, dv.u, dv.v, dv.w, dv.vis, dv.n, g, range, (int4 *)rec, (float2 *)visf,
                              (int *)active, (unsigned char *)marks, d.err, d.counters, (float4 *)feat);
    end_stage(ctx);
    begin_stage(ctx, "compact");
    launch_compact_bins(st, (const int *)active, range, (int *)slot_of_bin, (int *)bin_of_slot, counts,
                        (int *)tfirst, (int *)tcount, ntowers, tower_row_strips(S), pl.tune.group_items * ctx->sm_count,
                        (int *)gbegin,
                        (int *)gend, (int *)tgfirst, (int *)tgcount);
    end_stage(ctx);
    // Sub-grids are left zeroed by the previous pass's column stage; only
    // memory never cleared (new capacity, or after an overflowed pass) is zeroed.
    if (pl.zeroed_slots < (size_t)pl.slots_cap) {
        begin_stage(ctx, "zero_subgrids");
        RG_CUDA(cudaMemsetAsync(slots, 0, sizeof(float2) * (size_t)(sub_cells * pl.slots_cap), st));
        end_stage(ctx);
        pl.zeroed_slots = (size_t)pl.slots_cap;
    }
    if (lt) {
        begin_stage(ctx, "learned_gridding");
        if (dv.n > 0)
            launch_learned_towers(st, (const int4 *)rec, (const float2 *)visf, (const float4 *)feat, dv.n,
                                  (const int *)slot_of_bin, pl.slots_cap, (float2 *)slots, S, lt->P, lt->PB,
                                  lt->ksize, lt->inv_wmax, lt->scale, ctx->sm_count, d.err);
        end_stage(ctx);
    } else {
        begin_stage(ctx, "romein");
        if (dv.n > 0)
            launch_romein(st, (const int4 *)rec, (const float2 *)visf, dv.n, taps, (float2 *)slots,
                          (const int *)slot_of_bin, sub_cells, S, K, ctx->sm_count, pl.slots_cap,
                          pl.tune.romein_points, ilog2_int(S));
        end_stage(ctx);
    }
    begin_stage(ctx, "fft_cols_backward");
    launch_slot_masks(st, (const unsigned char *)marks, (const int *)bin_of_slot, counts, pl.slots_cap, S,
                      (unsigned *)masks);
    launch_sparse_cols(st, (float2 *)slots, (const unsigned *)masks, counts, pl.slots_cap, S, tw, ctx->sm_count);
    end_stage(ctx);
    begin_stage(ctx, "tower_rows");
    launch_tower_rows(st, (float2 *)slots, (const unsigned *)masks, (const int *)bin_of_slot, (const int *)gbegin,
                      (const int *)gend, range, counts, pl.slots_cap, pl.groups_cap, (const uint32_t *)ph,
                      (float2 *)partial, S, tw);
    end_stage(ctx);
    begin_stage(ctx, "tower_finish");
    launch_tower_finish(st, pl.groups_cap, (const int *)tgfirst, (const int *)tgcount, ntowers,
                        (const float2 *)partial, (float2 *)subimg, S, tw);
    end_stage(ctx);
    begin_stage(ctx, "fft_cols_forward");
    launch_fft32_cols(st, (float2 *)subimg, ntowers, S, -1, tw, (const int *)tcount);  // towers with data only
    end_stage(ctx);
    begin_stage(ctx, "add_back");
    launch_add_back(st, (const float2 *)subimg, (const int *)tcount, (double2 *)out_dev, N, S, M, chunk, nchunk,
                    (flags & RG_GRID_OVERWRITE) ? 1 : 0, range, counts, pl.slots_cap, pl.groups_cap, poison);
    end_stage(ctx);
    ctx->launches += 11;  // minmax, floors, prepare, compact, romein, masks, cols, rows, finish, cols, add-back
    RG_CHECK(check_launch("W-towers pass"));

    RG_CUDA(cudaMemcpyAsync(diag_host ? diag_host : ctx->pinned, d.err, 64, cudaMemcpyDeviceToHost, st));
    return RG_OK;
}

// After the stream has passed a wtowers_enqueue: capacities seen, overflow,
// input errors and the call statistics.
static rg_status wtowers_check(rg_context *ctx, TowerPlan &pl, bool *overflow, const void *diag_host = nullptr)
{
    const unsigned char *host = (const unsigned char *)(diag_host ? diag_host : ctx->pinned);
    unsigned err;
    unsigned long long ctr[2];
    int cnt[4], rng[3];
    std::memcpy(&err, host, 4);
    std::memcpy(ctr, host + 16, 16);
    std::memcpy(cnt, host + 32, 16);
    std::memcpy(rng, host + 48, 12);
    pl.seen_floors = rng[1];
    pl.seen_slots = cnt[0];
    pl.seen_groups = cnt[1];
    if (err & DERR_TIMEOUT) return fail(RG_ERR_CUDA, "a bounded wait for tensor-core work timed out");
    *overflow = (err & DERR_CAPACITY) || !rng[2] || cnt[0] > pl.slots_cap || cnt[1] > pl.groups_cap;
    if (*overflow) {
        pl.zeroed_slots = 0;  // some sub-grids may not have been consumed (cleared)
        return RG_OK;
    }
    if (err & DERR_NONFINITE) return fail(RG_ERR_INVALID_ARGUMENT, "non-finite u, v or w in the visibilities");
    if (err & DERR_PLANE_RANGE)
        return fail(RG_ERR_INVALID_ARGUMENT, "a visibility's w (or sub-cell index) falls outside the w-kernel table");
    ctx->stats[0] = (int64_t)ctr[0];
    ctx->stats[1] = cnt[0];
    ctx->stats[2] = cnt[2];
    ctx->stats[3] = rng[1];
    ctx->stats[4] = (int64_t)ctr[1];
    ctx->stats[6] = cnt[3];
    ctx->stats[7] = cnt[1];
    ctx->stats[8] = pl.tune.romein_points;
    ctx->stats[9] = pl.tune.group_items;
    return RG_OK;
}

static rg_status wtowers_pass(rg_context *ctx, const DevVis &dv, const float2 *taps, const rg_wkern *wkern,
                              const LearnedTaps *lt, double *out_dev, int N, double theta, int S, int M,
                              double winc, int flags, TowerPlan &pl, bool *overflow)
{
    RG_CHECK(wtowers_enqueue(ctx, dv, taps, wkern, lt, out_dev, N, theta, S, M, winc, flags, pl));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return wtowers_check(ctx, pl, overflow);
}

// Autotuner: coordinate search over the pass's schedule knobs — Romein grid
// points per thread (threads per CTA) and the row stage's floor-group size
// (work items per SM) — timing whole passes with CUDA events into a scratch
// grid.  Each candidate runs twice and the second run is timed.  The search
// runs once per shape, after the capacities are sized; results are per plan.
static rg_status wtowers_autotune(rg_context *ctx, const DevVis &dv, const float2 *taps, const rg_wkern *wkern,
                                  const LearnedTaps *lt, int N, double theta, int S, int M, double winc,
                                  TowerPlan &pl)
{
    const int K = lt ? lt->ksize : wkern->size;
    void *tmp;
    RG_CHECK(scratch(ctx, "tune_grid", sizeof(double2) * (size_t)N * N, &tmp));
    cudaEvent_t e0, e1;
    RG_CUDA(cudaEventCreate(&e0));
    RG_CUDA(cudaEventCreate(&e1));
    const bool prof = ctx->profiling;
    ctx->profiling = false;
    // A candidate whose floor groups outgrow the plan's capacity (more work
    // items per SM make more, smaller groups) is skipped: its pass wrote
    // nothing, and the plan keeps the capacities the caller's pass sized.
    auto time_pass = [&](float *ms) -> rg_status {
        bool overflow = false;
        for (int rep = 0; rep < 2; rep++) {
            RG_CUDA(cudaEventRecord(e0, ctx->stream));
            RG_CHECK(wtowers_pass(ctx, dv, taps, wkern, lt, (double *)tmp, N, theta, S, M, winc, RG_GRID_OVERWRITE,
                                  pl, &overflow));
            RG_CUDA(cudaEventRecord(e1, ctx->stream));
            RG_CUDA(cudaEventSynchronize(e1));
            if (overflow) {
                *ms = 1e30f;
                return RG_OK;
            }
        }
        RG_CUDA(cudaEventElapsedTime(ms, e0, e1));
        return RG_OK;
    };
    rg_status st = RG_OK;
    TowerTuning best = pl.tune;
    float best_ms = 1e30f;
    if (!lt) {  // Romein variants (the learned gridder has no points-per-thread knob)
        int cand[3], nc = 0;
        if (K == 16) { cand[0] = 2; cand[1] = 4; cand[2] = 8; nc = 3; }
        else if (K == 8) { cand[0] = 1; cand[1] = 2; cand[2] = 4; nc = 3; }
        else if (K == 32) { cand[0] = 4; cand[1] = 8; nc = 2; }
        for (int c = 0; c < nc && st == RG_OK; c++) {
            pl.tune.romein_points = cand[c];
            float ms = 0;
            st = time_pass(&ms);
            if (st == RG_OK && ms < best_ms) { best_ms = ms; best = pl.tune; }
        }
        pl.tune = best;
    }
    const int gcand[3] = {4, 8, 16};
    for (int c = 0; c < 3 && st == RG_OK; c++) {
        pl.tune.group_items = gcand[c];
        float ms = 0;
        st = time_pass(&ms);
        if (st == RG_OK && ms < best_ms) { best_ms = ms; best = pl.tune; }
    }
    pl.tune = best;
    pl.tuned = true;
    ctx->profiling = prof;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

// Graph replay of a whole pass: captured once per plan and set of device
// buffers (inputs, taps, output), then launched as one graph per call.
static void drop_graph(TowerPlan &pl)
{
    if (pl.graph_exec) cudaGraphExecDestroy(pl.graph_exec);
    pl.graph_exec = nullptr;
    pl.graph_key.clear();
}

// Capture failure is not an error of the call (its grid is already written):
// the plan simply keeps using ordinary launches.
static void capture_pass(rg_context *ctx, const DevVis &dv, const float2 *taps, const rg_wkern *wkern,
                         const LearnedTaps *lt, double *out_dev, int N, double theta, int S, int M, double winc,
                         int flags, TowerPlan &pl, const std::string &key)
{
    drop_graph(pl);
    const uint64_t gen0 = ctx->scratch_gen;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    const int launches0 = ctx->launches;
    const rg_status st = wtowers_enqueue(ctx, dv, taps, wkern, lt, out_dev, N, theta, S, M, winc, flags, pl);
    pl.graph_launches = ctx->launches - launches0;
    ctx->launches = launches0;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    cudaGetLastError();
    if (st == RG_OK && e == cudaSuccess && graph && ctx->scratch_gen == gen0 &&
        cudaGraphInstantiate(&pl.graph_exec, graph, 0) == cudaSuccess) {
        pl.graph_key = key;
        pl.graph_scratch_gen = ctx->scratch_gen;
    } else {
        cudaGetLastError();
        pl.graph_exec = nullptr;
    }
    if (graph) cudaGraphDestroy(graph);
}

// W-towers with table taps (lt == nullptr) or learned taps (wkern unused).
rg_status grid_wtowers_impl(rg_context *ctx, double *uvgrid, int grid_size, double theta, const rg_vis *vis,
                            const rg_wkern *wkern, const LearnedTaps *lt, int subgrid_size, int subgrid_margin,
                            double wincrement, int flags, const int32_t *part_of_tower, int part)
{
    if (!ctx || !uvgrid) return fail(RG_ERR_INVALID_ARGUMENT, "ctx and uvgrid must be non-NULL");
    if (grid_size < 2 || grid_size > 16384) return fail(RG_ERR_UNSUPPORTED, "grid_size must be in [2, 16384]");
    if (!(theta > 0.0) || !std::isfinite(theta)) return fail(RG_ERR_INVALID_ARGUMENT, "theta must be > 0");
    if (!(wincrement > 0.0) || !std::isfinite(wincrement))
        return fail(RG_ERR_INVALID_ARGUMENT, "wincrement must be > 0");
    RG_CHECK(check_vis(vis));
    if (!lt) RG_CHECK(check_wkern(wkern));
    const int S = subgrid_size, M = subgrid_margin, K = lt ? lt->ksize : wkern->size;
    if (lt && wincrement / 2 > lt->wmax)
        return fail(RG_ERR_INVALID_ARGUMENT, "the learned kernel's w range is narrower than wincrement / 2");
    // src/reference/grid.c:300-302
    if (M < K) return fail(RG_ERR_INVALID_ARGUMENT, "subgrid margin must be >= the kernel support");
    if (S % 2 || M % 2) return fail(RG_ERR_INVALID_ARGUMENT, "subgrid size and margin must be even");
    if (M >= S) return fail(RG_ERR_INVALID_ARGUMENT, "subgrid margin must be smaller than the subgrid");
    if (!fft32_supported(S)) return fail(RG_ERR_UNSUPPORTED, "subgrid size must be a power of two in [64, 1024]");
    RG_CUDA(cudaSetDevice(ctx->device));
    begin_call(ctx);
    const int N = grid_size;
    const int64_t cells = (int64_t)N * N;
    const int chunk = S - M;
    const int ntowers = (N / chunk + 1) * (N / chunk + 1);

    DevVis dv;
    begin_stage(ctx, "stage_in");
    RG_CHECK(stage_vis(ctx, vis, &dv));
    float2 *taps = nullptr;
    if (!lt) RG_CHECK(stage_taps(ctx, wkern, &taps, true));
    OutView ov;
    RG_CHECK(out_view(ctx, uvgrid, sizeof(double2) * (size_t)cells, "out_grid",
                      !(flags & RG_GRID_OVERWRITE), &ov));
    end_stage(ctx);

    // a share of a tower-partitioned observation: the selected towers as one
    // byte each in device memory, named by their fingerprint (a plan and its
    // captured graph keep pointing at the same selection)
    std::string selkey;
    const unsigned char *sel_dev = nullptr;
    if (part_of_tower) {
        std::vector<unsigned char> sel((size_t)ntowers);
        uint64_t h = 1469598103934665603ull;  // FNV-1a
        for (int t = 0; t < ntowers; t++) {
            sel[t] = part_of_tower[t] == part ? 1 : 0;
            h = (h ^ sel[t]) * 1099511628211ull;
        }
        char hb[40];
        std::snprintf(hb, sizeof(hb), "_sel%016llx", (unsigned long long)h);
        selkey = hb;
        const std::string name = "tower_sel" + selkey;
        const bool fresh = ctx->scratch.find(name) == ctx->scratch.end();
        void *p = nullptr;
        RG_CHECK(scratch(ctx, name.c_str(), (size_t)ntowers, &p));
        if (fresh) {
            RG_CUDA(cudaMemcpyAsync(p, sel.data(), (size_t)ntowers, cudaMemcpyHostToDevice, ctx->stream));
            RG_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        sel_dev = (const unsigned char *)p;
    }
    char keybuf[240];
    std::snprintf(keybuf, sizeof(keybuf), "%d_%d_%d_%.17g_%.17g_%lld_%c%s", N, S, M, theta, wincrement,
                  (long long)dv.n, lt ? 'L' : 'T', selkey.c_str());
    TowerPlan &pl = ctx->tower_plans[keybuf];
    pl.tower_sel = sel_dev;
    if (!pl.valid) {  // first call for this shape: generous capacities, learn the real sizes
        pl.floors_cap = 256;
        pl.slots_cap = ntowers * 16 + 64;
        pl.groups_cap = pl.slots_cap;
        pl.valid = true;
    }
    // Graph replay when nothing is profiled and every buffer lives on the
    // device: the same plan and the same buffers reuse one captured pass.
    char gkey[256];
    std::snprintf(gkey, sizeof(gkey), "%p_%p_%p_%p_%p_%p_%d", (const void *)dv.u, (const void *)dv.v,
                  (const void *)dv.w, (const void *)dv.vis, (const void *)taps, (void *)ov.dev, flags);
    const bool graphable = ctx->use_graphs && !ctx->profiling && dv.device && !ov.host;
    bool done = false;
    if (graphable && pl.graph_exec && pl.graph_key == gkey && pl.graph_scratch_gen == ctx->scratch_gen &&
        ctx->slots_owner == &pl && pl.zeroed_slots >= (size_t)pl.slots_cap) {
        RG_CUDA(cudaGraphLaunch(pl.graph_exec, ctx->stream));
        RG_CUDA(cudaStreamSynchronize(ctx->stream));
        bool overflow = false;
        RG_CHECK(wtowers_check(ctx, pl, &overflow));
        ctx->launches += pl.graph_launches;
        ctx->stats[10] = 1;
        if (overflow) {
            drop_graph(pl);  // the data outgrew the plan: size it again eagerly
            begin_call(ctx);
        } else {
            done = true;
        }
    }
    // A pass whose capacities overflow writes nothing to the grid (the add-back
    // checks the live counts), so it can simply be rerun with larger ones.
    for (int attempt = 0; attempt < 4 && !done; attempt++) {
        bool overflow = false;
        RG_CHECK(wtowers_pass(ctx, dv, taps, wkern, lt, (double *)ov.dev, N, theta, S, M, wincrement, flags, pl,
                              &overflow));
        if (!overflow) break;
        if (attempt == 3) return fail(RG_ERR_UNSUPPORTED, "W-towers capacities could not be sized");
        if (pl.seen_floors > (1 << 20) || (int64_t)pl.seen_floors * ntowers > ((int64_t)1 << 28))
            return fail(RG_ERR_UNSUPPORTED, "too many (tower, w-floor) bins; increase wincrement");
        pl.floors_cap = pl.seen_floors > pl.floors_cap ? pl.seen_floors + 8 : pl.floors_cap;
        pl.slots_cap = pl.seen_slots > pl.slots_cap ? pl.seen_slots + pl.seen_slots / 8 + 8 : pl.slots_cap;
        pl.groups_cap = pl.seen_groups > pl.groups_cap ? pl.seen_groups + pl.seen_groups / 8 + 8 : pl.groups_cap;
        drop_graph(pl);
        begin_call(ctx);
    }
    // shrink a first-call guess to the sizes seen (keeps memory proportional)
    if (!done && pl.slots_cap > pl.seen_slots + pl.seen_slots / 4 + 64) {
        pl.slots_cap = pl.seen_slots + pl.seen_slots / 8 + 8;
        pl.groups_cap = pl.seen_groups + pl.seen_groups / 8 + 8;
        drop_graph(pl);
    }
    if (!done && ctx->autotune && !pl.tuned && !ctx->profiling) {
        int64_t keep[11];
        std::memcpy(keep, ctx->stats, sizeof(keep));
        const int launches = ctx->launches;
        RG_CHECK(wtowers_autotune(ctx, dv, taps, wkern, lt, N, theta, S, M, wincrement, pl));
        std::memcpy(ctx->stats, keep, sizeof(keep));
        ctx->stats[8] = pl.tune.romein_points;
        ctx->stats[9] = pl.tune.group_items;
        ctx->launches = launches;
        drop_graph(pl);
    }
    if (!done && graphable && (!ctx->autotune || pl.tuned) && pl.zeroed_slots >= (size_t)pl.slots_cap)
        capture_pass(ctx, dv, taps, wkern, lt, (double *)ov.dev, N, theta, S, M, wincrement, flags, pl, gkey);
    begin_stage(ctx, "stage_out");
    RG_CHECK(finish_out(ctx, ov));
    end_stage(ctx);
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    collect_timings(ctx);
    ctx->stats[5] = ctx->launches;
    return RG_OK;
}

// Several observations of one shape in one call, pipelined over three
// streams: the inputs of later steps are copied in (copy_in) and the grids of
// earlier steps copied out (copy_out) while step k's pass runs (ctx->stream),
// with three sets of staging buffers.  Step 0 runs as an ordinary call (it sizes the plan,
// tunes and stages the kernel table, which the later steps reuse) unless an
// earlier call already sized and tuned the shape.  Each
// pass's diagnostics land in their own pinned slot; after the last step they
// are checked in order.  A pass that overflows its capacities writes nothing
// and stops the writes of every later pass of the batch (a device flag), and
// those steps are run again as ordinary calls.
static rg_status batch_streams(rg_context *ctx)
{
    if (!ctx->copy_in) RG_CUDA(cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking));
    if (!ctx->copy_out) RG_CUDA(cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking));
    for (int b = 0; b < rg_context::kBatchSets; b++)
        for (cudaEvent_t *e : {&ctx->ev_in[b], &ctx->ev_used[b], &ctx->ev_done[b], &ctx->ev_out[b]})
            if (!*e) RG_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return RG_OK;
}

rg_status grid_wtowers_batch_impl(rg_context *ctx, int count, double *const *uvgrids, int grid_size, double theta,
                                  const rg_vis *vis, const rg_wkern *wkern, int S, int M, double winc, int flags)
{
    if (!ctx || !uvgrids || !vis || count < 0) return fail(RG_ERR_INVALID_ARGUMENT, "bad batch arguments");
    if (count == 0) return RG_OK;
    bool same = true;
    for (int i = 0; i < count; i++) {
        RG_CHECK(check_vis(&vis[i]));
        if (!uvgrids[i]) return fail(RG_ERR_INVALID_ARGUMENT, "uvgrids must be non-NULL");
        same = same && vis[i].n == vis[0].n;
    }
    const int N = grid_size;
    const size_t grid_bytes = sizeof(double2) * (size_t)N * N;
    const int64_t n = vis[0].n;
    const size_t vb = sizeof(double) * (size_t)n;
    char keybuf[200];
    std::snprintf(keybuf, sizeof(keybuf), "%d_%d_%d_%.17g_%.17g_%lld_%c", N, S, M, theta, winc, (long long)n, 'T');
    // a shape already sized (and tuned) by an earlier call pipelines from step 0;
    // otherwise step 0 is an ordinary call that sizes and tunes it
    auto known = ctx->tower_plans.find(keybuf);
    const bool ready = known != ctx->tower_plans.end() && known->second.valid &&
                       (known->second.tuned || !ctx->autotune);
    int first = 0;
    if (!ready || !same || ctx->profiling) {
        RG_CHECK(grid_wtowers_impl(ctx, uvgrids[0], grid_size, theta, &vis[0], wkern, nullptr, S, M, winc, flags));
        first = 1;
    }
    if (count == first) return RG_OK;
    if (!same || ctx->profiling) {
        for (int i = 1; i < count; i++)
            RG_CHECK(grid_wtowers_impl(ctx, uvgrids[i], grid_size, theta, &vis[i], wkern, nullptr, S, M, winc, flags));
        return RG_OK;
    }
    RG_CHECK(check_wkern(wkern));
    RG_CUDA(cudaSetDevice(ctx->device));
    begin_call(ctx);
    RG_CHECK(batch_streams(ctx));
    TowerPlan &pl = ctx->tower_plans[keybuf];
    float2 *taps = nullptr;
    RG_CHECK(stage_taps(ctx, wkern, &taps, true));  // once for the batch (step 0 staged it already if it ran)
    void *poison = nullptr;  // set by the first pass that overflows; the later passes then write nothing
    RG_CHECK(scratch(ctx, "batch_poison", sizeof(int), &poison));
    RG_CUDA(cudaMemsetAsync(poison, 0, sizeof(int), ctx->stream));
    if (ctx->pinned_steps_bytes < (size_t)count * 64) {
        if (ctx->pinned_steps) cudaFreeHost(ctx->pinned_steps);
        ctx->pinned_steps = nullptr;
        ctx->pinned_steps_bytes = 0;
        RG_CUDA(cudaMallocHost(&ctx->pinned_steps, (size_t)count * 64));
        ctx->pinned_steps_bytes = (size_t)count * 64;
    }
    // Staging sets (kBatchSets) for inputs in host memory and for grids in
    // host memory.  With three, the upload of step i may start as soon as the
    // pass of step i-3 is done: two passes of slack for a copy that takes about
    // as long as one pass.
    constexpr int SETS = rg_context::kBatchSets;
    void *in[SETS][4], *outb[SETS];
    static const char *field[4] = {"u", "v", "w", "vis"};
    for (int b = 0; b < SETS; b++) {
        char name[32];
        for (int f = 0; f < 4; f++) {
            std::snprintf(name, sizeof(name), "batch_%s%d", field[f], b);
            RG_CHECK(scratch(ctx, name, f == 3 ? 2 * vb : vb, &in[b][f]));
        }
        std::snprintf(name, sizeof(name), "batch_out%d", b);
        RG_CHECK(scratch(ctx, name, grid_bytes, &outb[b]));
    }
    // the copy streams start after everything already on the context stream
    RG_CUDA(cudaEventRecord(ctx->ev_done[0], ctx->stream));
    RG_CUDA(cudaStreamWaitEvent(ctx->copy_in, ctx->ev_done[0], 0));
    RG_CUDA(cudaStreamWaitEvent(ctx->copy_out, ctx->ev_done[0], 0));
    // on any early return, leave no copy or pass of this batch in flight
    struct Quiesce {
        rg_context *c;
        ~Quiesce()
        {
            cudaStreamSynchronize(c->stream);
            cudaStreamSynchronize(c->copy_in);
            cudaStreamSynchronize(c->copy_out);
        }
    } quiesce{ctx};
    bool used[SETS] = {}, out_pending[SETS] = {};
    for (int i = first; i < count; i++) {
        const int b = i % SETS;
        const rg_vis &v = vis[i];
        const void *src[4] = {v.u, v.v, v.w, v.vis};
        const void *dev[4];
        // Input staging set b was last read by the pass of step i-SETS.  Its
        // output staging buffer is only rewritten by this step's pass, so the
        // wait for that step's grid copy-out goes on the pass, not on these
        // copies: uploads never queue behind downloads.
        if (used[b]) RG_CUDA(cudaStreamWaitEvent(ctx->copy_in, ctx->ev_used[b], 0));
        for (int f = 0; f < 4; f++) {
            if (n == 0 || is_device_pointer(src[f])) {
                dev[f] = src[f];
            } else {
                RG_CUDA(cudaMemcpyAsync(in[b][f], src[f], f == 3 ? 2 * vb : vb, cudaMemcpyHostToDevice,
                                        ctx->copy_in));
                dev[f] = in[b][f];
            }
        }
        DevVis dv;
        dv.u = (const double *)dev[0];
        dv.v = (const double *)dev[1];
        dv.w = (const double *)dev[2];
        dv.vis = (const double2 *)dev[3];
        dv.n = n;
        const bool host_out = !is_device_pointer(uvgrids[i]);
        double *out_dev = host_out ? (double *)outb[b] : uvgrids[i];
        if (host_out && !(flags & RG_GRID_OVERWRITE)) {
            // accumulating into a host grid: its upload rewrites the output staging buffer
            if (out_pending[b]) RG_CUDA(cudaStreamWaitEvent(ctx->copy_in, ctx->ev_out[b], 0));
            RG_CUDA(cudaMemcpyAsync(out_dev, uvgrids[i], grid_bytes, cudaMemcpyHostToDevice, ctx->copy_in));
        }
        RG_CUDA(cudaEventRecord(ctx->ev_in[b], ctx->copy_in));
        RG_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev_in[b], 0));
        if (host_out && out_pending[b])  // step i-SETS has left the output staging buffer
            RG_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev_out[b], 0));
        RG_CHECK(wtowers_enqueue(ctx, dv, (const float2 *)taps, wkern, nullptr, out_dev, N, theta, S, M, winc, flags,
                                 pl, (char *)ctx->pinned_steps + (size_t)i * 64, (int *)poison));
        RG_CUDA(cudaEventRecord(ctx->ev_used[b], ctx->stream));
        if (host_out) {
            RG_CUDA(cudaStreamWaitEvent(ctx->copy_out, ctx->ev_used[b], 0));
            RG_CUDA(cudaMemcpyAsync(uvgrids[i], out_dev, grid_bytes, cudaMemcpyDeviceToHost, ctx->copy_out));
            RG_CUDA(cudaEventRecord(ctx->ev_out[b], ctx->copy_out));
        }
        used[b] = true;
        out_pending[b] = host_out;
    }
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->copy_in));
    RG_CUDA(cudaStreamSynchronize(ctx->copy_out));
    // from the first step that overflowed on, nothing was written: those steps
    // run again as ordinary calls (which size the plan afresh)
    int redo = count;
    for (int i = first; i < count && redo == count; i++) {
        bool overflow = false;
        RG_CHECK(wtowers_check(ctx, pl, &overflow, (const char *)ctx->pinned_steps + (size_t)i * 64));
        if (overflow) redo = i;
    }
    for (int i = redo; i < count; i++)
        RG_CHECK(grid_wtowers_impl(ctx, uvgrids[i], grid_size, theta, &vis[i], wkern, nullptr, S, M, winc, flags));
    return RG_OK;
}

}  // namespace rg


extern "C" {

rg_status rg_grid_wtowers(rg_context *ctx, double *uvgrid, int grid_size, double theta,
                          const rg_vis *vis, const rg_wkern *wkern, int subgrid_size,
                          int subgrid_margin, double wincrement, int flags)
{
    return rg::grid_wtowers_impl(ctx, uvgrid, grid_size, theta, vis, wkern, nullptr, subgrid_size, subgrid_margin,
                                 wincrement, flags);
}

static rg_status check_towers_shape(int grid_size, double theta, int S, int M, double winc)
{
    if (grid_size < 2 || grid_size > 16384) return fail(RG_ERR_UNSUPPORTED, "grid_size must be in [2, 16384]");
    if (!(theta > 0.0) || !std::isfinite(theta)) return fail(RG_ERR_INVALID_ARGUMENT, "theta must be > 0");
    if (!(winc > 0.0) || !std::isfinite(winc)) return fail(RG_ERR_INVALID_ARGUMENT, "wincrement must be > 0");
    if (S % 2 || M % 2 || M < 0 || M >= S || S < 2)
        return fail(RG_ERR_INVALID_ARGUMENT, "subgrid size and margin must be even, 0 <= margin < subgrid");
    return RG_OK;
}

int rg_wtowers_tower_count(int grid_size, int subgrid_size, int subgrid_margin)
{
    const int chunk = subgrid_size - subgrid_margin;
    if (chunk <= 0 || grid_size < 1) return 0;
    const int nc = grid_size / chunk + 1;
    return nc * nc;
}

rg_status rg_wtowers_tower_loads(rg_context *ctx, int grid_size, double theta, const rg_vis *vis,
                                 int subgrid_size, int subgrid_margin, double wincrement, int64_t *vis_per_tower,
                                 int32_t *floors_per_tower, int ntowers)
{
    if (!ctx || !vis_per_tower || !floors_per_tower)
        return fail(RG_ERR_INVALID_ARGUMENT, "ctx and the output arrays must be non-NULL");
    RG_CHECK(check_towers_shape(grid_size, theta, subgrid_size, subgrid_margin, wincrement));
    RG_CHECK(check_vis(vis));
    const int S = subgrid_size, M = subgrid_margin, N = grid_size;
    const int chunk = S - M, nchunk = N / chunk + 1, nt = nchunk * nchunk;
    if (ntowers != nt)
        return fail(RG_ERR_INVALID_ARGUMENT, "ntowers must be rg_wtowers_tower_count(grid, subgrid, margin)");
    RG_CUDA(cudaSetDevice(ctx->device));
    begin_call(ctx);
    DevVis dv;
    RG_CHECK(stage_vis(ctx, vis, &dv));
    Diag d;
    RG_CHECK(diag_begin(ctx, &d));
    int *range = (int *)((char *)d.err + 48);
    // the floor count is known only on the device: size the bins for the
    // largest count the w range allows, read back once
    void *mm, *vc, *fl, *act;
    RG_CHECK(scratch(ctx, "wminmax", 16, &mm));
    RG_CHECK(scratch(ctx, "census_vis", sizeof(unsigned long long) * (size_t)nt, &vc));
    RG_CHECK(scratch(ctx, "census_floors", sizeof(int) * (size_t)nt, &fl));
    launch_minmax_w(ctx->stream, dv.u, dv.v, dv.w, dv.n, (double *)mm, d.err);
    double wr[2];
    RG_CUDA(cudaMemcpyAsync(wr, mm, sizeof(wr), cudaMemcpyDeviceToHost, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    const double nf = std::floor(wr[1] / wincrement + 0.5) - std::floor(wr[0] / wincrement + 0.5) + 1;
    if (!(nf >= 1) || nf * nt > (double)(1 << 28))
        return fail(RG_ERR_UNSUPPORTED, "too many (tower, w-floor) bins; increase wincrement");
    const int floors_cap = (int)nf;
    RG_CHECK(scratch(ctx, "census_active", sizeof(int) * (size_t)nt * floors_cap, &act));
    RG_CUDA(cudaMemsetAsync(act, 0, sizeof(int) * (size_t)nt * floors_cap, ctx->stream));
    RG_CUDA(cudaMemsetAsync(vc, 0, sizeof(unsigned long long) * (size_t)nt, ctx->stream));
    launch_w_floors(ctx->stream, (const double *)mm, wincrement, floors_cap, range, d.err);
    TowerGeom g;
    g.grid_size = N;
    g.subgrid = S;
    g.margin = M;
    g.chunk = chunk;
    g.nchunk = nchunk;
    g.ksize = 0;
    g.ov = 1;
    g.planes = 1;
    g.theta = theta;
    g.winc = wincrement;
    g.wk_wmin = 0.0;
    g.wk_wstep = 1.0;
    launch_tower_census(ctx->stream, dv.u, dv.v, dv.w, dv.n, g, range, (unsigned long long *)vc, (int *)act,
                        (int *)fl, nt, floors_cap, d.err);
    ctx->launches += 4;
    RG_CHECK(check_launch("W-towers tower census"));
    RG_CUDA(cudaMemcpyAsync(vis_per_tower, vc, sizeof(int64_t) * (size_t)nt, cudaMemcpyDeviceToHost, ctx->stream));
    RG_CUDA(cudaMemcpyAsync(floors_per_tower, fl, sizeof(int32_t) * (size_t)nt, cudaMemcpyDeviceToHost,
                            ctx->stream));
    RG_CHECK(diag_end(ctx, d, nullptr));
    return RG_OK;
}

rg_status rg_wtowers_partition(const int64_t *vis_per_tower, const int32_t *floors_per_tower, int ntowers,
                               int nparts, double vis_per_floor, int32_t *part_of_tower)
{
    if (!vis_per_tower || !floors_per_tower || !part_of_tower || ntowers < 0 || nparts < 1)
        return fail(RG_ERR_INVALID_ARGUMENT, "bad partition arguments");
    if (!(vis_per_floor >= 0.0) || !std::isfinite(vis_per_floor))
        return fail(RG_ERR_INVALID_ARGUMENT, "vis_per_floor must be finite and >= 0");
    const double wf = vis_per_floor > 0.0 ? vis_per_floor : 2400.0;
    // longest-processing-time first: towers by cost, largest first (ties by
    // index), each to the least loaded part (ties to the lowest part)
    std::vector<int> order((size_t)ntowers);
    std::vector<double> cost((size_t)ntowers);
    for (int t = 0; t < ntowers; t++) {
        order[t] = t;
        cost[t] = (double)vis_per_tower[t] + wf * (double)floors_per_tower[t];
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<double> load((size_t)nparts, 0.0);
    for (int t : order) {
        int best = 0;
        for (int p = 1; p < nparts; p++)
            if (load[p] < load[best]) best = p;
        part_of_tower[t] = best;
        load[best] += cost[t];
    }
    return RG_OK;
}

rg_status rg_grid_wtowers_part(rg_context *ctx, double *uvgrid, int grid_size, double theta, const rg_vis *vis,
                               const rg_wkern *wkern, int subgrid_size, int subgrid_margin, double wincrement,
                               int flags, const int32_t *part_of_tower, int part)
{
    if (!part_of_tower) return fail(RG_ERR_INVALID_ARGUMENT, "part_of_tower must be non-NULL");
    return rg::grid_wtowers_impl(ctx, uvgrid, grid_size, theta, vis, wkern, nullptr, subgrid_size, subgrid_margin,
                                 wincrement, flags, part_of_tower, part);
}

rg_status rg_grid_wtowers_batch(rg_context *ctx, int count, double *const *uvgrids, int grid_size, double theta,
                                const rg_vis *vis, const rg_wkern *wkern, int subgrid_size, int subgrid_margin,
                                double wincrement, int flags)
{
    return rg::grid_wtowers_batch_impl(ctx, count, uvgrids, grid_size, theta, vis, wkern, subgrid_size,
                                       subgrid_margin, wincrement, flags);
}

rg_status rg_weight(rg_context *ctx, int grid_size, double theta, const rg_vis *vis, double *vis_out)
{
    if (!ctx || !vis_out) return fail(RG_ERR_INVALID_ARGUMENT, "ctx and vis_out must be non-NULL");
    if (grid_size < 2) return fail(RG_ERR_INVALID_ARGUMENT, "grid_size must be >= 2");
    RG_CHECK(check_vis(vis));
    RG_CUDA(cudaSetDevice(ctx->device));
    DevVis dv;
    RG_CHECK(stage_vis(ctx, vis, &dv));
    const int64_t cells = (int64_t)grid_size * grid_size;
    void *count;
    RG_CHECK(scratch(ctx, "wcount", sizeof(unsigned) * (size_t)cells, &count));
    RG_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned) * (size_t)cells, ctx->stream));
    OutView ov;
    RG_CHECK(out_view(ctx, vis_out, sizeof(double2) * (size_t)dv.n, "out_vis", false, &ov));
    if (dv.n > 0) {
        launch_weight_count(ctx->stream, dv.u, dv.v, dv.n, grid_size, theta, (unsigned *)count);
        launch_weight_apply(ctx->stream, dv.u, dv.v, dv.vis, (double2 *)ov.dev, dv.n, grid_size, theta,
                            (const unsigned *)count);
        RG_CHECK(check_launch("weighting"));
    }
    RG_CHECK(finish_out(ctx, ov));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

rg_status rg_grid_simple(rg_context *ctx, double *uvgrid, int grid_size, double theta, const rg_vis *vis, int flags)
{
    if (!ctx || !uvgrid) return fail(RG_ERR_INVALID_ARGUMENT, "ctx and uvgrid must be non-NULL");
    if (grid_size < 2 || grid_size > 16384) return fail(RG_ERR_UNSUPPORTED, "grid_size must be in [2, 16384]");
    if (!(theta > 0.0) || !std::isfinite(theta)) return fail(RG_ERR_INVALID_ARGUMENT, "theta must be > 0");
    RG_CHECK(check_vis(vis));
    RG_CUDA(cudaSetDevice(ctx->device));
    begin_call(ctx);
    DevVis dv;
    RG_CHECK(stage_vis(ctx, vis, &dv));
    const int64_t cells = (int64_t)grid_size * grid_size;
    Diag d;
    RG_CHECK(diag_begin(ctx, &d));
    // accumulate into a scratch copy, so a call rejected for its data leaves
    // the caller's grid as it was
    void *acc;
    RG_CHECK(scratch(ctx, "simple_grid", sizeof(double2) * (size_t)cells, &acc));
    RG_CUDA(cudaMemsetAsync(acc, 0, sizeof(double2) * (size_t)cells, ctx->stream));
    if (dv.n > 0) {
        launch_simple_grid(ctx->stream, dv.u, dv.v, dv.vis, dv.n, grid_size, theta, (double2 *)acc, d.err);
        ctx->launches++;
        RG_CHECK(check_launch("simple gridding"));
    }
    RG_CHECK(diag_end(ctx, d, nullptr));
    OutView ov;
    RG_CHECK(out_view(ctx, uvgrid, sizeof(double2) * (size_t)cells, "out_grid", !(flags & RG_GRID_OVERWRITE), &ov));
    if (flags & RG_GRID_OVERWRITE)
        RG_CUDA(cudaMemcpyAsync(ov.dev, acc, sizeof(double2) * (size_t)cells, cudaMemcpyDeviceToDevice, ctx->stream));
    else
        launch_add_f64(ctx->stream, (const double2 *)acc, (double2 *)ov.dev, cells);
    RG_CHECK(check_launch("grid accumulation"));
    RG_CHECK(finish_out(ctx, ov));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->stats[0] = dv.n;
    ctx->stats[5] = ctx->launches;
    return RG_OK;
}

static rg_status grid_inplace(rg_context *ctx, double *uvgrid, int grid_size, int op)
{
    if (!ctx || !uvgrid) return fail(RG_ERR_INVALID_ARGUMENT, "ctx and uvgrid must be non-NULL");
    if (grid_size < 2 || (op == 1 && grid_size % 2))
        return fail(RG_ERR_INVALID_ARGUMENT, "grid_size must be >= 2 (and even for fft_shift)");
    RG_CUDA(cudaSetDevice(ctx->device));
    const int64_t cells = (int64_t)grid_size * grid_size;
    OutView ov;
    RG_CHECK(out_view(ctx, uvgrid, sizeof(double2) * (size_t)cells, "out_grid", true, &ov));
    if (op == 0) launch_make_hermitian(ctx->stream, (double2 *)ov.dev, grid_size);
    else launch_fft_shift(ctx->stream, (double2 *)ov.dev, grid_size);
    RG_CHECK(check_launch(op == 0 ? "make_hermitian" : "fft_shift"));
    RG_CHECK(finish_out(ctx, ov));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

rg_status rg_make_hermitian(rg_context *ctx, double *uvgrid, int grid_size)
{
    return grid_inplace(ctx, uvgrid, grid_size, 0);
}

rg_status rg_fft_shift(rg_context *ctx, double *uvgrid, int grid_size)
{
    return grid_inplace(ctx, uvgrid, grid_size, 1);
}

rg_status rg_image_from_grid(rg_context *ctx, double *uvgrid, int grid_size, double *image_out,
                             const double *taper_1d)
{
    if (!ctx || !uvgrid || !image_out) return fail(RG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!fft64_any_supported(grid_size) || grid_size % 2)
        return fail(RG_ERR_UNSUPPORTED, "image formation needs an even grid_size in [2, 4096]");
    RG_CUDA(cudaSetDevice(ctx->device));
    const int N = grid_size;
    const int64_t cells = (int64_t)N * N;
    OutView g;
    RG_CHECK(out_view(ctx, uvgrid, sizeof(double2) * (size_t)cells, "img_grid", true, &g));
    void *tmp;
    RG_CHECK(scratch(ctx, "img_tmp", sizeof(double2) * (size_t)cells, &tmp));
    const void *taper = nullptr;
    if (taper_1d) RG_CHECK(stage_in(ctx, taper_1d, sizeof(double) * N, "img_taper", &taper));
    OutView img;
    RG_CHECK(out_view(ctx, image_out, sizeof(double) * (size_t)cells, "img_out", false, &img));
    launch_make_hermitian(ctx->stream, (double2 *)g.dev, N);
    launch_fft_shift(ctx->stream, (double2 *)g.dev, N);
    void *work = nullptr;
    if (fft64_any_work_elems(N) > 0)
        RG_CHECK(scratch(ctx, "fft64_work", sizeof(double2) * (size_t)fft64_any_work_elems(N), &work));
    launch_fft64_2d(ctx->stream, (double2 *)g.dev, (double2 *)tmp, 1, N, N, -1, (double2 *)work);
    launch_fft_shift(ctx->stream, (double2 *)g.dev, N);
    launch_real_part(ctx->stream, (const double2 *)g.dev, (double *)img.dev, N, (const double *)taper);
    RG_CHECK(check_launch("image formation"));
    RG_CHECK(finish_out(ctx, g));
    RG_CHECK(finish_out(ctx, img));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

rg_status rg_fft2d(rg_context *ctx, void *data, int batch, int ny, int nx, int sign, int complex_bytes)
{
    if (!ctx || !data) return fail(RG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (batch < 1 || (sign != -1 && sign != 1)) return fail(RG_ERR_INVALID_ARGUMENT, "bad batch or sign");
    RG_CUDA(cudaSetDevice(ctx->device));
    const size_t bytes = (size_t)complex_bytes * batch * ny * nx;
    if (complex_bytes == 8) {
        if (ny != nx || !fft32_supported(nx))
            return fail(RG_ERR_UNSUPPORTED, "FP32 transforms need square power-of-two sizes in [64, 1024]");
        OutView ov;
        RG_CHECK(out_view(ctx, data, bytes, "fft_data", true, &ov));
        float2 *tw;
        RG_CHECK(get_twiddles32(ctx, nx, &tw));
        launch_fft32_rows(ctx->stream, (float2 *)ov.dev, (int64_t)batch * ny, nx, sign, tw);
        launch_fft32_cols(ctx->stream, (float2 *)ov.dev, batch, nx, sign, tw);
        RG_CHECK(check_launch("fft32"));
        RG_CHECK(finish_out(ctx, ov));
    } else if (complex_bytes == 16) {
        if (!fft64_any_supported(nx) || !fft64_any_supported(ny))
            return fail(RG_ERR_UNSUPPORTED, "FP64 transforms need sizes in [2, 4096]");
        OutView ov;
        RG_CHECK(out_view(ctx, data, bytes, "fft_data", true, &ov));
        void *tmp;
        RG_CHECK(scratch(ctx, "fft_tmp", bytes, &tmp));
        const int64_t wel = std::max(fft64_any_work_elems(nx), fft64_any_work_elems(ny));
        void *work = nullptr;
        if (wel > 0) RG_CHECK(scratch(ctx, "fft64_work", sizeof(double2) * (size_t)wel, &work));
        launch_fft64_2d(ctx->stream, (double2 *)ov.dev, (double2 *)tmp, batch, ny, nx, sign, (double2 *)work);
        RG_CHECK(check_launch("fft64"));
        RG_CHECK(finish_out(ctx, ov));
    } else {
        return fail(RG_ERR_INVALID_ARGUMENT, "complex_bytes must be 8 or 16");
    }
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

rg_status rg_dft_image(rg_context *ctx, double *image_out, int grid_size, double theta,
                       const rg_vis *vis, int precision, double factor)
{
    return rg_dft_image_rows(ctx, image_out, grid_size, theta, vis, precision, factor, 0, grid_size);
}

rg_status rg_dft_image_rows(rg_context *ctx, double *image_out, int grid_size, double theta,
                            const rg_vis *vis, int precision, double factor, int row0, int nrows)
{
    if (!ctx || !image_out) return fail(RG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (grid_size < 1 || grid_size > 65536) return fail(RG_ERR_INVALID_ARGUMENT, "bad grid_size");
    if (precision < 0 || precision > 2) return fail(RG_ERR_INVALID_ARGUMENT, "unknown precision mode");
    if (row0 < 0 || nrows < 0 || row0 > grid_size || nrows > grid_size - row0)
        return fail(RG_ERR_INVALID_ARGUMENT, "rows [row0, row0 + nrows) must lie in [0, grid_size)");
    RG_CHECK(check_vis(vis));
    RG_CUDA(cudaSetDevice(ctx->device));
    if (nrows == 0) return RG_OK;
    DevVis dv;
    RG_CHECK(stage_vis(ctx, vis, &dv));
    OutView ov;
    RG_CHECK(out_view(ctx, image_out, sizeof(double) * (size_t)nrows * grid_size, "dft_out", false, &ov));
    launch_dft(ctx->stream, dv.u, dv.v, dv.w, dv.vis, dv.n, (double *)ov.dev, grid_size, theta, precision,
               factor, ctx->sm_count, row0, nrows);
    RG_CHECK(check_launch("dft"));
    RG_CHECK(finish_out(ctx, ov));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

}  // extern "C"
