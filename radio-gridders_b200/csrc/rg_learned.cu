// C ABI of the learned w-kernel: network state, training, evaluation and the
// learned-tap W-projection gridder (kernels in k_mlp.cu).
#include <cmath>
#include <random>
#include <vector>

#include "rg_internal.h"

struct rg_mlp {
    int device = 0;
    int ksize = 16;
    double wmax = 2000.0;
    double out_scale = 0.05;
    int step = 0;
    float *P = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *loss = nullptr;
    void *PB = nullptr;
};

using namespace rg;

namespace {

rg_status upload_params(rg_context *ctx, rg_mlp *mlp, const float *params)
{
    const int np = mlp_param_count();
    const void *src;
    RG_CHECK(stage_in(ctx, params, sizeof(float) * np, "mlp_params_in", &src));
    RG_CUDA(cudaMemcpyAsync(mlp->P, src, sizeof(float) * np, cudaMemcpyDeviceToDevice, ctx->stream));
    launch_mlp_to_bf16(ctx->stream, mlp->P, mlp->PB);
    RG_CUDA(cudaMemsetAsync(mlp->m, 0, sizeof(float) * np, ctx->stream));
    RG_CUDA(cudaMemsetAsync(mlp->v, 0, sizeof(float) * np, ctx->stream));
    RG_CUDA(cudaMemsetAsync(mlp->grad, 0, sizeof(float) * np, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    mlp->step = 0;
    return RG_OK;
}

// Error word of the tensor-core kernels (DERR_TIMEOUT when a bounded wait
// gave up), zeroed before the launch and read after the stream has drained.
rg_status tc_err_begin(rg_context *ctx, unsigned **err)
{
    void *p;
    RG_CHECK(scratch(ctx, "tc_err", 16, &p));
    RG_CUDA(cudaMemsetAsync(p, 0, 16, ctx->stream));
    *err = (unsigned *)p;
    return RG_OK;
}

rg_status tc_err_end(rg_context *ctx, const unsigned *err)
{
    unsigned h = 0;
    RG_CUDA(cudaMemcpyAsync(&h, err, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h & DERR_TIMEOUT) return fail(RG_ERR_CUDA, "a bounded wait for tensor-core work timed out");
    return RG_OK;
}

rg_status check_mlp(rg_context *ctx, rg_mlp *mlp)
{
    if (!ctx || !mlp) return fail(RG_ERR_INVALID_ARGUMENT, "ctx and mlp must be non-NULL");
    if (ctx->device != mlp->device) return fail(RG_ERR_INVALID_ARGUMENT, "network lives on another device");
    return RG_OK;
}

}  // namespace

extern "C" {

int rg_mlp_param_count(void) { return mlp_param_count(); }

rg_status rg_mlp_create(rg_context *ctx, int ksize, double wmax, double out_scale, uint64_t seed, rg_mlp **out)
{
    if (!ctx || !out) return fail(RG_ERR_INVALID_ARGUMENT, "ctx and out must be non-NULL");
    if (ksize != 8 && ksize != 16) return fail(RG_ERR_UNSUPPORTED, "learned kernel support must be 8 or 16");
    if (!(wmax > 0.0) || !(out_scale > 0.0)) return fail(RG_ERR_INVALID_ARGUMENT, "wmax and out_scale must be > 0");
    RG_CUDA(cudaSetDevice(ctx->device));
    rg_mlp *mlp = new rg_mlp();
    mlp->device = ctx->device;
    mlp->ksize = ksize;
    mlp->wmax = wmax;
    mlp->out_scale = out_scale;
    const int np = mlp_param_count();
    if (cudaMalloc(&mlp->P, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&mlp->grad, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&mlp->m, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&mlp->v, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&mlp->loss, sizeof(float) * 4) != cudaSuccess ||
        cudaMalloc(&mlp->PB, 2 * (size_t)mlp_bf16_count()) != cudaSuccess) {
        cudaGetLastError();
        rg_mlp_destroy(mlp);
        return fail(RG_ERR_OUT_OF_MEMORY, "network allocation failed");
    }
    // He-normal initialisation of W1..W4 (fan-in 21 for W1), zero biases
    std::vector<float> h(np, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    auto fill = [&](int off, int rows, int cols, int fan_in, int live_rows) {
        const double sd = std::sqrt(2.0 / fan_in);
        for (int r = 0; r < rows; r++)
            for (int c = 0; c < cols; c++) h[off + r * cols + c] = r < live_rows ? (float)(sd * nd(rng)) : 0.f;
    };
    fill(0, 32, 128, 21, 21);
    fill(32 * 128 + 128, 128, 128, 128, 128);
    fill(32 * 128 + 128 + 128 * 128 + 128, 128, 128, 128, 128);
    fill(32 * 128 + 128 + 2 * (128 * 128 + 128), 128, 2, 128, 128);
    rg_status st = upload_params(ctx, mlp, h.data());
    if (st != RG_OK) {
        rg_mlp_destroy(mlp);
        return st;
    }
    *out = mlp;
    return RG_OK;
}

rg_status rg_mlp_destroy(rg_mlp *mlp)
{
    if (!mlp) return RG_OK;
    cudaSetDevice(mlp->device);
    cudaFree(mlp->P);
    cudaFree(mlp->grad);
    cudaFree(mlp->m);
    cudaFree(mlp->v);
    cudaFree(mlp->loss);
    cudaFree(mlp->PB);
    delete mlp;
    return RG_OK;
}

rg_status rg_mlp_set_params(rg_context *ctx, rg_mlp *mlp, const float *params)
{
    RG_CHECK(check_mlp(ctx, mlp));
    if (!params) return fail(RG_ERR_INVALID_ARGUMENT, "params is NULL");
    RG_CUDA(cudaSetDevice(ctx->device));
    return upload_params(ctx, mlp, params);
}

rg_status rg_mlp_get_params(rg_context *ctx, rg_mlp *mlp, float *params)
{
    RG_CHECK(check_mlp(ctx, mlp));
    if (!params) return fail(RG_ERR_INVALID_ARGUMENT, "params is NULL");
    RG_CUDA(cudaSetDevice(ctx->device));
    RG_CUDA(cudaMemcpyAsync(params, mlp->P, sizeof(float) * mlp_param_count(), cudaMemcpyDefault, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

rg_status rg_mlp_gradient(rg_context *ctx, rg_mlp *mlp, const float *samples, const float *targets, int n,
                          float *grad_out, float *loss_out)
{
    RG_CHECK(check_mlp(ctx, mlp));
    if (!samples || !targets || n < 1) return fail(RG_ERR_INVALID_ARGUMENT, "bad training batch");
    RG_CUDA(cudaSetDevice(ctx->device));
    const void *in, *tg;
    RG_CHECK(stage_in(ctx, samples, sizeof(float) * 5 * (size_t)n, "mlp_in", &in));
    RG_CHECK(stage_in(ctx, targets, sizeof(float) * 2 * (size_t)n, "mlp_tg", &tg));
    const int np = mlp_param_count();
    RG_CUDA(cudaMemsetAsync(mlp->grad, 0, sizeof(float) * np, ctx->stream));
    RG_CUDA(cudaMemsetAsync(mlp->loss, 0, sizeof(float), ctx->stream));
    launch_mlp_grad(ctx->stream, mlp->P, mlp->PB, (const float *)in, (const float2 *)tg, n, mlp->ksize,
                    (float)(1.0 / mlp->wmax), (float)(1.0 / mlp->out_scale), mlp->grad, mlp->loss);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp gradient");
    if (grad_out) RG_CUDA(cudaMemcpyAsync(grad_out, mlp->grad, sizeof(float) * np, cudaMemcpyDefault, ctx->stream));
    if (loss_out) RG_CUDA(cudaMemcpyAsync(loss_out, mlp->loss, sizeof(float), cudaMemcpyDefault, ctx->stream));
    RG_CUDA(cudaMemsetAsync(mlp->grad, 0, sizeof(float) * np, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

rg_status rg_mlp_train(rg_context *ctx, rg_mlp *mlp, const float *samples, const float *targets, int64_t n,
                       int batch, int steps, float lr, float *loss_out)
{
    RG_CHECK(check_mlp(ctx, mlp));
    if (!samples || !targets || n < 1 || batch < 1 || steps < 0)
        return fail(RG_ERR_INVALID_ARGUMENT, "bad training arguments");
    if (n > ((int64_t)1 << 30)) return fail(RG_ERR_UNSUPPORTED, "training set too large");
    RG_CUDA(cudaSetDevice(ctx->device));
    const void *in, *tg;
    // samples arrive as [5][n]; batches are taken as contiguous column ranges,
    // so copy them once into per-field device arrays
    RG_CHECK(stage_in(ctx, samples, sizeof(float) * 5 * (size_t)n, "mlp_train_in", &in));
    RG_CHECK(stage_in(ctx, targets, sizeof(float) * 2 * (size_t)n, "mlp_train_tg", &tg));
    void *bin;
    RG_CHECK(scratch(ctx, "mlp_batch_in", sizeof(float) * 5 * (size_t)batch, &bin));
    const int np = mlp_param_count();
    const float *fin = (const float *)in;
    for (int s = 0; s < steps; s++) {
        const int64_t b0 = ((int64_t)s * batch) % n;
        const int nb = (int)(b0 + batch <= n ? batch : n - b0);
        for (int f = 0; f < 5; f++)
            RG_CUDA(cudaMemcpyAsync((float *)bin + (size_t)f * nb, fin + (size_t)f * n + b0, sizeof(float) * nb,
                                    cudaMemcpyDeviceToDevice, ctx->stream));
        if (s == steps - 1) RG_CUDA(cudaMemsetAsync(mlp->loss, 0, sizeof(float), ctx->stream));
        launch_mlp_grad(ctx->stream, mlp->P, mlp->PB, (const float *)bin, (const float2 *)tg + b0, nb,
                        mlp->ksize, (float)(1.0 / mlp->wmax), (float)(1.0 / mlp->out_scale), mlp->grad,
                        mlp->loss);
        mlp->step++;
        launch_mlp_adam(ctx->stream, mlp->P, mlp->PB, mlp->grad, mlp->m, mlp->v, lr, mlp->step);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp training");
    (void)np;
    if (loss_out) RG_CUDA(cudaMemcpyAsync(loss_out, mlp->loss, sizeof(float), cudaMemcpyDefault, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

rg_status rg_mlp_eval(rg_context *ctx, rg_mlp *mlp, const float *samples, int64_t n, float *taps_out)
{
    RG_CHECK(check_mlp(ctx, mlp));
    if (!samples || !taps_out || n < 0 || n > ((int64_t)1 << 30))
        return fail(RG_ERR_INVALID_ARGUMENT, "bad evaluation arguments");
    RG_CUDA(cudaSetDevice(ctx->device));
    if (n == 0) return RG_OK;
    const void *in;
    RG_CHECK(stage_in(ctx, samples, sizeof(float) * 5 * (size_t)n, "mlp_eval_in", &in));
    void *out;
    const bool dev_out = is_device_pointer(taps_out);
    if (dev_out) out = taps_out;
    else RG_CHECK(scratch(ctx, "mlp_eval_out", sizeof(float) * 2 * (size_t)n, &out));
    unsigned *err;
    RG_CHECK(tc_err_begin(ctx, &err));
    launch_mlp_eval(ctx->stream, mlp->P, mlp->PB, (const float *)in, (int)n, mlp->ksize, (float)(1.0 / mlp->wmax),
                    (float)mlp->out_scale, (float2 *)out, ctx->sm_count, err);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "mlp evaluation");
    RG_CHECK(tc_err_end(ctx, err));
    if (!dev_out) RG_CUDA(cudaMemcpyAsync(taps_out, out, sizeof(float) * 2 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

rg_status rg_selftest_wait_timeout(rg_context *ctx)
{
    if (!ctx) return fail(RG_ERR_INVALID_ARGUMENT, "ctx must be non-NULL");
    RG_CUDA(cudaSetDevice(ctx->device));
    unsigned *err;
    RG_CHECK(tc_err_begin(ctx, &err));
    launch_mbar_timeout_probe(ctx->stream, err, 1ll << 22);  // ~2 ms of SM clock
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "wait self-test");
    return tc_err_end(ctx, err);
}

rg_status rg_grid_wprojection_learned(rg_context *ctx, rg_mlp *mlp, double *uvgrid, int grid_size, double theta,
                                      const rg_vis *vis, int flags)
{
    RG_CHECK(check_mlp(ctx, mlp));
    if (!uvgrid || !vis) return fail(RG_ERR_INVALID_ARGUMENT, "uvgrid and vis must be non-NULL");
    if (grid_size < 2 || grid_size > 16384) return fail(RG_ERR_UNSUPPORTED, "grid_size must be in [2, 16384]");
    if (!(theta > 0.0)) return fail(RG_ERR_INVALID_ARGUMENT, "theta must be > 0");
    if (vis->n < 0 || (vis->n > 0 && (!vis->u || !vis->v || !vis->w || !vis->vis)))
        return fail(RG_ERR_INVALID_ARGUMENT, "bad visibilities");
    RG_CUDA(cudaSetDevice(ctx->device));
    begin_call(ctx);
    const int N = grid_size;
    const int64_t cells = (int64_t)N * N;
    const size_t b = sizeof(double) * (size_t)vis->n;
    const void *u, *v, *w, *vz;
    begin_stage(ctx, "stage_in");
    RG_CHECK(stage_in(ctx, vis->u, b, "in_u", &u));
    RG_CHECK(stage_in(ctx, vis->v, b, "in_v", &v));
    RG_CHECK(stage_in(ctx, vis->w, b, "in_w", &w));
    RG_CHECK(stage_in(ctx, vis->vis, 2 * b, "in_vis", &vz));
    end_stage(ctx);
    void *grid32;
    RG_CHECK(scratch(ctx, "grid32", sizeof(float2) * (size_t)cells, &grid32));
    RG_CUDA(cudaMemsetAsync(grid32, 0, sizeof(float2) * (size_t)cells, ctx->stream));
    unsigned *err;
    RG_CHECK(tc_err_begin(ctx, &err));
    begin_stage(ctx, "learned_gridding");
    if (vis->n > 0)
        launch_learned_wproj(ctx->stream, (const double *)u, (const double *)v, (const double *)w,
                             (const double2 *)vz, vis->n, N, theta, mlp->P, mlp->PB, mlp->ksize,
                             (float)(1.0 / mlp->wmax), (float)mlp->out_scale, (float2 *)grid32, ctx->sm_count, err);
    end_stage(ctx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "learned gridding");
    RG_CHECK(tc_err_end(ctx, err));
    const bool dev = is_device_pointer(uvgrid);
    void *g = uvgrid;
    if (!dev) {
        RG_CHECK(scratch(ctx, "out_grid", sizeof(double2) * (size_t)cells, &g));
        if (!(flags & RG_GRID_OVERWRITE))
            RG_CUDA(cudaMemcpyAsync(g, uvgrid, sizeof(double2) * (size_t)cells, cudaMemcpyHostToDevice, ctx->stream));
    }
    launch_add_f32_to_f64(ctx->stream, (const float2 *)grid32, (double2 *)g, cells, (flags & RG_GRID_OVERWRITE) ? 1 : 0);
    if (!dev) RG_CUDA(cudaMemcpyAsync(uvgrid, g, sizeof(double2) * (size_t)cells, cudaMemcpyDeviceToHost, ctx->stream));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    collect_timings(ctx);
    ctx->stats[0] = vis->n;
    ctx->stats[5] = 2;
    return RG_OK;
}

rg_status rg_grid_wtowers_learned(rg_context *ctx, rg_mlp *mlp, double *uvgrid, int grid_size, double theta,
                                  const rg_vis *vis, int subgrid_size, int subgrid_margin, double wincrement,
                                  int flags)
{
    RG_CHECK(check_mlp(ctx, mlp));
    LearnedTaps lt;
    lt.P = mlp->P;
    lt.PB = mlp->PB;
    lt.ksize = mlp->ksize;
    lt.inv_wmax = (float)(1.0 / mlp->wmax);
    lt.scale = (float)mlp->out_scale;
    lt.wmax = mlp->wmax;
    return grid_wtowers_impl(ctx, uvgrid, grid_size, theta, vis, nullptr, &lt, subgrid_size, subgrid_margin,
                             wincrement, flags);
}

}  // extern "C"
