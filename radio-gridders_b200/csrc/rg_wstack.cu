// W-stacking predict (degridding): model visibilities of point sources from
// w-stacked FFTs of the sky and a separable 3-D de-convolution — the
// reference's wstack_predict (src/wstack/predict.cpp:396-562) and its CUDA
// version wstack_predict_cu_3D (src/wstack/predict.cu:808-1081), FP64.
//
//   1. sources snapped to the image grid (N = floor(theta lambda) pixels of
//      1/lambda) inside a grid padded to G = N round(0.5/x0) pixels, each
//      divided by the grid correction corr_lm(du l) corr_lm(du m) corr_n(dw n)
//      (predict.cpp:187-245);
//   2. plane p = quadrant-swapped FFT (sign -1) of the swapped sky times the
//      Fresnel pattern exp(2 pi i dw (1 - sqrt(1 - l^2 - m^2))) raised to
//      p - floor(planes/2) (predict.cpp:466-491: the reference steps the sky by
//      one more power per plane; here each plane's power is formed from the
//      exact phase, planes*dw*ph reduced modulo one turn in FP64);
//   3. per visibility, sum over support_w x support_uv^2 taps of the stack
//      weighted by conv_w x conv_uv x conv_uv at the visibility's sub-cell
//      offsets (src/wstack/wstack_common.h:423-484).
// All planes are one batched FP64 FFT on the device; the stack stays in HBM
// (planes x G^2 x 16 bytes) and every visibility is one warp.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "rg_internal.h"

namespace rg {
namespace {

struct SkyEntry {
    int64_t idx;  // row * G + column of the swapped (fft-shifted) sky
    double re;
    int x, y;     // pixel in the unpadded N x N image (for the Fresnel phase)
};

// plane p, shifted pixel of a source: value * exp(2 pi i (t0 + p) ph(x, y))
__global__ void wstack_scatter_kernel(const int64_t *__restrict__ idx, const double *__restrict__ val,
                                      const int2 *__restrict__ pix, int nsrc, int planes, int t0, int N, int G,
                                      double theta, double dw, double2 *__restrict__ stack)
{
    const int64_t total = (int64_t)nsrc * planes;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int s = (int)(k % nsrc), p = (int)(k / nsrc);
        const double l = theta * ((double)pix[s].x - N / 2) / N;
        const double m = theta * ((double)pix[s].y - N / 2) / N;
        const double ph = dw * (1.0 - sqrt(1.0 - l * l - m * m));
        const double turns = (double)(t0 + p) * ph;
        const double frac = turns - rint(turns);  // exact in FP64: one turn removed
        double sn, cs;
        sincospi(2.0 * frac, &sn, &cs);
        stack[(int64_t)p * G * G + idx[s]] = make_double2(val[s] * cs, val[s] * sn);
    }
}

// One warp per visibility: lanes over the support_uv^2 (u, v) taps, planes in
// turn, then a warp sum.
__global__ void wstack_degrid_kernel(const double2 *__restrict__ stack, const double *__restrict__ u,
                                     const double *__restrict__ v, const double *__restrict__ w, int64_t nvis,
                                     double du, double dw, int N, int G, int planes,
                                     const double *__restrict__ conv_uv, int suv, int ovuv,
                                     const double *__restrict__ conv_w, int sw, int ovw_n,
                                     double2 *__restrict__ out, unsigned *err)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < nvis; i += warps) {
        const double uu = u[i], vv = v[i], ww = w[i];
        if (!isfinite(uu) || !isfinite(vv) || !isfinite(ww)) {
            if (lane == 0) {
                out[i] = make_double2(0.0, 0.0);
                atomicOr(err, DERR_NONFINITE);
            }
            continue;
        }
        const double cu = ceil(uu / du), cv = ceil(vv / du), cw = ceil(ww / dw);
        if (fabs(cu) > 1e9 || fabs(cv) > 1e9 || fabs(cw) > 1e9) {  // far outside any stack
            if (lane == 0) {
                out[i] = make_double2(0.0, 0.0);
                atomicOr(err, DERR_GRID_RANGE);
            }
            continue;
        }
        const double flu = uu - cu * du, flv = vv - cv * du, flw = ww - cw * dw;
        const int ovu = (int)floor(fabs(flu) / du * ovuv);
        const int ovv = (int)floor(fabs(flv) / du * ovuv);
        const int ovw = (int)floor(fabs(flw) / dw * ovw_n);
        const int aa_h = suv / 2, aaw_h = sw / 2;
        const int64_t dus0 = (int64_t)cu + N - aa_h, dvs0 = (int64_t)cv + N - aa_h;
        const int64_t dws0 = (int64_t)cw + planes / 2 - aaw_h;
        if (dus0 < 0 || dus0 + suv > G || dvs0 < 0 || dvs0 + suv > G || dws0 < 0 || dws0 + sw > planes ||
            ovu >= ovuv || ovv >= ovuv || ovw >= ovw_n) {
            if (lane == 0) {
                out[i] = make_double2(0.0, 0.0);
                atomicOr(err, DERR_GRID_RANGE);
            }
            continue;
        }
        double2 acc = make_double2(0.0, 0.0);
        for (int a = 0; a < sw; a++) {
            const double gw = conv_w[sw * ovw + a];
            const double2 *plane = stack + (dws0 + a) * G * G;
            for (int t = lane; t < suv * suv; t += 32) {
                const int ty = t / suv, tx = t % suv;
                const double g = gw * conv_uv[suv * ovv + ty] * conv_uv[suv * ovu + tx];
                const double2 z = plane[(dvs0 + ty) * G + dus0 + tx];
                acc.x = fma(z.x, g, acc.x);
                acc.y = fma(z.y, g, acc.y);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        if (lane == 0) out[i] = acc;
    }
}

rg_status check_sepkern(const rg_sepkern *k, const char *name)
{
    if (!k || !k->data) return fail(RG_ERR_INVALID_ARGUMENT, std::string(name) + " is NULL");
    if (k->size < 1 || k->oversampling < 1 || (int64_t)k->size * k->oversampling > (1 << 26))
        return fail(RG_ERR_INVALID_ARGUMENT, std::string(name) + ": bad size or oversampling");
    return RG_OK;
}

// Host copy of a table (host or device pointer).
rg_status host_table(const rg_sepkern *k, std::vector<double> &out)
{
    out.resize((size_t)k->size * k->oversampling);
    RG_CUDA(cudaMemcpy(out.data(), k->data, sizeof(double) * out.size(), cudaMemcpyDefault));
    return RG_OK;
}

}  // namespace
}  // namespace rg

using namespace rg;

extern "C" rg_status rg_wstack_predict(rg_context *ctx, double theta, double lambda, const double *points,
                                       int npoints, const double *u, const double *v, const double *w,
                                       int64_t nvis, double du, double dw, double x0, const rg_sepkern *conv_uv,
                                       const rg_sepkern *conv_w, const rg_sepkern *corr_lm,
                                       const rg_sepkern *corr_n, double *vis_out)
{
    if (!ctx || (npoints > 0 && !points) || (nvis > 0 && (!u || !v || !w || !vis_out)))
        return fail(RG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (npoints < 0 || nvis < 0) return fail(RG_ERR_INVALID_ARGUMENT, "negative counts");
    if (!(theta > 0.0 && theta < 1.0) || !(lambda > 0.0) || !std::isfinite(lambda))
        return fail(RG_ERR_INVALID_ARGUMENT, "theta must be in (0, 1) and lambda > 0");
    if (!(du > 0.0) || !(dw > 0.0) || !std::isfinite(du) || !std::isfinite(dw))
        return fail(RG_ERR_INVALID_ARGUMENT, "du and dw must be finite and > 0");
    RG_CHECK(check_sepkern(conv_uv, "conv_uv"));
    RG_CHECK(check_sepkern(conv_w, "conv_w"));
    RG_CHECK(check_sepkern(corr_lm, "corr_lm"));
    RG_CHECK(check_sepkern(corr_n, "corr_n"));
    // the padded grid: the reference's round(0.5 / x0) (predict.cpp:410)
    if (!(x0 > 0.0 && x0 < 0.5)) return fail(RG_ERR_INVALID_ARGUMENT, "x0 must be in (0, 0.5)");
    const double x0ih = std::round(0.5 / x0);
    if (std::fabs(0.5 / x0 - x0ih) > 1e-9)
        return fail(RG_ERR_UNSUPPORTED, "0.5 / x0 must be an integer (the padding factor)");
    const int N = (int)std::floor(theta * lambda);
    const int G = (int)(x0ih * N);
    if (N < 2 || N % 2) return fail(RG_ERR_UNSUPPORTED, "floor(theta * lambda) must be even and >= 2");
    if (!fft64_any_supported(G)) return fail(RG_ERR_UNSUPPORTED, "the padded grid must be at most 4096 pixels");
    const int suv = conv_uv->size, sw = conv_w->size;
    const double max_w = std::sin(theta / 2) * std::sqrt(2.0 * ((double)N * N));
    const int planes = (int)std::ceil(max_w / dw) + sw + 1;  // predict.cpp:420-421
    const int t0 = -planes / 2;                               // predict.cpp:472
    const size_t g2 = (size_t)G * G;
    if ((double)g2 * planes * 16.0 * 2.2 > 120e9) return fail(RG_ERR_UNSUPPORTED, "w stack too large");
    RG_CUDA(cudaSetDevice(ctx->device));
    begin_call(ctx);

    // the quantised, grid-corrected sky (predict.cpp:187-245), summed per
    // pixel in source order, at its fft-shifted position
    std::vector<double> pts((size_t)2 * npoints), lm, nn;
    if (npoints > 0) RG_CUDA(cudaMemcpy(pts.data(), points, sizeof(double) * pts.size(), cudaMemcpyDefault));
    RG_CHECK(host_table(corr_lm, lm));
    RG_CHECK(host_table(corr_n, nn));
    const int lm_t = (int)lm.size(), n_t = (int)nn.size();
    const double lm_step = 1.0 / (double)lm_t, n_step = 1.0 / (double)n_t;
    const int gd = (G - N) / 2;
    std::vector<SkyEntry> sky;
    for (int i = 0; i < npoints; i++) {
        const double l = pts[2 * i], m = pts[2 * i + 1];
        if (!std::isfinite(l) || !std::isfinite(m)) return fail(RG_ERR_INVALID_ARGUMENT, "non-finite source position");
        const int lc = (int)std::floor((l / theta + 0.5) * (double)N);
        const int mc = (int)std::floor((m / theta + 0.5) * (double)N);
        if (lc < 0 || lc >= N || mc < 0 || mc >= N)
            return fail(RG_ERR_INVALID_ARGUMENT, "a source lies outside the image (|l|, |m| < theta / 2)");
        const double lq = (double)lc / lambda - theta / 2;
        const double mq = (double)mc / lambda - theta / 2;
        const double n = std::sqrt(1.0 - lq * lq - mq * mq) - 1.0;
        const int aau = (int)std::floor((du * lq) / lm_step) + lm_t / 2;
        const int aav = (int)std::floor((du * mq) / lm_step) + lm_t / 2;
        const int aaw = (int)std::floor((dw * n) / n_step) + n_t / 2;
        if (aau < 0 || aau >= lm_t || aav < 0 || aav >= lm_t || aaw < 0 || aaw >= n_t)
            return fail(RG_ERR_INVALID_ARGUMENT, "a source lies outside the grid-correction tables");
        double a = 1.0;
        a *= lm[aau];
        a *= lm[aav];
        a *= nn[aaw];
        const int col = (gd + lc + G / 2) % G, row = (gd + mc + G / 2) % G;
        const int64_t idx = (int64_t)row * G + col;
        bool merged = false;
        for (auto &e : sky)
            if (e.idx == idx) {
                e.re += 1.0 / a;
                merged = true;
                break;
            }
        if (!merged) sky.push_back({idx, 1.0 / a, lc, mc});
    }
    const int nsrc = (int)sky.size();
    std::vector<int64_t> hidx(nsrc);
    std::vector<double> hval(nsrc);
    std::vector<int2> hpix(nsrc);
    for (int s = 0; s < nsrc; s++) {
        hidx[s] = sky[s].idx;
        hval[s] = sky[s].re;
        hpix[s] = make_int2(sky[s].x, sky[s].y);
    }
    void *stack, *tmp, *sidx, *sval, *spix, *work = nullptr;
    RG_CHECK(scratch(ctx, "wstack_planes", sizeof(double2) * g2 * planes, &stack));
    RG_CHECK(scratch(ctx, "wstack_tmp", sizeof(double2) * g2 * planes, &tmp));
    RG_CHECK(scratch(ctx, "wstack_sky_idx", sizeof(int64_t) * (nsrc + 1), &sidx));
    RG_CHECK(scratch(ctx, "wstack_sky_val", sizeof(double) * (nsrc + 1), &sval));
    RG_CHECK(scratch(ctx, "wstack_sky_pix", sizeof(int2) * (nsrc + 1), &spix));
    if (fft64_any_work_elems(G) > 0)
        RG_CHECK(scratch(ctx, "fft64_work", sizeof(double2) * (size_t)fft64_any_work_elems(G), &work));
    const void *tuv, *tw;
    RG_CHECK(stage_in(ctx, conv_uv->data, sizeof(double) * (size_t)suv * conv_uv->oversampling, "wstack_conv_uv", &tuv));
    RG_CHECK(stage_in(ctx, conv_w->data, sizeof(double) * (size_t)sw * conv_w->oversampling, "wstack_conv_w", &tw));
    const void *du_p, *dv_p, *dw_p;
    RG_CHECK(stage_in(ctx, u, sizeof(double) * (size_t)nvis, "in_u", &du_p));
    RG_CHECK(stage_in(ctx, v, sizeof(double) * (size_t)nvis, "in_v", &dv_p));
    RG_CHECK(stage_in(ctx, w, sizeof(double) * (size_t)nvis, "in_w", &dw_p));
    OutView ov;
    RG_CHECK(out_view(ctx, vis_out, sizeof(double2) * (size_t)nvis, "wstack_vis", false, &ov));
    Diag d;
    RG_CHECK(diag_begin(ctx, &d));

    begin_stage(ctx, "wstack_sky");
    RG_CUDA(cudaMemsetAsync(stack, 0, sizeof(double2) * g2 * planes, ctx->stream));
    if (nsrc > 0) {
        RG_CUDA(cudaMemcpyAsync(sidx, hidx.data(), sizeof(int64_t) * nsrc, cudaMemcpyHostToDevice, ctx->stream));
        RG_CUDA(cudaMemcpyAsync(sval, hval.data(), sizeof(double) * nsrc, cudaMemcpyHostToDevice, ctx->stream));
        RG_CUDA(cudaMemcpyAsync(spix, hpix.data(), sizeof(int2) * nsrc, cudaMemcpyHostToDevice, ctx->stream));
        const int64_t tot = (int64_t)nsrc * planes;
        wstack_scatter_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 4096), 256, 0, ctx->stream>>>(
            (const int64_t *)sidx, (const double *)sval, (const int2 *)spix, nsrc, planes, t0, N, G, theta, dw,
            (double2 *)stack);
        ctx->launches++;
    }
    end_stage(ctx);
    begin_stage(ctx, "wstack_fft");
    launch_fft64_2d(ctx->stream, (double2 *)stack, (double2 *)tmp, planes, G, G, -1, (double2 *)work);
    for (int p = 0; p < planes; p++) launch_fft_shift(ctx->stream, (double2 *)stack + g2 * p, G);
    ctx->launches += 4 + planes;
    end_stage(ctx);
    begin_stage(ctx, "wstack_degrid");
    if (nvis > 0) {
        const int64_t blocks = std::min<int64_t>((nvis + 7) / 8, (int64_t)ctx->sm_count * 16);
        wstack_degrid_kernel<<<(unsigned)blocks, 256, 0, ctx->stream>>>(
            (const double2 *)stack, (const double *)du_p, (const double *)dv_p, (const double *)dw_p, nvis, du, dw,
            N, G, planes, (const double *)tuv, suv,
            conv_uv->oversampling, (const double *)tw, sw, conv_w->oversampling, (double2 *)ov.dev, d.err);
        ctx->launches++;
    }
    end_stage(ctx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "W-stacking predict launch");
    RG_CHECK(finish_out(ctx, ov));
    RG_CHECK(diag_end(ctx, d, nullptr));
    collect_timings(ctx);
    ctx->stats[0] = nvis;
    ctx->stats[3] = planes;
    ctx->stats[5] = ctx->launches;
    return RG_OK;
}
