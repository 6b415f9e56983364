// The w-kernel generator behind the C ABI: oversampled tap tables from a
// PSWF-tapered w-screen, in the layout the gridders index
// (kern_by_w[plane].data[(yf*ov + xf)*S*S + y*S + x], src/reference/grid.c:53-56).
//
// The reference has no generator of its own: its kernels come from the
// crocodile scripts as HDF5 files (README.md:25-26, loaded by
// src/common/hdf5.c:1362-1509).  This one is written from the mathematics:
//
//   s_w(l, m)  = A(l) A(m) exp(+2 pi i w (1 - sqrt(1 - l^2 - m^2)))
//                on an M x M screen, l = theta (i - M/2) / M,
//   K_w(p, q)  = 1/M^2 sum_ij s_w(l_i, m_j) exp(-2 pi i (p l_i + q m_j) / theta),
//   tap[plane][yf][xf][ty][tx] = K_w(tx - S/2 - xf/ov, ty - S/2 - yf/ov),
//
// A(x) = psi_0(c, 2x/theta), the zeroth prolate spheroidal wave function
// normalised to psi_0(0) = 1.  psi_0 is evaluated from its expansion in
// normalised Legendre polynomials, whose coefficients are the eigenvector of
// the smallest eigenvalue of a symmetric tridiagonal matrix (Bouwkamp 1947;
// Xiao, Rokhlin & Yarvin 2001); the eigenvalue is found by Sturm-sequence
// bisection and the eigenvector by inverse iteration (Wilkinson, The
// Algebraic Eigenvalue Problem, ch. 5 and 9).  The screen and the two
// non-uniform DFT sums run on the device in FP64.
#include <algorithm>
#include <cmath>
#include <vector>

#include "rg_internal.h"

namespace rg {
namespace {

// Tridiagonal matrix of the operator (1 - x^2) d2/dx2 - 2x d/dx - c^2 x^2 in
// the normalised even-degree Legendre basis sqrt(k + 1/2) P_k, k = 0, 2, ...
void pswf_matrix(double c, int nterms, std::vector<double> &d, std::vector<double> &e)
{
    d.resize(nterms);
    e.resize(nterms > 0 ? nterms - 1 : 0);
    const double c2 = c * c;
    for (int j = 0; j < nterms; j++) {
        const double k = 2.0 * j;
        d[j] = k * (k + 1) + c2 * (2 * k * (k + 1) - 1) / ((2 * k + 3) * (2 * k - 1));
        if (j + 1 < nterms) e[j] = c2 * (k + 1) * (k + 2) / ((2 * k + 3) * std::sqrt((2 * k + 1) * (2 * k + 5)));
    }
}

// Eigenvalues of the tridiagonal matrix below x (Sturm sequence of the LDL^T
// pivots).
int sturm_count(const std::vector<double> &d, const std::vector<double> &e, double x)
{
    int count = 0;
    double q = d[0] - x;
    if (q < 0) count++;
    for (size_t i = 1; i < d.size(); i++) {
        const double qq = q != 0.0 ? q : 1e-300;
        q = d[i] - x - e[i - 1] * e[i - 1] / qq;
        if (q < 0) count++;
    }
    return count;
}

// Solve (T - sigma I) y = b for tridiagonal T, Gaussian elimination with
// partial pivoting on the dense band (a small system: ~2c + 40 unknowns).
void shifted_solve(const std::vector<double> &d, const std::vector<double> &e, double sigma,
                   const std::vector<double> &b, std::vector<double> &y)
{
    const int n = (int)d.size();
    std::vector<double> a((size_t)n * n, 0.0), r(b);
    for (int i = 0; i < n; i++) {
        a[(size_t)i * n + i] = d[i] - sigma;
        if (i + 1 < n) a[(size_t)i * n + i + 1] = a[(size_t)(i + 1) * n + i] = e[i];
    }
    for (int col = 0; col < n; col++) {
        int piv = col;
        for (int i = col + 1; i < n; i++)
            if (std::fabs(a[(size_t)i * n + col]) > std::fabs(a[(size_t)piv * n + col])) piv = i;
        if (piv != col) {
            for (int j = 0; j < n; j++) std::swap(a[(size_t)col * n + j], a[(size_t)piv * n + j]);
            std::swap(r[col], r[piv]);
        }
        double p = a[(size_t)col * n + col];
        if (p == 0.0) p = a[(size_t)col * n + col] = 1e-300;  // exactly singular: any scaled eigenvector will do
        for (int i = col + 1; i < n; i++) {
            const double f = a[(size_t)i * n + col] / p;
            if (f == 0.0) continue;
            for (int j = col; j < n; j++) a[(size_t)i * n + j] -= f * a[(size_t)col * n + j];
            r[i] -= f * r[col];
        }
    }
    y.assign(n, 0.0);
    for (int i = n - 1; i >= 0; i--) {
        double s = r[i];
        for (int j = i + 1; j < n; j++) s -= a[(size_t)i * n + j] * y[j];
        y[i] = s / a[(size_t)i * n + i];
    }
}

// Expansion coefficients of psi_0(c, .) (unnormalised, any sign).
std::vector<double> pswf_coefficients(double c)
{
    const int nterms = (int)(2 * c + 40);
    std::vector<double> d, e;
    pswf_matrix(c, nterms, d, e);
    // Gershgorin interval, then bisection for the smallest eigenvalue
    double lo = d[0], hi = d[0];
    for (int i = 0; i < nterms; i++) {
        const double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i + 1 < nterms ? std::fabs(e[i]) : 0.0);
        lo = std::fmin(lo, d[i] - r);
        hi = std::fmax(hi, d[i] + r);
    }
    for (int it = 0; it < 200 && hi - lo > 1e-15 * std::fmax(1.0, std::fabs(lo) + std::fabs(hi)); it++) {
        const double mid = 0.5 * (lo + hi);
        if (sturm_count(d, e, mid) >= 1) hi = mid;
        else lo = mid;
    }
    const double lambda = 0.5 * (lo + hi);
    std::vector<double> x(nterms, 1.0), y;
    for (int it = 0; it < 6; it++) {
        shifted_solve(d, e, lambda, x, y);
        double nrm = 0.0;
        for (double v : y) nrm += v * v;
        nrm = std::sqrt(nrm);
        for (int i = 0; i < nterms; i++) x[i] = y[i] / nrm;
    }
    return x;
}

// psi_0(c, x) / psi_0(c, 0) from the coefficients, by the Legendre recurrence.
double pswf_value(const std::vector<double> &coef, double x)
{
    double p_prev = 1.0, p_cur = x;  // P_0, P_1
    double out = coef[0] * std::sqrt(0.5), at0 = coef[0] * std::sqrt(0.5);
    double q_prev = 1.0, q_cur = 0.0;  // the same at x = 0
    int deg = 1;
    for (size_t j = 1; j < coef.size(); j++) {
        const int k = 2 * (int)j;
        while (deg < k) {
            const double p_next = ((2 * deg + 1) * x * p_cur - deg * p_prev) / (deg + 1);
            const double q_next = (-(double)deg * q_prev) / (deg + 1);
            p_prev = p_cur;
            p_cur = p_next;
            q_prev = q_cur;
            q_cur = q_next;
            deg++;
        }
        out += coef[j] * std::sqrt(k + 0.5) * p_cur;
        at0 += coef[j] * std::sqrt(k + 0.5) * q_cur;
    }
    return out / at0;
}

// s[plane][j][i] = A_i A_j exp(+2 pi i w (1 - n)), FP64.
__global__ void wscreen_kernel(const double *__restrict__ w_planes, int planes, const double *__restrict__ taper,
                               int M, double theta, double2 *__restrict__ s)
{
    const int64_t total = (int64_t)planes * M * M;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(k % M), j = (int)((k / M) % M), p = (int)(k / ((int64_t)M * M));
        const double l = theta * (double)(i - M / 2) / M, m = theta * (double)(j - M / 2) / M;
        const double one_minus_n = 1.0 - sqrt(1.0 - (l * l + m * m));
        double sn, cs;
        sincospi(2.0 * w_planes[p] * one_minus_n, &sn, &cs);
        const double a = taper[i] * taper[j];
        s[k] = make_double2(a * cs, a * sn);
    }
}

// E[q][i] = exp(-2 pi i off_q (i - M/2) / M), off_q = t - S/2 - f/ov for
// q = f*S + t (sub-cell shift f, tap t).
__global__ void wkgen_phasors_kernel(int S, int ov, int M, double2 *__restrict__ E)
{
    const int total = ov * S * M;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int i = k % M, q = k / M;
        const int f = q / S, t = q % S;
        const double off = (double)(t - S / 2) - (double)f / ov;
        double sn, cs;
        sincospi(-2.0 * off * (double)(i - M / 2) / M, &sn, &cs);
        E[k] = make_double2(cs, sn);
    }
}

__device__ __forceinline__ double2 cmad(double2 a, double2 b, double2 acc)
{
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}

// T[plane][j][qx] = sum_i s[plane][j][i] E[qx][i]
__global__ void wkgen_rows_kernel(const double2 *__restrict__ s, const double2 *__restrict__ E, int planes, int M,
                                  int Q, double2 *__restrict__ T)
{
    const int64_t total = (int64_t)planes * M * Q;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int qx = (int)(k % Q);
        const int64_t pj = k / Q;  // plane * M + j
        const double2 *row = s + pj * M;
        const double2 *e = E + (int64_t)qx * M;
        double2 acc = make_double2(0.0, 0.0);
        for (int i = 0; i < M; i++) acc = cmad(row[i], e[i], acc);
        T[k] = acc;
    }
}

// data[plane][yf][xf][ty][tx] = 1/M^2 sum_j E[qy][j] T[plane][j][qx],
// qy = yf*S + ty, qx = xf*S + tx
__global__ void wkgen_cols_kernel(const double2 *__restrict__ T, const double2 *__restrict__ E, int planes, int M,
                                  int S, int ov, double2 *__restrict__ out)
{
    const int Q = ov * S;
    const int64_t total = (int64_t)planes * Q * Q;
    const double inv = 1.0 / ((double)M * M);
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        // output order [plane][yf][xf][ty][tx]
        const int tx = (int)(k % S);
        const int ty = (int)((k / S) % S);
        const int xf = (int)((k / ((int64_t)S * S)) % ov);
        const int yf = (int)((k / ((int64_t)S * S * ov)) % ov);
        const int p = (int)(k / ((int64_t)Q * Q));
        const int qx = xf * S + tx, qy = yf * S + ty;
        const double2 *e = E + (int64_t)qy * M;
        const double2 *t = T + (int64_t)p * M * Q + qx;
        double2 acc = make_double2(0.0, 0.0);
        for (int j = 0; j < M; j++) acc = cmad(e[j], t[(int64_t)j * Q], acc);
        out[k] = make_double2(acc.x * inv, acc.y * inv);
    }
}

}  // namespace
}  // namespace rg

using namespace rg;

extern "C" {

rg_status rg_pswf0(double c, const double *x, int64_t n, double *out)
{
    if (n < 0 || (n > 0 && (!x || !out))) return fail(RG_ERR_INVALID_ARGUMENT, "x and out must be non-NULL");
    if (!(c > 0.0) || !std::isfinite(c) || c > 1000.0) return fail(RG_ERR_INVALID_ARGUMENT, "c must be in (0, 1000]");
    const std::vector<double> coef = pswf_coefficients(c);
    for (int64_t k = 0; k < n; k++) {
        if (!(std::fabs(x[k]) <= 1.0)) return fail(RG_ERR_INVALID_ARGUMENT, "x must lie in [-1, 1]");
        out[k] = pswf_value(coef, x[k]);
    }
    return RG_OK;
}

rg_status rg_wkern_generate(rg_context *ctx, double theta, const double *w_planes, int plane_count, int size,
                            int oversampling, double c, int screen_pixels, double *data_out)
{
    if (!ctx || !w_planes || !data_out) return fail(RG_ERR_INVALID_ARGUMENT, "ctx, w_planes and data_out must be non-NULL");
    if (!(theta > 0.0) || !(theta < 2.0)) return fail(RG_ERR_INVALID_ARGUMENT, "theta must be in (0, 2)");
    if (plane_count < 1 || plane_count > 65536) return fail(RG_ERR_INVALID_ARGUMENT, "plane_count must be in [1, 65536]");
    if (size < 2 || size > 64 || size % 2) return fail(RG_ERR_INVALID_ARGUMENT, "size must be even, in [2, 64]");
    if (oversampling < 1 || oversampling > 128) return fail(RG_ERR_INVALID_ARGUMENT, "oversampling must be in [1, 128]");
    const int M = screen_pixels > 0 ? screen_pixels : 128;
    if (M < 4 || M > 4096 || M % 2) return fail(RG_ERR_INVALID_ARGUMENT, "screen_pixels must be even, in [4, 4096]");
    const double cc = c > 0.0 ? c : M_PI * (size - 2) / 2.0;
    if (!std::isfinite(cc) || cc > 1000.0) return fail(RG_ERR_INVALID_ARGUMENT, "c must be finite and <= 1000");
    for (int p = 0; p < plane_count; p++)
        if (!std::isfinite(w_planes[p])) return fail(RG_ERR_INVALID_ARGUMENT, "w planes must be finite");
    // the screen must stay inside the unit circle: (theta/2)^2 * 2 < 1
    RG_CUDA(cudaSetDevice(ctx->device));
    begin_call(ctx);
    const std::vector<double> coef = pswf_coefficients(cc);
    std::vector<double> taper(M);
    for (int i = 0; i < M; i++) taper[i] = pswf_value(coef, 2.0 * (double)(i - M / 2) / M);
    const int S = size, ov = oversampling, Q = ov * S;
    const int64_t ntaps = (int64_t)plane_count * Q * Q;
    void *d_w, *d_taper, *d_s, *d_E, *d_T;
    RG_CHECK(scratch(ctx, "wkgen_w", sizeof(double) * plane_count, &d_w));
    RG_CHECK(scratch(ctx, "wkgen_taper", sizeof(double) * M, &d_taper));
    RG_CHECK(scratch(ctx, "wkgen_screen", sizeof(double2) * (size_t)plane_count * M * M, &d_s));
    RG_CHECK(scratch(ctx, "wkgen_phasors", sizeof(double2) * (size_t)Q * M, &d_E));
    RG_CHECK(scratch(ctx, "wkgen_rows", sizeof(double2) * (size_t)plane_count * M * Q, &d_T));
    OutView ov_out;
    RG_CHECK(out_view(ctx, data_out, sizeof(double2) * (size_t)ntaps, "wkgen_out", false, &ov_out));
    RG_CUDA(cudaMemcpyAsync(d_w, w_planes, sizeof(double) * plane_count, cudaMemcpyHostToDevice, ctx->stream));
    RG_CUDA(cudaMemcpyAsync(d_taper, taper.data(), sizeof(double) * M, cudaMemcpyHostToDevice, ctx->stream));
    auto blocks = [](int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 32); };
    wscreen_kernel<<<blocks((int64_t)plane_count * M * M), 256, 0, ctx->stream>>>(
        (const double *)d_w, plane_count, (const double *)d_taper, M, theta, (double2 *)d_s);
    wkgen_phasors_kernel<<<blocks((int64_t)Q * M), 256, 0, ctx->stream>>>(S, ov, M, (double2 *)d_E);
    wkgen_rows_kernel<<<blocks((int64_t)plane_count * M * Q), 256, 0, ctx->stream>>>(
        (const double2 *)d_s, (const double2 *)d_E, plane_count, M, Q, (double2 *)d_T);
    wkgen_cols_kernel<<<blocks(ntaps), 256, 0, ctx->stream>>>((const double2 *)d_T, (const double2 *)d_E,
                                                              plane_count, M, S, ov, (double2 *)ov_out.dev);
    ctx->launches += 4;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "w-kernel generator launch");
    RG_CHECK(finish_out(ctx, ov_out));
    RG_CUDA(cudaStreamSynchronize(ctx->stream));
    return RG_OK;
}

}  // extern "C"
