// Direct Fourier transform imager.
//
//   image[y][x] = factor * sum_k Re(V_k exp(-2 pi i phi_k(x, y)))
//   phi = u l + v m + w (1 - n),  l = theta (x - N/2)/N, m = theta (y - N/2)/N
//
// the phase convention of the reference's calculate_dft_sum_flat
// (src/dft/dft_cuda.cu:15-39), with l taken from the column and u, v, w in
// wavelengths (its defects, src/dft/dft_cuda.cu:55-57 and :98-112, removed).
//
// A CTA owns a 32 x 32 pixel tile; each thread four pixels of one column.
// Rows [row0, row0 + nrows) only (a rank's share of a row-partitioned image):
// tiles start at row0, so a share that starts on a multiple of 32 computes its
// rows exactly as the whole image does.
// Visibilities are staged through shared memory 256 at a time.  Precision
// modes (the precision study):
//   FP64_REDUCED: per (tile, visibility) the phase at the tile centre phi0 is
//     formed and reduced modulo 1 in FP64 and folded into the visibility
//     (V' = V exp(-2 pi i phi0)); per pixel only the small increment
//     delta = u dl + v dm + w (n0 - n) is formed in FP32, reduced modulo 1, and
//     fed to the hardware sin/cos.  Partial sums are FP32 per batch of 256,
//     accumulated in FP64.
//   FP32_NAIVE: phi formed in FP32 from FP32 u, v, w, l, m, n, reduced in FP32.
//   FP64: phi, reduction and sin/cos all FP64.
#include "rg_internal.h"

namespace rg {

constexpr int TILE = 32, DFT_BATCH = 256, PIX = 4;

template <int MODE>
__global__ void __launch_bounds__(256) dft_kernel(const double *__restrict__ u,
                                                  const double *__restrict__ v,
                                                  const double *__restrict__ w,
                                                  const double2 *__restrict__ vis, int64_t nvis,
                                                  double *__restrict__ image, int N, double theta,
                                                  double factor, int row0, int nrows)
{
    // FP32 modes: (u, v, w, Re V) as one 16-byte entry and Im V beside it, so a
    // visibility is two shared-memory loads in the inner loop
    __shared__ float4 s4[DFT_BATCH];
    __shared__ float si[DFT_BATCH];
    __shared__ double du[DFT_BATCH], dv[DFT_BATCH], dw[DFT_BATCH], dr[DFT_BATCH], di[DFT_BATCH];
    const int tx = threadIdx.x % TILE, ty = threadIdx.x / TILE;  // ty in [0, 8)
    const int x0 = blockIdx.x * TILE, y0 = row0 + blockIdx.y * TILE;
    const int cx = x0 + TILE / 2, cy = y0 + TILE / 2;
    const double l0 = theta * (double)(cx - N / 2) / N;
    const double m0 = theta * (double)(cy - N / 2) / N;
    const double n0 = sqrt(1.0 - l0 * l0 - m0 * m0);

    const int x = x0 + tx;
    const double l = theta * (double)(x - N / 2) / N;
    double lp[PIX], mp[PIX], one_minus_n[PIX];
    float dl, dm[PIX], dn[PIX];
    dl = (float)(l - l0);
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        const int y = y0 + ty + 8 * p;
        lp[p] = l;
        mp[p] = theta * (double)(y - N / 2) / N;
        const double nn = sqrt(1.0 - l * l - mp[p] * mp[p]);
        one_minus_n[p] = 1.0 - nn;
        dm[p] = (float)(mp[p] - m0);
        dn[p] = (float)(n0 - nn);
    }
    double acc[PIX] = {0.0, 0.0, 0.0, 0.0};

    for (int64_t b0 = 0; b0 < nvis; b0 += DFT_BATCH) {
        const int cnt = (int)(nvis - b0 < DFT_BATCH ? nvis - b0 : DFT_BATCH);
        __syncthreads();
        if ((int)threadIdx.x < cnt) {
            const int64_t k = b0 + threadIdx.x;
            const double uu = u[k], vv = v[k], ww = w[k];
            const double2 z = vis[k];
            if (MODE == RG_DFT_FP64_REDUCED) {
                double ph = uu * l0 + vv * m0 + ww * (1.0 - n0);
                ph -= rint(ph);
                double s, c;
                sincospi(2.0 * ph, &s, &c);
                // V' = V exp(-2 pi i phi0)
                s4[threadIdx.x] = make_float4((float)uu, (float)vv, (float)ww, (float)(z.x * c + z.y * s));
                si[threadIdx.x] = (float)(z.y * c - z.x * s);
            } else if (MODE == RG_DFT_FP32_NAIVE) {
                s4[threadIdx.x] = make_float4((float)uu, (float)vv, (float)ww, (float)z.x);
                si[threadIdx.x] = (float)z.y;
            } else {
                du[threadIdx.x] = uu;
                dv[threadIdx.x] = vv;
                dw[threadIdx.x] = ww;
                dr[threadIdx.x] = z.x;
                di[threadIdx.x] = z.y;
            }
        }
        __syncthreads();
        if (MODE == RG_DFT_FP64) {
            double part[PIX] = {0.0, 0.0, 0.0, 0.0};
            for (int j = 0; j < cnt; j++) {
#pragma unroll
                for (int p = 0; p < PIX; p++) {
                    double ph = du[j] * lp[p] + dv[j] * mp[p] + dw[j] * one_minus_n[p];
                    ph -= rint(ph);
                    double s, c;
                    sincospi(2.0 * ph, &s, &c);
                    part[p] += dr[j] * c + di[j] * s;
                }
            }
#pragma unroll
            for (int p = 0; p < PIX; p++) acc[p] += part[p];
        } else {
            float part[PIX] = {0.f, 0.f, 0.f, 0.f};
            float fl[PIX], fm[PIX], fn[PIX];
#pragma unroll
            for (int p = 0; p < PIX; p++) {
                if (MODE == RG_DFT_FP32_NAIVE) {
                    fl[p] = (float)lp[p];
                    fm[p] = (float)mp[p];
                    fn[p] = (float)one_minus_n[p];
                } else {
                    fl[p] = dl;
                    fm[p] = dm[p];
                    fn[p] = dn[p];
                }
            }
#pragma unroll 4
            for (int j = 0; j < cnt; j++) {
                const float4 e = s4[j];
                const float uj = e.x, vj = e.y, wj = e.z, rj = e.w, ij = si[j];
#pragma unroll
                for (int p = 0; p < PIX; p++) {
                    float d = fmaf(uj, fl[p], fmaf(vj, fm[p], wj * fn[p]));
                    // nearest integer by the 1.5 * 2^23 shift (|d| < 2^22 turns):
                    // two adds on the FMA pipe instead of a rounding instruction
                    d -= (d + 12582912.f) - 12582912.f;
                    float s, c;
                    __sincosf(6.283185307179586f * d, &s, &c);
                    part[p] = fmaf(rj, c, fmaf(ij, s, part[p]));
                }
            }
#pragma unroll
            for (int p = 0; p < PIX; p++) acc[p] += (double)part[p];
        }
    }
#pragma unroll
    for (int p = 0; p < PIX; p++) {
        const int y = y0 + ty + 8 * p;
        if (x < N && y < row0 + nrows) image[(int64_t)(y - row0) * N + x] = factor * acc[p];
    }
}

void launch_dft(cudaStream_t s, const double *u, const double *v, const double *w,
                const double2 *vis, int64_t n, double *image, int grid_size, double theta,
                int precision, double factor, int sm_count, int row0, int nrows)
{
    (void)sm_count;
    if (nrows < 0) {
        row0 = 0;
        nrows = grid_size;
    }
    if (nrows == 0) return;
    dim3 grd((grid_size + TILE - 1) / TILE, (nrows + TILE - 1) / TILE);
    switch (precision) {
        case RG_DFT_FP32_NAIVE:
            dft_kernel<RG_DFT_FP32_NAIVE><<<grd, 256, 0, s>>>(u, v, w, vis, n, image, grid_size, theta, factor, row0,
                                                                 nrows);
            break;
        case RG_DFT_FP64:
            dft_kernel<RG_DFT_FP64><<<grd, 256, 0, s>>>(u, v, w, vis, n, image, grid_size, theta, factor, row0,
                                                                 nrows);
            break;
        default:
            dft_kernel<RG_DFT_FP64_REDUCED><<<grd, 256, 0, s>>>(u, v, w, vis, n, image, grid_size, theta, factor, row0,
                                                                 nrows);
            break;
    }
}

}  // namespace rg
