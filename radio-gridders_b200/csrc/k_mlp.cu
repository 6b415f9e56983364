// Learned w-kernel: a small MLP evaluated on tensor cores.
//
// Network (no counterpart in the reference; the reference reads quantised,
// oversampled w-kernel tables, src/reference/grid.c:157-185): 21 input features
// of a tap (w, sub-cell offsets du, dv, tap x, tap y and 16 Fourier features of
// the tap's offset from the visibility) -> 128 -> 128 -> 128 (SiLU) -> 2
// (complex tap / out_scale).  Layers 1-3 run as BF16 x BF16 -> FP32
// mma.sync.m16n8k16 tiles from shared memory; the 128 -> 2 output layer and all
// element-wise work are FP32.
//
// Parameters: one FP32 buffer, W1[32][128] (rows >= 21 unused), b1[128],
// W2[128][128], b2, W3[128][128], b3, W4[128][2], b4[2] (W[in][out]); plus BF16
// copies refreshed after every optimiser step: W1..W3 transposed (W^T[out][in],
// the forward pass's B operand, read as packed pairs along k) and W2, W3 as
// stored (the backward pass's W^T operand).
//
// Training: mlp_grad_kernel runs forward and backward for a tile of 64 samples
// entirely in shared memory and adds its weight gradients into an FP32
// gradient buffer with atomics; mlp_adam_kernel applies Adam and refreshes the
// BF16 copy.  Loss: mean over samples of |y - target / out_scale|^2.
#include <cuda_bf16.h>

#include "rg_internal.h"

namespace rg {

constexpr int MH = 128, MFIN = 32, MNFEAT = 21;
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + MFIN * MH;
constexpr int OFF_W2 = OFF_B1 + MH;
constexpr int OFF_B2 = OFF_W2 + MH * MH;
constexpr int OFF_W3 = OFF_B2 + MH;
constexpr int OFF_B3 = OFF_W3 + MH * MH;
constexpr int OFF_W4 = OFF_B3 + MH;
constexpr int OFF_B4 = OFF_W4 + MH * 2;
constexpr int MLP_NPARAM = OFF_B4 + 2;
// BF16 copy offsets: transposed W1..W3 (forward), then W2, W3 as stored (backward)
constexpr int BOFF_W1T = 0, BOFF_W2T = MFIN * MH, BOFF_W3T = BOFF_W2T + MH * MH;
constexpr int BOFF_W2 = BOFF_W3T + MH * MH, BOFF_W3 = BOFF_W2 + MH * MH, MLP_NBF16 = BOFF_W3 + MH * MH;

// padded shared-memory leading dimensions (bank-conflict free fragment access)
constexpr int LDF = MFIN + 8;  // features, bf16
constexpr int LDH = MH + 8;    // activations, bf16
constexpr int LDZ = MH + 8;    // pre-activations / gradients, fp32

using bf16 = __nv_bfloat16;

int mlp_param_count() { return MLP_NPARAM; }
int mlp_bf16_count() { return MLP_NBF16; }

__device__ __forceinline__ uint32_t pack_bf16(bf16 lo, bf16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Element (i, k) of A and (k, n) of B, with optional transposition of the
// stored row-major arrays.
template <bool T>
__device__ __forceinline__ bf16 at(const bf16 *M, int ld, int r, int c)
{
    return T ? M[c * ld + r] : M[r * ld + c];
}

// One warp accumulates the WM x WN tile at (m0, n0) of C = A(MxK) * B(KxN).
template <int WM, int WN, bool TA, bool TB>
__device__ __forceinline__ void warp_gemm(const bf16 *A, int lda, const bf16 *B, int ldb, int K,
                                          int m0, int n0, float (&acc)[WM / 16][WN / 8][4])
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t a[WM / 16][4];
#pragma unroll
        for (int mi = 0; mi < WM / 16; mi++) {
            const int r = m0 + mi * 16 + g;
            const int c = k0 + 2 * t;
            if (!TA) {
                a[mi][0] = *reinterpret_cast<const uint32_t *>(A + r * lda + c);
                a[mi][1] = *reinterpret_cast<const uint32_t *>(A + (r + 8) * lda + c);
                a[mi][2] = *reinterpret_cast<const uint32_t *>(A + r * lda + c + 8);
                a[mi][3] = *reinterpret_cast<const uint32_t *>(A + (r + 8) * lda + c + 8);
            } else {
                a[mi][0] = pack_bf16(at<true>(A, lda, r, c), at<true>(A, lda, r, c + 1));
                a[mi][1] = pack_bf16(at<true>(A, lda, r + 8, c), at<true>(A, lda, r + 8, c + 1));
                a[mi][2] = pack_bf16(at<true>(A, lda, r, c + 8), at<true>(A, lda, r, c + 9));
                a[mi][3] = pack_bf16(at<true>(A, lda, r + 8, c + 8), at<true>(A, lda, r + 8, c + 9));
            }
        }
#pragma unroll
        for (int ni = 0; ni < WN / 8; ni++) {
            const int n = n0 + ni * 8 + g;
            const int k = k0 + 2 * t;
            uint32_t b0, b1;
            if (TB) {
                b0 = *reinterpret_cast<const uint32_t *>(B + n * ldb + k);
                b1 = *reinterpret_cast<const uint32_t *>(B + n * ldb + k + 8);
            } else {
                b0 = pack_bf16(at<false>(B, ldb, k, n), at<false>(B, ldb, k + 1, n));
                b1 = pack_bf16(at<false>(B, ldb, k + 8, n), at<false>(B, ldb, k + 9, n));
            }
#pragma unroll
            for (int mi = 0; mi < WM / 16; mi++) mma_bf16(acc[mi][ni], a[mi][0], a[mi][1], a[mi][2], a[mi][3], b0, b1);
        }
    }
}

template <int WM, int WN>
__device__ __forceinline__ void zero_acc(float (&acc)[WM / 16][WN / 8][4])
{
#pragma unroll
    for (int mi = 0; mi < WM / 16; mi++)
#pragma unroll
        for (int ni = 0; ni < WN / 8; ni++)
#pragma unroll
            for (int e = 0; e < 4; e++) acc[mi][ni][e] = 0.f;
}

__device__ __forceinline__ float silu_f(float z) { return z / (1.f + __expf(-z)); }
// Inference SiLU: z * sigmoid(z) = z * (1 + tanh(z / 2)) / 2 with the hardware
// tanh approximation (one MUFU op; its ~2^-11 relative error is below the
// BF16 rounding of the activation it feeds).
__device__ __forceinline__ float silu_fast(float z)
{
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
    return 0.5f * z * (1.f + t);
}
__device__ __forceinline__ float dsilu_f(float z)
{
    const float s = 1.f / (1.f + __expf(-z));
    return s * (1.f + z * (1.f - s));
}

// Features of one tap (the definition in oracle/mlp_oracle.py).
__device__ __forceinline__ void tap_features(float w, float du, float dv, float tx, float ty, int ksize,
                                             float inv_wmax, bf16 *f)
{
    const float half = 0.5f * (float)ksize;
    const float p = tx - half - du, q = ty - half - dv;
    const float inv = 1.f / (half + 1.f);
    f[0] = __float2bfloat16(w * inv_wmax);
    f[1] = __float2bfloat16(2.f * du - 1.f);
    f[2] = __float2bfloat16(2.f * dv - 1.f);
    f[3] = __float2bfloat16(p / half);
    f[4] = __float2bfloat16(q / half);
#pragma unroll
    for (int k = 1; k <= 4; k++) {
        float s, c;
        sincospif((float)k * p * inv, &s, &c);
        f[5 + 2 * (k - 1)] = __float2bfloat16(c);
        f[6 + 2 * (k - 1)] = __float2bfloat16(s);
        sincospif((float)k * q * inv, &s, &c);
        f[13 + 2 * (k - 1)] = __float2bfloat16(c);
        f[14 + 2 * (k - 1)] = __float2bfloat16(s);
    }
#pragma unroll
    for (int k = MNFEAT; k < MFIN; k++) f[k] = __float2bfloat16(0.f);
}

// The same features from per-visibility tables: the Fourier terms depend on
// the tap only through p = tx - K/2 - du (q likewise), so a visibility needs
// them at K values of each; tab[t*8 + 2(k-1)], tab[t*8 + 2(k-1) + 1] = cos,
// sin(pi k p_t / (K/2 + 1)) for tap index t.
__device__ __forceinline__ void axis_table(float d, int t, int ksize, float *tab)
{
    const float half = 0.5f * (float)ksize;
    const float p = (float)t - half - d, inv = 1.f / (half + 1.f);
#pragma unroll
    for (int k = 1; k <= 4; k++) {
        float sn, cs;
        sincospif((float)k * p * inv, &sn, &cs);
        tab[t * 8 + 2 * (k - 1)] = cs;
        tab[t * 8 + 2 * (k - 1) + 1] = sn;
    }
}

__device__ __forceinline__ void tap_features_tab(float w, float du, float dv, int tx, int ty, int ksize,
                                                 float inv_wmax, const float *ptab, const float *qtab, bf16 *f)
{
    const float half = 0.5f * (float)ksize;
    const float p = (float)tx - half - du, q = (float)ty - half - dv;
    f[0] = __float2bfloat16(w * inv_wmax);
    f[1] = __float2bfloat16(2.f * du - 1.f);
    f[2] = __float2bfloat16(2.f * dv - 1.f);
    f[3] = __float2bfloat16(p / half);
    f[4] = __float2bfloat16(q / half);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        f[5 + j] = __float2bfloat16(ptab[tx * 8 + j]);
        f[13 + j] = __float2bfloat16(qtab[ty * 8 + j]);
    }
#pragma unroll
    for (int k = MNFEAT; k < MFIN; k++) f[k] = __float2bfloat16(0.f);
}

// Epilogue of a 32x32 (per warp) hidden-layer tile: z = acc + b; Z (fp32,
// optional) and H = bf16(silu(z)).
template <int WM, int WN, bool FAST = false>
__device__ __forceinline__ void hidden_epilogue(const float (&acc)[WM / 16][WN / 8][4], int m0, int n0,
                                                const float *__restrict__ bias, float *Z, bf16 *Hout)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mi = 0; mi < WM / 16; mi++)
#pragma unroll
        for (int ni = 0; ni < WN / 8; ni++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = m0 + mi * 16 + g + 8 * h;
                const int c = n0 + ni * 8 + 2 * t;
                const float z0 = acc[mi][ni][2 * h] + bias[c];
                const float z1 = acc[mi][ni][2 * h + 1] + bias[c + 1];
                if (Z) *reinterpret_cast<float2 *>(Z + r * LDZ + c) = make_float2(z0, z1);
                const float h0 = FAST ? silu_fast(z0) : silu_f(z0), h1 = FAST ? silu_fast(z1) : silu_f(z1);
                *reinterpret_cast<uint32_t *>(Hout + r * LDH + c) =
                    pack_bf16(__float2bfloat16(h0), __float2bfloat16(h1));
            }
}

// ---------------------------------------------------------------------------
// training
// ---------------------------------------------------------------------------
constexpr int TT = 64;  // samples per CTA

struct TrainSmem {
    bf16 F[TT * LDF];
    bf16 H[3][TT * LDH];
    float Z[3][TT * LDZ];
    float Y[TT * 2];
};

// in: [5][n] float (w, du, dv, tx, ty); target: [n] float2 (unscaled taps)
__global__ void __launch_bounds__(256) mlp_grad_kernel(const float *__restrict__ P, const bf16 *__restrict__ PB,
                                                       const float *__restrict__ in, const float2 *__restrict__ target,
                                                       int n, int ksize, float inv_wmax, float inv_scale,
                                                       float *__restrict__ grad, float *__restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem &S = *reinterpret_cast<TrainSmem *>(smem_raw);
    const int row0 = blockIdx.x * TT;
    const int warp = threadIdx.x >> 5;
    const float inv_n = 1.f / (float)n;

    if (threadIdx.x < TT) {
        const int i = row0 + threadIdx.x;
        if (i < n) {
            tap_features(in[i], in[n + i], in[2 * n + i], in[3 * n + i], in[4 * n + i], ksize, inv_wmax,
                         S.F + threadIdx.x * LDF);
        } else {
            for (int k = 0; k < MFIN; k++) S.F[threadIdx.x * LDF + k] = __float2bfloat16(0.f);
        }
    }
    __syncthreads();
    const int m0 = (warp >> 2) * 32, n0 = (warp & 3) * 32;
    const bf16 *WT[3] = {PB + BOFF_W1T, PB + BOFF_W2T, PB + BOFF_W3T};
    const bf16 *Wb[3] = {nullptr, PB + BOFF_W2, PB + BOFF_W3};
    const float *bias[3] = {P + OFF_B1, P + OFF_B2, P + OFF_B3};
    // forward, layers 1-3
    for (int L = 0; L < 3; L++) {
        float acc[2][4][4];
        zero_acc<32, 32>(acc);
        if (L == 0) warp_gemm<32, 32, false, true>(S.F, LDF, WT[0], MFIN, MFIN, m0, n0, acc);
        else warp_gemm<32, 32, false, true>(S.H[L - 1], LDH, WT[L], MH, MH, m0, n0, acc);
        hidden_epilogue<32, 32>(acc, m0, n0, bias[L], S.Z[L], S.H[L]);
        __syncthreads();
    }
    // output layer (fp32), loss, dy
    if (threadIdx.x < TT * 2) {
        const int r = threadIdx.x >> 1, c = threadIdx.x & 1;
        float y = P[OFF_B4 + c];
        for (int k = 0; k < MH; k++) y += __bfloat162float(S.H[2][r * LDH + k]) * P[OFF_W4 + k * 2 + c];
        const int i = row0 + r;
        float dy = 0.f;
        if (i < n) {
            const float2 tg = target[i];
            const float tv = (c == 0 ? tg.x : tg.y) * inv_scale;
            const float d = y - tv;
            atomicAdd(loss, d * d * inv_n);
            dy = 2.f * d * inv_n;
        }
        S.Y[r * 2 + c] = dy;
    }
    __syncthreads();
    // dW4, db4
    if (threadIdx.x < MH * 2) {
        const int k = threadIdx.x >> 1, c = threadIdx.x & 1;
        float s = 0.f;
        for (int r = 0; r < TT; r++) s += __bfloat162float(S.H[2][r * LDH + k]) * S.Y[r * 2 + c];
        atomicAdd(grad + OFF_W4 + k * 2 + c, s);
    }
    if (threadIdx.x < 2) {
        float s = 0.f;
        for (int r = 0; r < TT; r++) s += S.Y[r * 2 + threadIdx.x];
        atomicAdd(grad + OFF_B4 + threadIdx.x, s);
    }
    __syncthreads();
    // dz3 = (dy W4^T) * silu'(z3): fp32 into Z[2], bf16 into H[2]
    for (int e = threadIdx.x; e < TT * MH; e += blockDim.x) {
        const int r = e / MH, k = e % MH;
        const float dh = S.Y[r * 2] * P[OFF_W4 + k * 2] + S.Y[r * 2 + 1] * P[OFF_W4 + k * 2 + 1];
        const float dz = dh * dsilu_f(S.Z[2][r * LDZ + k]);
        S.Z[2][r * LDZ + k] = dz;
        S.H[2][r * LDH + k] = __float2bfloat16(dz);
    }
    __syncthreads();
    // layers 3, 2, 1 backward
    for (int L = 2; L >= 0; L--) {
        const bf16 *Hin = L == 0 ? S.F : S.H[L - 1];
        const int ldin = L == 0 ? LDF : LDH;
        const int fin = L == 0 ? MFIN : MH;
        const int woff = L == 0 ? OFF_W1 : (L == 1 ? OFF_W2 : OFF_W3);
        const int boff = L == 0 ? OFF_B1 : (L == 1 ? OFF_B2 : OFF_B3);
        // dW = Hin^T * dZ  (fin x 128, K = TT)
        if (fin == MH) {
            float acc[4][4][4];
            zero_acc<64, 32>(acc);
            const int wm0 = (warp >> 2) * 64, wn0 = (warp & 3) * 32;
            warp_gemm<64, 32, true, false>(Hin, ldin, S.H[L], LDH, TT, wm0, wn0, acc);
            const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
            for (int mi = 0; mi < 4; mi++)
#pragma unroll
                for (int ni = 0; ni < 4; ni++)
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int r = wm0 + mi * 16 + g + 8 * (e >> 1);
                        const int c = wn0 + ni * 8 + 2 * t + (e & 1);
                        atomicAdd(grad + woff + r * MH + c, acc[mi][ni][e]);
                    }
        } else {
            float acc[1][4][4];
            zero_acc<16, 32>(acc);
            const int wm0 = (warp >> 2) * 16, wn0 = (warp & 3) * 32;
            warp_gemm<16, 32, true, false>(Hin, ldin, S.H[L], LDH, TT, wm0, wn0, acc);
            const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
            for (int ni = 0; ni < 4; ni++)
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int r = wm0 + g + 8 * (e >> 1);
                    const int c = wn0 + ni * 8 + 2 * t + (e & 1);
                    if (r < MNFEAT) atomicAdd(grad + woff + r * MH + c, acc[0][ni][e]);
                }
        }
        // db
        if (threadIdx.x < MH) {
            float s = 0.f;
            for (int r = 0; r < TT; r++) s += S.Z[L][r * LDZ + threadIdx.x];
            atomicAdd(grad + boff + threadIdx.x, s);
        }
        if (L == 0) break;
        // dH_{L-1} = dZ_L * W_L^T, then dZ_{L-1} = dH * silu'(Z_{L-1})
        float acc[2][4][4];
        zero_acc<32, 32>(acc);
        warp_gemm<32, 32, false, true>(S.H[L], LDH, Wb[L], MH, MH, m0, n0, acc);
        __syncthreads();  // everyone is done reading H[L-1] (dW) and H[L] (this GEMM)
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int mi = 0; mi < 2; mi++)
#pragma unroll
            for (int ni = 0; ni < 4; ni++)
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int r = m0 + mi * 16 + g + 8 * h;
                    const int c = n0 + ni * 8 + 2 * t;
                    float *z = S.Z[L - 1] + r * LDZ + c;
                    const float d0 = acc[mi][ni][2 * h] * dsilu_f(z[0]);
                    const float d1 = acc[mi][ni][2 * h + 1] * dsilu_f(z[1]);
                    z[0] = d0;
                    z[1] = d1;
                    *reinterpret_cast<uint32_t *>(S.H[L - 1] + r * LDH + c) =
                        pack_bf16(__float2bfloat16(d0), __float2bfloat16(d1));
                }
        __syncthreads();
    }
}

// Write parameter i into the BF16 copies (transposed and as stored).
__device__ __forceinline__ void store_bf16_copies(bf16 *PB, int i, float p)
{
    const bf16 b = __float2bfloat16(p);
    if (i < OFF_B1) {
        const int k = i / MH, n = i % MH;
        PB[BOFF_W1T + n * MFIN + k] = b;
    } else if (i >= OFF_W2 && i < OFF_B2) {
        const int j = i - OFF_W2, k = j / MH, n = j % MH;
        PB[BOFF_W2T + n * MH + k] = b;
        PB[BOFF_W2 + j] = b;
    } else if (i >= OFF_W3 && i < OFF_B3) {
        const int j = i - OFF_W3, k = j / MH, n = j % MH;
        PB[BOFF_W3T + n * MH + k] = b;
        PB[BOFF_W3 + j] = b;
    }
}

// Adam (Kingma & Ba 2015) with bias correction; refreshes the BF16 copy and
// clears the gradient.
__global__ void mlp_adam_kernel(float *__restrict__ P, bf16 *__restrict__ PB, float *__restrict__ grad,
                                float *__restrict__ m, float *__restrict__ v, float lr, float b1,
                                float b2, float eps, float c1, float c2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x) {
        const float g = grad[i];
        const float mm = b1 * m[i] + (1.f - b1) * g;
        const float vv = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mm;
        v[i] = vv;
        float p = P[i] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
        if (i < OFF_B1 && (i / MH) >= MNFEAT) p = 0.f;  // padded W1 rows stay zero
        P[i] = p;
        grad[i] = 0.f;
        store_bf16_copies(PB, i, p);
    }
}

__global__ void mlp_to_bf16_kernel(const float *__restrict__ P, bf16 *__restrict__ PB)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x)
        store_bf16_copies(PB, i, P[i]);
}

// ---------------------------------------------------------------------------
// inference: 128 rows per pass
// ---------------------------------------------------------------------------
constexpr int IR = 128;

struct InferSmem {
    bf16 F[IR * LDF];
    bf16 H[2][IR * LDH];
    float2 Y[IR];
    float ftab[2][32 * 8];  // per-visibility Fourier terms (learned_scatter)
};

// Rows of S.F -> S.Y (taps / out_scale).  All threads of the block.
__device__ __forceinline__ void mlp_forward_rows(InferSmem &S, const float *__restrict__ P,
                                                 const bf16 *__restrict__ PB)
{
    const int warp = threadIdx.x >> 5;
    const int m0 = (warp >> 2) * 64, n0 = (warp & 3) * 32;
    {
        float acc[4][4][4];
        zero_acc<64, 32>(acc);
        warp_gemm<64, 32, false, true>(S.F, LDF, PB + BOFF_W1T, MFIN, MFIN, m0, n0, acc);
        hidden_epilogue<64, 32, true>(acc, m0, n0, P + OFF_B1, nullptr, S.H[0]);
    }
    __syncthreads();
    {
        float acc[4][4][4];
        zero_acc<64, 32>(acc);
        warp_gemm<64, 32, false, true>(S.H[0], LDH, PB + BOFF_W2T, MH, MH, m0, n0, acc);
        hidden_epilogue<64, 32, true>(acc, m0, n0, P + OFF_B2, nullptr, S.H[1]);
    }
    __syncthreads();
    {
        float acc[4][4][4];
        zero_acc<64, 32>(acc);
        warp_gemm<64, 32, false, true>(S.H[1], LDH, PB + BOFF_W3T, MH, MH, m0, n0, acc);
        hidden_epilogue<64, 32, true>(acc, m0, n0, P + OFF_B3, nullptr, S.H[0]);
    }
    __syncthreads();
    // output layer: two threads per row, half of k each, combined by shuffle
    {
        const int r = threadIdx.x >> 1, half = threadIdx.x & 1;
        float y0 = 0.f, y1 = 0.f;
        const bf16 *h = S.H[0] + r * LDH + half * 64;
        const float *w4 = P + OFF_W4 + half * 64 * 2;
#pragma unroll 8
        for (int k = 0; k < 64; k++) {
            const float hv = __bfloat162float(h[k]);
            y0 = fmaf(hv, w4[2 * k], y0);
            y1 = fmaf(hv, w4[2 * k + 1], y1);
        }
        y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
        y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
        if (half == 0) S.Y[r] = make_float2(y0 + P[OFF_B4], y1 + P[OFF_B4 + 1]);
    }
    __syncthreads();
}

// Evaluate taps at arbitrary inputs: in [5][n] -> out float2 (scaled taps).
__global__ void __launch_bounds__(256) mlp_eval_kernel(const float *__restrict__ P, const bf16 *__restrict__ PB,
                                                       const float *__restrict__ in, int n, int ksize,
                                                       float inv_wmax, float scale, float2 *__restrict__ out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InferSmem &S = *reinterpret_cast<InferSmem *>(smem_raw);
    for (int base = blockIdx.x * IR; base < n; base += gridDim.x * IR) {
        if (threadIdx.x < IR) {
            const int i = base + threadIdx.x;
            if (i < n) tap_features(in[i], in[n + i], in[2 * n + i], in[3 * n + i], in[4 * n + i], ksize,
                                    inv_wmax, S.F + threadIdx.x * LDF);
            else
                for (int k = 0; k < MFIN; k++) S.F[threadIdx.x * LDF + k] = __float2bfloat16(0.f);
        }
        __syncthreads();
        mlp_forward_rows(S, P, PB);
        if (threadIdx.x < IR && base + threadIdx.x < n) {
            const float2 y = S.Y[threadIdx.x];
            out[base + threadIdx.x] = make_float2(y.x * scale, y.y * scale);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// W-projection with learned taps.  Per visibility: x = theta u, cell =
// floor(x), du = x - cell (continuous — no oversampling quantisation);
// footprint column cell - K/2 + tx; taps from the network at (w, du, dv, tx,
// ty); grid[idx] += vis * conj(tap) with the reference's linear index rule
// (dropped outside [0, N^2)).  K = 16: two 128-row passes per visibility.
// ---------------------------------------------------------------------------
// One visibility: taps from the network in passes of IR rows, each scattered
// as grid[goff + ty*ld + tx] += vis * conj(tap) where the index lies in
// [0, limit).  All threads of the CTA take part (barriers inside).
__device__ __forceinline__ void learned_scatter(InferSmem &S, const float *__restrict__ P,
                                                const bf16 *__restrict__ PB, float wf, float du, float dv,
                                                float vr, float vi, float2 *grid, int64_t goff, int64_t ld,
                                                int64_t limit, int ksize, float inv_wmax, float scale,
                                                int strip_lg = 0)
{
    const int taps = ksize * ksize;
    if (threadIdx.x < ksize) axis_table(du, threadIdx.x, ksize, S.ftab[0]);
    else if (threadIdx.x >= 32 && threadIdx.x < 32 + ksize) axis_table(dv, threadIdx.x - 32, ksize, S.ftab[1]);
    __syncthreads();
    for (int t0 = 0; t0 < taps; t0 += IR) {
        if (threadIdx.x < IR) {
            const int t = t0 + threadIdx.x;
            if (t < taps)
                tap_features_tab(wf, du, dv, t % ksize, t / ksize, ksize, inv_wmax, S.ftab[0], S.ftab[1],
                                 S.F + threadIdx.x * LDF);
            else
                for (int k = 0; k < MFIN; k++) S.F[threadIdx.x * LDF + k] = __float2bfloat16(0.f);
        }
        __syncthreads();
        mlp_forward_rows(S, P, PB);
        if (threadIdx.x < IR) {
            const int t = t0 + threadIdx.x;
            const float2 k = S.Y[threadIdx.x];
            const float kr = k.x * scale, ki = k.y * scale;
            const int64_t idx = goff + (int64_t)(t / ksize) * ld + (t % ksize);
            if (t < taps && idx >= 0 && idx < limit)
                atomicAdd(grid + (strip_lg ? (int64_t)strip_addr((int)idx, strip_lg) : idx),
                          make_float2(vr * kr + vi * ki, vi * kr - vr * ki));
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) learned_wproj_kernel(
    const double *__restrict__ u, const double *__restrict__ v, const double *__restrict__ w,
    const double2 *__restrict__ vis, int64_t nvis, int N, double theta, const float *__restrict__ P,
    const bf16 *__restrict__ PB, int ksize, float inv_wmax, float scale, float2 *__restrict__ grid)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InferSmem &S = *reinterpret_cast<InferSmem *>(smem_raw);
    for (int64_t i = blockIdx.x; i < nvis; i += gridDim.x) {
        const double x = theta * u[i], y = theta * v[i];
        const double cx = floor(x), cy = floor(y);
        const double2 vz = vis[i];
        const int64_t goff = ((int64_t)cy - ksize / 2 + N / 2) * N + ((int64_t)cx - ksize / 2 + N / 2);
        learned_scatter(S, P, PB, (float)w[i], (float)(x - cx), (float)(y - cy), (float)vz.x, (float)vz.y, grid,
                        goff, N, (int64_t)N * N, ksize, inv_wmax, scale);
    }
}

// ---------------------------------------------------------------------------
// W-towers with learned taps: the records of the tower binning (sub-grid slot
// via slot_of_bin, footprint origin in the sub-grid) and the continuous
// offsets feat = {w - w_mid, du, dv}; same scatter as above into the slot's
// S x S sub-grid.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) learned_towers_kernel(
    const int4 *__restrict__ rec, const float2 *__restrict__ visf, const float4 *__restrict__ feat, int64_t nvis,
    const int *__restrict__ slot_of_bin, int slot_cap, float2 *__restrict__ slots, int sub,
    const float *__restrict__ P, const bf16 *__restrict__ PB, int ksize, float inv_wmax, float scale)
{
    const int strip_lg = __ffs(sub) - 1;  // sub-grids are strip-major (strip_addr)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InferSmem &S = *reinterpret_cast<InferSmem *>(smem_raw);
    const int64_t cells = (int64_t)sub * sub;
    for (int64_t i = blockIdx.x; i < nvis; i += gridDim.x) {
        const int4 r = rec[i];
        if (r.x < 0) continue;  // uniform across the CTA
        const int slot = slot_of_bin[r.x];
        if (slot >= slot_cap) continue;
        const float4 f = feat[i];
        const float2 vz = visf[i];
        learned_scatter(S, P, PB, f.x, f.y, f.z, vz.x, vz.y, slots + (int64_t)slot * cells, r.y, sub, cells, ksize,
                        inv_wmax, scale, strip_lg);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_mlp_grad(cudaStream_t s, const float *P, const void *PB, const float *in, const float2 *target,
                     int n, int ksize, float inv_wmax, float inv_scale, float *grad, float *loss)
{
    const size_t sm = sizeof(TrainSmem);
    cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    mlp_grad_kernel<<<(n + TT - 1) / TT, 256, sm, s>>>(P, (const bf16 *)PB, in, target, n, ksize, inv_wmax,
                                                       inv_scale, grad, loss);
}

void launch_mlp_adam(cudaStream_t s, float *P, void *PB, float *grad, float *m, float *v, float lr, int step)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    mlp_adam_kernel<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(P, (bf16 *)PB, grad, m, v, lr, b1, b2, 1e-8f, c1, c2);
}

void launch_mlp_to_bf16(cudaStream_t s, const float *P, void *PB)
{
    mlp_to_bf16_kernel<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(P, (bf16 *)PB);
}

void launch_mlp_eval(cudaStream_t s, const float *P, const void *PB, const float *in, int n, int ksize,
                     float inv_wmax, float scale, float2 *out, int sm_count)
{
    const size_t sm = sizeof(InferSmem);
    cudaFuncSetAttribute(mlp_eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int blocks = (n + IR - 1) / IR;
    if (blocks > sm_count * 4) blocks = sm_count * 4;
    if (blocks < 1) blocks = 1;
    mlp_eval_kernel<<<blocks, 256, sm, s>>>(P, (const bf16 *)PB, in, n, ksize, inv_wmax, scale, out);
}

void launch_learned_towers(cudaStream_t s, const int4 *rec, const float2 *visf, const float4 *feat, int64_t n,
                           const int *slot_of_bin, int slot_cap, float2 *slots, int subgrid, const float *P,
                           const void *PB, int ksize, float inv_wmax, float scale, int sm_count)
{
    const size_t sm = sizeof(InferSmem);
    cudaFuncSetAttribute(learned_towers_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int64_t blocks = n < (int64_t)sm_count * 4 ? n : (int64_t)sm_count * 4;
    if (blocks < 1) blocks = 1;
    learned_towers_kernel<<<(unsigned)blocks, 256, sm, s>>>(rec, visf, feat, n, slot_of_bin, slot_cap, slots, subgrid,
                                                            P, (const bf16 *)PB, ksize, inv_wmax, scale);
}

void launch_learned_wproj(cudaStream_t s, const double *u, const double *v, const double *w,
                          const double2 *vis, int64_t n, int N, double theta, const float *P, const void *PB,
                          int ksize, float inv_wmax, float scale, float2 *grid, int sm_count)
{
    const size_t sm = sizeof(InferSmem);
    cudaFuncSetAttribute(learned_wproj_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int64_t blocks = n < (int64_t)sm_count * 4 ? n : (int64_t)sm_count * 4;
    if (blocks < 1) blocks = 1;
    learned_wproj_kernel<<<(unsigned)blocks, 256, sm, s>>>(u, v, w, vis, n, N, theta, P, (const bf16 *)PB,
                                                           ksize, inv_wmax, scale, grid);
}

}  // namespace rg
