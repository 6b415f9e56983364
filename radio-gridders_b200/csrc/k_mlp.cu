// Learned w-kernel: a small MLP evaluated on tensor cores.
//
// Network (no counterpart in the reference; the reference reads quantised,
// oversampled w-kernel tables, src/reference/grid.c:157-185): 21 input features
// of a tap (w, sub-cell offsets du, dv, tap x, tap y and 16 Fourier features of
// the tap's offset from the visibility) -> 128 -> 128 -> 128 (SiLU) -> 2
// (complex tap / out_scale).  Layers 1-3 are tensor-core products with FP32
// accumulation: in inference (evaluation and both gridders) FP16 tcgen05 MMAs
// with TMEM accumulators, in training BF16 mma.sync.m16n8k16 tiles (the
// backward pass needs the activations and gradients in registers and shared
// memory anyway); the 128 -> 2 output layer is FP32.
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
#include <cuda_fp16.h>

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
__device__ __forceinline__ float dsilu_f(float z)
{
    const float s = 1.f / (1.f + __expf(-z));
    return s * (1.f + z * (1.f - s));
}

// A feature or activation as the tensor cores' element type: BF16 in
// training, FP16 in inference.
template <class T> __device__ __forceinline__ T to_elem(float x);
template <> __device__ __forceinline__ bf16 to_elem<bf16>(float x) { return __float2bfloat16(x); }
template <> __device__ __forceinline__ __half to_elem<__half>(float x) { return __float2half_rn(x); }

// Features of one tap (the definition in oracle/mlp_oracle.py).
template <class T>
__device__ __forceinline__ void tap_features(float w, float du, float dv, float tx, float ty, int ksize,
                                             float inv_wmax, T *f)
{
    const float half = 0.5f * (float)ksize;
    const float p = tx - half - du, q = ty - half - dv;
    const float inv = 1.f / (half + 1.f);
    f[0] = to_elem<T>(w * inv_wmax);
    f[1] = to_elem<T>(2.f * du - 1.f);
    f[2] = to_elem<T>(2.f * dv - 1.f);
    f[3] = to_elem<T>(p / half);
    f[4] = to_elem<T>(q / half);
#pragma unroll
    for (int k = 1; k <= 4; k++) {
        float s, c;
        sincospif((float)k * p * inv, &s, &c);
        f[5 + 2 * (k - 1)] = to_elem<T>(c);
        f[6 + 2 * (k - 1)] = to_elem<T>(s);
        sincospif((float)k * q * inv, &s, &c);
        f[13 + 2 * (k - 1)] = to_elem<T>(c);
        f[14 + 2 * (k - 1)] = to_elem<T>(s);
    }
#pragma unroll
    for (int k = MNFEAT; k < MFIN; k++) f[k] = to_elem<T>(0.f);
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

template <class T>
__device__ __forceinline__ void tap_features_tab(float w, float du, float dv, int tx, int ty, int ksize,
                                                 float inv_wmax, const float *ptab, const float *qtab, T *f)
{
    const float half = 0.5f * (float)ksize;
    const float p = (float)tx - half - du, q = (float)ty - half - dv;
    f[0] = to_elem<T>(w * inv_wmax);
    f[1] = to_elem<T>(2.f * du - 1.f);
    f[2] = to_elem<T>(2.f * dv - 1.f);
    f[3] = to_elem<T>(p / half);
    f[4] = to_elem<T>(q / half);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        f[5 + j] = to_elem<T>(ptab[tx * 8 + j]);
        f[13 + j] = to_elem<T>(qtab[ty * 8 + j]);
    }
#pragma unroll
    for (int k = MNFEAT; k < MFIN; k++) f[k] = to_elem<T>(0.f);
}

// Epilogue of a 32x32 (per warp) hidden-layer tile: z = acc + b; Z (fp32,
// optional) and H = bf16(silu(z)).
template <int WM, int WN>
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
                *reinterpret_cast<uint32_t *>(Hout + r * LDH + c) =
                    pack_bf16(__float2bfloat16(silu_f(z0)), __float2bfloat16(silu_f(z1)));
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
// Inference on the 5th-generation tensor cores (tcgen05).  Rows (taps) go in
// tiles of 128; each hidden layer is an M = 128, N = 128 FP16 x FP16 -> FP32
// product issued as K = 16 steps by one thread from shared-memory operands
// into an accumulator in tensor memory (TMEM), and its epilogue (bias, SiLU,
// FP16 pack back into shared memory as the next layer's A operand) is done by
// the tile's 128 threads, each owning one TMEM lane (row).  The 128 -> 2
// output layer runs in FP32 in the last epilogue.
//
// Inference computes in FP16 where training used BF16.  The weights are the
// BF16-rounded ones the training forward pass used (converted exactly): the
// network was fitted through those, and the unrounded FP32 master weights are
// a slightly different function whose error is systematic across taps.
// Features and activations are FP16 (11-bit instead of 8-bit mantissas), and
// the SiLU runs on packed pairs — one f32 -> f16x2 conversion and one
// tanh.approx.f16x2 per two activations, half the transcendental-unit work of
// the BF16 form.
//
// A CTA (one per SM) holds one copy of W1..W3 (72 KB) and runs TC_GROUPS
// independent tile groups of four warps, each with its own feature / hidden
// buffers, mbarrier and 128 TMEM columns: while one group's epilogue runs on
// the CUDA cores, another group's MMAs run on the tensor core.
//
// Operands use the K-major layout without swizzle: 8-row x 16-byte core
// matrices, rows 16 bytes apart, the two core matrices of a K = 16 step
// 128 bytes apart (leading byte offset), 8-row groups K * 16 bytes apart
// (stride byte offset).
// ---------------------------------------------------------------------------
constexpr int IR = 128;  // rows per tile
constexpr int TC_GROUPS = 4;
constexpr int TC_THREADS = TC_GROUPS * IR;
constexpr int TC_KMAX = 16;  // largest kernel support (feature tables)

__host__ __device__ constexpr int core_off(int row, int k, int K)
{
    return (row >> 3) * (K * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

struct TcSmem {
    alignas(16) unsigned char W1[MH * MFIN * 2];  // B operands: W^T [out][in], K-major, FP16
    alignas(16) unsigned char W2[MH * MH * 2];
    alignas(16) unsigned char W3[MH * MH * 2];
    // A of layers 2, 3 (activations); its first IR * MFIN * 2 bytes are also
    // layer 1's A (features): layer 1's MMA has completed before its epilogue
    // writes activations, and the next tile's features are stored after the
    // layer-3 MMA (the last reader of the activations) has completed.
    alignas(16) unsigned char H[TC_GROUPS][IR * MH * 2];
    float hb[3][MH];                                         // b1..b3 / 2
    float2 w4[MH];
    float ftab[TC_GROUPS][2][TC_KMAX * 8];  // per-visibility Fourier terms
    unsigned long long bar[TC_GROUPS];
    int abort_flag[TC_GROUPS];
    uint32_t tmem_base;
};
static_assert(sizeof(TcSmem) <= 227 * 1024, "tensor-core inference shared memory");

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), descriptor version 1, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and B
// FP16 (bits 7-9, 10-12 = 0), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t kIdescF16 = (1u << 4) | ((uint32_t)(MH >> 3) << 17) | ((uint32_t)(IR >> 4) << 24);

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(kIdescF16), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void group_sync(int g)
{
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(IR) : "memory");
}

// Bounded wait for the completion of the mbarrier phase with this parity
// (by default 2^32 SM clocks, about two seconds); false when it did not
// complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit = 1ll << 32)
{
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// 32 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: the
// warp reads lanes 32 (warp % 4) .. + 31).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
          "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
          "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}
// Wait for this thread's TMEM loads; v is tied to the wait so that no use of
// the loaded registers is scheduled before it.
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&v)[32])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]),
                   "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]),
                   "+r"(v[14]), "+r"(v[15]), "+r"(v[16]), "+r"(v[17]), "+r"(v[18]), "+r"(v[19]), "+r"(v[20]),
                   "+r"(v[21]), "+r"(v[22]), "+r"(v[23]), "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]),
                   "+r"(v[28]), "+r"(v[29]), "+r"(v[30]), "+r"(v[31])
                 :
                 : "memory");
}

// The MH accumulator columns of this thread's TMEM lane in chunks of 32:
// fn(c, v) for chunk c, with chunk c + 1 loading while chunk c is processed.
template <class Fn>
__device__ __forceinline__ void tmem_row_chunks(uint32_t taddr, Fn &&fn)
{
    static_assert(MH == 128, "four chunks of 32 columns");
    uint32_t a[32], b[32];
    tmem_ld32(taddr, a);
    tmem_wait_ld(a);
    tmem_ld32(taddr + 32, b);
    fn(0, a);
    tmem_wait_ld(b);
    tmem_ld32(taddr + 64, a);
    fn(1, b);
    tmem_wait_ld(a);
    tmem_ld32(taddr + 96, b);
    fn(2, a);
    tmem_wait_ld(b);
    fn(3, b);
}

// SiLU of a pair from the half pre-activations hz = z / 2:
// z sigmoid(z) = hz (1 + tanh hz), in FP16 with the hardware tanh
// approximation (relative error ~2^-11, the FP16 rounding of its result).
__device__ __forceinline__ uint32_t silu2_half(float hz0, float hz1)
{
    const __half2 h = __floats2half2_rn(hz0, hz1);
    uint32_t hu = *reinterpret_cast<const uint32_t *>(&h), t;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(hu));
    const __half2 r = __hfma2(h, *reinterpret_cast<const __half2 *>(&t), h);
    return *reinterpret_cast<const uint32_t *>(&r);
}

// One 16-byte core-matrix row of W^T in FP16: W^T[n][k0 .. k0+7] of the BF16
// copy (transposed, K columns), converted exactly.
__device__ __forceinline__ void stage_wt(unsigned char *dst, const bf16 *__restrict__ WT, int n, int k0, int K)
{
    const uint4 in = *reinterpret_cast<const uint4 *>(WT + n * K + k0);
    const uint32_t w[4] = {in.x, in.y, in.z, in.w};
    uint32_t q[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const __half2 h = __floats2half2_rn(__uint_as_float(w[j] << 16), __uint_as_float(w[j] & 0xFFFF0000u));
        q[j] = *reinterpret_cast<const uint32_t *>(&h);
    }
    *reinterpret_cast<uint4 *>(dst + core_off(n, k0, K)) = make_uint4(q[0], q[1], q[2], q[3]);
}

// CTA prologue: weights into the core-matrix layout, biases, mbarriers and
// TMEM columns (warp 0 allocates TC_GROUPS * 128 columns).
__device__ __forceinline__ void tc_prologue(TcSmem &S, const float *__restrict__ P, const bf16 *__restrict__ PB)
{
    for (int c = threadIdx.x; c < MH * (MFIN / 8); c += blockDim.x)
        stage_wt(S.W1, PB + BOFF_W1T, c / (MFIN / 8), (c % (MFIN / 8)) * 8, MFIN);
    for (int c = threadIdx.x; c < MH * (MH / 8); c += blockDim.x) {
        stage_wt(S.W2, PB + BOFF_W2T, c / (MH / 8), (c % (MH / 8)) * 8, MH);
        stage_wt(S.W3, PB + BOFF_W3T, c / (MH / 8), (c % (MH / 8)) * 8, MH);
    }
    for (int n = threadIdx.x; n < MH; n += blockDim.x) {
        S.hb[0][n] = 0.5f * P[OFF_B1 + n];
        S.hb[1][n] = 0.5f * P[OFF_B2 + n];
        S.hb[2][n] = 0.5f * P[OFF_B3 + n];
        S.w4[n] = make_float2(P[OFF_W4 + 2 * n], P[OFF_W4 + 2 * n + 1]);
    }
    if (threadIdx.x < TC_GROUPS) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar[threadIdx.x])) : "memory");
        S.abort_flag[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (threadIdx.x < 32) {
        constexpr uint32_t cols = TC_GROUPS * IR <= 256 ? 256 : 512;
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&S.tmem_base)),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

__device__ __forceinline__ void tc_epilogue(TcSmem &S)
{
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc_fence_after();
        constexpr uint32_t cols = TC_GROUPS * IR <= 256 ? 256 : 512;
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem_base), "r"(cols)
                     : "memory");
    }
}

// Row r of a tile: features into the group's A buffer (core layout, K = 32).
__device__ __forceinline__ void tc_store_features(unsigned char *F, int r, const __half (&f)[MFIN])
{
#pragma unroll
    for (int j = 0; j < MFIN / 8; j++)
        *reinterpret_cast<uint4 *>(F + core_off(r, 8 * j, MFIN)) = *reinterpret_cast<const uint4 *>(f + 8 * j);
}

// Issue one hidden layer (K / 16 MMA steps) and commit it to the group's
// mbarrier.  One thread.
__device__ __forceinline__ void tc_issue_layer(uint32_t d_tmem, const unsigned char *A, const unsigned char *B, int K,
                                               uint32_t bar)
{
    tc_fence_after();
    const uint32_t a = smem_u32(A), b = smem_u32(B);
    for (int s = 0; s < K / 16; s++)
        umma_f16(d_tmem, umma_desc(a + s * 256, 128, K * 16), umma_desc(b + s * 256, 128, K * 16), s > 0);
    umma_commit(bar);
}

// Hidden epilogue of row r: TMEM accumulator -> SiLU(z + b) as FP16 into H.
__device__ __forceinline__ void tc_hidden_epilogue(uint32_t taddr, const float *__restrict__ hb, unsigned char *H,
                                                   int r)
{
    tmem_row_chunks(taddr, [&](int c, const uint32_t(&v)[32]) {
        uint32_t pk[16];
#pragma unroll
        for (int j = 0; j < 16; j++)
            pk[j] = silu2_half(fmaf(__uint_as_float(v[2 * j]), 0.5f, hb[c * 32 + 2 * j]),
                               fmaf(__uint_as_float(v[2 * j + 1]), 0.5f, hb[c * 32 + 2 * j + 1]));
#pragma unroll
        for (int j = 0; j < 4; j++)
            *reinterpret_cast<uint4 *>(H + core_off(r, c * 32 + 8 * j, MH)) =
                make_uint4(pk[4 * j], pk[4 * j + 1], pk[4 * j + 2], pk[4 * j + 3]);
    });
}

// Output epilogue of row r: SiLU(z + b3) (FP16 pairs), times W4, plus b4.
__device__ __forceinline__ float2 tc_output_epilogue(uint32_t taddr, const float *__restrict__ hb,
                                                     const float2 *__restrict__ w4, float2 b4)
{
    float y0 = b4.x, y1 = b4.y;
    tmem_row_chunks(taddr, [&](int c, const uint32_t(&v)[32]) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint32_t hp = silu2_half(fmaf(__uint_as_float(v[2 * j]), 0.5f, hb[c * 32 + 2 * j]),
                                           fmaf(__uint_as_float(v[2 * j + 1]), 0.5f, hb[c * 32 + 2 * j + 1]));
            const float2 h = __half22float2(*reinterpret_cast<const __half2 *>(&hp));
            const float2 wa = w4[c * 32 + 2 * j], wb = w4[c * 32 + 2 * j + 1];
            y0 = fmaf(h.x, wa.x, fmaf(h.y, wb.x, y0));
            y1 = fmaf(h.x, wa.y, fmaf(h.y, wb.y, y1));
        }
    });
    return make_float2(y0, y1);
}

// The network on the 128 feature rows the group has just stored in S.H[g]:
// returns row r's output (tap / out_scale).  All threads of group g.  On a
// wait that timed out the error word gets DERR_TIMEOUT and *ok turns false
// for the whole group (read after a group barrier).
__device__ __forceinline__ float2 tc_tile(TcSmem &S, int g, int r, uint32_t &phase, float2 b4,
                                          unsigned *__restrict__ err, bool *ok)
{
    const uint32_t bar = smem_u32(&S.bar[g]);
    const uint32_t d_tmem = S.tmem_base + (uint32_t)(g * IR);
    const uint32_t taddr = d_tmem + ((uint32_t)((r >> 5) * 32) << 16);
    float2 y = make_float2(0.f, 0.f);
    fence_async_smem();
    tc_fence_before();
    group_sync(g);
    if (S.abort_flag[g]) {
        *ok = false;
        return y;
    }
#pragma unroll 1
    for (int layer = 0; layer < 3; layer++) {
        if (r == 0) {
            if (layer == 0) tc_issue_layer(d_tmem, S.H[g], S.W1, MFIN, bar);
            else tc_issue_layer(d_tmem, S.H[g], layer == 1 ? S.W2 : S.W3, MH, bar);
        }
        if (!mbar_wait(bar, phase)) {
            S.abort_flag[g] = 1;
            atomicOr(err, DERR_TIMEOUT);
        }
        phase ^= 1u;
        tc_fence_after();
        if (layer < 2) {
            tc_hidden_epilogue(taddr, S.hb[layer], S.H[g], r);
            fence_async_smem();
            tc_fence_before();
            group_sync(g);
            if (S.abort_flag[g]) {
                *ok = false;
                return y;
            }
        } else {
            y = tc_output_epilogue(taddr, S.hb[2], S.w4, b4);
        }
    }
    return y;
}

// Evaluate taps at arbitrary inputs: in [5][n] -> out float2 (scaled taps).
__global__ void __launch_bounds__(TC_THREADS, 1) mlp_eval_kernel(const float *__restrict__ P,
                                                                  const bf16 *__restrict__ PB,
                                                                  const float *__restrict__ in, int n, int ksize,
                                                                  float inv_wmax, float scale,
                                                                  float2 *__restrict__ out, unsigned *err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TcSmem &S = *reinterpret_cast<TcSmem *>(smem_raw);
    tc_prologue(S, P, PB);
    const int g = threadIdx.x / IR, r = threadIdx.x % IR;
    const float2 b4 = make_float2(P[OFF_B4], P[OFF_B4 + 1]);
    uint32_t phase = 0;
    bool ok = true;
    for (int base = (blockIdx.x * TC_GROUPS + g) * IR; base < n && ok; base += gridDim.x * TC_GROUPS * IR) {
        const int i = base + r;
        __align__(16) __half f[MFIN];
        if (i < n) tap_features(in[i], in[n + i], in[2 * n + i], in[3 * n + i], in[4 * n + i], ksize, inv_wmax, f);
        else
            for (int k = 0; k < MFIN; k++) f[k] = __float2half_rn(0.f);
        tc_store_features(S.H[g], r, f);
        const float2 y = tc_tile(S, g, r, phase, b4, err, &ok);
        if (ok && i < n) out[i] = make_float2(y.x * scale, y.y * scale);
    }
    tc_epilogue(S);
}

// ---------------------------------------------------------------------------
// Gridding with learned taps.  A visibility's K x K taps are K*K / 128 tiles
// (one half-filled tile for K = 8); tap t = ty * K + tx of the tile row is
// scattered as grid[goff + ty * ld + tx] += vis * conj(tap) where that index
// lies in [0, limit) — or, when axes is set, where column col0 + tx and row
// row0 + ty both lie in [0, ld).  The groups of a CTA take visibilities in
// turn.
// ---------------------------------------------------------------------------
struct LearnedVis {
    float wf, du, dv, vr, vi;
    float2 *grid;
    int64_t goff, ld, limit;
    int col0, row0;
    bool axes;
};

// W-projection: x = theta u, cell = floor(x), du = x - cell (continuous — no
// oversampling quantisation); footprint column cell - K/2 + tx; taps whose
// column or row leaves the grid are dropped (the reference GPU gridder's
// per-axis check, src/grid/grid_cuda.cu:25-41).
struct WprojVisSource {
    const double *u, *v, *w;
    const double2 *vis;
    int N, ksize;
    double theta;
    float2 *grid;
    __device__ bool get(int64_t i, LearnedVis &o) const
    {
        const double x = theta * u[i], y = theta * v[i];
        const double cx = floor(x), cy = floor(y);
        const double2 vz = vis[i];
        o.goff = ((int64_t)cy - ksize / 2 + N / 2) * N + ((int64_t)cx - ksize / 2 + N / 2);
        o.wf = (float)w[i];
        o.du = (float)(x - cx);
        o.dv = (float)(y - cy);
        o.vr = (float)vz.x;
        o.vi = (float)vz.y;
        o.grid = grid;
        o.ld = N;
        o.limit = (int64_t)N * N;
        o.col0 = (int)cx - ksize / 2 + N / 2;
        o.row0 = (int)cy - ksize / 2 + N / 2;
        o.axes = true;
        return true;
    }
};

// W-towers: the records of the tower binning (sub-grid slot via slot_of_bin,
// footprint origin in the sub-grid) and the continuous offsets
// feat = {w - w_mid, du, dv}; scattered into the slot's strip-major S x S
// sub-grid.
struct TowersVisSource {
    const int4 *rec;
    const float2 *visf;
    const float4 *feat;
    const int *slot_of_bin;
    int slot_cap, sub;
    float2 *slots;
    __device__ bool get(int64_t i, LearnedVis &o) const
    {
        const int4 r = rec[i];
        if (r.x < 0) return false;
        const int slot = slot_of_bin[r.x];
        if (slot >= slot_cap) return false;
        const float4 f = feat[i];
        const float2 vz = visf[i];
        o.wf = f.x;
        o.du = f.y;
        o.dv = f.z;
        o.vr = vz.x;
        o.vi = vz.y;
        o.grid = slots + (int64_t)slot * sub * sub;
        o.goff = r.y;
        o.ld = sub;
        o.limit = (int64_t)sub * sub;
        o.col0 = o.row0 = 0;
        o.axes = false;
        return true;
    }
};

template <class Src>
__global__ void __launch_bounds__(TC_THREADS, 1) learned_grid_kernel(Src src, int64_t nvis, const float *__restrict__ P,
                                                                      const bf16 *__restrict__ PB, int ksize,
                                                                      float inv_wmax, float scale, int strip_lg,
                                                                      unsigned *err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TcSmem &S = *reinterpret_cast<TcSmem *>(smem_raw);
    tc_prologue(S, P, PB);
    const int g = threadIdx.x / IR, r = threadIdx.x % IR;
    const float2 b4 = make_float2(P[OFF_B4], P[OFF_B4 + 1]);
    const int taps = ksize * ksize;
    uint32_t phase = 0;
    bool ok = true;
    for (int64_t i = (int64_t)blockIdx.x * TC_GROUPS + g; i < nvis && ok; i += (int64_t)gridDim.x * TC_GROUPS) {
        LearnedVis o;
        if (!src.get(i, o)) continue;  // uniform across the group
        // the previous visibility's last tile read the tables before its barriers
        if (r < ksize) axis_table(o.du, r, ksize, S.ftab[g][0]);
        else if (r >= 32 && r < 32 + ksize) axis_table(o.dv, r - 32, ksize, S.ftab[g][1]);
        group_sync(g);
        for (int t0 = 0; t0 < taps && ok; t0 += IR) {
            const int t = t0 + r;
            __align__(16) __half f[MFIN];
            if (t < taps)
                tap_features_tab(o.wf, o.du, o.dv, t % ksize, t / ksize, ksize, inv_wmax, S.ftab[g][0],
                                 S.ftab[g][1], f);
            else
                for (int k = 0; k < MFIN; k++) f[k] = __float2half_rn(0.f);
            tc_store_features(S.H[g], r, f);
            const float2 y = tc_tile(S, g, r, phase, b4, err, &ok);
            const float kr = y.x * scale, ki = y.y * scale;
            const int64_t idx = o.goff + (int64_t)(t / ksize) * o.ld + (t % ksize);
            const bool inside = o.axes ? ((unsigned)(o.col0 + t % ksize) < (unsigned)o.ld &&
                                          (unsigned)(o.row0 + t / ksize) < (unsigned)o.ld)
                                       : (idx >= 0 && idx < o.limit);
            if (ok && t < taps && inside)
                atomicAdd(o.grid + (strip_lg ? (int64_t)strip_addr((int)idx, strip_lg) : idx),
                          make_float2(o.vr * kr + o.vi * ki, o.vi * kr - o.vr * ki));
        }
    }
    tc_epilogue(S);
}

// Self-test of the bounded wait: one CTA waits on an mbarrier that nothing
// arrives on, for `limit` SM clocks, and reports DERR_TIMEOUT like the
// inference kernels do.
__global__ void mbar_timeout_probe_kernel(unsigned *err, long long limit)
{
    __shared__ unsigned long long bar;
    if (threadIdx.x == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)) : "memory");
    __syncthreads();
    if (!mbar_wait(smem_u32(&bar), 0, limit)) atomicOr(err, DERR_TIMEOUT);
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

void launch_mbar_timeout_probe(cudaStream_t s, unsigned *err, long long limit)
{
    mbar_timeout_probe_kernel<<<1, 64, 0, s>>>(err, limit);
}

static int tc_blocks(int64_t groups_of_work, int sm_count)
{
    int64_t b = (groups_of_work + TC_GROUPS - 1) / TC_GROUPS;
    if (b > sm_count) b = sm_count;
    return b < 1 ? 1 : (int)b;
}

void launch_mlp_eval(cudaStream_t s, const float *P, const void *PB, const float *in, int n, int ksize,
                     float inv_wmax, float scale, float2 *out, int sm_count, unsigned *err)
{
    const size_t sm = sizeof(TcSmem);
    cudaFuncSetAttribute(mlp_eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    mlp_eval_kernel<<<tc_blocks((n + IR - 1) / IR, sm_count), TC_THREADS, sm, s>>>(P, (const bf16 *)PB, in, n, ksize,
                                                                                  inv_wmax, scale, out, err);
}

void launch_learned_towers(cudaStream_t s, const int4 *rec, const float2 *visf, const float4 *feat, int64_t n,
                           const int *slot_of_bin, int slot_cap, float2 *slots, int subgrid, const float *P,
                           const void *PB, int ksize, float inv_wmax, float scale, int sm_count, unsigned *err)
{
    const size_t sm = sizeof(TcSmem);
    auto kern = learned_grid_kernel<TowersVisSource>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    TowersVisSource src{rec, visf, feat, slot_of_bin, slot_cap, subgrid, slots};
    int strip_lg = 0;
    while ((1 << strip_lg) < subgrid) strip_lg++;  // sub-grids are strip-major (strip_addr)
    kern<<<tc_blocks(n, sm_count), TC_THREADS, sm, s>>>(src, n, P, (const bf16 *)PB, ksize, inv_wmax, scale,
                                                        strip_lg, err);
}

void launch_learned_wproj(cudaStream_t s, const double *u, const double *v, const double *w,
                          const double2 *vis, int64_t n, int N, double theta, const float *P, const void *PB,
                          int ksize, float inv_wmax, float scale, float2 *grid, int sm_count, unsigned *err)
{
    const size_t sm = sizeof(TcSmem);
    auto kern = learned_grid_kernel<WprojVisSource>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    WprojVisSource src{u, v, w, vis, N, ksize, theta, grid};
    kern<<<tc_blocks(n, sm_count), TC_THREADS, sm, s>>>(src, n, P, (const bf16 *)PB, ksize, inv_wmax, scale, 0, err);
}

}  // namespace rg
