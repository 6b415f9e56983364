// Device building blocks for the project's own FFTs (FP32 complex).
//
// A length-N transform, N = N1 * 32, is computed in four steps (Bailey's
// four-step method): 32-point transforms in registers over the stride-N1
// subsequences, a twiddle multiply W_N^(n1 k2), an exchange through shared
// memory, and N1-point transforms in registers.  Register transforms are
// radix-2 decimation-in-frequency with compile-time indices, so all data stays
// in registers; outputs come out in bit-reversed order and are stored to their
// natural positions.  Twiddles are FP64-computed values rounded to FP32.
#pragma once

#include <cuda_runtime.h>

namespace rg {

// exp(-2 pi i k / 32), k = 0..15, as FP32 literals (cos/sin evaluated in
// FP64 and rounded).  Called with compile-time k only, so it folds to
// immediates.
__device__ __forceinline__ float2 tw32(int k)
{
    switch (k) {
        case 0: return make_float2(1.0f, -0.0f);
        case 1: return make_float2(0.9807852506637573f, -0.19509032368659973f);
        case 2: return make_float2(0.9238795042037964f, -0.3826834261417389f);
        case 3: return make_float2(0.8314695954322815f, -0.5555702447891235f);
        case 4: return make_float2(0.7071067690849304f, -0.7071067690849304f);
        case 5: return make_float2(0.5555702447891235f, -0.8314695954322815f);
        case 6: return make_float2(0.3826834261417389f, -0.9238795042037964f);
        case 7: return make_float2(0.19509032368659973f, -0.9807852506637573f);
        case 8: return make_float2(6.123234262925839e-17f, -1.0f);
        case 9: return make_float2(-0.19509032368659973f, -0.9807852506637573f);
        case 10: return make_float2(-0.3826834261417389f, -0.9238795042037964f);
        case 11: return make_float2(-0.5555702447891235f, -0.8314695954322815f);
        case 12: return make_float2(-0.7071067690849304f, -0.7071067690849304f);
        case 13: return make_float2(-0.8314695954322815f, -0.5555702447891235f);
        case 14: return make_float2(-0.9238795042037964f, -0.3826834261417389f);
        case 15: return make_float2(-0.9807852506637573f, -0.19509032368659973f);
        default: return make_float2(0.f, 0.f);
    }
}

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

__host__ __device__ constexpr int bitrevc(int x, int bits)
{
    int r = 0;
    for (int b = 0; b < bits; b++) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

__device__ __forceinline__ float2 caddf(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

// In-register radix-2 DIF transform of N <= 32 points, sign SIGN (-1 forward,
// +1 backward), unnormalised.  On return a[j] = X[bitrev(j)].
template <int N, int SIGN>
__device__ __forceinline__ void reg_fft(float2 (&a)[N])
{
#pragma unroll
    for (int span = N / 2; span >= 1; span >>= 1) {
#pragma unroll
        for (int g = 0; g < N; g += 2 * span) {
#pragma unroll
            for (int j = 0; j < span; j++) {
                const float2 x = a[g + j], y = a[g + j + span];
                a[g + j] = make_float2(x.x + y.x, x.y + y.y);
                const float2 d = make_float2(x.x - y.x, x.y - y.y);
                if (j == 0) {
                    a[g + j + span] = d;
                } else {
                    const int k = j * (32 / (2 * span));
                    if (k == 8) {  // exp(-+ i pi / 2)
                        a[g + j + span] = SIGN < 0 ? make_float2(d.y, -d.x) : make_float2(-d.y, d.x);
                    } else {
                        float2 t = tw32(k);
                        if (SIGN > 0) t.y = -t.y;
                        a[g + j + span] = cmulf(d, t);
                    }
                }
            }
        }
    }
}

}  // namespace rg
