// Device building blocks for the project's own FFTs (FP32 complex).
//
// A length-N transform, N = N1 * 32, is computed in four steps (Bailey's
// four-step method): 32-point transforms in registers over the stride-N1
// subsequences, a twiddle multiply W_N^(n1 k2), an exchange through shared
// memory, and N1-point transforms in registers.  Register transforms are
// radix-2 with compile-time indices, so all data stays in registers; outputs
// come out in bit-reversed order and are stored to their natural positions.
// Twiddles are FP64-computed values rounded to FP32.
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

// exp(-2 pi i k / 32), k = 1..15 except 8, as scale x (1 + i ratio) when
// |cos| >= |sin| (scale = cos, ratio = tan) or scale x (ratio + i) otherwise
// (scale = sin, ratio = cot): |ratio| <= 1.  FP64-evaluated, rounded to FP32;
// compile-time k only.
struct TanTwiddle {
    float scale, ratio;
    bool cot;
};
__device__ __forceinline__ TanTwiddle tw32_tan(int k)
{
    switch (k) {
        case 1: return {0.9807852506637573f, -0.1989123672246933f, false};
        case 2: return {0.9238795042037964f, -0.4142135679721832f, false};
        case 3: return {0.8314695954322815f, -0.6681786179542542f, false};
        case 4: return {0.7071067690849304f, -1.0f, false};
        case 5: return {-0.8314695954322815f, -0.6681786179542542f, true};
        case 6: return {-0.9238795042037964f, -0.4142135679721832f, true};
        case 7: return {-0.9807852506637573f, -0.1989123672246933f, true};
        case 9: return {-0.9807852506637573f, 0.1989123672246933f, true};
        case 10: return {-0.9238795042037964f, 0.4142135679721832f, true};
        case 11: return {-0.8314695954322815f, 0.6681786179542542f, true};
        case 12: return {-0.7071067690849304f, 1.0f, true};
        case 13: return {-0.8314695954322815f, 0.6681786179542542f, false};
        case 14: return {-0.9238795042037964f, 0.4142135679721832f, false};
        case 15: return {-0.9807852506637573f, 0.1989123672246933f, false};
        default: return {1.0f, 0.0f, false};
    }
}

// In-register radix-2 transforms of N <= 32 points, sign SIGN (-1 forward,
// +1 backward), unnormalised.  On return a[j] = X[bitrev(j)].
//
// reg_fft_dif: decimation in frequency, twiddles as complex multiplies.
template <int N, int SIGN>
__device__ __forceinline__ void reg_fft_dif(float2 (&a)[N])
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

// reg_fft: decimation in time over the view v[i] = a[bitrev(i)] (x in bit-reversed
// order, so v ends in natural order, which is a[j] = X[bitrev(j)]); the view
// is compile-time register renaming.  A twiddled butterfly x +- w y with
// w = scale (1 + i ratio) takes u = y (1 + i ratio) in two fused multiply-adds
// and x +- scale u in two more on packed FP32 pairs (the tangent form of
// Goedecker, SIAM J. Sci. Comput. 18 (1997), for multiply-add units); an
// untwiddled one is one packed add and one packed multiply-add by -1 (exact).
// Four instructions per twiddled butterfly and two per untwiddled one, against
// eight and four for complex multiplies and scalar additions, with the same
// results as their scalar forms.  It holds about ten more registers than
// reg_fft_dif: the kernels whose occupancy those registers would cut (the
// batched row and column transforms) keep the DIF form, the sub-grid stages
// take this one.
template <int N, int SIGN>
__device__ __forceinline__ void reg_fft(float2 (&a)[N])
{
    constexpr int LB = ilog2c(N);
#pragma unroll
    for (int span = 1; span < N; span <<= 1) {
#pragma unroll
        for (int g = 0; g < N; g += 2 * span) {
#pragma unroll
            for (int j = 0; j < span; j++) {
                const int p = bitrevc(g + j, LB), q = bitrevc(g + j + span, LB);
                const float2 x = a[p], y = a[q];
                const int k = j * (32 / (2 * span));  // w = exp(SIGN 2 pi i k / 32)
                if (k == 0) {  // x + y, x - y = y (-1) + x
                    a[p] = __fadd2_rn(x, y);
                    a[q] = __ffma2_rn(y, make_float2(-1.f, -1.f), x);
                } else if (k == 8) {  // w = -+ i
                    const float2 wy = SIGN < 0 ? make_float2(y.y, -y.x) : make_float2(-y.y, y.x);
                    a[p] = make_float2(x.x + wy.x, x.y + wy.y);
                    a[q] = make_float2(x.x - wy.x, x.y - wy.y);
                } else {
                    const TanTwiddle t = tw32_tan(k);
                    const float c = t.scale, r = t.ratio;
                    // u = y (1 + i r) or y (r + i); SIGN > 0 takes the conjugates,
                    // y (1 - i r) or y (r - i)
                    float2 u;
                    if (!t.cot)
                        u = SIGN < 0 ? make_float2(fmaf(-r, y.y, y.x), fmaf(r, y.x, y.y))
                                     : make_float2(fmaf(r, y.y, y.x), fmaf(-r, y.x, y.y));
                    else
                        u = SIGN < 0 ? make_float2(fmaf(r, y.x, -y.y), fmaf(r, y.y, y.x))
                                     : make_float2(fmaf(r, y.x, y.y), fmaf(r, y.y, -y.x));
                    a[p] = __ffma2_rn(make_float2(c, c), u, x);
                    a[q] = __ffma2_rn(make_float2(-c, -c), u, x);
                }
            }
        }
    }
}

}  // namespace rg
