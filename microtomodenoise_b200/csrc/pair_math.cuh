// Packed-pair FP32 arithmetic and the exact per-offset weight step shared by
// the plain FP32 filter kernels (filter_kernels.cu, filter_column.cu).
#pragma once

#include <cuda_runtime.h>

namespace inlm {

// Packed-pair arithmetic (sm_100 f32x2: one FADD2/FMUL2 instruction does two
// IEEE round-to-nearest operations; measured on B200 it issues in one slot but
// gives no more FP32 lane throughput than two scalar instructions, so the gain
// is issue slots left for the loads around it). ptxas fuses an FMUL2 whose
// result feeds an FADD2 into one FFMA2 even with explicit .rn modifiers, which
// would round once instead of twice; scalar products feeding paired sums (or
// paired products feeding only products) keep every rounding of the
// reference, so the kernels below never let an FMUL2 result reach an addition.
// A pair is a 64-bit register holding (element 0, element 1).
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
// Paired product; its result must only feed multiplications (see above).
__device__ __forceinline__ f32x2 mul2_to_mul(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
// Fused pair a*b + c, one rounding per lane (FFMA2): the fused FP32 form only.
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
    f32x2 d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ float2 unpack2(f32x2 a) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(a));
    return r;
}
__device__ __forceinline__ f32x2 splat2(float v) { return pack2(v, v); }
// Two scalar products as a pair (safe to feed add2).
__device__ __forceinline__ f32x2 mul_pair(float a0, float a1, float b) {
    return pack2(__fmul_rn(a0, b), __fmul_rn(a1, b));
}
__device__ __forceinline__ f32x2 mul_pair(float2 a, float2 b) {
    return pack2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
}

// One offset's weight and accumulation for a voxel pair, exactly as the
// reference CPU filter rounds it: x = dist*m; Pade[3/3] (120 + 60x + 12x*x +
// x*x*x) / (120 - 60x + 12x*x - x*x*x) with the products that feed sums
// scalar and the sums paired; w = x > -3.56648 ? quotient : 0; acc += w*raw,
// wsum += w, wmax = max(wmax, w). Both quotients are always formed and then
// selected: a division under the cutoff test becomes a divergent branch (10%
// slower).
__device__ __forceinline__ void exact_weight_pair(f32x2 dist, f32x2 m2, float2 rsv, f32x2& acc,
                                                  f32x2& wsum, float& wmax0, float& wmax1) {
    const f32x2 c12 = splat2(12.f), c120 = splat2(120.f);
    const f32x2 x = mul2_to_mul(dist, m2);
    const float2 xs = unpack2(x);
    const float2 x12 = unpack2(mul2_to_mul(c12, x));
    const float2 xx = unpack2(mul2_to_mul(x, x));
    const f32x2 ta = mul_pair(xs, make_float2(60.f, 60.f));
    const f32x2 tb = mul_pair(x12, xs);
    const f32x2 tc = mul_pair(xx, xs);
    const float2 num = unpack2(add2(add2(add2(c120, ta), tb), tc));
    const float2 den = unpack2(sub2(add2(sub2(c120, ta), tb), tc));
    const float q0 = __fdiv_rn(num.x, den.x), q1 = __fdiv_rn(num.y, den.y);
    const float w0 = (xs.x > -3.56648f) ? q0 : 0.0f;
    const float w1 = (xs.y > -3.56648f) ? q1 : 0.0f;
    acc = add2(acc, mul_pair(make_float2(w0, w1), rsv));
    wsum = add2(wsum, pack2(w0, w1));
    wmax0 = fmaxf(wmax0, w0);
    wmax1 = fmaxf(wmax1, w1);
}

// The fused FP32 form of the same step: Pade[3/3] in Horner form with fused
// pairs, 120 + x(60 + x(12 + x)) over 120 + x(-60 + x(12 - x)), a fast
// division, and w*raw fused into its sum (not bit-identical to the
// reference; within 1e-4 relative except where a weight crosses the cutoff).
__device__ __forceinline__ void fused_weight_pair(f32x2 dist, f32x2 m2, float2 rsv, f32x2& acc,
                                                  f32x2& wsum, float& wmax0, float& wmax1) {
    const f32x2 c12 = splat2(12.f), c120 = splat2(120.f), c60 = splat2(60.f), cm60 = splat2(-60.f);
    const f32x2 x = mul2_to_mul(dist, m2);
    const float2 xs = unpack2(x);
    const f32x2 num = fma2(x, fma2(x, add2(c12, x), c60), c120);
    const f32x2 den = fma2(x, fma2(x, sub2(c12, x), cm60), c120);
    const float2 nu = unpack2(num), de = unpack2(den);
    const float q0 = __fdividef(nu.x, de.x), q1 = __fdividef(nu.y, de.y);
    const float w0 = (xs.x > -3.56648f) ? q0 : 0.0f;
    const float w1 = (xs.y > -3.56648f) ? q1 : 0.0f;
    const f32x2 wp = pack2(w0, w1);
    acc = fma2(wp, pack2(rsv.x, rsv.y), acc);
    wsum = add2(wsum, wp);
    wmax0 = fmaxf(wmax0, w0);
    wmax1 = fmaxf(wmax1, w1);
}

}  // namespace inlm
