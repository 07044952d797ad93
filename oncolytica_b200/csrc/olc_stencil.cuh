// The explicit 7-point update of one voxel in FP32, scalar and on pairs of
// voxels, shared by the FP32 and 16-bit stencil kernels:
//   u = c + r * (((x- + x+) + (y- + y+)) + (z- + z+) - 6 c)
//   out = max(u * inv_decay, 0),   inv_decay = 1 / (1 + lambda dt/S)
// every operation separately rounded to nearest (the oracle's C arithmetic
// compiled without contraction).
#pragma once
#include "olc_device.cuh"
#include "../../include/olc.h"

namespace olc {

__device__ __forceinline__ float stencil_update(float xm, float xp, float ym, float yp, float zm, float zp, float c,
                                                float r, float inv_decay) {
    const float s = __fadd_rn(__fadd_rn(__fadd_rn(xm, xp), __fadd_rn(ym, yp)), __fadd_rn(zm, zp));
    const float u = __fadd_rn(c, __fmul_rn(r, __fsub_rn(s, __fmul_rn(6.0f, c))));
    return fmaxf(__fmul_rn(u, inv_decay), 0.0f);
}

// Paired FP32: sm_100's add/sub/mul.rn.f32x2 round each half exactly like the
// scalar .rn instruction.  The assembler does, however, fuse a paired multiply
// that feeds a paired add or subtract into one fused multiply-add (one
// rounding instead of two; measured on B200), so every product that feeds a
// sum is formed with scalar __fmul_rn; the sums and the final product (which
// only feeds the clamp) are paired.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk2(float lo, float hi) {
    f32x2 d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ float2 upk2(f32x2 d) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(d));
    return make_float2(lo, hi);
}
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
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// stencil_update on two voxels at once (every argument a pair).
__device__ __forceinline__ float2 stencil_update2(f32x2 xm, f32x2 xp, f32x2 ym, f32x2 yp, f32x2 zm, f32x2 zp,
                                                  f32x2 c, f32x2 r2, f32x2 id2) {
    const f32x2 s = add2(add2(add2(xm, xp), add2(ym, yp)), add2(zm, zp));
    const float2 cc = upk2(c);
    const float2 d = upk2(sub2(s, pk2(__fmul_rn(6.0f, cc.x), __fmul_rn(6.0f, cc.y))));
    const float2 rr = upk2(r2);
    const f32x2 u = add2(c, pk2(__fmul_rn(rr.x, d.x), __fmul_rn(rr.y, d.y)));
    const float2 w = upk2(mul2(u, id2));
    return make_float2(fmaxf(w.x, 0.0f), fmaxf(w.y, 0.0f));
}

// Four consecutive x voxels: centre row c, rows ym/yp, planes zm/zp, and the
// left/right neighbours xl/xr of the group.
__device__ __forceinline__ float4 stencil_update4(float xl, float xr, float4 c, float4 ym, float4 yp, float4 zm,
                                                  float4 zp, float r, float inv_decay) {
    const f32x2 r2 = pk2(r, r), id2 = pk2(inv_decay, inv_decay);
    const f32x2 mid = pk2(c.y, c.z);  // x+1 of the first pair, x-1 of the second
    const float2 a = stencil_update2(pk2(xl, c.x), mid, pk2(ym.x, ym.y), pk2(yp.x, yp.y), pk2(zm.x, zm.y),
                                     pk2(zp.x, zp.y), pk2(c.x, c.y), r2, id2);
    const float2 b = stencil_update2(mid, pk2(c.w, xr), pk2(ym.z, ym.w), pk2(yp.z, yp.w), pk2(zm.z, zm.w),
                                     pk2(zp.z, zp.w), pk2(c.z, c.w), r2, id2);
    return make_float4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// The update of the 16-bit field storages: the same sums, with the two
// products fused into their sums (one rounding each):
//   u = fma(r, fma(-6, c, s), c),   out = max(u * inv_decay, 0)
// on eight consecutive x voxels (four pairs); the oracle restates it with C's
// correctly rounded fmaf.
__device__ __forceinline__ void stencil_update8_fma(float xl, float xr, const float (&c)[8], const float (&ym)[8],
                                                    const float (&yp)[8], const float (&zm)[8], const float (&zp)[8],
                                                    float r, float inv_decay, float (&out)[8]) {
    const f32x2 r2 = pk2(r, r), id2 = pk2(inv_decay, inv_decay), m6 = pk2(-6.0f, -6.0f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int e = 2 * k;
        const f32x2 cc = pk2(c[e], c[e + 1]);
        // the x sums as two scalar adds: their operands are shifted by one
        // voxel, so as a pair they would straddle register pairs
        const float sx0 = __fadd_rn(k == 0 ? xl : c[e - 1], c[e + 1]);
        const float sx1 = __fadd_rn(c[e], k == 3 ? xr : c[e + 2]);
        const f32x2 s = add2(add2(pk2(sx0, sx1), add2(pk2(ym[e], ym[e + 1]), pk2(yp[e], yp[e + 1]))),
                             add2(pk2(zm[e], zm[e + 1]), pk2(zp[e], zp[e + 1])));
        const float2 w = upk2(mul2(fma2(r2, fma2(m6, cc, s), cc), id2));
        out[e] = fmaxf(w.x, 0.0f);
        out[e + 1] = fmaxf(w.y, 0.0f);
    }
}

// stencil_update8_fma on the working values of an encoded 16-bit field
// (OLC_ENC_*): OLC_ENC_DEFICIT updates deficits s = b - f, whose decay adds
// dec_sub = b (1 - inv_decay) and whose clamp [0, b] is the image of f in
// [0, b]:  out = min(max(fma(u, inv_decay, dec_sub), 0), b);  the other
// encodings update values as stencil_update8_fma does (OLC_ENC_OFFSET3
// clamps to [0, b] when it encodes).
template <int EN>
__device__ __forceinline__ void stencil_update8_enc(float xl, float xr, const float (&c)[8], const float (&ym)[8],
                                                    const float (&yp)[8], const float (&zm)[8],
                                                    const float (&zp)[8], float r, float inv_decay, float dec_sub,
                                                    float b, float (&out)[8]) {
    if (EN != OLC_ENC_DEFICIT) {
        stencil_update8_fma(xl, xr, c, ym, yp, zm, zp, r, inv_decay, out);
        return;
    }
    const f32x2 r2 = pk2(r, r), id2 = pk2(inv_decay, inv_decay), m6 = pk2(-6.0f, -6.0f),
                ds2 = pk2(dec_sub, dec_sub);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int e = 2 * k;
        const f32x2 cc = pk2(c[e], c[e + 1]);
        const float sx0 = __fadd_rn(k == 0 ? xl : c[e - 1], c[e + 1]);
        const float sx1 = __fadd_rn(c[e], k == 3 ? xr : c[e + 2]);
        const f32x2 s = add2(add2(pk2(sx0, sx1), add2(pk2(ym[e], ym[e + 1]), pk2(yp[e], yp[e + 1]))),
                             add2(pk2(zm[e], zm[e + 1]), pk2(zp[e], zp[e + 1])));
        const float2 w = upk2(fma2(fma2(r2, fma2(m6, cc, s), cc), id2, ds2));
        out[e] = fminf(fmaxf(w.x, 0.0f), b);
        out[e + 1] = fminf(fmaxf(w.y, 0.0f), b);
    }
}

// Eight consecutive x voxels (four pairs): centre row c, rows ym/yp, planes
// zm/zp, and the neighbours xl/xr left and right of the group.
__device__ __forceinline__ void stencil_update8(float xl, float xr, const float (&c)[8], const float (&ym)[8],
                                                const float (&yp)[8], const float (&zm)[8], const float (&zp)[8],
                                                float r, float inv_decay, float (&out)[8]) {
    const f32x2 r2 = pk2(r, r), id2 = pk2(inv_decay, inv_decay);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int e = 2 * k;
        const float2 v = stencil_update2(pk2(k == 0 ? xl : c[e - 1], c[e]), pk2(c[e + 1], k == 3 ? xr : c[e + 2]),
                                         pk2(ym[e], ym[e + 1]), pk2(yp[e], yp[e + 1]), pk2(zm[e], zm[e + 1]),
                                         pk2(zp[e], zp[e + 1]), pk2(c[e], c[e + 1]), r2, id2);
        out[e] = v.x;
        out[e + 1] = v.y;
    }
}

}  // namespace olc
