// BF16 / FP16 storage of fields: conversions to and from FP32 (round to
// nearest even) and 4-element vector loads and stores.  Bits are handled as
// unsigned short.
#pragma once
#include "olc_device.cuh"
#include "../../include/olc.h"

namespace olc {

template <int ST>
struct Store16;

template <>
struct Store16<OLC_FIELD_BF16> {
    static __device__ __forceinline__ float to_f(unsigned short h) { return __uint_as_float((olc_u32)h << 16); }
    // round to nearest even on the FP32 bit pattern (values here are finite)
    static __device__ __forceinline__ unsigned short from_f(float f) {
        unsigned short h;
        asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(h) : "f"(f));
        return h;
    }
};

template <>
struct Store16<OLC_FIELD_F16> {
    static __device__ __forceinline__ float to_f(unsigned short h) {
        float f;
        asm("{ .reg .b16 t; mov.b16 t, %1; cvt.f32.f16 %0, t; }" : "=f"(f) : "h"(h));
        return f;
    }
    static __device__ __forceinline__ unsigned short from_f(float f) {
        unsigned short h;
        asm("{ .reg .b16 t; cvt.rn.f16.f32 t, %1; mov.b16 %0, t; }" : "=h"(h) : "f"(f));
        return h;
    }
};

// BF16 with stochastic rounding in the substeps: same storage as BF16
template <>
struct Store16<OLC_FIELD_BF16_SR> : Store16<OLC_FIELD_BF16> {};

// Stochastic BF16 rounding of a finite non-negative value with 32 random bits:
// the low 16 bits of the FP32 pattern plus 16 random bits carry into the kept
// half with probability equal to the discarded fraction.
__device__ __forceinline__ unsigned short olc_bf16_sr(float f, olc_u32 rnd) {
    return (unsigned short)((__float_as_uint(f) + (rnd & 0xffffu)) >> 16);
}

// Random bits of voxel v (index within its grid) for one substep: `key` mixes
// the step, substep and field (olc_sr_key).
__device__ __forceinline__ olc_u32 olc_sr_key(olc_u32 step, int sub, int field) {
    return olc_fmix32((step << 8) ^ (olc_u32)sub ^ ((olc_u32)field << 24));
}
__device__ __forceinline__ olc_u32 olc_sr_bits(unsigned long long v, olc_u32 key) {
    return olc_fmix32((olc_u32)v * 0x9E3779B1u ^ key);
}

template <int ST>
__device__ __forceinline__ float4 load4(const unsigned short* p) {
    const uint2 raw = *reinterpret_cast<const uint2*>(p);
    return make_float4(Store16<ST>::to_f((unsigned short)(raw.x & 0xffffu)), Store16<ST>::to_f((unsigned short)(raw.x >> 16)),
                       Store16<ST>::to_f((unsigned short)(raw.y & 0xffffu)), Store16<ST>::to_f((unsigned short)(raw.y >> 16)));
}

// Stores four values at voxel index v (stochastic rounding for ST = BF16_SR).
template <int ST>
__device__ __forceinline__ void store4_at(unsigned short* p, float4 v, unsigned long long vi, olc_u32 key) {
    if (ST == OLC_FIELD_BF16_SR) {
        const olc_u32 lo = (olc_u32)olc_bf16_sr(v.x, olc_sr_bits(vi, key)) |
                           ((olc_u32)olc_bf16_sr(v.y, olc_sr_bits(vi + 1, key)) << 16);
        const olc_u32 hi = (olc_u32)olc_bf16_sr(v.z, olc_sr_bits(vi + 2, key)) |
                           ((olc_u32)olc_bf16_sr(v.w, olc_sr_bits(vi + 3, key)) << 16);
        *reinterpret_cast<uint2*>(p) = make_uint2(lo, hi);
        return;
    }
    const olc_u32 lo = (olc_u32)Store16<ST>::from_f(v.x) | ((olc_u32)Store16<ST>::from_f(v.y) << 16);
    const olc_u32 hi = (olc_u32)Store16<ST>::from_f(v.z) | ((olc_u32)Store16<ST>::from_f(v.w) << 16);
    *reinterpret_cast<uint2*>(p) = make_uint2(lo, hi);
}

template <int ST>
__device__ __forceinline__ void store4(unsigned short* p, float4 v) {
    const olc_u32 lo = (olc_u32)Store16<ST>::from_f(v.x) | ((olc_u32)Store16<ST>::from_f(v.y) << 16);
    const olc_u32 hi = (olc_u32)Store16<ST>::from_f(v.z) | ((olc_u32)Store16<ST>::from_f(v.w) << 16);
    *reinterpret_cast<uint2*>(p) = make_uint2(lo, hi);
}


}  // namespace olc
