// BF16 / FP16 storage of fields: conversions to and from FP32 (round to
// nearest even, or stochastic for the _SR types) and 8-element vector loads
// and stores.  Bits are handled as unsigned short.
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

// BF16 / FP16 with stochastic rounding in the substeps: same storage
template <>
struct Store16<OLC_FIELD_BF16_SR> : Store16<OLC_FIELD_BF16> {};
template <>
struct Store16<OLC_FIELD_F16_SR> : Store16<OLC_FIELD_F16> {};

template <int ST>
struct IsSR {
    static constexpr bool value = ST == OLC_FIELD_BF16_SR || ST == OLC_FIELD_F16_SR;
};

// Stochastic BF16 rounding of a finite non-negative value with 32 random bits:
// the low 16 bits of the FP32 pattern plus 16 random bits carry into the kept
// half with probability equal to the discarded fraction.
__device__ __forceinline__ unsigned short olc_bf16_sr(float f, olc_u32 rnd) {
    return (unsigned short)((__float_as_uint(f) + (rnd & 0xffffu)) >> 16);
}


// Random bits for one substep: `key` mixes the step, substep and field
// (fmix32, once per launch); voxels 2p and 2p+1 of a grid share one 32-bit
// word x = ((p ^ key) * 0x9E3779B1) ^ (x >> 15) (a multiplicative hash with
// one xorshift), voxel 2p taking its low and voxel 2p+1 its high 16 bits.
__device__ __forceinline__ olc_u32 olc_sr_key(olc_u32 step, int sub, int field) {
    return olc_fmix32((step << 8) ^ (olc_u32)sub ^ ((olc_u32)field << 24));
}
__device__ __forceinline__ olc_u32 olc_sr_pair(unsigned long long pair, olc_u32 key) {
    olc_u32 x = ((olc_u32)pair ^ key) * 0x9E3779B1u;
    return x ^ (x >> 15);
}

// Eight consecutive values (16 bytes): load to FP32, store with rounding at
// voxel index vi (a multiple of 8; stochastic for the _SR types).
template <int ST>
__device__ __forceinline__ void load8(const unsigned short* p, float (&f)[8]) {
    const uint4 raw = *reinterpret_cast<const uint4*>(p);
    const olc_u32 w[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        f[2 * k] = Store16<ST>::to_f((unsigned short)(w[k] & 0xffffu));
        f[2 * k + 1] = Store16<ST>::to_f((unsigned short)(w[k] >> 16));
    }
}

// Two FP32 values -> one word of two 16-bit values (a in the low half, b in
// the high half).  cvt.*x2 converts its first source into the high half.
template <int ST>
__device__ __forceinline__ olc_u32 pack2(float a, float b) {
    olc_u32 d;
    if (ST == OLC_FIELD_BF16 || ST == OLC_FIELD_BF16_SR)
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
    else
        asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
    return d;
}

// The same with stochastic rounding, by the conversion's random-bits form:
// the low half (a) takes bits 15..0 of rnd (BF16) or 12..0 (FP16), the high
// half (b) bits 31..16 or 28..16; a value rounds away from zero when the top
// of its discarded bits plus those random bits carries (olc_bf16_sr for BF16).
template <int ST>
__device__ __forceinline__ olc_u32 pack2_sr(float a, float b, olc_u32 rnd) {
    olc_u32 d;
    if (ST == OLC_FIELD_BF16_SR)
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(b), "f"(a), "r"(rnd));
    else
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(b), "f"(a), "r"(rnd));
    return d;
}

// Eight values (16 bytes) stored at voxel index vi (a multiple of 8), rounded
// to nearest even or, for the _SR types, stochastically with the pair hash.
template <int ST>
__device__ __forceinline__ void store8_at(unsigned short* p, const float (&v)[8], unsigned long long vi, olc_u32 key) {
    olc_u32 w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        w[k] = IsSR<ST>::value ? pack2_sr<ST>(v[2 * k], v[2 * k + 1], olc_sr_pair((vi >> 1) + k, key))
                               : pack2<ST>(v[2 * k], v[2 * k + 1]);
    *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
}

}  // namespace olc
