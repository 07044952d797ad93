// BF16 / FP16 storage of fields: conversions to and from FP32 (round to
// nearest even, or stochastic for the _SR types) and 8-element vector loads
// and stores.  Bits are handled as unsigned short.
#pragma once
#include <type_traits>

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

// ------------------------------------------------------------------ encodings
// What a 16-bit element holds (OLC_ENC_*, olc.h).  Kernels work on the
// "working" value of an element: the deficit b - f for OLC_ENC_DEFICIT (the
// 7-point update is linear, so substeps and residuals stay in that domain),
// the field value f otherwise.  `Codec` gathers the per-encoding steps.
struct EncConst {
    float b, half_b, quarter_b, upper_q;
};

template <int ST, int EN>
struct Codec {
    // working value of one element
    static __device__ __forceinline__ float work(unsigned short h, const EncConst& k) {
        if (EN != OLC_ENC_OFFSET3) return Store16<ST>::to_f(h);
        // magnitude with the sign (bit 15) kept and bit 14 cleared, plus
        // (b/2) x (bit 15 + bit 14): codes 00 -> m, 01 -> b/2 + m,
        // 10 -> b/2 - m, 11 -> b - m
        // The offset (b/2 per set flag bit; both products and their sum are
        // exact) is formed with selects: an integer-to-float conversion runs
        // on the quarter-rate conversion pipe and bounded the substep.
        const float m = Store16<ST>::to_f((unsigned short)(h & 0xBFFFu));
        const float o15 = (h & 0x8000u) ? k.half_b : 0.0f;
        const float o14 = (h & 0x4000u) ? k.half_b : 0.0f;
        return __fadd_rn(m, __fadd_rn(o15, o14));
    }
    // field value from a working value
    static __device__ __forceinline__ float phys_of_work(float w, const EncConst& k) {
        return EN == OLC_ENC_DEFICIT ? __fsub_rn(k.b, w) : w;
    }
    static __device__ __forceinline__ float phys(unsigned short h, const EncConst& k) {
        return phys_of_work(work(h, k), k);
    }
    // OLC_ENC_OFFSET3: magnitude to round and the code bits of a value f,
    // clamped to [0, b]; every subtraction is exact (Sterbenz)
    static __device__ __forceinline__ float split3(float f, const EncConst& k, olc_u32* code) {
        f = fminf(fmaxf(f, 0.0f), k.b);
        if (f < k.quarter_b) {
            *code = 0u;
            return fabsf(f);
        }
        if (f > k.upper_q) {
            *code = 0xC000u;
            return __fsub_rn(k.b, f);
        }
        const float d = __fsub_rn(f, k.half_b);
        *code = d < 0.0f ? 0x8000u : 0x4000u;
        return fabsf(d);
    }
    // two working values -> one word (a low, b high), nearest or stochastic
    static __device__ __forceinline__ olc_u32 pack(float a, float b, const EncConst& k, bool sr, olc_u32 rnd) {
        if (EN != OLC_ENC_OFFSET3) return sr ? pack2_sr<ST>(a, b, rnd) : pack2<ST>(a, b);
        olc_u32 ca, cb;
        const float ma = split3(a, k, &ca), mb = split3(b, k, &cb);
        return (sr ? pack2_sr<ST>(ma, mb, rnd) : pack2<ST>(ma, mb)) | ca | (cb << 16);
    }
    // one working value -> one element, to nearest
    static __device__ __forceinline__ unsigned short enc_rn(float w, const EncConst& k) {
        if (EN != OLC_ENC_OFFSET3) return Store16<ST>::from_f(w);
        olc_u32 c;
        const float m = split3(w, k, &c);
        return (unsigned short)(Store16<ST>::from_f(m) | c);
    }
};

// Eight elements (16 bytes) to working values.
template <int ST, int EN>
__device__ __forceinline__ void load8w(const unsigned short* p, float (&f)[8], const EncConst& k) {
    if (EN != OLC_ENC_OFFSET3) {
        load8<ST>(p, f);
        return;
    }
    const uint4 raw = *reinterpret_cast<const uint4*>(p);
    const olc_u32 w[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        f[2 * q] = Codec<ST, EN>::work((unsigned short)(w[q] & 0xffffu), k);
        f[2 * q + 1] = Codec<ST, EN>::work((unsigned short)(w[q] >> 16), k);
    }
}

// Eight working values stored at voxel index vi (a multiple of 8).
template <int ST, int EN>
__device__ __forceinline__ void store8w_at(unsigned short* p, const float (&v)[8], unsigned long long vi,
                                           olc_u32 key, const EncConst& k) {
    olc_u32 w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
        w[q] = Codec<ST, EN>::pack(v[2 * q], v[2 * q + 1], k, IsSR<ST>::value,
                                   IsSR<ST>::value ? olc_sr_pair((vi >> 1) + q, key) : 0u);
    *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
}

// The per-step reaction of one interior voxel (FS: a FieldStep): working value
// w = work(h) + residual; the uptake f <- f / (1 + K dt) and the step's decay
// f <- f * decay_step (round-to-nearest storages; 1 otherwise), rounded to
// nearest with the new residual kept.  For OLC_ENC_DEFICIT (w = b - f) the
// same maps are w <- (w + b K dt) / (1 + K dt), w <- w * decay_step +
// b (1 - decay_step), which leave a voxel with K = 0 and no decay unchanged.
template <int ST, int EN, class FS>
__device__ __forceinline__ void react_voxel(unsigned short& h, float& comp, float kv, const FS& fs,
                                            const EncConst& k) {
    float val = __fadd_rn(Codec<ST, EN>::work(h, k), comp);
    if (EN == OLC_ENC_DEFICIT) {
        if (kv != 0.0f) {
            const float kd = __fmul_rn(kv, fs.sink_dt);
            val = __fdiv_rn(__fadd_rn(val, __fmul_rn(k.b, kd)), __fadd_rn(1.0f, kd));
        }
        val = __fmaf_rn(val, fs.decay_step, fs.dec_step);
    } else {
        if (kv != 0.0f) val = __fdiv_rn(val, __fadd_rn(1.0f, __fmul_rn(kv, fs.sink_dt)));
        val = __fmul_rn(val, fs.decay_step);
    }
    h = Codec<ST, EN>::enc_rn(val, k);
    comp = __fsub_rn(val, Codec<ST, EN>::work(h, k));
}

// A voxel's field value with its residual (reductions, metrics).
template <int ST, int EN>
__device__ __forceinline__ float phys_with_residual(unsigned short h, float comp, const EncConst& k) {
    return Codec<ST, EN>::phys_of_work(__fadd_rn(Codec<ST, EN>::work(h, k), comp), k);
}

// Host side: calls f(storage, encoding) with both as std::integral_constant,
// for the runtime 16-bit storage type and encoding of a field.
template <class F>
inline void with_storage16(int storage, int encoding, F&& f) {
    auto by_enc = [&](auto st) {
        if (encoding == OLC_ENC_DEFICIT)
            f(st, std::integral_constant<int, OLC_ENC_DEFICIT>{});
        else if (encoding == OLC_ENC_OFFSET3)
            f(st, std::integral_constant<int, OLC_ENC_OFFSET3>{});
        else
            f(st, std::integral_constant<int, OLC_ENC_VALUE>{});
    };
    if (storage == OLC_FIELD_BF16)
        by_enc(std::integral_constant<int, OLC_FIELD_BF16>{});
    else if (storage == OLC_FIELD_BF16_SR)
        by_enc(std::integral_constant<int, OLC_FIELD_BF16_SR>{});
    else if (storage == OLC_FIELD_F16_SR)
        by_enc(std::integral_constant<int, OLC_FIELD_F16_SR>{});
    else
        by_enc(std::integral_constant<int, OLC_FIELD_F16>{});
}

// The reaction and the reductions round to nearest: a stochastic-rounding
// storage type shares its base type's kernels there.
template <int ST>
struct BaseOf {
    static constexpr int value = ST == OLC_FIELD_BF16_SR ? OLC_FIELD_BF16 : ST == OLC_FIELD_F16_SR ? OLC_FIELD_F16 : ST;
};

}  // namespace olc
