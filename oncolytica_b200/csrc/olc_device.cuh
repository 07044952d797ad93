// Device-side helpers shared by the prebuilt kernels (libolc.so) and by the
// NVRTC-compiled rule kernels.  Plain C types only, so the header compiles
// both under nvcc and under NVRTC (which has no host standard library).
//
// Reference semantics restated here:
//   * xorshift32 RNG and its float mapping  — framework/src/oncolytica/gpu/compiler/template.wgsl:75-82
//     (identical to NextRand, engine/assets/shaders/tumor_sim.wgsl:194-200)
//   * random unit direction                 — template.wgsl:84-98
//   * hierarchical Morton keys              — template.wgsl:100-132,
//     framework/src/oncolytica/core/runtime/_geometry.py:14-47
#pragma once

typedef unsigned int olc_u32;
typedef int olc_i32;
typedef unsigned long long olc_u64;

// ---------------------------------------------------------------- status bits
// A device status word collects non-fatal conditions; kernels never trap.
#define OLC_ST_CAPACITY      0x1u   // births dropped: agent capacity reached
#define OLC_ST_TIMEOUT       0x2u   // a bounded spin-wait gave up
#define OLC_ST_MULTI_DIVIDE  0x4u   // a rule called divide() twice in one call
#define OLC_ST_BAD_KEY       0x8u   // key outside the bin table (never expected)

// Spin limit for decoupled look-back waits.  Every wait is bounded; on expiry
// the kernel records OLC_ST_TIMEOUT and continues with what it has.
#define OLC_SPIN_LIMIT (1u << 22)

// ---------------------------------------------------------------- RNG
// xorshift32 (shifts 13, 17, 5) followed by u32 -> f32 (round to nearest) and
// an exact scale by 2^-32.  The result lies in [0, 1] (it can round to 1.0).
__device__ __forceinline__ float olc_next_rand(olc_u32& s) {
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return __fmul_rn(__uint2float_rn(s), 2.3283064365386963e-10f);
}

// Unit vector from two draws: z = 2 r1 - 1, phi = 2 pi r2,
// (sqrt(max(0, 1 - z^2)) cos phi, ... sin phi, z).
__device__ __forceinline__ float3 olc_rand_dir(olc_u32& s) {
    float r1 = olc_next_rand(s);
    float r2 = olc_next_rand(s);
    float z = __fsub_rn(__fmul_rn(r1, 2.0f), 1.0f);
    float phi = __fmul_rn(r2, 6.283185307179586f);
    float rxy = sqrtf(fmaxf(0.0f, __fsub_rn(1.0f, __fmul_rn(z, z))));
    return make_float3(__fmul_rn(rxy, cosf(phi)), __fmul_rn(rxy, sinf(phi)), z);
}

// MurmurHash3's 32-bit finaliser (fmix32), a published integer mixer.
__device__ __host__ __forceinline__ olc_u32 olc_fmix32(olc_u32 h) {
    h ^= h >> 16; h *= 0x85EBCA6Bu;
    h ^= h >> 13; h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

// Initial per-agent RNG state: MurmurHash3's 32-bit finaliser (fmix32, a
// published integer mixer) of seed*golden + index, forced odd so it is never
// the xorshift fixed point 0.
__device__ __host__ __forceinline__ olc_u32 olc_seed_rng(olc_u32 seed, olc_u32 index) {
    olc_u32 h = seed * 0x9E3779B9u + index;
    h ^= h >> 16; h *= 0x85EBCA6Bu;
    h ^= h >> 13; h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h | 1u;
}

// Child RNG state: parent state at the divide() call xor 0x12345678
// (engine/assets/shaders/tumor_sim.wgsl:694).
#define OLC_CHILD_RNG_XOR 0x12345678u

// ---------------------------------------------------------------- Morton keys
__device__ __host__ __forceinline__ olc_u32 olc_interleave9(olc_u32 v) {
    olc_u32 x = v & 0x1ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__device__ __host__ __forceinline__ olc_u32 olc_chem_key(int cx, int cy, int cz) {
    return olc_interleave9((olc_u32)cx) | (olc_interleave9((olc_u32)cy) << 1) |
           (olc_interleave9((olc_u32)cz) << 2);
}

// Tissue (bin) key: Morton key of the coarse coordinate c/2, shifted by 3,
// with the parity of each axis in the low 3 bits.
__device__ __host__ __forceinline__ olc_u32 olc_tissue_key(int cx, int cy, int cz) {
    olc_u32 j = olc_chem_key(cx / 2, cy / 2, cz / 2);
    olc_u32 i = (olc_u32)(cx & 1) | ((olc_u32)(cy & 1) << 1) | ((olc_u32)(cz & 1) << 2);
    return (j << 3) | i;
}

// The tissue key splits into one term per axis, OR-ed:
//   olc_tissue_key(x, y, z) = olc_tissue_axis(x, 0) | olc_tissue_axis(y, 1) | olc_tissue_axis(z, 2)
// (the coarse coordinate's interleaved bits above the three parity bits), so
// a walk over the 27 Moore bins needs 9 interleaves instead of 81.
__device__ __host__ __forceinline__ olc_u32 olc_tissue_axis(int c, int axis) {
    return (olc_interleave9((olc_u32)(c >> 1)) << (3 + axis)) | ((olc_u32)(c & 1) << axis);
}

// Bin coordinate of one position component: trunc(p / vs) with an IEEE
// (correctly rounded) divide, clamped to [0, dim-1].  NaN maps to 0.
__device__ __forceinline__ int olc_bin_coord(float p, float vs, int dim) {
    float q = __fdiv_rn(p, vs);
    int c = __float2int_rz(q);
    c = c < 0 ? 0 : c;
    c = c > dim - 1 ? dim - 1 : c;
    return c;
}

// ---------------------------------------------------------------- memory order
__device__ __forceinline__ olc_u32 olc_ld_relaxed(const olc_u32* p) {
    olc_u32 v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void olc_st_relaxed(olc_u32* p, olc_u32 v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Decoupled look-back words: 2 flag bits over a 30-bit count.
#define OLC_LB_AGG    0x40000000u
#define OLC_LB_PREFIX 0x80000000u
#define OLC_LB_MASK   0x3fffffffu

// Waits (bounded: `limit` polls) for the tile-`t` word to carry a flag, then
// returns it; on expiry it records OLC_ST_TIMEOUT and returns an empty prefix.
__device__ __forceinline__ olc_u32 olc_lb_wait(const olc_u32* word, olc_u32* status,
                                               olc_u32 limit = OLC_SPIN_LIMIT) {
    olc_u32 v = olc_ld_relaxed(word);
    olc_u32 spins = 0;
    while ((v & (OLC_LB_AGG | OLC_LB_PREFIX)) == 0u) {
        if (++spins > limit) {
            atomicOr(status, OLC_ST_TIMEOUT);
            return OLC_LB_PREFIX;  // count 0, treated as a prefix so the walk ends
        }
        __nanosleep(32);
        v = olc_ld_relaxed(word);
    }
    return v;
}

// Exclusive prefix of `count` over all earlier tiles for one lane of
// look-back state (`words` points at this lane's column; stride between
// tiles is `stride` words).  Publishes this tile's aggregate first and its
// inclusive prefix afterwards.
__device__ __forceinline__ olc_u32 olc_lookback(olc_u32* words, olc_u32 stride, olc_u32 tile,
                                                olc_u32 count, olc_u32* status,
                                                olc_u32 limit = OLC_SPIN_LIMIT) {
    if (tile == 0) {
        olc_st_relaxed(words, OLC_LB_PREFIX | count);
        return 0;
    }
    olc_st_relaxed(words + (olc_u64)tile * stride, OLC_LB_AGG | count);
    olc_u32 excl = 0;
    int t = (int)tile - 1;
    while (t >= 0) {
        olc_u32 v = olc_lb_wait(words + (olc_u64)t * stride, status, limit);
        excl += v & OLC_LB_MASK;
        if (v & OLC_LB_PREFIX) break;
        --t;
    }
    olc_st_relaxed(words + (olc_u64)tile * stride, OLC_LB_PREFIX | (excl + count));
    return excl;
}

// ---------------------------------------------------------------- mbarrier waits
// One poll of phase `parity` of the shared-memory mbarrier at `bar`.
__device__ __forceinline__ bool olc_mbar_try_wait(olc_u32 bar, olc_u32 parity) {
    olc_u32 ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for a TMA tile's mbarrier phase: true once the phase
// completed.  After `limit` polls the thread records OLC_ST_TIMEOUT, polls up
// to `limit` more times so that a copy still in flight can land before the
// block's shared memory is released, and returns false (the caller returns).
__device__ __forceinline__ bool olc_mbar_wait_bounded(olc_u32 bar, olc_u32 parity, olc_u32* status,
                                                      olc_u32 limit = OLC_SPIN_LIMIT) {
    for (olc_u32 it = 0; it < limit; ++it)
        if (olc_mbar_try_wait(bar, parity)) return true;
    atomicOr(status, OLC_ST_TIMEOUT);
    for (olc_u32 it = 0; it < limit && !olc_mbar_try_wait(bar, parity); ++it) {
    }
    return false;
}
