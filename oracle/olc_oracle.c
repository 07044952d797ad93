/*
 * olc_oracle.c — CPU oracle for the Oncolytica step (TEST INFRASTRUCTURE,
 * see olc_oracle.h).  Each function cites the reference lines it restates.
 * Build: oracle/build.py (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include "olc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int nthreads_or_all(int nt) {
#ifdef _OPENMP
    return nt > 0 ? nt : omp_get_max_threads();
#else
    (void)nt;
    return 1;
#endif
}

/* ------------------------------------------------------------------ RNG */

/* framework/src/oncolytica/gpu/compiler/template.wgsl:75-82 (_next_rand):
 * s ^= s << 13; s ^= s >> 17; s ^= s << 5; return f32(s) * 2.3283064365386963e-10 */
float orc_next_rand(uint32_t* state) {
    uint32_t s = *state;
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    *state = s;
    return (float)s * 2.3283064365386963e-10f;
}

/* template.wgsl:84-98 (_rand_dir) */
void orc_rand_dir(uint32_t* state, float out[3]) {
    float r1 = orc_next_rand(state);
    float r2 = orc_next_rand(state);
    float z = r1 * 2.0f - 1.0f;
    float phi = r2 * 6.283185307179586f;
    float t = 1.0f - z * z;
    float rxy = sqrtf(t > 0.0f ? t : 0.0f);
    out[0] = rxy * cosf(phi);
    out[1] = rxy * sinf(phi);
    out[2] = z;
}

uint32_t orc_seed_rng(uint32_t seed, uint32_t index) {
    uint32_t h = seed * 0x9E3779B9u + index;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h | 1u;
}

void orc_rng_batch(uint32_t* states, uint32_t n, int draws, float* out, float* dirs) {
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t s = states[i];
        for (int k = 0; k < draws; ++k) out[(size_t)i * draws + k] = orc_next_rand(&s);
        if (dirs) orc_rand_dir(&s, dirs + 3 * (size_t)i);
        states[i] = s;
    }
}

/* ------------------------------------------------------------------ keys */

/* template.wgsl:100-107, _geometry.py:14-21 */
uint32_t orc_interleave9(uint32_t v) {
    uint32_t x = v & 0x1ffu;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

/* template.wgsl:109-114, _geometry.py:24-30 */
uint32_t orc_chem_key(int cx, int cy, int cz) {
    return orc_interleave9((uint32_t)cx) | (orc_interleave9((uint32_t)cy) << 1) |
           (orc_interleave9((uint32_t)cz) << 2);
}

/* template.wgsl:116-128, _geometry.py:33-42 */
uint32_t orc_tissue_key(int cx, int cy, int cz) {
    uint32_t j = orc_chem_key(cx / 2, cy / 2, cz / 2);
    uint32_t i = (uint32_t)(cx & 1) | ((uint32_t)(cy & 1) << 1) | ((uint32_t)(cz & 1) << 2);
    return (j << 3) | i;
}

/* template.wgsl:180 computes i32(pos / vs); this build clamps to the grid */
int orc_bin_coord(float p, float vs, int dim) {
    float q = p / vs;
    int c;
    if (q != q) c = 0;
    else if (q >= 2147483520.0f) c = 2147483647;
    else if (q <= -2147483648.0f) c = -2147483647 - 1;
    else c = (int)q; /* truncation toward zero */
    if (c < 0) c = 0;
    if (c > dim - 1) c = dim - 1;
    return c;
}

/* template.wgsl:174-186 (the key of Kernel_CountAndOffset); dead rows take
 * tissue_key(dims), the key die() produces (_stmt_translator.py:431-440). */
void orc_keys(const float* x, const float* y, const float* z, const uint8_t* dead, uint32_t n,
              const int32_t dims[3], float vs, uint32_t* keys) {
    const uint32_t sentinel = orc_tissue_key(dims[0], dims[1], dims[2]);
    for (uint32_t i = 0; i < n; ++i) {
        if (dead && dead[i]) {
            keys[i] = sentinel;
            continue;
        }
        int cx = orc_bin_coord(x[i], vs, dims[0]);
        int cy = orc_bin_coord(y[i], vs, dims[1]);
        int cz = orc_bin_coord(z[i], vs, dims[2]);
        keys[i] = orc_tissue_key(cx, cy, cz);
    }
}

/* ------------------------------------------------------------------ sort */

/* Stable sort by key: LSD radix with 16-bit digits (counting sort per digit).
 * The reference's scatter (template.wgsl:335-343) places a row at
 * start[key] + local_offset with an atomic local offset; the deterministic
 * refinement keeps equal keys in input order. */
void orc_sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, uint32_t n) {
    uint32_t* ka = (uint32_t*)malloc((size_t)n * 4 + 4);
    uint32_t* va = (uint32_t*)malloc((size_t)n * 4 + 4);
    uint32_t* cnt = (uint32_t*)malloc(65536 * 4);
    for (uint32_t i = 0; i < n; ++i) {
        ka[i] = kin[i];
        va[i] = vin ? vin[i] : i;
    }
    for (int pass = 0; pass < 2; ++pass) {
        const int sh = 16 * pass;
        memset(cnt, 0, 65536 * 4);
        for (uint32_t i = 0; i < n; ++i) cnt[(ka[i] >> sh) & 0xffffu]++;
        uint32_t run = 0;
        for (int d = 0; d < 65536; ++d) {
            uint32_t c = cnt[d];
            cnt[d] = run;
            run += c;
        }
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t o = cnt[(ka[i] >> sh) & 0xffffu]++;
            kout[o] = ka[i];
            vout[o] = va[i];
        }
        if (pass == 0) {
            memcpy(ka, kout, (size_t)n * 4);
            memcpy(va, vout, (size_t)n * 4);
        }
    }
    free(ka);
    free(va);
    free(cnt);
}

/* VoxelTable startIndex / count (template.wgsl:42-45, 228-329) as ranges */
void orc_bin_ranges(const uint32_t* keys, uint32_t n, uint32_t n_bins, uint32_t* ranges) {
    memset(ranges, 0, (size_t)n_bins * 8);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t k = keys[i];
        if (k >= n_bins) continue;
        if (i == 0 || keys[i - 1] != k) ranges[2 * (size_t)k] = i;
        if (i + 1 == n || keys[i + 1] != k) ranges[2 * (size_t)k + 1] = i + 1;
    }
}

/* ------------------------------------------------------------------ fields */

/* engine/assets/shaders/tumor_sim.wgsl:387-412 (implicit sink) and :414-446
 * (7-point Laplacian, Dirichlet faces), substeps as chemistry_rule(iterations=S). */
int orc_diffuse(float* f, float* tmp, float* sink, const int32_t dims[3], float dx, float dt, float D,
                float decay, float boundary, int substeps, int nthreads) {
    return orc_diffuse_pinned(f, tmp, sink, dims, dx, dt, D, decay, boundary, substeps, NULL, 0, 0.0f, nthreads);
}

/* orc_diffuse with pinned voxels: after every substep the voxels listed in
 * `pins` (x-fastest indices) hold `pin_value` — the engine's vessel mask
 * (engine/assets/shaders/tumor_sim.wgsl:366-380, 430-433: voxels inside the
 * vessel cylinder are stored as 1.0 by every diffusion pass). */
int orc_diffuse_pinned(float* f, float* tmp, float* sink, const int32_t dims[3], float dx, float dt, float D,
                       float decay, float boundary, int substeps, const uint32_t* pins, uint32_t n_pins,
                       float pin_value, int nthreads) {
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    const int nt = nthreads_or_all(nthreads);
    if (substeps < 1) return -1;
    const float dts = dt / (float)substeps;
    const float r = D * dts / (dx * dx);
    if (r > 1.0f / 6.0f + 1e-7f) return -1;
    const float inv_decay = 1.0f / (1.0f + decay * dts);
    const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
    if (sink) {
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    size_t v = (size_t)z * sz + (size_t)y * sy + x;
                    float k = sink[v];
                    if (k != 0.0f) {
                        int face = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
                        if (!face) f[v] = f[v] / (1.0f + k * dt);
                        sink[v] = 0.0f;
                    }
                }
    }
    float* cur = f;
    float* nxt = tmp;
    for (int s = 0; s < substeps; ++s) {
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y) {
                size_t row = (size_t)z * sz + (size_t)y * sy;
                for (int x = 0; x < nx; ++x) {
                    size_t v = row + x;
                    if (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1) {
                        nxt[v] = boundary;
                        continue;
                    }
                    float c = cur[v];
                    float s1 = (cur[v - 1] + cur[v + 1]) + (cur[v - sy] + cur[v + sy]);
                    float s2 = s1 + (cur[v - sz] + cur[v + sz]);
                    float u = c + r * (s2 - 6.0f * c);
                    float o = u * inv_decay;
                    nxt[v] = o > 0.0f ? o : 0.0f;
                }
            }
        for (uint32_t k = 0; k < n_pins; ++k) nxt[pins[k]] = pin_value;
        float* t = cur;
        cur = nxt;
        nxt = t;
    }
    if (cur != f) memcpy(f, cur, (size_t)nx * ny * nz * 4);
    return 0;
}

/* ------------------------------------------------------------------ 16-bit field storage */
/* The precision tier of the CUDA path (olc_field16.cu), restated: fields stored
 * as BF16 (storage 1) or FP16 (storage 2), every update in FP32 with
 * round-to-nearest-even back to storage.  Per step: a reaction pass
 * (value + residual, uptake, the step's decay (1 + lambda dt/S)^-S, residual
 * kept in comp), then S substeps without decay; faces pinned.  Storages 3 and
 * 4 (stochastic rounding) keep the FP32 scheme's decay in every substep
 * (u * 1/(1 + lambda dt/S)) and no decay in the reaction pass.  The substep
 * fuses its two products: u = fmaf(r, fmaf(-6, c, s), c) (C's fmaf rounds
 * once, as the GPU's fused multiply-add). */
static float bf16_to_f(uint16_t h) {
    uint32_t u = (uint32_t)h << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}
static uint16_t f_to_bf16(float f) { /* finite values: RN-even on the bit pattern */
    uint32_t u;
    memcpy(&u, &f, 4);
    return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}
static float h16_to_f(uint16_t h, int storage) {
    if (storage == 1 || storage == 3) return bf16_to_f(h);  /* 2 and 4: FP16 */
    _Float16 x;
    memcpy(&x, &h, 2);
    return (float)x;
}
static uint16_t f_to_h16(float f, int storage) {
    if (storage == 1 || storage == 3) return f_to_bf16(f);
    _Float16 x = (_Float16)f;
    uint16_t h;
    memcpy(&h, &x, 2);
    return h;
}

/* Stochastic BF16 rounding of the substeps (storage 3): key = fmix32((step <<
 * 8) ^ substep ^ (field << 24)); voxels 2p, 2p+1 share x = (p ^ key) *
 * 0x9E3779B1, x ^= x >> 15, voxel 2p taking the low and 2p+1 the high 16 bits;
 * the low 16 FP32 bits plus those random bits carry into the kept half with
 * probability equal to the discarded fraction. */
static uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}
static uint16_t f_to_bf16_sr(float f, uint32_t rnd) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return (uint16_t)((u + (rnd & 0xffffu)) >> 16);
}

/* FP32 -> FP16 rounded toward zero (IEEE binary16; finite inputs, results
 * past the largest finite FP16 clamp to it), from the bit pattern. */
static uint16_t f_to_f16_rz(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    const uint16_t sign = (uint16_t)((u >> 16) & 0x8000u);
    const int e = (int)((u >> 23) & 0xffu) - 127;
    const uint32_t m = u & 0x7fffffu;
    if (((u >> 23) & 0xffu) == 0u) return sign; /* zero and FP32 subnormals */
    if (e > 15) return (uint16_t)(sign | 0x7bffu);
    if (e >= -14) return (uint16_t)(sign | (uint16_t)((e + 15) << 10) | (uint16_t)(m >> 13));
    if (e < -24) return sign;
    return (uint16_t)(sign | (uint16_t)((0x800000u | m) >> (uint32_t)(-1 - e))); /* |f| * 2^24, truncated */
}

/* Stochastic FP16 rounding (storage 4) of a finite value: the value rounded
 * toward zero, plus one unit in the last place when the top 13 of the bits
 * below that place plus 13 random bits carry (normal results drop 13 FP32
 * mantissa bits; subnormal results drop more, and their top 13 are used).
 * The random bits come from the same pair hash as storage 3 (voxel 2p: bits
 * 12..0 of the pair word, voxel 2p+1: bits 28..16). */
static uint16_t f_to_f16_sr(float f, uint32_t rnd) {
    uint32_t u;
    memcpy(&u, &f, 4);
    const uint16_t h = f_to_f16_rz(f);
    const int ebits = (int)((u >> 23) & 0xffu);
    if (ebits == 0 || (h & 0x7fffu) == 0x7bffu) return h; /* zero / FP32 subnormal, or at the FP16 maximum */
    const int e = ebits - 127;
    const uint32_t m = (u & 0x7fffffu) | 0x800000u;
    uint32_t top13;
    if (e >= -14) {
        top13 = m & 0x1fffu; /* 13 dropped mantissa bits */
    } else {
        const int sh = -1 - e; /* bits of m below the subnormal unit 2^-24 (>= 14) */
        if (sh > 24 + 13) return h;
        top13 = sh >= 13 ? (uint32_t)(((uint64_t)m & ((1ull << sh) - 1ull)) >> (sh - 13)) : 0u;
    }
    return (top13 + (rnd & 0x1fffu) >= 0x2000u) ? (uint16_t)(h + 1u) : h;
}

void orc_round16(const float* in, uint16_t* out, size_t n, int storage, const uint32_t* rnd) {
    for (size_t i = 0; i < n; ++i) {
        if (storage == 3)
            out[i] = f_to_bf16_sr(in[i], rnd[i]);
        else if (storage == 4)
            out[i] = f_to_f16_sr(in[i], rnd[i]);
        else if (storage == 5)
            out[i] = f_to_f16_rz(in[i]);
        else
            out[i] = f_to_h16(in[i], storage);
    }
}

/* Encodings of 16-bit elements (olc.h OLC_ENC_*): 0 the value, 1 the deficit
 * b - f (the kernels' working value is then the deficit), 2 f minus the
 * offset o in {0, b/2, b} nearest f, o and the sign in bits 15 and 14
 * (oncolytica_b200/csrc/olc_store16.cuh: Codec). */
typedef struct {
    float b, hb, qb, uq;
} Enc16;
static Enc16 enc16_consts(float b) {
    Enc16 k;
    k.b = b;
    k.hb = 0.5f * b;
    k.qb = 0.25f * b;
    k.uq = b - k.qb;
    return k;
}
static float work16(uint16_t h, int storage, int enc, const Enc16* k) {
    if (enc != 2) return h16_to_f(h, storage);
    const float m = h16_to_f((uint16_t)(h & 0xBFFFu), storage);
    const uint32_t units = (uint32_t)(h >> 15) + (uint32_t)((h >> 14) & 1u);
    return m + (float)units * k->hb;
}
static float phys_of_work16(float w, int enc, const Enc16* k) { return enc == 1 ? k->b - w : w; }
static float split3(float f, const Enc16* k, uint16_t* code) {
    f = f > 0.0f ? f : 0.0f;
    f = f < k->b ? f : k->b;
    if (f < k->qb) {
        *code = 0;
        return fabsf(f);
    }
    if (f > k->uq) {
        *code = 0xC000u;
        return k->b - f;
    }
    const float d = f - k->hb;
    *code = d < 0.0f ? 0x8000u : 0x4000u;
    return fabsf(d);
}
static uint16_t enc16_rn(float w, int storage, int enc, const Enc16* k) {
    if (enc != 2) return f_to_h16(w, storage);
    uint16_t c;
    const float m = split3(w, k, &c);
    return (uint16_t)(f_to_h16(m, storage) | c);
}
static uint16_t enc16_sr(float w, int storage, int enc, const Enc16* k, uint32_t rb) {
    uint16_t c = 0;
    const float m = enc == 2 ? split3(w, k, &c) : w;
    return (uint16_t)((storage == 3 ? f_to_bf16_sr(m, rb) : f_to_f16_sr(m, rb)) | c);
}

void orc_encode16(const float* f, uint16_t* out, size_t n, int storage, int encoding, float boundary) {
    const Enc16 k = enc16_consts(boundary);
    for (size_t i = 0; i < n; ++i) out[i] = enc16_rn(encoding == 1 ? boundary - f[i] : f[i], storage, encoding, &k);
}

void orc_decode16(const uint16_t* h, const float* comp, float* out, size_t n, int storage, int encoding,
                  float boundary) {
    const Enc16 k = enc16_consts(boundary);
    for (size_t i = 0; i < n; ++i) {
        float w = work16(h[i], storage, encoding, &k);
        if (comp) w = w + comp[i];
        out[i] = phys_of_work16(w, encoding, &k);
    }
}

int orc_diffuse16e(uint16_t* f, uint16_t* tmp, float* sink, float* comp, const int32_t dims[3], float dx, float dt,
                   float D, float decay, float boundary, int substeps, int storage, int encoding, uint32_t step,
                   int field, int nthreads) {
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    const int nt = nthreads_or_all(nthreads);
    if (substeps < 1 || storage < 1 || storage > 4 || encoding < 0 || encoding > 2) return -1;
    if (encoding != 0 && !(boundary > 0.0f)) return -1;
    if (encoding == 2 && boundary > 4.0f) return -1;
    const float dts = dt / (float)substeps;
    const float r = D * dts / (dx * dx);
    if (r > 1.0f / 6.0f + 1e-7f) return -1;
    const int sr = storage == 3 || storage == 4;
    const float decay_step = sr ? 1.0f : (float)pow(1.0 + (double)decay * (double)dts, -(double)substeps);
    const float inv_decay = sr ? 1.0f / (1.0f + decay * dts) : 1.0f;
    const Enc16 k = enc16_consts(boundary);
    const float dec_sub = boundary * (1.0f - inv_decay);
    const float dec_step = boundary * (1.0f - decay_step);
    /* the faces hold the boundary: value as stored, deficit 0, or b exactly */
    const float face_w =
        encoding == 1 ? 0.0f : (encoding == 2 ? boundary : h16_to_f(f_to_h16(boundary, storage), storage));
    const uint16_t bh = enc16_rn(face_w, storage, encoding, &k);
    const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                size_t v = (size_t)z * sz + (size_t)y * sy + x;
                float kv = sink ? sink[v] : 0.0f;
                if (sink) sink[v] = 0.0f;
                if (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1) continue;
                float val = work16(f[v], storage, encoding, &k) + comp[v];
                if (encoding == 1) {
                    if (kv != 0.0f) {
                        const float kd = kv * dt;
                        val = (val + boundary * kd) / (1.0f + kd);
                    }
                    val = fmaf(val, decay_step, dec_step);
                } else {
                    if (kv != 0.0f) val = val / (1.0f + kv * dt);
                    val = val * decay_step;
                }
                uint16_t h = enc16_rn(val, storage, encoding, &k);
                f[v] = h;
                comp[v] = val - work16(h, storage, encoding, &k);
            }
    uint16_t* cur = f;
    uint16_t* nxt = tmp;
    for (int s = 0; s < substeps; ++s) {
        const uint32_t key = fmix32((step << 8) ^ (uint32_t)s ^ ((uint32_t)field << 24));
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y) {
                size_t row = (size_t)z * sz + (size_t)y * sy;
                for (int x = 0; x < nx; ++x) {
                    size_t v = row + x;
                    if (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1) {
                        nxt[v] = bh;
                        continue;
                    }
                    float c = work16(cur[v], storage, encoding, &k);
                    float s1 = (work16(cur[v - 1], storage, encoding, &k) + work16(cur[v + 1], storage, encoding, &k)) +
                               (work16(cur[v - sy], storage, encoding, &k) +
                                work16(cur[v + sy], storage, encoding, &k));
                    float s2 = s1 + (work16(cur[v - sz], storage, encoding, &k) +
                                     work16(cur[v + sz], storage, encoding, &k));
                    float u = fmaf(r, fmaf(-6.0f, c, s2), c);
                    if (encoding == 1) {
                        u = fmaf(u, inv_decay, dec_sub);
                        u = u > 0.0f ? u : 0.0f;
                        u = u < boundary ? u : boundary;
                    } else {
                        u = u * inv_decay;
                        u = u > 0.0f ? u : 0.0f;
                    }
                    if (sr) {
                        uint32_t xr = ((uint32_t)(v >> 1) ^ key) * 0x9E3779B1u;
                        xr ^= xr >> 15;
                        const uint32_t rb = (v & 1) ? (xr >> 16) : (xr & 0xffffu);
                        nxt[v] = enc16_sr(u, storage, encoding, &k, rb);
                    } else {
                        nxt[v] = enc16_rn(u, storage, encoding, &k);
                    }
                }
            }
        uint16_t* t = cur;
        cur = nxt;
        nxt = t;
    }
    if (cur != f) memcpy(f, cur, (size_t)nx * ny * nz * 2);
    return 0;
}

int orc_diffuse16(uint16_t* f, uint16_t* tmp, float* sink, float* comp, const int32_t dims[3], float dx, float dt,
                  float D, float decay, float boundary, int substeps, int storage, uint32_t step, int field,
                  int nthreads) {
    return orc_diffuse16e(f, tmp, sink, comp, dims, dx, dt, D, decay, boundary, substeps, storage, 0, step, field,
                          nthreads);
}

/* The field schemes evaluated in FP64, the reference against which each
 * storage type's field error is measured.  split = 0: the FP32 scheme
 * (orc_diffuse: decay in every substep); split = 1: the 16-bit scheme's
 * arithmetic (uptake and the step's decay (1 + lambda dt/S)^-S once, then
 * substeps without decay), so the difference of the two FP64 results is the
 * splitting error alone. */
int orc_diffuse_f64(double* f, double* tmp, const float* sink, const int32_t dims[3], double dx, double dt, double D,
                    double decay, double boundary, int substeps, int split, int nthreads) {
    const int nx = dims[0], ny = dims[1], nz = dims[2];
    const int nt = nthreads_or_all(nthreads);
    if (substeps < 1) return -1;
    const double dts = dt / substeps;
    const double r = D * dts / (dx * dx);
    const double inv_decay = split ? 1.0 : 1.0 / (1.0 + decay * dts);
    const double decay_step = split ? pow(1.0 + decay * dts, -(double)substeps) : 1.0;
    const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
    if (sink || split) {
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int z = 1; z < nz - 1; ++z)
            for (int y = 1; y < ny - 1; ++y)
                for (int x = 1; x < nx - 1; ++x) {
                    size_t v = (size_t)z * sz + (size_t)y * sy + x;
                    if (sink) f[v] = f[v] / (1.0 + (double)sink[v] * dt);
                    f[v] *= decay_step;
                }
    }
    double* cur = f;
    double* nxt = tmp;
    for (int s = 0; s < substeps; ++s) {
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y) {
                size_t row = (size_t)z * sz + (size_t)y * sy;
                for (int x = 0; x < nx; ++x) {
                    size_t v = row + x;
                    if (x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1) {
                        nxt[v] = boundary;
                        continue;
                    }
                    double c = cur[v];
                    double s2 = ((cur[v - 1] + cur[v + 1]) + (cur[v - sy] + cur[v + sy])) + (cur[v - sz] + cur[v + sz]);
                    double u = (c + r * (s2 - 6.0 * c)) * inv_decay;
                    nxt[v] = u > 0.0 ? u : 0.0;
                }
            }
        double* t = cur;
        cur = nxt;
        nxt = t;
    }
    if (cur != f) memcpy(f, cur, (size_t)nx * ny * nz * 8);
    return 0;
}

/* ------------------------------------------------------------------ contact */

/* engine/assets/shaders/tumor_sim.wgsl:505-628, overdamped (see olc_contact.cu) */
void orc_contact(const float* posr, const uint32_t* ranges, uint32_t n, const int32_t tdims[3], float tvs,
                 float stiffness, float mobility, float max_disp, float dt, const float lo[3], const float hi[3],
                 float* xo, float* yo, float* zo, int nthreads) {
    const int nt = nthreads_or_all(nthreads);
    const float md = mobility * dt;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const float* p = posr + 4 * (size_t)i;
        if (p[3] < 0.0f) continue;
        const int cx = orc_bin_coord(p[0], tvs, tdims[0]);
        const int cy = orc_bin_coord(p[1], tvs, tdims[1]);
        const int cz = orc_bin_coord(p[2], tvs, tdims[2]);
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        for (int dz = -1; dz <= 1; ++dz) {
            const int nz = cz + dz;
            if (nz < 0 || nz >= tdims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int ny = cy + dy;
                if (ny < 0 || ny >= tdims[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = cx + dx;
                    if (nx < 0 || nx >= tdims[0]) continue;
                    const uint32_t k = orc_tissue_key(nx, ny, nz);
                    const uint32_t s = ranges[2 * (size_t)k], e = ranges[2 * (size_t)k + 1];
                    for (uint32_t j = s; j < e; ++j) {
                        if (j == i) continue;
                        const float* q = posr + 4 * (size_t)j;
                        if (q[3] < 0.0f) continue;
                        const float ddx = p[0] - q[0], ddy = p[1] - q[1], ddz = p[2] - q[2];
                        const float d2 = (ddx * ddx + ddy * ddy) + ddz * ddz;
                        const float rsum = p[3] + q[3];
                        const float dist = sqrtf(d2);
                        if (!(dist < rsum)) continue;
                        const float ov = rsum - dist;
                        const float f = (stiffness * ov) * sqrtf(ov);
                        if (dist < 1e-5f) {
                            fx = fx + (i < j ? -f : f);
                        } else {
                            const float sc = f / dist;
                            fx = fx + ddx * sc;
                            fy = fy + ddy * sc;
                            fz = fz + ddz * sc;
                        }
                    }
                }
            }
        }
        float mx = fx * md, my = fy * md, mz = fz * md;
        const float len = sqrtf((mx * mx + my * my) + mz * mz);
        if (len > max_disp) {
            const float sc = max_disp / len;
            mx = mx * sc;
            my = my * sc;
            mz = mz * sc;
        }
        float nx = p[0] + mx, ny = p[1] + my, nz = p[2] + mz;
        xo[i] = fminf(fmaxf(nx, lo[0]), hi[0]);
        yo[i] = fminf(fmaxf(ny, lo[1]), hi[1]);
        zo[i] = fminf(fmaxf(nz, lo[2]), hi[2]);
    }
}

/* Restates k_contact_mech: the walk, order and rounding of orc_contact, with
 * the engine's necrotic factor and adhesion branch
 * (engine/assets/shaders/tumor_sim.wgsl:552-569) and its damped velocity
 * integration (:606-625). */
static float orc_field_at(const float* f, const int32_t d[3], int x, int y, int z) {
    return f[((size_t)z * d[1] + y) * d[0] + x];
}

/* Central difference 0.5 (f(v + e) - f(v - e)), neighbours clamped to the grid. */
static void orc_grad(const float* f, const int32_t d[3], int x, int y, int z, float g[3]) {
    const int xm = x > 0 ? x - 1 : 0, xp = x < d[0] - 1 ? x + 1 : d[0] - 1;
    const int ym = y > 0 ? y - 1 : 0, yp = y < d[1] - 1 ? y + 1 : d[1] - 1;
    const int zm = z > 0 ? z - 1 : 0, zp = z < d[2] - 1 ? z + 1 : d[2] - 1;
    g[0] = 0.5f * (orc_field_at(f, d, xp, y, z) - orc_field_at(f, d, xm, y, z));
    g[1] = 0.5f * (orc_field_at(f, d, x, yp, z) - orc_field_at(f, d, x, ym, z));
    g[2] = 0.5f * (orc_field_at(f, d, x, y, zp) - orc_field_at(f, d, x, y, zm));
}

void orc_contact_mech(const float* posr, const uint32_t* ranges, uint32_t n, const int32_t tdims[3], float tvs,
                      float stiffness, float mobility, float max_disp, float dt, const float lo[3], const float hi[3],
                      const int32_t* state, float necrotic_factor, float adh_k, float adh_range, float* vx,
                      float* vy, float* vz, float damping, float max_speed, float* xo, float* yo, float* zo,
                      int nthreads) {
    orc_contact_motion(posr, ranges, n, tdims, tvs, stiffness, mobility, max_disp, dt, lo, hi, state,
                       necrotic_factor, adh_k, adh_range, vx, vy, vz, damping, max_speed, NULL, NULL, NULL, NULL,
                       NULL, 0.0f, 0.0f, 0.0f, 0, NULL, NULL, NULL, xo, yo, zo, nthreads);
}

void orc_contact_motion(const float* posr, const uint32_t* ranges, uint32_t n, const int32_t tdims[3], float tvs,
                        float stiffness, float mobility, float max_disp, float dt, const float lo[3],
                        const float hi[3], const int32_t* state, float necrotic_factor, float adh_k,
                        float adh_range, float* vx, float* vy, float* vz, float damping, float max_speed,
                        const int32_t* species, uint32_t* rng, const float* o2, const float* glu,
                        const int32_t* cdims, float cvs, float chemo_force, float impulse, int n_species,
                        const float* sp_o2, const float* sp_glu, const float* sp_move, float* xo, float* yo,
                        float* zo, int nthreads) {
    const int nt = nthreads_or_all(nthreads);
    const int adh = adh_k != 0.0f && adh_range > 0.0f;
    const float k_nec = stiffness * necrotic_factor;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        const float* p = posr + 4 * (size_t)i;
        if (p[3] < 0.0f) continue;
        const int nec_i = state && state[i] == 3;
        const int cx = orc_bin_coord(p[0], tvs, tdims[0]);
        const int cy = orc_bin_coord(p[1], tvs, tdims[1]);
        const int cz = orc_bin_coord(p[2], tvs, tdims[2]);
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        for (int dz = -1; dz <= 1; ++dz) {
            const int nz = cz + dz;
            if (nz < 0 || nz >= tdims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int ny = cy + dy;
                if (ny < 0 || ny >= tdims[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = cx + dx;
                    if (nx < 0 || nx >= tdims[0]) continue;
                    const uint32_t k = orc_tissue_key(nx, ny, nz);
                    const uint32_t s = ranges[2 * (size_t)k], e = ranges[2 * (size_t)k + 1];
                    for (uint32_t j = s; j < e; ++j) {
                        if (j == i) continue;
                        const float* q = posr + 4 * (size_t)j;
                        if (q[3] < 0.0f) continue;
                        const float ddx = p[0] - q[0], ddy = p[1] - q[1], ddz = p[2] - q[2];
                        const float d2 = (ddx * ddx + ddy * ddy) + ddz * ddz;
                        const float rsum = p[3] + q[3];
                        const float reach = adh ? rsum + adh_range : rsum;
                        const float dist = sqrtf(d2);
                        if (!(dist < reach)) continue;
                        const int nec = nec_i || (state && state[j] == 3);
                        if (dist < rsum) {
                            const float ov = rsum - dist;
                            const float f = ((nec ? k_nec : stiffness) * ov) * sqrtf(ov);
                            if (dist < 1e-5f) {
                                fx = fx + (i < j ? -f : f);
                            } else {
                                const float sc = f / dist;
                                fx = fx + ddx * sc;
                                fy = fy + ddy * sc;
                                fz = fz + ddz * sc;
                            }
                        } else if (!nec) {
                            const float gap = dist - rsum;
                            const float fall = 0.5f * (1.0f + cosf((3.14159f * gap) / adh_range));
                            const float sc = (adh_k * fall) / dist;
                            fx = fx - ddx * sc;
                            fy = fy - ddy * sc;
                            fz = fz - ddz * sc;
                        }
                    }
                }
            }
        }
        /* active motion of a non-necrotic agent (tumor_sim.wgsl:584-604) */
        if (!nec_i && n_species > 0 && (o2 || glu || rng)) {
            int sp = species ? species[i] : 0;
            sp = sp < 0 ? 0 : (sp >= n_species ? n_species - 1 : sp);
            if (o2 || glu) {
                const int gx = orc_bin_coord(p[0], cvs, cdims[0]);
                const int gy = orc_bin_coord(p[1], cvs, cdims[1]);
                const int gz = orc_bin_coord(p[2], cvs, cdims[2]);
                float g0[3] = {0.0f, 0.0f, 0.0f}, g1[3] = {0.0f, 0.0f, 0.0f};
                if (o2) orc_grad(o2, cdims, gx, gy, gz, g0);
                if (glu) orc_grad(glu, cdims, gx, gy, gz, g1);
                fx = fx + (g0[0] * sp_o2[sp] + g1[0] * sp_glu[sp]) * chemo_force;
                fy = fy + (g0[1] * sp_o2[sp] + g1[1] * sp_glu[sp]) * chemo_force;
                fz = fz + (g0[2] * sp_o2[sp] + g1[2] * sp_glu[sp]) * chemo_force;
            }
            if (rng) {
                float r[3];
                orc_rand_dir(&rng[i], r);
                fx = fx + (r[0] * sp_move[sp]) * impulse;
                fy = fy + (r[1] * sp_move[sp]) * impulse;
                fz = fz + (r[2] * sp_move[sp]) * impulse;
            }
        }
        float mx, my, mz;
        if (!vx) {
            const float md = mobility * dt;
            mx = fx * md;
            my = fy * md;
            mz = fz * md;
            const float len = sqrtf((mx * mx + my * my) + mz * mz);
            if (len > max_disp) {
                const float sc = max_disp / len;
                mx = mx * sc;
                my = my * sc;
                mz = mz * sc;
            }
        } else {
            const float damp = nec_i ? damping * 2.0f : damping;
            float ux = vx[i], uy = vy[i], uz = vz[i];
            ux = ux + (fx - ux * damp) * dt;
            uy = uy + (fy - uy * damp) * dt;
            uz = uz + (fz - uz * damp) * dt;
            const float speed = sqrtf((ux * ux + uy * uy) + uz * uz);
            if (speed > max_speed) {
                ux = (ux / speed) * max_speed;
                uy = (uy / speed) * max_speed;
                uz = (uz / speed) * max_speed;
            }
            vx[i] = ux;
            vy[i] = uy;
            vz[i] = uz;
            mx = ux * dt;
            my = uy * dt;
            mz = uz * dt;
        }
        xo[i] = fminf(fmaxf(p[0] + mx, lo[0]), hi[0]);
        yo[i] = fminf(fmaxf(p[1] + my, lo[1]), hi[1]);
        zo[i] = fminf(fmaxf(p[2] + mz, lo[2]), hi[2]);
    }
}

/* ------------------------------------------------------------------ tumour workload */

size_t orc_tumour_sizeof(void) { return sizeof(OrcTumour); }

int orc_tumour_fields(OrcTumour* t, int nthreads) {
    if (orc_diffuse(t->o2, t->o2_tmp, t->o2_sink, t->cdims, t->cvs, t->dt, t->D_o2, 0.0f, t->bnd_o2, t->S_o2,
                    nthreads))
        return -1;
    if (t->has_drug &&
        orc_diffuse(t->drug, t->drug_tmp, NULL, t->cdims, t->cvs, t->dt, t->D_drug, t->decay_drug, t->bnd_drug,
                    t->S_drug, nthreads))
        return -1;
    return 0;
}

#define ST_PROLIF 1
#define ST_QUIESCENT 2
#define ST_NECROTIC 3

/* Grid + compaction, the tumour rule (restated from workloads.py's DSL), contact. */
int orc_tumour_agents(OrcTumour* t, int nthreads) {
    const int nt = nthreads_or_all(nthreads);
    const uint32_t rows = t->n, cap = t->cap;
    const uint32_t sentinel = orc_tissue_key(t->tdims[0], t->tdims[1], t->tdims[2]);
    uint32_t* keys = (uint32_t*)malloc((size_t)rows * 4 + 4);
    uint32_t* skeys = (uint32_t*)malloc((size_t)rows * 4 + 4);
    uint32_t* perm = (uint32_t*)malloc((size_t)rows * 4 + 4);
    uint32_t* ranges = (uint32_t*)malloc((size_t)sentinel * 8 + 8);
    if (!keys || !skeys || !perm || !ranges) return -1;

    /* keys + stable sort + compaction (template.wgsl:152-186, 335-343) */
    orc_keys(t->x, t->y, t->z, t->dead, rows, t->tdims, t->tvs, keys);
    orc_sort_pairs(keys, NULL, skeys, perm, rows);
    uint32_t dead = 0;
    for (uint32_t i = 0; i < rows; ++i) dead += t->dead[i] ? 1u : 0u;
    const uint32_t n = rows - dead;
    orc_bin_ranges(skeys, rows, sentinel, ranges);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        uint32_t i = (uint32_t)ii, s = perm[i];
        t->x2[i] = t->x[s];
        t->y2[i] = t->y[s];
        t->z2[i] = t->z[s];
        t->radius2[i] = t->radius[s];
        t->volume2[i] = t->volume[s];
        t->state2[i] = t->state[s];
        t->rng2[i] = t->rng[s];
    }
#define SWAPP(a, b)     \
    do {                \
        void* _t = (a); \
        (a) = (b);      \
        (b) = _t;       \
    } while (0)
    SWAPP(t->x, t->x2);
    SWAPP(t->y, t->y2);
    SWAPP(t->z, t->z2);
    SWAPP(t->radius, t->radius2);
    SWAPP(t->volume, t->volume2);
    SWAPP(t->state, t->state2);
    SWAPP(t->rng, t->rng2);
    memset(t->dead, 0, rows ? rows : 1);
    t->deaths = dead;

    /* the rule, per agent */
    int32_t* dep = (int32_t*)malloc((size_t)n * 4 + 4);
    uint8_t* born = (uint8_t*)malloc((size_t)n + 1);
    float* child = (float*)malloc((size_t)n * 16 + 16); /* x y z volume */
    uint32_t* child_rng = (uint32_t*)malloc((size_t)n * 4 + 4);
    const float* o2f = t->o2;
    const float* drugf = t->drug;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        dep[i] = -1;
        born[i] = 0;
        if (t->state[i] == ST_NECROTIC) continue;
        const int cx = orc_bin_coord(t->x[i], t->cvs, t->cdims[0]);
        const int cy = orc_bin_coord(t->y[i], t->cvs, t->cdims[1]);
        const int cz = orc_bin_coord(t->z[i], t->cvs, t->cdims[2]);
        const size_t idx = ((size_t)cz * t->cdims[1] + cy) * t->cdims[0] + cx;
        const float o2 = o2f[idx];
        if (o2 <= t->o2_necrotic) {
            t->state[i] = ST_NECROTIC;
            continue;
        }
        uint32_t rng = t->rng[i];
        if (t->death_k > 0.0f) {
            float rr = orc_next_rand(&rng);
            if (rr < t->death_k * drugf[idx]) {
                t->dead[i] = 1;
                t->rng[i] = rng;
                continue;
            }
        }
        dep[i] = (int32_t)idx;
        if (o2 <= t->o2_quiescent) {
            t->state[i] = ST_QUIESCENT;
            t->rng[i] = rng;
            continue;
        }
        t->state[i] = ST_PROLIF;
        float v = t->volume[i];
        v = v + (t->growth * v) * t->dt;
        t->volume[i] = v;
        if (v > t->v_div) {
            const float half = v * 0.5f;
            t->volume[i] = half;
            float d[3];
            orc_rand_dir(&rng, d);
            const float hr = t->radius[i] * 0.5f;
            const float ox = d[0] * hr, oy = d[1] * hr, oz = d[2] * hr;
            child[4 * (size_t)i + 0] = t->x[i] + ox;
            child[4 * (size_t)i + 1] = t->y[i] + oy;
            child[4 * (size_t)i + 2] = t->z[i] + oz;
            child[4 * (size_t)i + 3] = half;
            t->x[i] = t->x[i] - ox;
            t->y[i] = t->y[i] - oy;
            t->z[i] = t->z[i] - oz;
            child_rng[i] = rng ^ 0x12345678u;
            born[i] = 1;
        }
        t->rng[i] = rng;
    }
    /* uptake deposits (equal rates, so any summation order gives these bits) */
    for (uint32_t i = 0; i < n; ++i)
        if (dep[i] >= 0) t->o2_sink[dep[i]] += t->uptake;
    /* births at n + exclusive scan of birth flags in parent order */
    uint32_t b = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!born[i]) continue;
        uint32_t slot = n + b;
        if (slot < cap) {
            t->x[slot] = child[4 * (size_t)i + 0];
            t->y[slot] = child[4 * (size_t)i + 1];
            t->z[slot] = child[4 * (size_t)i + 2];
            t->volume[slot] = child[4 * (size_t)i + 3];
            t->radius[slot] = t->radius[i];
            t->state[slot] = ST_PROLIF;
            t->rng[slot] = child_rng[i];
            t->dead[slot] = 0;
            ++b;
        }
    }
    t->births = b;
    /* contact over the live rows with post-rule positions (dead: radius -1) */
    float* posr = (float*)malloc((size_t)n * 16 + 16);
    for (uint32_t i = 0; i < n; ++i) {
        posr[4 * (size_t)i + 0] = t->x[i];
        posr[4 * (size_t)i + 1] = t->y[i];
        posr[4 * (size_t)i + 2] = t->z[i];
        posr[4 * (size_t)i + 3] = t->dead[i] ? -1.0f : t->radius[i];
    }
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = t->lo[k] + t->margin;
        hi[k] = t->hi[k] - t->margin;
    }
    orc_contact(posr, ranges, n, t->tdims, t->tvs, t->stiffness, t->mobility, t->max_disp, t->dt, lo, hi, t->x,
                t->y, t->z, nt);
    t->n = n + b;
    free(posr);
    free(dep);
    free(born);
    free(child);
    free(child_rng);
    free(keys);
    free(skeys);
    free(perm);
    free(ranges);
    return 0;
}

int orc_tumour_step(OrcTumour* t, int nthreads) {
    if (orc_tumour_fields(t, nthreads)) return -1;
    return orc_tumour_agents(t, nthreads);
}
