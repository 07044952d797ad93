// Runtime for rule kernels: the argument block every rule kernel receives and
// the device functions the translated rule bodies call.  Compiled twice: by
// nvcc into libolc.so (for the layout of OlcRuleParams) and by NVRTC together
// with the CUDA C that oncolytica_b200.compiler emits for a model.
//
// Reference semantics restated:
//   * per-agent rule wrapper: load agent, local RNG, body, store RNG, write
//     the Out buffer (framework/src/oncolytica/gpu/compiler/_shader_builder.py:207-221)
//   * die() removes the agent at the next sort; divide() appends a child
//     (framework/src/oncolytica/gpu/compiler/translator/_stmt_translator.py:431-453),
//     here at a deterministic slot: rows + exclusive scan of births in parent order.
//   * Moore neighbourhood of the agent's bin, out-of-range bins skipped, self
//     skipped (_stmt_translator.py:459-491; offsets template.wgsl:11-21).
//   * chemistry_at / tissue_at: nearest voxel, clamped to the grid
//     (framework/src/oncolytica/core/utils/_types.py:314-346).
#pragma once
#include "olc_device.cuh"

#define OLC_MAX_AGENT_COLS 64
#define OLC_MAX_FIELD_COLS 8
#define OLC_MAX_RULE_KERNELS 16

// Device counter block (u32 words).
#define OLC_CTR_N          0    // live agents after this step's sort
#define OLC_CTR_DEAD       1    // dead rows removed by this step's sort
#define OLC_CTR_STATUS     2    // sticky OLC_ST_* bits
#define OLC_CTR_DEAD_TMP   3    // dead rows counted by the key kernel
#define OLC_CTR_ROWS       4    // rows entering this step's sort (live + dead)
#define OLC_CTR_FIELD_STEP 5    // steps whose grid stage has run (salt of stochastic rounding)
#define OLC_CTR_SORT_TILE  8    // 4 words: tile counters of the sort passes
#define OLC_CTR_RULE_TILE  12   // OLC_MAX_RULE_KERNELS words: tile counters
#define OLC_CTR_BIRTHS     28   // OLC_MAX_RULE_KERNELS words: births per rule
#define OLC_CTR_AGENT_STEPS 60  // 2 words (u64): sum of N over steps
#define OLC_CTR_WORDS      64

#define OLC_RULE_THREADS 256

// Batched mode: one record per simulation, in device memory.  Every
// simulation of a batch runs the same model; geometry, parameters, metric
// accumulators, field grids and bin table differ.
struct OlcSimDesc {
    int tdims[3];
    float tvs;
    int cdims[3];
    float cvs;
    float lo[3];                   // contact clamp box (domain shrunk by the margin)
    float hi[3];
    float center[3];               // radial-profile centre
    float bin_width;               // radial-profile bin width
    olc_u32 ranges_base;           // first entry of this simulation in the shared bin table
    olc_u32 params_off;            // bytes into the params blob
    olc_u32 metrics_off;           // bytes into the metric accumulators
    olc_u32 substeps_mask;         // bit f: field f takes an odd number of substeps
    olc_u32 step_base;             // handle steps run before this simulation joined (serving pool)
    unsigned long long field_off;  // first voxel of this simulation in every field buffer
};

struct OlcRuleParams {
    const void* in[OLC_MAX_AGENT_COLS];
    void* out[OLC_MAX_AGENT_COLS];
    const void* field[OLC_MAX_FIELD_COLS];  // current grid of each field (storage per field_type)
    float* sink[OLC_MAX_FIELD_COLS];
    const olc_u32* ranges;        // bin table, 2 words per key
    unsigned char* life;          // 0 alive, 1 dead (removed at the next sort)
    float4* posr;                 // (x, y, z, radius) for the contact pass, or null
    olc_u32* counters;            // OLC_CTR_* block
    olc_u32* birth_lb;            // look-back words of this rule kernel
    const unsigned char* params;  // Params blob
    void* metrics;                // metric accumulators
    const unsigned char* tissue;  // tissue grid columns (Morton-indexed), or null
    int tdims[3];
    float tvs;
    int cdims[3];
    float cvs;
    olc_u32 capacity;
    olc_u32 n_cols;
    int radius_col;
    float radius_const;
    int rule_index;
    int n_tissue_cols;
    olc_u32 tissue_stride;        // bytes between tissue columns
    int pad;
    // batched mode (sims != null): per-simulation records, the agent-column
    // tables in device memory, the second buffer of every field and the
    // buffer parity of every (simulation, field)
    const OlcSimDesc* sims;
    const void* const* cols_in;
    void* const* cols_out;
    const void* field_alt[OLC_MAX_FIELD_COLS];
    const unsigned char* fpar;
    int n_fields;
    int sim_col;
    int field_type[OLC_MAX_FIELD_COLS];  // OLC_FIELD_* storage | (OLC_ENC_* << 8)
    float field_bval[OLC_MAX_FIELD_COLS];  // boundary value (the encodings' b)
    // tissue / chemistry rules: the buffers a voxel rule writes; it reads
    // `tissue` and `field` (the state before the rule: every voxel sees its
    // neighbours' previous values)
    unsigned char* tissue_out;
    void* field_out[OLC_MAX_FIELD_COLS];
    // batched chemistry rules: the members' field tiles (member, tile x, y, z
    // of vtile[0] x vtile[1] x vtile[2] voxels) a voxel kernel walks
    const uint4* vtiles;
    olc_u32 n_vtiles;
    int vtile[3];
};

// What a rule body sees of one simulation of a batch (batched mode).  Member
// names follow OlcRuleParams, so the same helpers serve both.
struct OlcSimView {
    const void* const* in;
    void* const* out;
    const void* field[OLC_MAX_FIELD_COLS];
    int field_type[OLC_MAX_FIELD_COLS];
    float field_bval[OLC_MAX_FIELD_COLS];
    void* field_out[OLC_MAX_FIELD_COLS];  // the member's other buffer (chemistry rules write it)
    float* sink[OLC_MAX_FIELD_COLS];
    const olc_u32* ranges;
    float4* posr;
    const unsigned char* params;
    void* metrics;
    const unsigned char* tissue;
    int tdims[3];
    float tvs;
    int cdims[3];
    float cvs;
    int n_tissue_cols;
    olc_u32 tissue_stride;
};

__device__ __forceinline__ OlcSimView olc_sim_view(const OlcRuleParams& P, olc_u32 sim) {
    const OlcSimDesc& d = P.sims[sim];
    OlcSimView V;
    V.in = P.cols_in;
    V.out = P.cols_out;
#pragma unroll
    for (int f = 0; f < OLC_MAX_FIELD_COLS; ++f) {
        const bool alt = f < P.n_fields && P.fpar[sim * (olc_u32)P.n_fields + f] != 0;
        const unsigned char* base = static_cast<const unsigned char*>(alt ? P.field_alt[f] : P.field[f]);
        V.field_type[f] = P.field_type[f];
        V.field_bval[f] = P.field_bval[f];
        V.field[f] = base ? base + d.field_off * (P.field_type[f] ? 2u : 4u) : nullptr;
        unsigned char* other = static_cast<unsigned char*>(const_cast<void*>(alt ? P.field[f] : P.field_alt[f]));
        V.field_out[f] = other ? other + d.field_off * (P.field_type[f] ? 2u : 4u) : nullptr;
        V.sink[f] = P.sink[f] ? P.sink[f] + d.field_off : nullptr;
    }
    V.ranges = P.ranges + 2ull * d.ranges_base;
    V.posr = P.posr;
    V.params = P.params + d.params_off;
    V.metrics = static_cast<unsigned char*>(P.metrics) + d.metrics_off;
    V.tissue = nullptr;  // tissue grids are not bound in batched mode
    for (int k = 0; k < 3; ++k) {
        V.tdims[k] = d.tdims[k];
        V.cdims[k] = d.cdims[k];
    }
    V.tvs = d.tvs;
    V.cvs = d.cvs;
    V.n_tissue_cols = 0;
    V.tissue_stride = 0;
    return V;
}

// Rows processed by rule kernel k: live agents plus children of earlier rules.
__device__ __forceinline__ olc_u32 olc_rule_rows(const olc_u32* ctr, int k) {
    olc_u32 r = ctr[OLC_CTR_N];
    for (int j = 0; j < k; ++j) r += ctr[OLC_CTR_BIRTHS + j];
    return r;
}

// Rows in use after all rules of the step (children are stored only below
// the capacity, so the sum never exceeds it).
__device__ __forceinline__ olc_u32 olc_total_rows(const olc_u32* ctr) {
    olc_u32 r = ctr[OLC_CTR_N];
    for (int j = 0; j < OLC_MAX_RULE_KERNELS; ++j) r += ctr[OLC_CTR_BIRTHS + j];
    return r;
}

// ------------------------------------------------------------- vector helpers
struct olc_vec3 {
    float x, y, z;
};
struct olc_ivec3 {
    int x, y, z;
};

__device__ __forceinline__ olc_vec3 olc_v3(float x, float y, float z) { olc_vec3 v; v.x = x; v.y = y; v.z = z; return v; }
__device__ __forceinline__ olc_ivec3 olc_iv3(int x, int y, int z) { olc_ivec3 v; v.x = x; v.y = y; v.z = z; return v; }
__device__ __forceinline__ olc_vec3 operator+(olc_vec3 a, olc_vec3 b) { return olc_v3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ olc_vec3 operator-(olc_vec3 a, olc_vec3 b) { return olc_v3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ olc_vec3 operator*(olc_vec3 a, olc_vec3 b) { return olc_v3(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z)); }
__device__ __forceinline__ olc_vec3 operator*(olc_vec3 a, float s) { return olc_v3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)); }
__device__ __forceinline__ olc_vec3 operator*(float s, olc_vec3 a) { return olc_v3(__fmul_rn(s, a.x), __fmul_rn(s, a.y), __fmul_rn(s, a.z)); }
__device__ __forceinline__ olc_vec3 operator/(olc_vec3 a, float s) { return olc_v3(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)); }
__device__ __forceinline__ olc_vec3 operator-(olc_vec3 a) { return olc_v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ bool operator==(olc_vec3 a, olc_vec3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
__device__ __forceinline__ bool operator!=(olc_vec3 a, olc_vec3 b) { return !(a == b); }
__device__ __forceinline__ olc_ivec3 operator+(olc_ivec3 a, olc_ivec3 b) { return olc_iv3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ olc_ivec3 operator-(olc_ivec3 a, olc_ivec3 b) { return olc_iv3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ olc_ivec3 operator*(olc_ivec3 a, olc_ivec3 b) { return olc_iv3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ olc_ivec3 operator*(olc_ivec3 a, int s) { return olc_iv3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ olc_ivec3 operator*(int s, olc_ivec3 a) { return olc_iv3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ olc_ivec3 operator-(olc_ivec3 a) { return olc_iv3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ bool operator==(olc_ivec3 a, olc_ivec3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
__device__ __forceinline__ bool operator!=(olc_ivec3 a, olc_ivec3 b) { return !(a == b); }

// ------------------------------------------------------------- ol.math
// Each helper evaluates its formula with separately rounded IEEE operations,
// so results match a float32 CPU evaluation of the same formula.
__device__ __forceinline__ float olc_dot(olc_vec3 a, olc_vec3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float olc_length_sq(olc_vec3 v) { return olc_dot(v, v); }
__device__ __forceinline__ float olc_length(olc_vec3 v) { return sqrtf(olc_dot(v, v)); }
__device__ __forceinline__ float olc_distance_sq(olc_vec3 a, olc_vec3 b) { return olc_length_sq(a - b); }
__device__ __forceinline__ float olc_distance(olc_vec3 a, olc_vec3 b) { return olc_length(a - b); }
__device__ __forceinline__ olc_vec3 olc_normalize(olc_vec3 v) {
    float n = olc_length(v);
    if (n == 0.0f) return olc_v3(0.0f, 0.0f, 0.0f);
    float inv = __fdiv_rn(1.0f, n);
    return v * inv;
}
__device__ __forceinline__ olc_vec3 olc_cross(olc_vec3 a, olc_vec3 b) {
    return olc_v3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
                  __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
                  __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ olc_vec3 olc_reflect(olc_vec3 v, olc_vec3 n) {
    float d = __fmul_rn(2.0f, olc_dot(v, n));
    return v - n * d;
}
__device__ __forceinline__ float olc_lerp(float a, float b, float t) { return __fadd_rn(a, __fmul_rn(__fsub_rn(b, a), t)); }
__device__ __forceinline__ olc_vec3 olc_lerp_vec(olc_vec3 a, olc_vec3 b, float t) {
    float it = __fsub_rn(1.0f, t);
    return olc_v3(__fadd_rn(__fmul_rn(a.x, it), __fmul_rn(b.x, t)),
                  __fadd_rn(__fmul_rn(a.y, it), __fmul_rn(b.y, t)),
                  __fadd_rn(__fmul_rn(a.z, it), __fmul_rn(b.z, t)));
}
__device__ __forceinline__ float olc_clampf(float v, float lo, float hi) { return fmaxf(lo, fminf(hi, v)); }
__device__ __forceinline__ int olc_clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ olc_vec3 olc_clampv(olc_vec3 v, olc_vec3 lo, olc_vec3 hi) {
    return olc_v3(olc_clampf(v.x, lo.x, hi.x), olc_clampf(v.y, lo.y, hi.y), olc_clampf(v.z, lo.z, hi.z));
}
__device__ __forceinline__ float olc_sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ int olc_signi(int x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }
__device__ __forceinline__ float olc_smoothstep(float e0, float e1, float x) {
    float t = olc_clampf(__fdiv_rn(__fsub_rn(x, e0), __fsub_rn(e1, e0)), 0.0f, 1.0f);
    return __fmul_rn(__fmul_rn(t, t), __fsub_rn(3.0f, __fmul_rn(2.0f, t)));
}
__device__ __forceinline__ float olc_step_fn(float edge, float x) { return x < edge ? 0.0f : 1.0f; }
__device__ __forceinline__ float olc_fract(float x) { return __fsub_rn(x, floorf(x)); }
// Python semantics for // and % on integers and floats.
__device__ __forceinline__ int olc_floordiv_i(int a, int b) {
    int q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
    return q;
}
__device__ __forceinline__ int olc_mod_i(int a, int b) {
    int r = a % b;
    if (r != 0 && ((r < 0) != (b < 0))) r += b;
    return r;
}
__device__ __forceinline__ float olc_floordiv_f(float a, float b) { return floorf(__fdiv_rn(a, b)); }
__device__ __forceinline__ float olc_mod_f(float a, float b) {
    float r = fmodf(a, b);
    if (r != 0.0f && ((r < 0.0f) != (b < 0.0f))) r = __fadd_rn(r, b);
    return r;
}

// ------------------------------------------------------------- grid lookups
template <class PT>
__device__ __forceinline__ olc_u32 olc_chem_index(const PT& P, olc_vec3 p) {
    int cx = olc_bin_coord(p.x, P.cvs, P.cdims[0]);
    int cy = olc_bin_coord(p.y, P.cvs, P.cdims[1]);
    int cz = olc_bin_coord(p.z, P.cvs, P.cdims[2]);
    return ((olc_u32)cz * (olc_u32)P.cdims[1] + (olc_u32)cy) * (olc_u32)P.cdims[0] + (olc_u32)cx;
}

template <class PT>
__device__ __forceinline__ olc_u32 olc_tissue_index(const PT& P, olc_vec3 p) {
    int tx = olc_bin_coord(p.x, P.tvs, P.tdims[0]);
    int ty = olc_bin_coord(p.y, P.tvs, P.tdims[1]);
    int tz = olc_bin_coord(p.z, P.tvs, P.tdims[2]);
    return olc_tissue_key(tx, ty, tz);
}

template <class PT>
__device__ __forceinline__ olc_ivec3 olc_tissue_coord(const PT& P, olc_vec3 p) {
    return olc_iv3(olc_bin_coord(p.x, P.tvs, P.tdims[0]), olc_bin_coord(p.y, P.tvs, P.tdims[1]),
                   olc_bin_coord(p.z, P.tvs, P.tdims[2]));
}

// 16-bit field storage: BF16 is the top half of an FP32 pattern; FP16 is
// widened with the exact PTX conversion.
__device__ __forceinline__ float olc_bf16_to_float(unsigned short h) { return __uint_as_float((olc_u32)h << 16); }
__device__ __forceinline__ float olc_f16_to_float(unsigned short h) {
    float f;
    asm("{ .reg .b16 t; mov.b16 t, %1; cvt.f32.f16 %0, t; }" : "=f"(f) : "h"(h));
    return f;
}

// Value of one 16-bit element of a field with type word t = storage |
// (encoding << 8) and boundary value b.  Storage 2 and 4 are FP16, 1 and 3
// BF16; encodings (olc.h OLC_ENC_*): 0 the value, 1 the deficit b - value,
// 2 the value minus an offset in {0, b/2, b} named by bits 15 and 14.
__device__ __forceinline__ float olc_field16_value(unsigned short h, int t, float b) {
    const int st = t & 0xff, en = t >> 8;
    const bool f16 = st == 2 || st == 4;
    if (en == 2) {
        const unsigned short mh = (unsigned short)(h & 0xBFFFu);
        const float m = f16 ? olc_f16_to_float(mh) : olc_bf16_to_float(mh);
        const olc_u32 units = (olc_u32)(h >> 15) + (olc_u32)((h >> 14) & 1u);
        return __fadd_rn(m, __fmul_rn((float)units, __fmul_rn(0.5f, b)));
    }
    const float v = f16 ? olc_f16_to_float(h) : olc_bf16_to_float(h);
    return en == 1 ? __fsub_rn(b, v) : v;
}

// Value at voxel v of a field in any storage (type word and boundary as above).
__device__ __forceinline__ float olc_field_value(const void* p, int t, float b, olc_u32 v) {
    if (t == 0) return static_cast<const float*>(p)[v];
    return olc_field16_value(static_cast<const unsigned short*>(p)[v], t, b);
}

// Field value at voxel v of field f, whatever its storage.
template <class PT>
__device__ __forceinline__ float olc_field_at(const PT& P, int f, olc_u32 v) {
    const void* p = P.field[f];
    if (!p) return 0.0f;
    return olc_field_value(p, P.field_type[f], P.field_bval[f], v);
}

// Deposit into a field's sink (sum of first-order uptake rates of a voxel).
template <class PT>
__device__ __forceinline__ void olc_deposit(const PT& P, int field, olc_vec3 p, float rate) {
    float* s = P.sink[field];
    if (s) atomicAdd(s + olc_chem_index(P, p), rate);
}

template <typename T, class PT>
__device__ __forceinline__ T olc_param(const PT& P, int offset) {
    return *reinterpret_cast<const T*>(P.params + offset);
}

template <typename T, class PT>
__device__ __forceinline__ T olc_col_in(const PT& P, int col, olc_u32 i) {
    return reinterpret_cast<const T*>(P.in[col])[i];
}

template <typename T, class PT>
__device__ __forceinline__ void olc_col_out(const PT& P, int col, olc_u32 i, T v) {
    reinterpret_cast<T*>(P.out[col])[i] = v;
}

template <typename T, class PT>
__device__ __forceinline__ T olc_tissue_col(const PT& P, int col, olc_u32 key) {
    return reinterpret_cast<const T*>(P.tissue + (size_t)col * P.tissue_stride)[key];
}
template <typename T>
__device__ __forceinline__ void olc_tissue_col_out(const OlcRuleParams& P, int col, olc_u32 key, T v) {
    reinterpret_cast<T*>(P.tissue_out + (size_t)col * P.tissue_stride)[key] = v;
}
// Chemistry rules: FP32 fields only (the host checks the storage).
__device__ __forceinline__ float olc_field_in(const OlcRuleParams& P, int f, olc_u32 v) {
    return static_cast<const float*>(P.field[f])[v];
}
template <class PT>
__device__ __forceinline__ void olc_field_out(const PT& P, int f, olc_u32 v, float x) {
    static_cast<float*>(P.field_out[f])[v] = x;
}

// Metric accumulators: one 4-byte word per metric field.  Integer adds are
// reduced across the converged lanes that target the same word first (in a
// batch, lanes of one warp can belong to different simulations), so each
// group issues one atomic.
template <class PT>
__device__ __forceinline__ void olc_metric_add_i(const PT& P, int slot, int v) {
    int* dst = reinterpret_cast<int*>(P.metrics) + slot;
    const olc_u32 m = __match_any_sync(__activemask(), reinterpret_cast<unsigned long long>(dst));
    const int s = __reduce_add_sync(m, v);
    if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && s != 0) atomicAdd(dst, s);
}
template <class PT>
__device__ __forceinline__ void olc_metric_add_u(const PT& P, int slot, olc_u32 v) {
    olc_u32* dst = reinterpret_cast<olc_u32*>(P.metrics) + slot;
    const olc_u32 m = __match_any_sync(__activemask(), reinterpret_cast<unsigned long long>(dst));
    const olc_u32 s = __reduce_add_sync(m, v);
    if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && s != 0u) atomicAdd(dst, s);
}
template <class PT>
__device__ __forceinline__ void olc_metric_add_f(const PT& P, int slot, float v) {
    if (v != 0.0f) atomicAdd(reinterpret_cast<float*>(P.metrics) + slot, v);
}

#ifdef OLC_SOLO_METRIC_WORDS
// Solo handles: every lane of a block adds to the same words, so a metric
// rule accumulates into the block's words in shared memory (its kernel clears
// them first and adds them to the handle's words once at its end); integer
// adds are still reduced across the converged lanes first.
__shared__ olc_u32 olc_s_metrics[OLC_SOLO_METRIC_WORDS];
__device__ __forceinline__ void olc_metric_add_i(const OlcRuleParams&, int slot, int v) {
    const olc_u32 m = __activemask();
    const int s = __reduce_add_sync(m, v);
    if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && s != 0) atomicAdd(reinterpret_cast<int*>(olc_s_metrics) + slot, s);
}
__device__ __forceinline__ void olc_metric_add_u(const OlcRuleParams&, int slot, olc_u32 v) {
    const olc_u32 m = __activemask();
    const olc_u32 s = __reduce_add_sync(m, v);
    if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && s != 0u) atomicAdd(olc_s_metrics + slot, s);
}
__device__ __forceinline__ void olc_metric_add_f(const OlcRuleParams&, int slot, float v) {
    if (v != 0.0f) atomicAdd(reinterpret_cast<float*>(olc_s_metrics) + slot, v);
}
#endif

// Block-wide birth scan + decoupled look-back.  Returns the row of this
// thread's child (or 0xffffffff when it has none).  All threads must call it.
__device__ __forceinline__ olc_u32 olc_birth_slot(const OlcRuleParams& P, bool born, olc_u32 tile,
                                                  olc_u32 base_rows, olc_u32* s_warp, olc_u32* s_excl) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    olc_u32 ballot = __ballot_sync(0xffffffffu, born);
    olc_u32 before = __popc(ballot & ((1u << lane) - 1u));
    if (lane == 0) s_warp[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
        olc_u32 total = 0;
        for (int w = 0; w < OLC_RULE_THREADS / 32; ++w) {
            olc_u32 c = s_warp[w];
            s_warp[w] = total;
            total += c;
        }
        olc_u32 excl = olc_lookback(P.birth_lb, 1u, tile, total, P.counters + OLC_CTR_STATUS);
        // Children past the capacity are dropped (and flagged); only stored
        // children count, so the row count never exceeds the capacity.
        olc_u32 first = base_rows + excl;
        olc_u32 room = P.capacity > first ? P.capacity - first : 0u;
        olc_u32 stored = total < room ? total : room;
        if (stored) atomicAdd(P.counters + OLC_CTR_BIRTHS + P.rule_index, stored);
        if (stored < total) atomicOr(P.counters + OLC_CTR_STATUS, OLC_ST_CAPACITY);
        *s_excl = excl;
    }
    __syncthreads();
    olc_u32 slot = base_rows + *s_excl + s_warp[warp] + before;
    return born ? slot : 0xffffffffu;
}
