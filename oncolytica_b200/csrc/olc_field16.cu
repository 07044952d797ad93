// Diffusion-reaction of a field stored as BF16 or FP16 (the precision tier;
// no counterpart in the reference, whose fields are FP32 textures).
//
// Per step:
//   reaction  (once):  v = f + comp;  v /= 1 + K dt (uptake, if any);
//                      v *= (1 + lambda dt/S)^-S (the step's decay);
//                      f = round16(v);  comp = v - f          (FP32, RN-even)
//   diffusion (S substeps): c' = round16(max(c + r (S6 - 6 c), 0)) with the
//                      sum S6 = ((xm + xp) + (ym + yp)) + (zm + zp) in FP32;
//                      outer faces pinned to round16(boundary); round16 is to
//                      nearest even, or stochastic for OLC_FIELD_BF16_SR and
//                      OLC_FIELD_F16_SR
//                      (hash bits of voxel, step, substep and field).
// comp carries each voxel's rounding residual of the reaction into the next
// step (compensated summation), so small uptake and decay terms are not lost
// to the 8- or 11-bit mantissa.  The substeps round every result; their
// error is what the FP64 comparison reports.  Every operation is separately
// rounded, so the CPU restatement reproduces the bits.
#include "olc_internal.h"
#include "olc_stencil.cuh"
#include "olc_store16.cuh"

#include <cuda.h>

namespace olc {

namespace {

__device__ __forceinline__ olc_u32 smem_addr(const void* p) {
    return static_cast<olc_u32>(__cvta_generic_to_shared(p));
}


}  // namespace

// The encoding constants of a field step.
__host__ __device__ __forceinline__ EncConst enc_const(const FieldStep& fs) {
    EncConst k;
    k.b = fs.bval;
    k.half_b = fs.half_b;
    k.quarter_b = fs.quarter_b;
    k.upper_q = fs.upper_q;
    return k;
}

// ------------------------------------------------------------------ reaction
template <int ST, int EN>
__global__ void __launch_bounds__(256) k_react16(unsigned short* __restrict__ f, float* __restrict__ K,
                                                 float* __restrict__ comp, const FieldStep fs) {
    const int nx = fs.dims[0], ny = fs.dims[1], nz = fs.dims[2];
    const size_t nvox = (size_t)nx * ny * nz;
    const EncConst ek = enc_const(fs);
    const bool aligned = ((reinterpret_cast<uintptr_t>(f) & 7u) | (reinterpret_cast<uintptr_t>(comp) & 15u) |
                          (reinterpret_cast<uintptr_t>(K) & 15u)) == 0u;
    if ((nx & 3) == 0 && aligned) {
        // four voxels of one row per thread, 8- and 16-byte accesses; the
        // arithmetic per voxel is the scalar loop's below
        const size_t nq = nvox / 4;
        for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nq; q += (size_t)gridDim.x * blockDim.x) {
            const size_t v0 = 4 * q;
            const int x0 = (int)(v0 % (size_t)nx);
            const size_t t = v0 / (size_t)nx;
            const int y = (int)(t % (size_t)ny);
            const int z = (int)(t / (size_t)ny);
            const bool face_yz = y == 0 || z == 0 || y == ny - 1 || z == nz - 1;
            float kv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (K) {
                const float4 k4 = *reinterpret_cast<const float4*>(K + v0);
                kv[0] = k4.x;
                kv[1] = k4.y;
                kv[2] = k4.z;
                kv[3] = k4.w;
                if (k4.x != 0.0f || k4.y != 0.0f || k4.z != 0.0f || k4.w != 0.0f)
                    *reinterpret_cast<float4*>(K + v0) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
            if (face_yz) continue;
            const uint2 h2 = *reinterpret_cast<const uint2*>(f + v0);
            const float4 c4 = *reinterpret_cast<const float4*>(comp + v0);
            unsigned short h[4] = {(unsigned short)(h2.x & 0xffffu), (unsigned short)(h2.x >> 16),
                                   (unsigned short)(h2.y & 0xffffu), (unsigned short)(h2.y >> 16)};
            float c[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int x = x0 + e;
                if (x == 0 || x == nx - 1) continue;
                react_voxel<ST, EN>(h[e], c[e], kv[e], fs, ek);
            }
            *reinterpret_cast<uint2*>(f + v0) =
                make_uint2((olc_u32)h[0] | ((olc_u32)h[1] << 16), (olc_u32)h[2] | ((olc_u32)h[3] << 16));
            *reinterpret_cast<float4*>(comp + v0) = make_float4(c[0], c[1], c[2], c[3]);
        }
        return;
    }
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < nvox; v += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(v % (size_t)nx);
        const size_t t = v / (size_t)nx;
        const int y = (int)(t % (size_t)ny);
        const int z = (int)(t / (size_t)ny);
        const bool face = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
        float k = 0.0f;
        if (K) {
            k = K[v];
            if (k != 0.0f) K[v] = 0.0f;
        }
        if (face) continue;
        unsigned short h = f[v];
        float c = comp[v];
        react_voxel<ST, EN>(h, c, k, fs, ek);
        f[v] = h;
        comp[v] = c;
    }
}

void launch_react16(void* f, float* sink, float* comp, const FieldStep& fs, cudaStream_t s) {
    const size_t nvox = (size_t)fs.dims[0] * fs.dims[1] * fs.dims[2];
    size_t blocks = (nvox + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    with_storage16(fs.storage, fs.encoding, [&](auto st, auto en) {
        k_react16<BaseOf<decltype(st)::value>::value, decltype(en)::value>
            <<<(unsigned)blocks, 256, 0, s>>>(static_cast<unsigned short*>(f), sink, comp, fs);
    });
}

// ------------------------------------------------------------------ diffusion substep
// The TMA tile of k_substep_x4 on 16-bit storage, eight voxels per thread: a
// CTA of 8 x TYR threads owns a 64 x TYR x TZ block; the TMA box is
// 80 x (TYR+2) x (TZ+2) elements with x starting 8 columns early (16-byte
// alignment of 2-byte elements).  Per eight voxels a thread issues 16-byte
// shared loads of the centre, y and z rows, two 2-byte loads of the x
// neighbours and one 16-byte store, as many instructions per byte as the
// 4-wide FP32 kernel.
namespace t16 {
constexpr int TX = 64, HX = 8, WX = TX + 2 * HX;  // 80 elements, 160 bytes
constexpr int TYR = 16, TZ = 8, WY = TYR + 2, WZ = TZ + 2;
constexpr int THREADS = 8 * TYR;
constexpr unsigned BYTES = WX * WY * WZ * 2;
constexpr size_t SMEM = BYTES + 16 + 128;
}  // namespace t16

// The working value the Dirichlet faces hold (OLC_ENC_*): the boundary as
// stored, its deficit 0, or b itself (OLC_ENC_OFFSET3 stores it exactly).
template <int ST, int EN>
__device__ __forceinline__ float face_work(float bval) {
    if (EN == OLC_ENC_DEFICIT) return 0.0f;
    if (EN == OLC_ENC_OFFSET3) return bval;
    return Store16<ST>::to_f(Store16<ST>::from_f(bval));
}

// The 64 x TYR x TZ output block at (x0, y0, z0) from its staged 16-bit box
// (stochastic-rounding key given), on the working values of encoding EN.
template <int ST, int EN>
__device__ __forceinline__ void t16_tile(const unsigned short* tile, unsigned short* __restrict__ out, int x0, int y0,
                                         int z0, int nx, int ny, int nz, const FieldStep& fs, olc_u32 key) {
    using namespace t16;
    const int g = threadIdx.x & 7, ty = threadIdx.x >> 3;
    const int x = x0 + 8 * g, y = y0 + ty;
    // lanes past the grid still load (inside the box), but store nothing
    const bool active = x < nx && y < ny;
    const EncConst k = enc_const(fs);
    const float r = fs.r, inv_decay = fs.inv_decay, dec_sub = fs.dec_sub;
    const bool edge_y = y == 0 || y == ny - 1;
    const bool ex0 = x == 0, ex7 = x + 7 == nx - 1;
    constexpr int PS = WY * WX;
    const unsigned short* col = tile + (ty + 1) * WX + HX + 8 * g;
    float zm[8], c[8], zp[8], ym[8], yp[8], v[8];
    load8w<ST, EN>(col, zm, k);
    load8w<ST, EN>(col + PS, c, k);
    const size_t sz = (size_t)nx * ny;
    unsigned short* o = out + (size_t)z0 * sz + (size_t)y * nx + x;
    const float bf = face_work<ST, EN>(fs.bval);
    unsigned long long vi = (unsigned long long)z0 * sz + (unsigned long long)y * nx + x;
#pragma unroll
    for (int lz = 1; lz <= TZ; ++lz) {
        const int z = z0 + lz - 1;
        if (z >= nz) break;
        const unsigned short* pc = col + lz * PS;
        load8w<ST, EN>(pc + PS, zp, k);
        load8w<ST, EN>(pc - WX, ym, k);
        load8w<ST, EN>(pc + WX, yp, k);
        // x neighbours of the group from shared memory (2-byte loads with a
        // 4-way bank conflict; lane shuffles of the neighbours' registers
        // measured 14 % slower on B200)
        const float xl = Codec<ST, EN>::work(pc[-1], k), xr = Codec<ST, EN>::work(pc[8], k);
        stencil_update8_enc<EN>(xl, xr, c, ym, yp, zm, zp, r, inv_decay, dec_sub, k.b, v);
        if (edge_y || z == 0 || z == nz - 1) {
#pragma unroll
            for (int e = 0; e < 8; ++e) v[e] = bf;
        } else {
            if (ex0) v[0] = bf;
            if (ex7) v[7] = bf;
        }
        if (active) store8w_at<ST, EN>(o, v, vi, key, k);
        o += sz;
        vi += sz;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            zm[e] = c[e];
            c[e] = zp[e];
        }
    }
}

template <int ST, int EN>
__global__ void __launch_bounds__(t16::THREADS) k_substep16(const __grid_constant__ CUtensorMap in_map,
                                                           unsigned short* __restrict__ out, const FieldStep fs,
                                                           olc_u32* status, int rev, const olc_u32* step_ctr,
                                                           olc_u32 step_host, int sub, int field) {
    using namespace t16;
    extern __shared__ unsigned char t16_raw[];
    const olc_u32 pad = (128u - (smem_addr(t16_raw) & 127u)) & 127u;
    unsigned short* tile = reinterpret_cast<unsigned short*>(t16_raw + pad);
    const olc_u32 bar = smem_addr(t16_raw + pad + BYTES);
    const int bx = rev ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
    const int by = rev ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
    const int bz = rev ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
    const int x0 = bx * TX, y0 = by * TYR, z0 = bz * TZ;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(tile)),
            "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(x0 - HX), "r"(y0 - 1), "r"(z0 - 1), "r"(bar)
            : "memory");
    }
    // bounded wait for the tile (olc_mbar_wait_bounded records a timeout);
    // a warp leaves as a whole (the tile has no block-wide barrier)
    const bool tile_ready = olc_mbar_wait_bounded(bar, 0, status);
    if (__any_sync(0xffffffffu, !tile_ready)) return;
    t16_tile<ST, EN>(tile, out, x0, y0, z0, fs.dims[0], fs.dims[1], fs.dims[2], fs,
                     olc_sr_key(step_ctr ? *step_ctr : step_host, sub, field));
}

// ------------------------------------------------------------------ batched substep
// k_substep16's tile on one member of a batch (as k_substep_batch_x4 does for
// FP32): tile list entry blockIdx.x names the member and the tile, the
// member's tensor maps come from a table in device memory, and the
// stochastic-rounding key counts the member's own steps.
static_assert(t16::TX == BATCH_T16_TX && t16::TYR == BATCH_T16_TY && t16::TZ == BATCH_T16_TZ, "batched 16-bit tile");

template <int ST, int EN>
__global__ void __launch_bounds__(t16::THREADS) k_substep_batch_t16(
    const uint4* __restrict__ tiles, const OlcSimDesc* __restrict__ sims, const FieldStep* __restrict__ steps,
    const CUtensorMap* __restrict__ maps, int field, int n_fields, const unsigned char* __restrict__ fpar, int sub,
    unsigned short* fa, unsigned short* fb, const olc_u32* step_ctr, olc_u32* status) {
    using namespace t16;
    extern __shared__ unsigned char t16_raw[];
    const olc_u32 pad = (128u - (smem_addr(t16_raw) & 127u)) & 127u;
    unsigned short* tile = reinterpret_cast<unsigned short*>(t16_raw + pad);
    const olc_u32 bar = smem_addr(t16_raw + pad + BYTES);
    const uint4 t = tiles[blockIdx.x];
    const OlcSimDesc& d = sims[t.x];
    const size_t j = (size_t)t.x * n_fields + field;
    const FieldStep fs = steps[j];
    const bool flip = ((fpar[j] ^ (unsigned)sub) & 1u) != 0u;
    const CUtensorMap* map = maps + 2 * j + (flip ? 1 : 0);
    unsigned short* out = (flip ? fa : fb) + d.field_off;
    const int x0 = (int)t.y * TX, y0 = (int)t.z * TYR, z0 = (int)t.w * TZ;
    // programmatic dependent launch: the next substep's CTAs may start their
    // prologue (tile entry, member record, parity, barrier set-up: nothing the
    // previous launch writes) during this launch's last wave; every access to
    // field data follows griddepcontrol.wait
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(tile)),
            "l"(reinterpret_cast<unsigned long long>(map)), "r"(x0 - HX), "r"(y0 - 1), "r"(z0 - 1), "r"(bar)
            : "memory");
    }
    // bounded wait for the tile (olc_mbar_wait_bounded records a timeout);
    // a warp leaves as a whole (the tile has no block-wide barrier)
    const bool tile_ready = olc_mbar_wait_bounded(bar, 0, status);
    if (__any_sync(0xffffffffu, !tile_ready)) return;
    t16_tile<ST, EN>(tile, out, x0, y0, z0, d.cdims[0], d.cdims[1], d.cdims[2], fs,
                     olc_sr_key(*step_ctr - d.step_base, sub, field));
}

template <int ST, int EN>
static void launch_bt16(const uint4* tiles, olc_u32 n_tiles, const OlcSimDesc* sims, const FieldStep* steps,
                        const CUtensorMap* maps, int field, int n_fields, const unsigned char* fpar, int sub,
                        void* fa, void* fb, const olc_u32* step_ctr, olc_u32* status, cudaStream_t s) {
    using namespace t16;
    static int configured_mask = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 32 && !(configured_mask & (1 << dev))) {
        cudaFuncSetAttribute(k_substep_batch_t16<ST, EN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
        configured_mask |= 1 << dev;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_tiles);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_substep_batch_t16<ST, EN>, tiles, sims, steps, maps, field, n_fields, fpar, sub,
                       static_cast<unsigned short*>(fa), static_cast<unsigned short*>(fb), step_ctr, status);
}

void launch_substep_batch_t16(const BatchArgs& b, int storage, int encoding, const uint4* tiles, olc_u32 n_tiles,
                              const FieldStep* steps, const CUtensorMap* maps, int field, int n_fields,
                              const unsigned char* fpar, int sub, void* fa, void* fb, const olc_u32* step_ctr,
                              olc_u32* status, cudaStream_t s) {
    if (n_tiles == 0) return;
    with_storage16(storage, encoding, [&](auto st, auto en) {
        launch_bt16<decltype(st)::value, decltype(en)::value>(tiles, n_tiles, b.sims, steps, maps, field, n_fields,
                                                              fpar, sub, fa, fb, step_ctr, status, s);
    });
}

bool make_field_maps16(FieldMaps16* m, void* a, void* b, const int dims[3]) {
    using namespace t16;
    m->ok = false;
    const cuuint32_t box[3] = {WX, WY, WZ};
    if (!encode_map_elems(&m->map[0], a, dims, box, 2) || !encode_map_elems(&m->map[1], b, dims, box, 2)) return false;
    m->ok = true;
    return true;
}

template <int ST, int EN>
static void launch_sub16(const CUtensorMap& map, void* out, const FieldStep& fs, olc_u32* status, int rev,
                         const olc_u32* step_ctr, olc_u32 step_host, int sub, int field, cudaStream_t s) {
    using namespace t16;
    static int configured_mask = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 32 && !(configured_mask & (1 << dev))) {
        cudaFuncSetAttribute(k_substep16<ST, EN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
        configured_mask |= 1 << dev;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((fs.dims[0] + TX - 1) / TX, (fs.dims[1] + TYR - 1) / TYR, (fs.dims[2] + TZ - 1) / TZ);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_substep16<ST, EN>, map, static_cast<unsigned short*>(out), fs, status, rev, step_ctr,
                       step_host, sub, field);
}

void* run_substeps16(void* a, void* b, const FieldMaps16& m, int a_index, const FieldStep& fs, olc_u32* status,
                     const olc_u32* step_ctr, olc_u32 step_host, int field, cudaStream_t s) {
    void* bufs[2];
    bufs[a_index] = a;
    bufs[1 - a_index] = b;
    int cur = a_index;
    for (int i = 0; i < fs.substeps; ++i) {
        with_storage16(fs.storage, fs.encoding, [&](auto st, auto en) {
            launch_sub16<decltype(st)::value, decltype(en)::value>(m.map[cur], bufs[1 - cur], fs, status, i & 1,
                                                                   step_ctr, step_host, i, field, s);
        });
        cur = 1 - cur;
    }
    return bufs[cur];
}

// ------------------------------------------------------------------ reductions
// Mass (FP64 sum of value + residual), minimum and maximum of a 16-bit field;
// one block partial per block, summed in a fixed order by the last block (as
// k_reduce_field).
template <int ST, int EN>
__global__ void __launch_bounds__(256) k_reduce_field16(const unsigned short* __restrict__ f,
                                                        const float* __restrict__ comp, size_t nvox, int slot,
                                                        OlcReductions* out, double* partials, olc_u32* ticket,
                                                        const EncConst ek) {
    __shared__ double s_v[3][8];
    __shared__ bool s_last;
    double sum = 0.0, mn = 1e300, mx = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nvox; i += (size_t)gridDim.x * blockDim.x) {
        const double v = (double)phys_with_residual<ST, EN>(f[i], comp ? comp[i] : 0.0f, ek);
        sum += v;
        mn = fmin(mn, v);
        mx = fmax(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_v[0][warp] = sum;
        s_v[1][warp] = mn;
        s_v[2][warp] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0, a = 1e300, b = 0.0;
        for (int w = 0; w < 8; ++w) {
            t += s_v[0][w];
            a = fmin(a, s_v[1][w]);
            b = fmax(b, s_v[2][w]);
        }
        atomicMin(reinterpret_cast<unsigned long long*>(&out->field_min[slot]), (unsigned long long)__double_as_longlong(a));
        atomicMax(reinterpret_cast<unsigned long long*>(&out->field_max[slot]), (unsigned long long)__double_as_longlong(b));
        partials[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) t += __ldcg(partials + b);
        out->field_mass[slot] = t;
        *ticket = 0u;
    }
}

void launch_reduce_field16(const void* f, const float* comp, const FieldStep& fs, int slot, OlcReductions* out,
                           const RedScratch& rs, cudaStream_t s) {
    const size_t nvox = (size_t)fs.dims[0] * fs.dims[1] * fs.dims[2];
    size_t blocks = (nvox + 255) / 256;
    if (blocks == 0) blocks = 1;
    if (blocks > RED_MAX_BLOCKS) blocks = RED_MAX_BLOCKS;
    double* part = rs.partials + (size_t)(4 + slot) * RED_MAX_BLOCKS;
    olc_u32* ticket = rs.tickets + 1 + slot;
    const unsigned short* p = static_cast<const unsigned short*>(f);
    const EncConst ek = enc_const(fs);
    with_storage16(fs.storage, fs.encoding, [&](auto st, auto en) {
        k_reduce_field16<BaseOf<decltype(st)::value>::value, decltype(en)::value>
            <<<(unsigned)blocks, 256, 0, s>>>(p, comp, nvox, slot, out, part, ticket, ek);
    });
}

}  // namespace olc
