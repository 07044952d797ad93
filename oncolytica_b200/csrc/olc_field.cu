// Diffusion-reaction of one chemistry field.
//
// Reference arithmetic (engine/assets/shaders/tumor_sim.wgsl):
//   * Kernel_ApplyReaction :387-412 — implicit first-order sink,
//       f <- f / (1 + K dt), K = sum of the uptake rates deposited in the voxel
//   * Kernel_DiffusionSolver :414-446 — explicit 7-point Laplacian with the
//       outer faces pinned to the boundary value (Dirichlet)
// and the framework's substep mechanism chemistry_rule(iterations=S)
// (framework/src/oncolytica/gpu/runtime/_gpu_backend.py:134-142).
//
// One substep of an interior voxel, every operation separately rounded so the
// CPU restatement reproduces it bit for bit:
//   s   = ((xm + xp) + (ym + yp)) + (zm + zp)
//   u   = c + r * (s - 6 c)
//   out = max(u * inv_decay, 0),   inv_decay = 1 / (1 + lambda dt/S)
#include "olc_internal.h"
#include "olc_stencil.cuh"

#include <cuda.h>  // CUtensorMap (types only; the encoder comes from cudaGetDriverEntryPoint)

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace olc {

bool make_field_step(const OlcDiffusion& d, const int dims[3], float dx, float dt, FieldStep* out,
                     std::string* err) {
    if (d.substeps < 1) {
        *err = "substeps must be >= 1";
        return false;
    }
    for (int i = 0; i < 3; ++i) {
        if (dims[i] < 3) {
            *err = "field dims must be >= 3";
            return false;
        }
    }
    if (!(dx > 0.0f) || !(dt >= 0.0f) || d.diffusion < 0.0f || d.decay < 0.0f) {
        *err = "dx must be > 0 and dt, diffusion, decay >= 0";
        return false;
    }
    const float dts = dt / (float)d.substeps;
    const float r = d.diffusion * dts / (dx * dx);
    if (r > 1.0f / 6.0f + 1e-7f) {
        *err = "explicit diffusion unstable: D*dt/(S*dx^2) = " + std::to_string(r) +
               " > 1/6; raise substeps";
        return false;
    }
    if (d.storage < OLC_FIELD_F32 || d.storage > OLC_FIELD_F16_SR) {
        *err = "storage must be OLC_FIELD_F32, OLC_FIELD_BF16, OLC_FIELD_F16, OLC_FIELD_BF16_SR or OLC_FIELD_F16_SR";
        return false;
    }
    if (d.storage != OLC_FIELD_F32 && dims[0] % 8 != 0) {
        *err = "16-bit field storage needs an x extent that is a multiple of 8";
        return false;
    }
    if (d.encoding < OLC_ENC_VALUE || d.encoding > OLC_ENC_OFFSET3) {
        *err = "encoding must be OLC_ENC_VALUE, OLC_ENC_DEFICIT or OLC_ENC_OFFSET3";
        return false;
    }
    if (d.encoding != OLC_ENC_VALUE && d.storage == OLC_FIELD_F32) {
        *err = "encodings apply to 16-bit storage only (FP32 fields use OLC_ENC_VALUE)";
        return false;
    }
    if (d.encoding == OLC_ENC_DEFICIT && !(d.boundary > 0.0f && d.boundary <= 65504.0f)) {
        *err = "OLC_ENC_DEFICIT needs 0 < boundary <= 65504";
        return false;
    }
    if (d.encoding == OLC_ENC_OFFSET3 && !(d.boundary > 0.0f && d.boundary <= 4.0f)) {
        *err = "OLC_ENC_OFFSET3 needs 0 < boundary <= 4 (the offset flags use the top two bits)";
        return false;
    }
    for (int i = 0; i < 3; ++i) out->dims[i] = dims[i];
    out->r = r;
    out->bval = d.boundary;
    out->sink_dt = dt;
    out->substeps = d.substeps;
    out->storage = d.storage;
    if (d.storage == OLC_FIELD_F32 || d.storage == OLC_FIELD_BF16_SR || d.storage == OLC_FIELD_F16_SR) {
        // every substep decays (stochastic rounding keeps the small decrements)
        out->inv_decay = 1.0f / (1.0f + d.decay * dts);
        out->decay_step = 1.0f;
    } else {
        // round to nearest would lose the small per-substep decrements: decay
        // leaves the substeps and is applied once per step by the reaction pass
        out->inv_decay = 1.0f;
        out->decay_step = (float)std::pow(1.0 + (double)d.decay * (double)dts, -(double)d.substeps);
    }
    // the encodings' constants, each one FP32 operation (the oracle repeats them)
    const float b = d.boundary;
    out->encoding = d.encoding;
    out->dec_sub = b * (1.0f - out->inv_decay);
    out->dec_step = b * (1.0f - out->decay_step);
    out->half_b = 0.5f * b;
    out->quarter_b = 0.25f * b;
    out->upper_q = b - out->quarter_b;
    return true;
}

// f <- f / (1 + K dt) on interior voxels, K <- 0 everywhere.  With nx a
// multiple of 4 and 16-byte aligned buffers each thread takes four voxels of
// a row (16-byte loads of K; f is read and written only where K != 0).
__global__ void __launch_bounds__(256) k_sink(float* __restrict__ f, float* __restrict__ K, int nx, int ny,
                                              int nz, float dt) {
    const size_t nvox = (size_t)nx * ny * nz;
    if ((nx & 3) == 0 && ((reinterpret_cast<uintptr_t>(f) | reinterpret_cast<uintptr_t>(K)) & 15u) == 0) {
        const size_t nq = nvox / 4;
        for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nq; q += (size_t)gridDim.x * blockDim.x) {
            const float4 k4 = *reinterpret_cast<const float4*>(K + 4 * q);
            if (k4.x == 0.0f && k4.y == 0.0f && k4.z == 0.0f && k4.w == 0.0f) continue;
            const size_t v0 = 4 * q;
            const int x0 = (int)(v0 % (size_t)nx);
            const size_t t = v0 / (size_t)nx;
            const int y = (int)(t % (size_t)ny);
            const int z = (int)(t / (size_t)ny);
            if (!(y == 0 || z == 0 || y == ny - 1 || z == nz - 1)) {
                float4 f4 = *reinterpret_cast<const float4*>(f + v0);
                float* fv = &f4.x;
                const float* kv = &k4.x;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int x = x0 + e;
                    if (kv[e] != 0.0f && x != 0 && x != nx - 1)
                        fv[e] = __fdiv_rn(fv[e], __fadd_rn(1.0f, __fmul_rn(kv[e], dt)));
                }
                *reinterpret_cast<float4*>(f + v0) = f4;
            }
            *reinterpret_cast<float4*>(K + v0) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        return;
    }
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < nvox;
         v += (size_t)gridDim.x * blockDim.x) {
        float k = K[v];
        if (k != 0.0f) {
            int x = (int)(v % (size_t)nx);
            size_t t = v / (size_t)nx;
            int y = (int)(t % (size_t)ny);
            int z = (int)(t / (size_t)ny);
            bool face = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
            if (!face) f[v] = __fdiv_rn(f[v], __fadd_rn(1.0f, __fmul_rn(k, dt)));
            K[v] = 0.0f;
        }
    }
}

// One substep.  A block covers a 32 x 8 column patch and ZC planes; each
// thread walks its column in z with the z neighbours in registers.
template <int BX, int BY, int ZC>
__global__ void __launch_bounds__(BX* BY) k_substep(const float* __restrict__ in, float* __restrict__ out,
                                                   int nx, int ny, int nz, float r, float inv_decay,
                                                   float bval) {
    const int x = blockIdx.x * BX + threadIdx.x;
    const int y = blockIdx.y * BY + threadIdx.y;
    const int z0 = blockIdx.z * ZC;
    if (x >= nx || y >= ny || z0 >= nz) return;
    const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
    const bool edge_xy = x == 0 || y == 0 || x == nx - 1 || y == ny - 1;
    const int z1 = min(z0 + ZC, nz);
    size_t idx = (size_t)z0 * sz + (size_t)y * sy + x;
    float zm = z0 > 0 ? __ldg(in + idx - sz) : 0.0f;
    float c = __ldg(in + idx);
    for (int z = z0; z < z1; ++z, idx += sz) {
        float zp = (z + 1 < nz) ? __ldg(in + idx + sz) : 0.0f;
        float o;
        if (edge_xy || z == 0 || z == nz - 1) {
            o = bval;
        } else {
            float xm = __ldg(in + idx - 1), xp = __ldg(in + idx + 1);
            float ym = __ldg(in + idx - sy), yp = __ldg(in + idx + sy);
            float s = __fadd_rn(__fadd_rn(__fadd_rn(xm, xp), __fadd_rn(ym, yp)), __fadd_rn(zm, zp));
            float u = __fadd_rn(c, __fmul_rn(r, __fsub_rn(s, __fmul_rn(6.0f, c))));
            o = fmaxf(__fmul_rn(u, inv_decay), 0.0f);
        }
        out[idx] = o;
        zm = c;
        c = zp;
    }
}

__device__ __forceinline__ olc_u32 smem_u32(const void* p) {
    return static_cast<olc_u32>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------- 4-wide TMA tile path
// k_substep_x4<TYR, TZ>: the same single substep with each thread owning four
// consecutive x voxels of a row, so the x neighbours of the inner voxels are
// already in registers and the z, y rows come from shared memory as 16-byte
// vectors.  A CTA of 16 x TYR threads owns a 64 x TYR x TZ block of outputs;
// one TMA box (72 x (TYR+2) x (TZ+2) floats, x starting 4 columns early so it
// is 16-byte aligned) holds the block and its halo.  Per four voxels a thread
// issues three 128-bit and two 32-bit shared loads and one 128-bit store; the
// arithmetic per voxel is k_substep's (same operations, same order,
// separately rounded), so results equal it bit for bit.  Needs nx % 4 == 0,
// which the TMA row-stride rule already imposes.  The tile (TYR rows, TZ
// planes) is a tuning choice per handle (OlcTuning, chosen by measurement).
template <int TYR, int TZ>
struct X4Shape {
    static constexpr int TX = 64, HX = 4, WX = TX + 2 * HX, WY = TYR + 2, WZ = TZ + 2;
    static constexpr int THREADS = 16 * TYR;
    static constexpr unsigned BYTES = (unsigned)(WX * WY * WZ * 4);
    static constexpr size_t SMEM = BYTES + 16 + 128;  // tile + mbarrier + alignment slack
};

// L2 eviction priority of a tile's accesses (a cache policy for the
// .L2::cache_hint forms): the planes a field keeps resident across substeps
// are read and written with evict_last, the rest with evict_first, so the
// streamed planes do not push the kept ones out; evict_normal when nothing is
// kept.
__device__ __forceinline__ unsigned long long l2_policy(int keep, bool kept) {
    unsigned long long pol;
    if (!keep)
        asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol));
    else if (kept)
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    else
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void st_hint4(float* p, float4 v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w), "l"(pol)
                 : "memory");
}

// The 64 x TYR x TZ output block at (x0, y0, z0) from its staged box (stores
// with cache policy pol).
template <int TYR, int TZ>
__device__ __forceinline__ void x4_tile(const float* tile, float* __restrict__ out, int x0, int y0, int z0, int nx,
                                        int ny, int nz, float r, float inv_decay, float bval,
                                        unsigned long long pol) {
    using S = X4Shape<TYR, TZ>;
    const int g = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int x = x0 + 4 * g, y = y0 + ty;
    if (x >= nx || y >= ny) return;
    const bool edge_y = y == 0 || y == ny - 1;
    const bool ex0 = x == 0, ex3 = x + 3 == nx - 1;
    constexpr int PS = S::WY * S::WX;  // plane stride (floats)
    const float* col = tile + (ty + 1) * S::WX + S::HX + 4 * g;  // plane 0 of this thread's four voxels
    float4 zm = *reinterpret_cast<const float4*>(col);
    float4 c = *reinterpret_cast<const float4*>(col + PS);
    const size_t sz = (size_t)nx * ny;
    float* o = out + (size_t)z0 * sz + (size_t)y * nx + x;
#pragma unroll 4
    for (int lz = 1; lz <= TZ; ++lz) {
        const int z = z0 + lz - 1;
        if (z >= nz) break;
        const float* pc = col + lz * PS;
        const float4 zp = *reinterpret_cast<const float4*>(pc + PS);
        const float4 ym = *reinterpret_cast<const float4*>(pc - S::WX);
        const float4 yp = *reinterpret_cast<const float4*>(pc + S::WX);
        const float xl = pc[-1], xr = pc[4];
        float4 v = stencil_update4(xl, xr, c, ym, yp, zm, zp, r, inv_decay);
        if (edge_y || z == 0 || z == nz - 1) {
            v = make_float4(bval, bval, bval, bval);
        } else {
            if (ex0) v.x = bval;
            if (ex3) v.w = bval;
        }
        st_hint4(o, v, pol);
        o += sz;
        zm = c;
        c = zp;
    }
}

// keep: planes [0, keep) of both buffers are the field's L2-resident slab
// (0: no eviction hints).
template <int TYR, int TZ>
__global__ void __launch_bounds__(16 * TYR, 1) k_substep_x4(const __grid_constant__ CUtensorMap in_map,
                                                        float* __restrict__ out, int nx, int ny, int nz, float r,
                                                        float inv_decay, float bval, olc_u32* status, int rev,
                                                        int keep) {
    using S = X4Shape<TYR, TZ>;
    extern __shared__ unsigned char x4_raw[];
    const olc_u32 pad = (128u - (smem_u32(x4_raw) & 127u)) & 127u;
    float* tile = reinterpret_cast<float*>(x4_raw + pad);
    const olc_u32 bar_a = smem_u32(x4_raw + pad + S::BYTES);
    // rev != 0 walks the tiles in reverse launch order, so a substep starts on
    // the tiles the previous one wrote last, while they are still in L2
    const int bx = rev ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
    const int by = rev ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
    const int bz = rev ? gridDim.z - 1 - blockIdx.z : blockIdx.z;
    const int x0 = bx * S::TX, y0 = by * TYR, z0 = bz * TZ;
    // programmatic dependent launch, as in k_substep_tma
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const unsigned long long pol = l2_policy(keep, z0 < keep);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(S::BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint "
            "[%0], [%1, {%2, %3, %4}], [%5], %6;" ::"r"(smem_u32(tile)),
            "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(x0 - S::HX), "r"(y0 - 1), "r"(z0 - 1),
            "r"(bar_a), "l"(pol)
            : "memory");
    }
    // bounded wait for the tile (olc_mbar_wait_bounded records a timeout)
    if (!olc_mbar_wait_bounded(bar_a, 0, status)) return;
    x4_tile<TYR, TZ>(tile, out, x0, y0, z0, nx, ny, nz, r, inv_decay, bval, pol);
}

// ---------------------------------------------------------------- two substeps per pass
// k_substep_pair<NT>: two substeps in one pass (temporal blocking), for FP32
// fields whose rows fit one TMA box (nx <= 256, nx % 4 == 0).  A CTA owns
// full-width rows [y0, y0 + TY) and planes [z0, z0 + ZL) and marches up z.
// Each thread owns four consecutive x voxels of one row of the intermediate
// (first-substep) field, which covers the CTA's rows plus one on each side
// (MR = TY + 2 rows, MR = NT / (nx / 4)); full rows need no x halo.
//   * Input planes z0-2 .. z0+ZL+1 (TY + 4 rows each, one TMA box per plane)
//     stream through a ring of PAIR_RING shared-memory slots, each refilled as
//     soon as every thread is past its last read of it.
//   * Step p computes intermediate plane p (7-point update of the input, the
//     thread's own column of planes p-1 and p held in registers) into one of
//     three intermediate planes in shared memory and keeps it in registers;
//     after the step's one barrier it computes output plane p-1 from the
//     intermediate planes p-2, p-1 (registers), p (registers) and the x/y
//     neighbours of plane p-1 (shared memory).
// Every voxel of both substeps is computed with stencil_update4 and the
// boundary rule of x4_tile (faces hold bval), so the output equals two
// k_substep_x4 launches bit for bit; intermediate rows and planes outside
// the grid are never read by an output inside it.  DRAM traffic is one read
// and one write of the field per two substeps.
constexpr int PAIR_RING = 4;

__host__ __device__ inline int pair_round32(int v) { return (v + 31) & ~31; }

// Shared memory of k_substep_pair for a row width and output rows per CTA.
__host__ __device__ inline int pair_slot_floats(int nx, int ty) { return pair_round32(nx * (ty + 4)); }
__host__ __device__ inline int pair_mid_floats(int nx, int ty) { return pair_round32(nx * (ty + 2)); }
inline size_t pair_smem_bytes(int nx, int ty) {
    return (size_t)(PAIR_RING * pair_slot_floats(nx, ty) + 3 * pair_mid_floats(nx, ty)) * 4 + 8 * PAIR_RING + 128;
}

template <int NT>
__global__ void __launch_bounds__(NT, 1024 / NT) k_substep_pair(const __grid_constant__ CUtensorMap in_map,
                                                               float* __restrict__ out, int nx, int ny, int nz,
                                                               float r, float inv_decay, float bval,
                                                               olc_u32* status, int rev, int ty, int zl) {
    extern __shared__ unsigned char pair_raw[];
    const olc_u32 pad = (128u - (smem_u32(pair_raw) & 127u)) & 127u;
    float* ring = reinterpret_cast<float*>(pair_raw + pad);
    const int slot_f = pair_slot_floats(nx, ty), mid_f = pair_mid_floats(nx, ty);
    float* mid = ring + PAIR_RING * slot_f;
    const olc_u32 bar0 = smem_u32(mid + 3 * mid_f);
    const int by = rev ? gridDim.x - 1 - blockIdx.x : blockIdx.x;
    const int bz = rev ? gridDim.y - 1 - blockIdx.y : blockIdx.y;
    const int y0 = by * ty, z0 = bz * zl;
    const int z_end = min(z0 + zl, nz);
    const int nq = z_end - z0 + 4;  // input planes z0-2 .. z_end+1
    const olc_u32 plane_bytes = (olc_u32)(nx * (ty + 4) * 4);
    const int G = nx >> 2, MR = ty + 2;
    const int mr = threadIdx.x / G, g = threadIdx.x - mr * G;
    const bool live = mr < MR;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        for (int k = 0; k < PAIR_RING; ++k)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8 * k) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");
    // input plane z0 - 2 + q lives in slot q % PAIR_RING; its mbarrier phase is (q / PAIR_RING) & 1
    int issued = 0;  // thread 0: planes issued so far
    auto issue_upto = [&](int last_free) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (; issued < nq && issued - PAIR_RING <= last_free; ++issued) {
            const olc_u32 bar = bar0 + 8 * (issued % PAIR_RING);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(plane_bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(ring + (issued % PAIR_RING) * slot_f)),
                "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(0), "r"(y0 - 2), "r"(z0 - 2 + issued),
                "r"(bar)
                : "memory");
        }
    };
    auto wait_plane = [&](int q) {
        return olc_mbar_wait_bounded(bar0 + 8 * (q % PAIR_RING), (olc_u32)((q / PAIR_RING) & 1), status);
    };
    if (threadIdx.x == 0) issue_upto(-1);
    const int row_off = (mr + 1) * nx + 4 * g;  // this thread's voxels in an input slot
    const int y = y0 - 1 + mr, x = 4 * g;
    const bool y_face = y <= 0 || y >= ny - 1;  // rows outside the grid too (never read)
    const bool ex0 = x == 0, ex3 = x + 3 == nx - 1;
    const bool out_row = live && mr >= 1 && mr <= MR - 2 && y < ny;
    const float4 b4 = make_float4(bval, bval, bval, bval);
    const size_t sz = (size_t)nx * ny;
    bool ok = wait_plane(0) && wait_plane(1);
    float4 in_zm = b4, in_c = b4, mid_a = b4, mid_b = b4;
    if (live) {
        in_zm = *reinterpret_cast<const float4*>(ring + row_off);
        in_c = *reinterpret_cast<const float4*>(ring + slot_f + row_off);
    }
    for (int p = z0 - 1, i = 0; p <= z_end; ++p, ++i) {
        const int qn = i + 2;  // input plane p + 1
        ok = ok && wait_plane(qn);
        float4 v = b4;
        if (live) {
            const float* pc = ring + ((qn - 1) % PAIR_RING) * slot_f + row_off;
            const float4 zp = *reinterpret_cast<const float4*>(ring + (qn % PAIR_RING) * slot_f + row_off);
            const float4 ym = *reinterpret_cast<const float4*>(pc - nx);
            const float4 yp = *reinterpret_cast<const float4*>(pc + nx);
            v = stencil_update4(pc[-1], pc[4], in_c, ym, yp, in_zm, zp, r, inv_decay);
            if (y_face || p <= 0 || p >= nz - 1) {
                v = b4;
            } else {
                if (ex0) v.x = bval;
                if (ex3) v.w = bval;
            }
            *reinterpret_cast<float4*>(mid + (i % 3) * mid_f + mr * nx + 4 * g) = v;
            in_zm = in_c;
            in_c = zp;
        }
        if (__syncthreads_or(!ok)) {
            // a plane never arrived: let the copies still in flight land, then leave
            if (threadIdx.x == 0)
                for (int q = issued > PAIR_RING ? issued - PAIR_RING : 0; q < issued; ++q)
                    for (olc_u32 it = 0; it < OLC_SPIN_LIMIT; ++it)
                        if (olc_mbar_try_wait(bar0 + 8 * (q % PAIR_RING), (olc_u32)((q / PAIR_RING) & 1))) break;
            return;
        }
        if (threadIdx.x == 0) issue_upto(qn - 1);  // input plane p is read for the last time
        if (p - 1 >= z0 && out_row) {
            const int z = p - 1;
            const float* mb = mid + ((i + 2) % 3) * mid_f + mr * nx + 4 * g;  // intermediate plane p - 1
            const float4 ym = *reinterpret_cast<const float4*>(mb - nx);
            const float4 yp = *reinterpret_cast<const float4*>(mb + nx);
            float4 o = stencil_update4(mb[-1], mb[4], mid_b, ym, yp, mid_a, v, r, inv_decay);
            if (y == 0 || y == ny - 1 || z == 0 || z == nz - 1) {
                o = b4;
            } else {
                if (ex0) o.x = bval;
                if (ex3) o.w = bval;
            }
            *reinterpret_cast<float4*>(out + (size_t)z * sz + (size_t)y * nx + x) = o;
        }
        mid_a = mid_b;
        mid_b = v;
    }
}

// The CTA shape of k_substep_pair<nt> on a field: output rows per CTA (0 when
// the field does not fit: nx > 256, nx % 4 != 0, or fewer than three
// intermediate rows).
int pair_rows(int nt, const int dims[3]) {
    if (nt <= 0 || dims[0] > 256 || dims[0] % 4 != 0 || dims[0] < 8) return 0;
    const int mr = nt / (dims[0] / 4);
    if (mr < 3) return 0;
    return std::min(std::min(mr - 2, dims[1]), 252);  // a box is at most 256 rows
}

bool pair_threads_known(int nt) { return nt == 0 || nt == 128 || nt == 256 || nt == 512 || nt == 1024; }

// ---------------------------------------------------------------- batched substep
// TMA box of a member's tensor map for the batched 16-bit substep.
void batch_substep_box(int storage, cuuint32_t box[3]) {
    (void)storage;
    box[0] = BATCH_T16_TX + 16;
    box[1] = BATCH_T16_TY + 2;
    box[2] = BATCH_T16_TZ + 2;
}

namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}
}  // namespace

bool encode_map_elems(CUtensorMap* map, void* base, const int dims[3], const cuuint32_t box[3], int elem_bytes) {
    if (elem_bytes != 2 && elem_bytes != 4) return false;
    if (((size_t)dims[0] * elem_bytes) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0) return false;
    if (((size_t)box[0] * elem_bytes) % 16 != 0) return false;
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t gdim[3] = {(cuuint64_t)dims[0], (cuuint64_t)dims[1], (cuuint64_t)dims[2]};
    cuuint64_t gstride[2] = {(cuuint64_t)dims[0] * elem_bytes, (cuuint64_t)dims[0] * dims[1] * elem_bytes};
    cuuint32_t estride[3] = {1, 1, 1};
    return fn(map, elem_bytes == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, gdim,
              gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static bool encode_map(CUtensorMap* map, float* base, const int dims[3], const cuuint32_t box[3]) {
    if ((dims[0] * 4) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0) return false;
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t gdim[3] = {(cuuint64_t)dims[0], (cuuint64_t)dims[1], (cuuint64_t)dims[2]};
    cuuint64_t gstride[2] = {(cuuint64_t)dims[0] * 4, (cuuint64_t)dims[0] * dims[1] * 4};
    cuuint32_t estride[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, gdim, gstride, box, estride,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The 4-wide tiles compiled in (TYR, TZ); OlcTuning.stencil_tile_{y,z} picks
// one per handle (default (8, 8): on B200 with a 256^3 FP32 field 21.2 us per
// substep against 21.5 for (16, 8) and 22.1 for (8, 16)).
#define OLC_VX_SHAPES(X) X(8, 8) X(16, 8) X(8, 16) X(16, 4)

bool stencil_tile_known(int tile_y, int tile_z) {
    bool known = false;
#define OLC_VX_MATCH(p, q) known = known || (tile_y == p && tile_z == q);
    OLC_VX_SHAPES(OLC_VX_MATCH)
#undef OLC_VX_MATCH
    return known;
}

template <int NT>
static int pair_default_planes(const int dims[3], int ty);

bool make_field_maps(FieldMaps* m, float* a, float* b, const int dims[3], int tile_y, int tile_z, int pair_threads,
                     int pair_planes, int keep_pct) {
    m->ok = false;
    m->pair_nt = m->pair_ty = m->pair_zl = 0;
    if (!stencil_tile_known(tile_y, tile_z) || !pair_threads_known(pair_threads) || pair_planes < 0 ||
        keep_pct < 0 || keep_pct > 100)
        return false;
    m->keep = (int)((long long)dims[2] * keep_pct / 100);
    m->VY = tile_y;
    m->VZ = tile_z;
    const cuuint32_t boxv[3] = {72, (cuuint32_t)(tile_y + 2), (cuuint32_t)(tile_z + 2)};
    if (!encode_map(&m->vec[0], a, dims, boxv) || !encode_map(&m->vec[1], b, dims, boxv)) return false;
    m->ok = true;
    // two substeps per pass where the rows fit one box (else single passes)
    const int ty = pair_threads ? pair_rows(pair_threads, dims) : 0;
    if (ty > 0) {
        const cuuint32_t boxp[3] = {(cuuint32_t)dims[0], (cuuint32_t)(ty + 4), 1};
        if (encode_map(&m->pair[0], a, dims, boxp) && encode_map(&m->pair[1], b, dims, boxp)) {
            m->pair_nt = pair_threads;
            m->pair_ty = ty;
            m->pair_zl = pair_planes ? pair_planes
                         : pair_threads == 128 ? pair_default_planes<128>(dims, ty)
                         : pair_threads == 256 ? pair_default_planes<256>(dims, ty)
                         : pair_threads == 512 ? pair_default_planes<512>(dims, ty)
                                               : pair_default_planes<1024>(dims, ty);
        }
    }
    return true;
}

template <int TYR, int TZ>
static void launch_x4(const CUtensorMap& map, float* out, const FieldStep& fs, olc_u32* status, int rev,
                      int keep, cudaStream_t s) {
    using S = X4Shape<TYR, TZ>;
    static int configured_mask = 0;  // per device (up to 32)
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 32 && !(configured_mask & (1 << dev))) {
        cudaFuncSetAttribute(k_substep_x4<TYR, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        configured_mask |= 1 << dev;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((fs.dims[0] + S::TX - 1) / S::TX, (fs.dims[1] + TYR - 1) / TYR, (fs.dims[2] + TZ - 1) / TZ);
    cfg.blockDim = dim3(S::THREADS);
    cfg.dynamicSmemBytes = S::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_substep_x4<TYR, TZ>, map, out, fs.dims[0], fs.dims[1], fs.dims[2], fs.r,
                       fs.inv_decay, fs.bval, status, rev, keep);
}

template <int NT>
static void configure_pair() {
    static int configured_mask = 0;  // per device (up to 32)
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 32 && !(configured_mask & (1 << dev))) {
        cudaFuncSetAttribute(k_substep_pair<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        configured_mask |= 1 << dev;
    }
}

// Planes per CTA of k_substep_pair<NT>: as few as keep every CTA of the grid
// resident in one wave (at least 8, so the z halo stays a small share).
template <int NT>
static int pair_default_planes(const int dims[3], int ty) {
    configure_pair<NT>();
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_substep_pair<NT>, NT, pair_smem_bytes(dims[0], ty));
    const int slots = std::max(1, per_sm) * std::max(1, sms);
    const int gy = (dims[1] + ty - 1) / ty;
    const int chunks = std::max(1, slots / gy);
    return std::max(8, (dims[2] + chunks - 1) / chunks);
}

template <int NT>
static void launch_pair_nt(const FieldMaps& m, int cur, float* out, const FieldStep& fs, olc_u32* status, int rev,
                           cudaStream_t s) {
    configure_pair<NT>();
    const int ny = fs.dims[1], nz = fs.dims[2], ty = m.pair_ty, zl = m.pair_zl;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((ny + ty - 1) / ty, (nz + zl - 1) / zl, 1);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = pair_smem_bytes(fs.dims[0], ty);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_substep_pair<NT>, m.pair[cur], out, fs.dims[0], ny, nz, fs.r, fs.inv_decay, fs.bval,
                       status, rev, ty, zl);
}

static void launch_pair(const FieldMaps& m, int cur, float* out, const FieldStep& fs, olc_u32* status, int rev,
                        cudaStream_t s) {
    switch (m.pair_nt) {
        case 128: launch_pair_nt<128>(m, cur, out, fs, status, rev, s); break;
        case 256: launch_pair_nt<256>(m, cur, out, fs, status, rev, s); break;
        case 512: launch_pair_nt<512>(m, cur, out, fs, status, rev, s); break;
        default: launch_pair_nt<1024>(m, cur, out, fs, status, rev, s); break;
    }
}

static void launch_single(const FieldMaps& m, int cur, float* out, const FieldStep& fs, olc_u32* status, int rev,
                          cudaStream_t s) {
#define OLC_VX_LAUNCH(p, q)                                   \
    if (m.VY == p && m.VZ == q) {                             \
        launch_x4<p, q>(m.vec[cur], out, fs, status, rev, m.keep, s); \
        return;                                               \
    }
    OLC_VX_SHAPES(OLC_VX_LAUNCH)
#undef OLC_VX_LAUNCH
}

// Pinned voxels (the engine's vessel mask): after a substep, the listed
// voxels of its output hold the pin value.
__global__ void __launch_bounds__(256) k_pin(float* __restrict__ f, const olc_u32* __restrict__ idx, olc_u32 n,
                                             float value) {
    for (olc_u32 k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) f[idx[k]] = value;
}

void launch_pins(float* f, const Pins* pins, cudaStream_t s) {
    if (!pins || pins->n == 0) return;
    olc_u32 blocks = (pins->n + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_pin<<<blocks, 256, 0, s>>>(f, pins->idx, pins->n, pins->value);
}

// S substeps, one launch each; every other substep walks its tiles in reverse
// order, so it starts on the tiles the previous one wrote last (still in L2).
float* run_substeps_tma(float* a, float* b, const FieldMaps& m, int a_index, const FieldStep& fs, olc_u32* status,
                        cudaStream_t s, const Pins* pins) {
    float* bufs[2];
    bufs[a_index] = a;
    bufs[1 - a_index] = b;
    int cur = a_index;
    int i = 0;
    if (m.pair_nt && !(pins && pins->n)) {
        // two substeps per launch (pinned voxels are re-pinned after every
        // substep, so fields with pins take single passes)
        for (; i + 1 < fs.substeps; i += 2) {
            launch_pair(m, cur, bufs[1 - cur], fs, status, (i >> 1) & 1, s);
            cur = 1 - cur;
        }
    }
    for (; i < fs.substeps; ++i) {
        launch_single(m, cur, bufs[1 - cur], fs, status, i & 1, s);
        launch_pins(bufs[1 - cur], pins, s);
        cur = 1 - cur;
    }
    return bufs[cur];
}

int substep_launches(const FieldMaps& m, const FieldStep& fs, const Pins* pins) {
    if (pins && pins->n) return 2 * fs.substeps;
    if (m.ok && m.pair_nt) return fs.substeps / 2 + (fs.substeps & 1);
    return fs.substeps;
}

// Status word of the stateless stage entry points (bounded waits report here).
__device__ olc_u32 g_stage_status;

olc_u32* stage_status_word() {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_stage_status) != cudaSuccess) return nullptr;
    return static_cast<olc_u32*>(p);
}

void launch_sink(float* f, float* sink, const FieldStep& fs, cudaStream_t s) {
    if (!sink) return;
    const size_t nvox = (size_t)fs.dims[0] * fs.dims[1] * fs.dims[2];
    size_t blocks = (nvox + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_sink<<<(unsigned)blocks, 256, 0, s>>>(f, sink, fs.dims[0], fs.dims[1], fs.dims[2], fs.sink_dt);
}

void launch_substep(const float* in, float* out, const FieldStep& fs, cudaStream_t s) {
    constexpr int BX = 32, BY = 8, ZC = 16;
    dim3 grid((fs.dims[0] + BX - 1) / BX, (fs.dims[1] + BY - 1) / BY, (fs.dims[2] + ZC - 1) / ZC);
    k_substep<BX, BY, ZC><<<grid, dim3(BX, BY), 0, s>>>(in, out, fs.dims[0], fs.dims[1], fs.dims[2], fs.r,
                                                       fs.inv_decay, fs.bval);
}

float* run_substeps(float* a, float* b, const FieldStep& fs, cudaStream_t s, const Pins* pins) {
    float* cur = a;
    float* nxt = b;
    for (int i = 0; i < fs.substeps; ++i) {
        launch_substep(cur, nxt, fs, s);
        launch_pins(nxt, pins, s);
        float* t = cur;
        cur = nxt;
        nxt = t;
    }
    return cur;
}

float* run_field_step(float* a, float* b, float* sink, const FieldStep& fs, cudaStream_t s, const Pins* pins) {
    launch_sink(a, sink, fs, s);
    float* cur = a;
    float* nxt = b;
    for (int i = 0; i < fs.substeps; ++i) {
        launch_substep(cur, nxt, fs, s);
        launch_pins(nxt, pins, s);
        float* t = cur;
        cur = nxt;
        nxt = t;
    }
    return cur;
}

}  // namespace olc
