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

// f <- f / (1 + K dt) on interior voxels, K <- 0 everywhere.
__global__ void __launch_bounds__(256) k_sink(float* __restrict__ f, float* __restrict__ K, int nx, int ny,
                                              int nz, float dt) {
    const size_t nvox = (size_t)nx * ny * nz;
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

// ---------------------------------------------------------------- TMA tile path
// A CTA owns a TX x TY x TZ block of outputs.  One cp.async.bulk.tensor.3d
// copy brings the block plus its halo (HX = 4 in x so the box starts on a
// 16-byte boundary, 1 in y and z) into shared memory; completion is signalled
// on an mbarrier (bounded wait).  Each thread then walks its column in z with
// the z neighbours in registers and the x/y neighbours read from shared memory,
// and stores its outputs with coalesced 128-byte rows.  Out-of-range parts of
// the box (domain faces) are zero-filled by the TMA unit; they only feed
// boundary voxels, which are pinned to the boundary value.
namespace tma {
constexpr int TX = 32, TY = 8, TZ = 16, HX = 4;
constexpr int WX = TX + 2 * HX, WY = TY + 2, WZ = TZ + 2;
constexpr unsigned BYTES = WX * WY * WZ * 4;
}  // namespace tma

__device__ __forceinline__ olc_u32 smem_u32(const void* p) {
    return static_cast<olc_u32>(__cvta_generic_to_shared(p));
}


__global__ void __launch_bounds__(256) k_substep_tma(const __grid_constant__ CUtensorMap in_map,
                                                     float* __restrict__ out, int nx, int ny, int nz, float r,
                                                     float inv_decay, float bval, olc_u32* status) {
    using namespace tma;
    __shared__ alignas(128) float tile[WZ][WY][WX];
    __shared__ alignas(8) unsigned long long bar;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
    const olc_u32 bar_a = smem_u32(&bar);
    // Programmatic dependent launch: the next substep may start its launch once
    // every block of this one is running; it waits (griddepcontrol.wait) for
    // this grid to finish before touching memory.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    // the input is the previous substep's output: wait for that grid
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(&tile[0][0][0])),
            "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(x0 - HX), "r"(y0 - 1), "r"(z0 - 1), "r"(bar_a)
            : "memory");
    }
    // bounded wait for the tile (olc_mbar_wait_bounded records a timeout)
    if (!olc_mbar_wait_bounded(bar_a, 0, status)) return;
    const int x = x0 + tx, y = y0 + ty;
    if (x >= nx || y >= ny) return;
    const bool edge_xy = x == 0 || y == 0 || x == nx - 1 || y == ny - 1;
    const size_t sz = (size_t)nx * ny;
    const int lx = tx + HX, ly = ty + 1;
    float zm = tile[0][ly][lx];
    float c = tile[1][ly][lx];
    float* o = out + (size_t)z0 * sz + (size_t)y * nx + x;
#pragma unroll 4
    for (int lz = 1; lz <= TZ; ++lz) {
        const int z = z0 + lz - 1;
        if (z >= nz) break;
        const float zp = tile[lz + 1][ly][lx];
        float v;
        if (edge_xy || z == 0 || z == nz - 1) {
            v = bval;
        } else {
            const float xm = tile[lz][ly][lx - 1], xp = tile[lz][ly][lx + 1];
            const float ym = tile[lz][ly - 1][lx], yp = tile[lz][ly + 1][lx];
            const float s = __fadd_rn(__fadd_rn(__fadd_rn(xm, xp), __fadd_rn(ym, yp)), __fadd_rn(zm, zp));
            const float u = __fadd_rn(c, __fmul_rn(r, __fsub_rn(s, __fmul_rn(6.0f, c))));
            v = fmaxf(__fmul_rn(u, inv_decay), 0.0f);
        }
        *o = v;
        o += sz;
        zm = c;
        c = zp;
    }
}

// ---------------------------------------------------------------- 4-wide TMA tile path
// k_substep_x4<TYR, TZ>: the same single substep with each thread owning four
// consecutive x voxels of a row, so the x neighbours of the inner voxels are
// already in registers and the z, y rows come from shared memory as 16-byte
// vectors.  A CTA of 16 x TYR threads owns a 64 x TYR x TZ block of outputs;
// one TMA box (72 x (TYR+2) x (TZ+2) floats, x starting 4 columns early so it
// is 16-byte aligned) holds the block and its halo.  Per four voxels a thread
// issues three 128-bit and two 32-bit shared loads and one 128-bit store; the
// arithmetic per voxel is unchanged (same operations, same order, separately
// rounded), so results equal k_substep_tma bit for bit.  Needs nx % 4 == 0,
// which the TMA row-stride rule already imposes.
template <int TYR, int TZ>
struct X4Shape {
    static constexpr int TX = 64, HX = 4, WX = TX + 2 * HX, WY = TYR + 2, WZ = TZ + 2;
    static constexpr int THREADS = 16 * TYR;
    static constexpr unsigned BYTES = (unsigned)(WX * WY * WZ * 4);
    static constexpr size_t SMEM = BYTES + 16 + 128;  // tile + mbarrier + alignment slack
};

// The 64 x TYR x TZ output block at (x0, y0, z0) from its staged box.
template <int TYR, int TZ>
__device__ __forceinline__ void x4_tile(const float* tile, float* __restrict__ out, int x0, int y0, int z0, int nx,
                                        int ny, int nz, float r, float inv_decay, float bval) {
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
        *reinterpret_cast<float4*>(o) = v;
        o += sz;
        zm = c;
        c = zp;
    }
}

template <int TYR, int TZ>
__global__ void __launch_bounds__(16 * TYR, 1) k_substep_x4(const __grid_constant__ CUtensorMap in_map,
                                                        float* __restrict__ out, int nx, int ny, int nz, float r,
                                                        float inv_decay, float bval, olc_u32* status, int rev) {
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
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(S::BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(tile)),
            "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(x0 - S::HX), "r"(y0 - 1), "r"(z0 - 1),
            "r"(bar_a)
            : "memory");
    }
    // bounded wait for the tile (olc_mbar_wait_bounded records a timeout)
    if (!olc_mbar_wait_bounded(bar_a, 0, status)) return;
    x4_tile<TYR, TZ>(tile, out, x0, y0, z0, nx, ny, nz, r, inv_decay, bval);
}

// ---------------------------------------------------------------- batched substep
// TMA box of a member's tensor map for the batched 16-bit substep.
void batch_substep_box(int storage, cuuint32_t box[3]) {
    (void)storage;
    box[0] = BATCH_T16_TX + 16;
    box[1] = BATCH_T16_TY + 2;
    box[2] = BATCH_T16_TZ + 2;
}

// ---------------------------------------------------------------- persistent pipeline
// k_substep_pipe<TYR, TZ, NS>: the 4-wide substep as a persistent kernel.  The
// grid holds as many CTAs as fit on the GPU at once; CTA b takes tiles b,
// b + G, b + 2G, ... (so the tiles in flight at any moment form one
// contiguous slab of the field, as a wave of k_substep_x4 does), through a
// ring of NS shared-memory stages: while it computes tile k, the TMA loads of
// tiles k+1 .. k+NS-1 are in flight.  One barrier per tile both makes the
// timeout decision uniform and tells thread 0 that the stage read last is
// free for the next load.  Same tile arithmetic as k_substep_x4.
template <int TYR, int TZ, int NS>
struct PipeShape {
    using S = X4Shape<TYR, TZ>;
    static constexpr size_t SMEM = (size_t)NS * S::BYTES + 8 * NS + 128;
};

template <int TYR, int TZ, int NS>
__global__ void __launch_bounds__(16 * TYR, 1) k_substep_pipe(const __grid_constant__ CUtensorMap in_map,
                                                             float* __restrict__ out, int nx, int ny, int nz,
                                                             float r, float inv_decay, float bval, olc_u32* status,
                                                             int rev) {
    using S = X4Shape<TYR, TZ>;
    extern __shared__ unsigned char pipe_raw[];
    const olc_u32 pad = (128u - (smem_u32(pipe_raw) & 127u)) & 127u;
    float* stages = reinterpret_cast<float*>(pipe_raw + pad);
    const olc_u32 bar0 = smem_u32(pipe_raw + pad + (size_t)NS * S::BYTES);
    const int ntx = (nx + S::TX - 1) / S::TX, nty = (ny + TYR - 1) / TYR, ntz = (nz + TZ - 1) / TZ;
    const int ntiles = ntx * nty * ntz;
    const int G = (int)gridDim.x;
    const int mine = ((int)blockIdx.x < ntiles) ? (ntiles - (int)blockIdx.x + G - 1) / G : 0;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        for (int k = 0; k < NS; ++k) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8 * k) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");
    auto origin = [&](int k, int* x0, int* y0, int* z0) {
        int t = (int)blockIdx.x + k * G;
        if (rev) t = ntiles - 1 - t;
        *x0 = (t % ntx) * S::TX;
        t /= ntx;
        *y0 = (t % nty) * TYR;
        *z0 = (t / nty) * TZ;
    };
    auto issue = [&](int k) {  // thread 0: TMA load of this CTA's k-th tile into stage k % NS
        if (k >= mine) return;
        int x0, y0, z0;
        origin(k, &x0, &y0, &z0);
        const olc_u32 bar = bar0 + 8 * (k % NS);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(S::BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(stages + (size_t)(k % NS) * (S::BYTES / 4))),
            "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(x0 - S::HX), "r"(y0 - 1), "r"(z0 - 1), "r"(bar)
            : "memory");
    };
    if (threadIdx.x == 0)
        for (int k = 0; k < NS; ++k) issue(k);
    for (int k = 0; k < mine; ++k) {
        const olc_u32 bar = bar0 + 8 * (k % NS), parity = (olc_u32)((k / NS) & 1);
        bool ok = false;
        for (olc_u32 it = 0; it < OLC_SPIN_LIMIT; ++it) {
            if (olc_mbar_try_wait(bar, parity)) {
                ok = true;
                break;
            }
        }
        if (__syncthreads_or(!ok)) {
            // loads k .. k+NS-2 (k+NS-1 once k = 0) may still be in flight: give
            // each a bounded chance to land before the shared memory is released
            if (threadIdx.x == 0) {
                atomicOr(status, OLC_ST_TIMEOUT);
                const int last = min(mine - 1, k == 0 ? NS - 1 : k + NS - 2);
                for (int j = k; j <= last; ++j)
                    for (olc_u32 it = 0;
                         it < OLC_SPIN_LIMIT && !olc_mbar_try_wait(bar0 + 8 * (j % NS), (olc_u32)((j / NS) & 1)); ++it) {
                    }
            }
            return;
        }
        // every thread is past tile k-1: its stage may be refilled
        if (threadIdx.x == 0 && k > 0) issue(k - 1 + NS);
        int x0, y0, z0;
        origin(k, &x0, &y0, &z0);
        x4_tile<TYR, TZ>(stages + (size_t)(k % NS) * (S::BYTES / 4), out, x0, y0, z0, nx, ny, nz, r, inv_decay,
                         bval);
    }
}

// ---------------------------------------------------------------- two substeps per pass
// k_substep_t2<TYR, ZC, NS>: two substeps in one pass over HBM, marching in z.
// A CTA owns a 64 x TYR column patch of outputs over ZC planes.  Input planes
// (80 x (TYR+4) floats: x from x0-8 so the box is 16-byte aligned, y from
// y0-2) stream through a ring of NS shared-memory slots by TMA, NS-2 planes
// ahead of use.  For each plane the CTA first computes the intermediate
// (first-substep) plane over the patch grown by one voxel in x and y (18
// four-wide groups x TYR+2 rows) into a ring of four shared planes, then the
// output plane two planes behind it from three intermediate planes, and
// stores that.  Every voxel of both levels goes through the single-substep
// update (same operations, same order) with the face voxels pinned, so one
// pass equals two k_substep_x4 launches bit for bit.  Intermediate voxels
// outside the domain are computed from the TMA zero fill and only feed face
// outputs, which are pinned.
template <int TYR, int ZC, int NS>
struct T2Shape {
    static constexpr int TX = 64;
    static constexpr int PW = 80, PH = TYR + 4;  // input plane (floats)
    static constexpr int LW = 72, LH = TYR + 2;  // intermediate plane
    static constexpr unsigned PBYTES = (unsigned)(PW * PH * 4);
    static constexpr unsigned LBYTES = (unsigned)(LW * LH * 4);
    static constexpr int L1_TASKS = 18 * LH, L2_TASKS = 16 * TYR;
    static constexpr int THREADS = ((L1_TASKS > L2_TASKS ? L1_TASKS : L2_TASKS) + 31) / 32 * 32;
    static constexpr size_t SMEM = (size_t)NS * PBYTES + 4 * (size_t)LBYTES + 8 * NS + 128;
};

// Four voxels at `c` (16-byte aligned) of a plane with row stride `W`, with
// the planes below and above at the same offsets `zm`, `zp`.
template <int W>
__device__ __forceinline__ float4 update4(const float* zm, const float* c, const float* zp, float r,
                                          float inv_decay) {
    const float4 cc = *reinterpret_cast<const float4*>(c);
    const float4 m = *reinterpret_cast<const float4*>(zm);
    const float4 p = *reinterpret_cast<const float4*>(zp);
    const float4 ym = *reinterpret_cast<const float4*>(c - W);
    const float4 yp = *reinterpret_cast<const float4*>(c + W);
    const float xl = c[-1], xr = c[4];
    return stencil_update4(xl, xr, cc, ym, yp, m, p, r, inv_decay);
}

// Face voxels of the group starting at x (row y, plane z) take the boundary value.
__device__ __forceinline__ float4 pin_faces(float4 v, int x, int y, int z, int nx, int ny, int nz, float bval) {
    if (y == 0 || y == ny - 1 || z == 0 || z == nz - 1) return make_float4(bval, bval, bval, bval);
    if (x == 0) v.x = bval;
    if (x + 3 == nx - 1) v.w = bval;
    return v;
}

template <int TYR, int ZC, int NS>
__global__ void __launch_bounds__(T2Shape<TYR, ZC, NS>::THREADS, 1) k_substep_t2(
    const __grid_constant__ CUtensorMap in_map, float* __restrict__ out, int nx, int ny, int nz, float r,
    float inv_decay, float bval, olc_u32* status, int rev) {
    using S = T2Shape<TYR, ZC, NS>;
    static_assert(NS >= 4, "the ring holds the three planes in use plus at least one in flight");
    extern __shared__ unsigned char t2_raw[];
    const olc_u32 pad = (128u - (smem_u32(t2_raw) & 127u)) & 127u;
    float* pin = reinterpret_cast<float*>(t2_raw + pad);                          // NS input planes
    float* mid = reinterpret_cast<float*>(t2_raw + pad + (size_t)NS * S::PBYTES);  // 4 intermediate planes
    const olc_u32 bar0 = smem_u32(t2_raw + pad + (size_t)NS * S::PBYTES + 4 * (size_t)S::LBYTES);
    // tile order: x fastest, then y, then z chunk; reversed when rev != 0
    const int ntx = (nx + S::TX - 1) / S::TX, nty = (ny + TYR - 1) / TYR;
    int t = rev ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
    const int x0 = (t % ntx) * S::TX;
    t /= ntx;
    const int y0 = (t % nty) * TYR;
    const int z0 = (t / nty) * ZC;
    constexpr int NP = ZC + 4;  // input planes z0-2 .. z0+ZC+1
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (threadIdx.x == 0) {
        for (int k = 0; k < NS; ++k) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8 * k) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");
    auto issue = [&](int sidx) {  // thread 0: TMA load of input plane z0-2+sidx into slot sidx % NS
        if (sidx >= NP) return;
        const olc_u32 bar = bar0 + 8 * (sidx % NS);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(S::PBYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(pin + (size_t)(sidx % NS) * (S::PBYTES / 4))),
            "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(x0 - 8), "r"(y0 - 2), "r"(z0 - 2 + sidx), "r"(bar)
            : "memory");
    };
    auto wait_plane = [&](int sidx) -> bool {
        const olc_u32 bar = bar0 + 8 * (sidx % NS), parity = (olc_u32)((sidx / NS) & 1);
        for (olc_u32 it = 0; it < OLC_SPIN_LIMIT; ++it)
            if (olc_mbar_try_wait(bar, parity)) return true;
        return false;
    };
    if (threadIdx.x == 0)
        for (int k = 0; k < NS; ++k) issue(k);
    // this thread's intermediate task (group g1 of 18, row r1 of TYR+2) and output task
    const int tid = threadIdx.x;
    const bool has1 = tid < S::L1_TASKS, has2 = tid < S::L2_TASKS;
    const int g1 = tid % 18, r1 = tid / 18;
    const int g2 = tid & 15, r2 = tid >> 4;
    const int x1 = x0 - 4 + 4 * g1, y1 = y0 - 1 + r1;
    const int x2 = x0 + 4 * g2, y2 = y0 + r2;
    const int poff = (r1 + 1) * S::PW + 4 + 4 * g1;  // intermediate voxel's centre in an input plane
    const int moff1 = r1 * S::LW + 4 * g1;           // its slot in an intermediate plane
    const int moff2 = (r2 + 1) * S::LW + 4 + 4 * g2;  // output voxel's centre in an intermediate plane
    const size_t sz = (size_t)nx * ny;
    // Iteration u computes intermediate plane u (input planes u..u+2) and
    // output plane u-3 (intermediate planes u-3..u-1, finished in earlier
    // iterations): the two are independent, so one barrier per iteration
    // suffices; before it every thread has waited for input plane u+3, which
    // the next iteration needs, and after it thread 0 refills input plane u's
    // slot (last read by intermediate plane u).
    auto fail = [&](int from, int last_issued) {  // thread 0: these planes may still be in flight
        atomicOr(status, OLC_ST_TIMEOUT);
        for (int sidx = from; sidx <= last_issued && sidx < NP; ++sidx) wait_plane(sidx);
    };
    {
        const bool ok = wait_plane(0) && wait_plane(1) && wait_plane(2);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) fail(0, NS - 1);
            return;
        }
    }
    for (int u = 0; u <= ZC + 2; ++u) {
        if (u < ZC + 2 && has1) {
            const float* pm = pin + (size_t)(u % NS) * (S::PBYTES / 4) + poff;
            const float* pc = pin + (size_t)((u + 1) % NS) * (S::PBYTES / 4) + poff;
            const float* pp = pin + (size_t)((u + 2) % NS) * (S::PBYTES / 4) + poff;
            float4 v = update4<S::PW>(pm, pc, pp, r, inv_decay);
            v = pin_faces(v, x1, y1, z0 - 1 + u, nx, ny, nz, bval);
            *reinterpret_cast<float4*>(mid + (size_t)(u & 3) * (S::LBYTES / 4) + moff1) = v;
        }
        if (u >= 3 && has2) {
            const int z = z0 + u - 3;
            if (z < nz && x2 < nx && y2 < ny) {
                const float* mm = mid + (size_t)((u - 3) & 3) * (S::LBYTES / 4) + moff2;
                const float* mc = mid + (size_t)((u - 2) & 3) * (S::LBYTES / 4) + moff2;
                const float* mp = mid + (size_t)((u - 1) & 3) * (S::LBYTES / 4) + moff2;
                float4 v = update4<S::LW>(mm, mc, mp, r, inv_decay);
                v = pin_faces(v, x2, y2, z, nx, ny, nz, bval);
                *reinterpret_cast<float4*>(out + (size_t)z * sz + (size_t)y2 * nx + x2) = v;
            }
        }
        const bool ok = (u + 3 < NP) ? wait_plane(u + 3) : true;
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) fail(u + 3, u - 1 + NS);  // issued so far: planes < u + NS
            return;
        }
        if (threadIdx.x == 0) issue(u + NS);
    }
}

// ---------------------------------------------------------------- temporal blocking
// k_substep_tb<T, TY, TZ> advances a 32 x TY x TZ block of outputs by T
// substeps in one pass over HBM.  One TMA box brings the block plus a halo of
// T planes (4 columns in x, for 16-byte alignment) into shared buffer A;
// level t = 1..T-1 is computed on the block grown by T-t in every direction
// into the other buffer (A and B alternate); level T is stored to global
// memory.  Every voxel of every level goes through the same separately
// rounded update as k_substep, so T substeps here equal T launches of it bit
// for bit.  Voxels outside the domain are never read by interior voxels
// (faces are pinned), so the TMA zero fill beyond the faces is harmless.
template <int T, int TY, int TZ>
struct TbShape {
    static constexpr int TX = 32, HX = 4;
    static constexpr int W0 = TX + 2 * HX, H0 = TY + 2 * T, D0 = TZ + 2 * T;
    static constexpr int size0 = W0 * H0 * D0;
    // largest level >= 1 region (level 1)
    static constexpr int W1 = TX + 2 * (T - 1), H1 = TY + 2 * (T - 1), D1 = TZ + 2 * (T - 1);
    static constexpr int size1 = W1 * H1 * D1;
    static constexpr int sizeA = (size0 > size1 ? size0 : size1);
    static constexpr size_t smem_bytes = (size_t)(((sizeA + 31) / 32) * 32 + size1) * 4 + 16;
};

template <int T, int TY, int TZ>
__global__ void __launch_bounds__(256) k_substep_tb(const __grid_constant__ CUtensorMap in_map,
                                                    float* __restrict__ out, int nx, int ny, int nz, float r,
                                                    float inv_decay, float bval, olc_u32* status) {
    using S = TbShape<T, TY, TZ>;
    constexpr int TX = S::TX;
    extern __shared__ __align__(128) float smem_raw[];
    // TMA destinations want 128-byte alignment: round the dynamic base up
    float* const smem = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    float* const bufA = smem;
    float* const bufB = smem + ((S::sizeA + 31) / 32) * 32;
    unsigned long long* bar =
        reinterpret_cast<unsigned long long*>((reinterpret_cast<uintptr_t>(bufB + S::size1) + 7) & ~uintptr_t(7));
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
    const olc_u32 bar_a = smem_u32(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a),
                     "r"((olc_u32)(S::size0 * 4))
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(bufA)),
            "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(x0 - S::HX), "r"(y0 - T), "r"(z0 - T),
            "r"(bar_a)
            : "memory");
    }
    // bounded wait for the tile (olc_mbar_wait_bounded records a timeout)
    if (!olc_mbar_wait_bounded(bar_a, 0, status)) return;

    // levels 1 .. T-1 in shared memory
    const float* src = bufA;
    int sw = S::W0, sh = S::H0;           // source dims
    int sox = x0 - S::HX, soy = y0 - T, soz = z0 - T;  // source origin (global coords)
#pragma unroll
    for (int t = 1; t < T; ++t) {
        float* dst = (t & 1) ? bufB : bufA;
        const int g = T - t;
        const int dw = TX + 2 * g, dh = TY + 2 * g, dd = TZ + 2 * g;
        const int dox = x0 - g, doy = y0 - g, doz = z0 - g;
        for (int col = threadIdx.x; col < dw * dh; col += blockDim.x) {
            const int cx = col % dw, cy = col / dw;
            const int gx = dox + cx, gy = doy + cy;
            const int sx = gx - sox, sy = gy - soy;
            const bool edge_xy = gx <= 0 || gy <= 0 || gx >= nx - 1 || gy >= ny - 1;
            int sidx = ((doz - soz - 1) * sh + sy) * sw + sx;
            float zm = src[sidx];
            sidx += sw * sh;
            float c = src[sidx];
            float* d = dst + cy * dw + cx;
            for (int cz = 0; cz < dd; ++cz) {
                const int gz = doz + cz;
                const float zp = src[sidx + sw * sh];
                float v;
                if (edge_xy || gz <= 0 || gz >= nz - 1) {
                    v = bval;
                } else {
                    const float xm = src[sidx - 1], xp = src[sidx + 1];
                    const float ym = src[sidx - sw], yp = src[sidx + sw];
                    const float s = __fadd_rn(__fadd_rn(__fadd_rn(xm, xp), __fadd_rn(ym, yp)), __fadd_rn(zm, zp));
                    const float u = __fadd_rn(c, __fmul_rn(r, __fsub_rn(s, __fmul_rn(6.0f, c))));
                    v = fmaxf(__fmul_rn(u, inv_decay), 0.0f);
                }
                d[cz * dw * dh] = v;
                zm = c;
                c = zp;
                sidx += sw * sh;
            }
        }
        __syncthreads();
        src = dst;
        sw = dw;
        sh = dh;
        sox = dox;
        soy = doy;
        soz = doz;
    }

    // level T: the block's outputs, one column per thread
    for (int col = threadIdx.x; col < TX * TY; col += blockDim.x) {
        const int cx = col % TX, cy = col / TX;
        const int gx = x0 + cx, gy = y0 + cy;
        if (gx >= nx || gy >= ny) continue;
        const int sx = gx - sox, sy = gy - soy;
        const bool edge_xy = gx == 0 || gy == 0 || gx == nx - 1 || gy == ny - 1;
        int sidx = ((z0 - soz - 1) * sh + sy) * sw + sx;
        float zm = src[sidx];
        sidx += sw * sh;
        float c = src[sidx];
        float* o = out + ((size_t)z0 * ny + gy) * nx + gx;
        const size_t sz = (size_t)nx * ny;
        for (int cz = 0; cz < TZ; ++cz) {
            const int gz = z0 + cz;
            if (gz >= nz) break;
            const float zp = src[sidx + sw * sh];
            float v;
            if (edge_xy || gz == 0 || gz == nz - 1) {
                v = bval;
            } else {
                const float xm = src[sidx - 1], xp = src[sidx + 1];
                const float ym = src[sidx - sw], yp = src[sidx + sw];
                const float s = __fadd_rn(__fadd_rn(__fadd_rn(xm, xp), __fadd_rn(ym, yp)), __fadd_rn(zm, zp));
                const float u = __fadd_rn(c, __fmul_rn(r, __fsub_rn(s, __fmul_rn(6.0f, c))));
                v = fmaxf(__fmul_rn(u, inv_decay), 0.0f);
            }
            *o = v;
            o += sz;
            zm = c;
            c = zp;
            sidx += sw * sh;
        }
    }
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

// Temporal-block shapes compiled in; OLC_TB="T,TY,TZ" selects one (default 2,8,16).
#define OLC_TB_SHAPES(X) X(2, 8, 16) X(2, 8, 32) X(2, 16, 16) X(3, 8, 16) X(3, 16, 16) X(4, 16, 16) X(2, 4, 32)

// Default T = 1: on B200 the single-substep TMA kernel (26.9 us per 256^3 FP32
// substep) beats every temporal block measured (T=2: 32 us, T=3: 40 us; the
// intermediate levels make the kernel shared-memory bound at low occupancy).
static void tb_from_env(FieldMaps* m) {
    m->T = 1;
    m->TY = 8;
    m->TZ = 16;
    const char* v = getenv("OLC_TB");
    if (!v) return;
    int T = 0, TY = 0, TZ = 0;
    if (sscanf(v, "%d,%d,%d", &T, &TY, &TZ) != 3) return;
    bool known = T == 1;
#define OLC_TB_MATCH(a, b, c) known = known || (T == a && TY == b && TZ == c);
    OLC_TB_SHAPES(OLC_TB_MATCH)
#undef OLC_TB_MATCH
    if (known) {
        m->T = T;
        m->TY = TY;
        m->TZ = TZ;
    }
}

// 4-wide single-substep shapes compiled in (TYR, TZ); OLC_VX="TYR,TZ" selects
// one, OLC_VX=0 the scalar k_substep_tma.
#define OLC_VX_SHAPES(X) X(16, 8) X(16, 4) X(8, 8) X(8, 16) X(16, 16) X(32, 4)

// Default (8, 8): on B200 with a 256^3 FP32 field, 21.2 us per substep against
// 21.5 for (16, 8), 22.1 for (8, 16) and 25.4 for the scalar kernel.
static void vx_from_env(FieldMaps* m) {
    m->VY = 8;
    m->VZ = 8;
    const char* v = getenv("OLC_VX");
    if (!v) return;
    int a = 0, b = 0;
    if (sscanf(v, "%d,%d", &a, &b) != 2) {
        m->VY = m->VZ = 0;
        return;
    }
    bool known = false;
#define OLC_VX_MATCH(p, q) known = known || (a == p && b == q);
    OLC_VX_SHAPES(OLC_VX_MATCH)
#undef OLC_VX_MATCH
    if (known) {
        m->VY = a;
        m->VZ = b;
    }
}

// Persistent pipeline shapes compiled in (TYR, TZ, NS); OLC_PIPE="TYR,TZ,NS"
// selects one, OLC_PIPE=0 the one-tile-per-CTA kernels.
#define OLC_PIPE_SHAPES(X) X(8, 8, 2) X(8, 8, 3) X(8, 8, 4) X(16, 4, 2) X(16, 4, 3) X(16, 8, 2) X(32, 4, 2)

static void pipe_from_env(FieldMaps* m) {
    m->PY = 0;
    m->PZ = 0;
    m->PN = 0;
    const char* v = getenv("OLC_PIPE");
    if (!v) return;
    int a = 0, b = 0, c = 0;
    if (sscanf(v, "%d,%d,%d", &a, &b, &c) != 3) return;
    bool known = false;
#define OLC_PIPE_MATCH(p, q, n) known = known || (a == p && b == q && c == n);
    OLC_PIPE_SHAPES(OLC_PIPE_MATCH)
#undef OLC_PIPE_MATCH
    if (known) {
        m->PY = a;
        m->PZ = b;
        m->PN = c;
    }
}

// Two-substep shapes compiled in (TYR, ZC, NS); OLC_T2="TYR,ZC,NS" selects
// one, OLC_T2=0 runs one substep per pass.
#define OLC_T2_SHAPES(X) X(8, 16, 6) X(8, 32, 6) X(12, 16, 6) X(12, 32, 6) X(16, 16, 6) X(16, 32, 6) X(8, 32, 8) X(8, 16, 8) X(16, 16, 8)

// Off by default: on B200 with a 256^3 FP32 field the best shape, (16,16,8),
// takes 27.1 us per substep against 21.0 for k_substep_x4.  It halves the
// DRAM traffic but executes 2.3x the instructions of two single passes (the
// intermediate plane covers the patch plus a one-voxel ring, and every plane
// costs a barrier and a TMA wait), so it is issue-bound.
static void t2_from_env(FieldMaps* m) {
    m->T2Y = m->T2Z = m->T2N = 0;
    const char* v = getenv("OLC_T2");
    if (!v) return;
    int a = 0, b = 0, c = 0;
    if (sscanf(v, "%d,%d,%d", &a, &b, &c) != 3) {
        m->T2Y = m->T2Z = m->T2N = 0;
        return;
    }
    bool known = false;
#define OLC_T2_MATCH(p, q, n) known = known || (a == p && b == q && c == n);
    OLC_T2_SHAPES(OLC_T2_MATCH)
#undef OLC_T2_MATCH
    if (known) {
        m->T2Y = a;
        m->T2Z = b;
        m->T2N = c;
    }
}

bool make_field_maps(FieldMaps* m, float* a, float* b, const int dims[3]) {
    using namespace tma;
    m->ok = false;
    tb_from_env(m);
    vx_from_env(m);
    pipe_from_env(m);
    t2_from_env(m);
    const cuuint32_t box1[3] = {WX, WY, WZ};
    if (!encode_map(&m->single[0], a, dims, box1) || !encode_map(&m->single[1], b, dims, box1)) return false;
    if (m->VY > 0) {
        const cuuint32_t boxv[3] = {72, (cuuint32_t)(m->VY + 2), (cuuint32_t)(m->VZ + 2)};
        if (!encode_map(&m->vec[0], a, dims, boxv) || !encode_map(&m->vec[1], b, dims, boxv)) m->VY = m->VZ = 0;
    }
    if (m->T2Y > 0) {
        const cuuint32_t boxt[3] = {80, (cuuint32_t)(m->T2Y + 4), 1};
        if (!encode_map(&m->t2[0], a, dims, boxt) || !encode_map(&m->t2[1], b, dims, boxt)) m->T2Y = 0;
    }
    if (m->PY > 0) {
        const cuuint32_t boxp[3] = {72, (cuuint32_t)(m->PY + 2), (cuuint32_t)(m->PZ + 2)};
        if (!encode_map(&m->pipe[0], a, dims, boxp) || !encode_map(&m->pipe[1], b, dims, boxp)) m->PY = 0;
    }
    if (m->T > 1) {
        const cuuint32_t boxT[3] = {(cuuint32_t)(32 + 8), (cuuint32_t)(m->TY + 2 * m->T),
                                    (cuuint32_t)(m->TZ + 2 * m->T)};
        if (!encode_map(&m->block[0], a, dims, boxT) || !encode_map(&m->block[1], b, dims, boxT)) m->T = 1;
    }
    m->ok = true;
    return true;
}

template <int T, int TY, int TZ>
static void launch_tb(const CUtensorMap& map, float* out, const FieldStep& fs, olc_u32* status, cudaStream_t s) {
    using S = TbShape<T, TY, TZ>;
    const int bytes = (int)S::smem_bytes + 128;
    static int configured_mask = 0;  // per device (up to 32)
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 32 && !(configured_mask & (1 << dev))) {
        cudaFuncSetAttribute(k_substep_tb<T, TY, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        configured_mask |= 1 << dev;
    }
    dim3 grid((fs.dims[0] + 31) / 32, (fs.dims[1] + TY - 1) / TY, (fs.dims[2] + TZ - 1) / TZ);
    k_substep_tb<T, TY, TZ><<<grid, 256, bytes, s>>>(map, out, fs.dims[0], fs.dims[1], fs.dims[2], fs.r,
                                                     fs.inv_decay, fs.bval, status);
}

static void launch_block(const FieldMaps& m, const CUtensorMap& map, float* out, const FieldStep& fs,
                         olc_u32* status, cudaStream_t s) {
#define OLC_TB_LAUNCH(a, b, c)                              \
    if (m.T == a && m.TY == b && m.TZ == c) {               \
        launch_tb<a, b, c>(map, out, fs, status, s);        \
        return;                                             \
    }
    OLC_TB_SHAPES(OLC_TB_LAUNCH)
#undef OLC_TB_LAUNCH
}

void launch_substep_tma(const CUtensorMap& in_map, float* out, const FieldStep& fs, olc_u32* status,
                        cudaStream_t s) {
    using namespace tma;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((fs.dims[0] + TX - 1) / TX, (fs.dims[1] + TY - 1) / TY, (fs.dims[2] + TZ - 1) / TZ);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_substep_tma, in_map, out, fs.dims[0], fs.dims[1], fs.dims[2], fs.r, fs.inv_decay,
                       fs.bval, status);
}

template <int TYR, int TZ>
static void launch_x4(const CUtensorMap& map, float* out, const FieldStep& fs, olc_u32* status, int rev,
                      cudaStream_t s) {
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
                       fs.inv_decay, fs.bval, status, rev);
}

template <int TYR, int TZ, int NS>
static void launch_pipe(const CUtensorMap& map, float* out, const FieldStep& fs, olc_u32* status, int rev,
                        cudaStream_t s) {
    using P = PipeShape<TYR, TZ, NS>;
    static int configured_mask = 0;  // per device (up to 32)
    static int per_sm[32] = {};
    static int sms[32] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 32) return;
    if (!(configured_mask & (1 << dev))) {
        cudaFuncSetAttribute(k_substep_pipe<TYR, TZ, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::SMEM);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[dev], k_substep_pipe<TYR, TZ, NS>, 16 * TYR, P::SMEM);
        cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
        if (per_sm[dev] < 1) per_sm[dev] = 1;
        configured_mask |= 1 << dev;
    }
    const int ntiles = ((fs.dims[0] + 63) / 64) * ((fs.dims[1] + TYR - 1) / TYR) * ((fs.dims[2] + TZ - 1) / TZ);
    const int gmax = per_sm[dev] * sms[dev];
    // as many CTAs as fit, then evened out so every CTA takes the same number of tiles (+-1)
    const int per_cta = (ntiles + gmax - 1) / gmax;
    const int grid = (ntiles + per_cta - 1) / per_cta;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(16 * TYR);
    cfg.dynamicSmemBytes = P::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_substep_pipe<TYR, TZ, NS>, map, out, fs.dims[0], fs.dims[1], fs.dims[2], fs.r,
                       fs.inv_decay, fs.bval, status, rev);
}

static void launch_single(const FieldMaps& m, int cur, float* out, const FieldStep& fs, olc_u32* status, int rev,
                          cudaStream_t s) {
#define OLC_PIPE_LAUNCH(p, q, n)                                  \
    if (m.PY == p && m.PZ == q && m.PN == n) {                    \
        launch_pipe<p, q, n>(m.pipe[cur], out, fs, status, rev, s); \
        return;                                                   \
    }
    OLC_PIPE_SHAPES(OLC_PIPE_LAUNCH)
#undef OLC_PIPE_LAUNCH
#define OLC_VX_LAUNCH(p, q)                                \
    if (m.VY == p && m.VZ == q) {                          \
        launch_x4<p, q>(m.vec[cur], out, fs, status, rev, s); \
        return;                                            \
    }
    OLC_VX_SHAPES(OLC_VX_LAUNCH)
#undef OLC_VX_LAUNCH
    launch_substep_tma(m.single[cur], out, fs, status, s);
}

template <int TYR, int ZC, int NS>
static void launch_t2(const CUtensorMap& map, float* out, const FieldStep& fs, olc_u32* status, int rev,
                      cudaStream_t s) {
    using S = T2Shape<TYR, ZC, NS>;
    static int configured_mask = 0;  // per device (up to 32)
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 32 && !(configured_mask & (1 << dev))) {
        cudaFuncSetAttribute(k_substep_t2<TYR, ZC, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        configured_mask |= 1 << dev;
    }
    const int tiles = ((fs.dims[0] + S::TX - 1) / S::TX) * ((fs.dims[1] + TYR - 1) / TYR) * ((fs.dims[2] + ZC - 1) / ZC);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(tiles);
    cfg.blockDim = dim3(S::THREADS);
    cfg.dynamicSmemBytes = S::SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_substep_t2<TYR, ZC, NS>, map, out, fs.dims[0], fs.dims[1], fs.dims[2], fs.r,
                       fs.inv_decay, fs.bval, status, rev);
}

static bool launch_pair(const FieldMaps& m, int cur, float* out, const FieldStep& fs, olc_u32* status, int rev,
                        cudaStream_t s) {
#define OLC_T2_LAUNCH(p, q, n)                                   \
    if (m.T2Y == p && m.T2Z == q && m.T2N == n) {                \
        launch_t2<p, q, n>(m.t2[cur], out, fs, status, rev, s);  \
        return true;                                             \
    }
    OLC_T2_SHAPES(OLC_T2_LAUNCH)
#undef OLC_T2_LAUNCH
    return false;
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

float* run_substeps_tma(float* a, float* b, const FieldMaps& m, int a_index, const FieldStep& fs, olc_u32* status,
                        cudaStream_t s, const Pins* pins) {
    float* bufs[2];
    bufs[a_index] = a;
    bufs[1 - a_index] = b;
    int cur = a_index;
    int left = fs.substeps;
    // alternate the tile order between substeps (OLC_STENCIL_ORDER=forward keeps one order)
    const char* order = getenv("OLC_STENCIL_ORDER");
    const bool alternate = !(order && std::string(order) == "forward");
    int launch = 0;
    const bool pinned = pins && pins->n > 0;  // pins go between substeps: one substep per launch
    while (left > 0) {
        const int rev = alternate ? (launch & 1) : 0;
        if (!pinned && m.T2Y > 0 && left >= 2 && launch_pair(m, cur, bufs[1 - cur], fs, status, rev, s)) {
            left -= 2;
        } else if (!pinned && m.T > 1 && left >= m.T) {
            launch_block(m, m.block[cur], bufs[1 - cur], fs, status, s);
            left -= m.T;
        } else {
            launch_single(m, cur, bufs[1 - cur], fs, status, rev, s);
            launch_pins(bufs[1 - cur], pins, s);
            left -= 1;
        }
        cur = 1 - cur;
        ++launch;
    }
    return bufs[cur];
}

int launches_for(const FieldMaps& m, int substeps) {
    if (m.T2Y > 0) return substeps / 2 + substeps % 2;
    if (m.T <= 1) return substeps;
    return substeps / m.T + substeps % m.T;
}

bool stencil_tma_enabled() {
    const char* v = getenv("OLC_STENCIL");
    return !(v && std::string(v) == "plain");
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
