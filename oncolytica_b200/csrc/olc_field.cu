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

#include <cuda.h>  // CUtensorMap (types only; the encoder comes from cudaGetDriverEntryPoint)

#include <cmath>
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
    for (int i = 0; i < 3; ++i) out->dims[i] = dims[i];
    out->r = r;
    out->inv_decay = 1.0f / (1.0f + d.decay * dts);
    out->bval = d.boundary;
    out->sink_dt = dt;
    out->substeps = d.substeps;
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

__device__ __forceinline__ bool mbar_try_wait(olc_u32 bar, olc_u32 parity) {
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

__global__ void __launch_bounds__(256) k_substep_tma(const __grid_constant__ CUtensorMap in_map,
                                                     float* __restrict__ out, int nx, int ny, int nz, float r,
                                                     float inv_decay, float bval, olc_u32* status) {
    using namespace tma;
    __shared__ alignas(128) float tile[WZ][WY][WX];
    __shared__ alignas(8) unsigned long long bar;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
    const olc_u32 bar_a = smem_u32(&bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(&tile[0][0][0])),
            "l"(reinterpret_cast<unsigned long long>(&in_map)), "r"(x0 - HX), "r"(y0 - 1), "r"(z0 - 1), "r"(bar_a)
            : "memory");
    }
    // bounded wait for the tile
    bool ready = false;
    for (olc_u32 it = 0; it < OLC_SPIN_LIMIT; ++it) {
        if (mbar_try_wait(bar_a, 0)) {
            ready = true;
            break;
        }
    }
    if (!ready) {
        if (threadIdx.x == 0) atomicOr(status, OLC_ST_TIMEOUT);
        // give the copy in flight a second bounded chance to land before the
        // block's shared memory is released
        for (olc_u32 it = 0; it < OLC_SPIN_LIMIT && !mbar_try_wait(bar_a, 0); ++it) {
        }
        return;
    }
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

bool make_field_map(CUtensorMap* map, float* base, const int dims[3]) {
    using namespace tma;
    if ((dims[0] * 4) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0) return false;
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t gdim[3] = {(cuuint64_t)dims[0], (cuuint64_t)dims[1], (cuuint64_t)dims[2]};
    cuuint64_t gstride[2] = {(cuuint64_t)dims[0] * 4, (cuuint64_t)dims[0] * dims[1] * 4};
    cuuint32_t box[3] = {WX, WY, WZ};
    cuuint32_t estride[3] = {1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, gdim, gstride, box, estride,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void launch_substep_tma(const CUtensorMap& in_map, float* out, const FieldStep& fs, olc_u32* status,
                        cudaStream_t s) {
    using namespace tma;
    dim3 grid((fs.dims[0] + TX - 1) / TX, (fs.dims[1] + TY - 1) / TY, (fs.dims[2] + TZ - 1) / TZ);
    k_substep_tma<<<grid, 256, 0, s>>>(in_map, out, fs.dims[0], fs.dims[1], fs.dims[2], fs.r, fs.inv_decay,
                                       fs.bval, status);
}

float* run_substeps_tma(float* a, float* b, const CUtensorMap& map_a, const CUtensorMap& map_b,
                        const FieldStep& fs, olc_u32* status, cudaStream_t s) {
    float* cur = a;
    for (int i = 0; i < fs.substeps; ++i) {
        const bool from_a = cur == a;
        launch_substep_tma(from_a ? map_a : map_b, from_a ? b : a, fs, status, s);
        cur = from_a ? b : a;
    }
    return cur;
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

float* run_substeps(float* a, float* b, const FieldStep& fs, cudaStream_t s) {
    float* cur = a;
    float* nxt = b;
    for (int i = 0; i < fs.substeps; ++i) {
        launch_substep(cur, nxt, fs, s);
        float* t = cur;
        cur = nxt;
        nxt = t;
    }
    return cur;
}

float* run_field_step(float* a, float* b, float* sink, const FieldStep& fs, cudaStream_t s) {
    launch_sink(a, sink, fs, s);
    float* cur = a;
    float* nxt = b;
    for (int i = 0; i < fs.substeps; ++i) {
        launch_substep(cur, nxt, fs, s);
        float* t = cur;
        cur = nxt;
        nxt = t;
    }
    return cur;
}

}  // namespace olc
