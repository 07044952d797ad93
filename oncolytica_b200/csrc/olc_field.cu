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
    bool ready = false;
    for (olc_u32 it = 0; it < OLC_SPIN_LIMIT; ++it) {
        if (mbar_try_wait(bar_a, 0)) {
            ready = true;
            break;
        }
    }
    if (!ready) {
        if (threadIdx.x == 0) atomicOr(status, OLC_ST_TIMEOUT);
        for (olc_u32 it = 0; it < OLC_SPIN_LIMIT && !mbar_try_wait(bar_a, 0); ++it) {
        }
        return;
    }

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

bool make_field_maps(FieldMaps* m, float* a, float* b, const int dims[3]) {
    using namespace tma;
    m->ok = false;
    tb_from_env(m);
    const cuuint32_t box1[3] = {WX, WY, WZ};
    if (!encode_map(&m->single[0], a, dims, box1) || !encode_map(&m->single[1], b, dims, box1)) return false;
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

float* run_substeps_tma(float* a, float* b, const FieldMaps& m, int a_index, const FieldStep& fs, olc_u32* status,
                        cudaStream_t s) {
    float* bufs[2];
    bufs[a_index] = a;
    bufs[1 - a_index] = b;
    int cur = a_index;
    int left = fs.substeps;
    while (left > 0) {
        if (m.T > 1 && left >= m.T) {
            launch_block(m, m.block[cur], bufs[1 - cur], fs, status, s);
            left -= m.T;
        } else {
            launch_substep_tma(m.single[cur], bufs[1 - cur], fs, status, s);
            left -= 1;
        }
        cur = 1 - cur;
    }
    return bufs[cur];
}

int launches_for(const FieldMaps& m, int substeps) {
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
