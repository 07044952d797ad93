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

#include <cmath>

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
