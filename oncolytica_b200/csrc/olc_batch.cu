// Batched mode: many independent simulations of one model advance in one
// launch per stage.  No counterpart in the reference, which runs one
// simulation per engine.
//
// Layout.  Agents of every simulation share the agent columns; a `_sim`
// column holds each row's simulation index.  The sort key is
// (simulation << key_shift) | bin key, so after the stable sort the rows are
// simulation-major and, inside a simulation, in exactly the order a solo run
// of that simulation produces (same bin keys, ties in the same pre-sort
// order: survivors first, then children in parent order).  Dead rows get the
// key n_sims << key_shift and sort behind every simulation.  The bin table is
// the concatenation of the simulations' tables (OlcSimDesc::ranges_base).
// Each field buffer is the concatenation of the simulations' grids
// (OlcSimDesc::field_off); which of the field's two buffers holds a
// simulation's current grid is a per-(simulation, field) parity byte, since
// simulations take different numbers of substeps.
//
// Every kernel here computes, for each simulation, the same values with the
// same operations as the solo kernels (olc_grid.cu, olc_contact.cu,
// olc_field.cu), so each simulation of a batch reproduces its solo run bit for
// bit.  The FP64 sums of the per-simulation reductions are accumulated with
// atomics and are exact only up to their order.
#include "olc_internal.h"
#include "olc_store16.cuh"

namespace olc {

static unsigned sm_blocks(int per_sm) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return (unsigned)(sms * per_sm);
}

static unsigned grid_cap(olc_u64 n, int threads, unsigned cap) {
    olc_u64 b = (n + threads - 1) / threads;
    if (b == 0) b = 1;
    return (unsigned)(b < cap ? b : cap);
}

// ------------------------------------------------------------------ keys
__device__ __forceinline__ void hist_add_b(olc_u32 (*sh)[RADIX], olc_u32 key, int passes) {
    const olc_u32 active = __activemask();
    const int lane = threadIdx.x & 31;
    for (int p = 0; p < passes; ++p) {
        olc_u32 d = (key >> (8 * p)) & 0xffu;
        olc_u32 peers = __match_any_sync(active, d);
        if ((peers & ((1u << lane) - 1u)) == 0u) atomicAdd(&sh[p][d], (olc_u32)__popc(peers));
    }
}

__global__ void __launch_bounds__(256) k_keys_batch(const float* __restrict__ x, const float* __restrict__ y,
                                                    const float* __restrict__ z, const olc_u32* __restrict__ sim,
                                                    const unsigned char* __restrict__ dead, const olc_u32* counters,
                                                    const OlcSimDesc* __restrict__ sims, int shift,
                                                    olc_u32 sentinel, olc_u32* __restrict__ keys,
                                                    olc_u32* __restrict__ hist, int passes, olc_u32* dead_ctr) {
    __shared__ olc_u32 sh[MAX_PASSES][RADIX];
    __shared__ olc_u32 s_dead;
    const olc_u32 n = olc_total_rows(counters);
    for (int i = threadIdx.x; i < MAX_PASSES * RADIX; i += blockDim.x) (&sh[0][0])[i] = 0u;
    if (threadIdx.x == 0) s_dead = 0u;
    __syncthreads();
    olc_u32 my_dead = 0;
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        olc_u32 k;
        if (dead[i]) {
            k = sentinel;
            ++my_dead;
        } else {
            const olc_u32 s = sim[i];
            const OlcSimDesc& d = sims[s];
            const int cx = olc_bin_coord(x[i], d.tvs, d.tdims[0]);
            const int cy = olc_bin_coord(y[i], d.tvs, d.tdims[1]);
            const int cz = olc_bin_coord(z[i], d.tvs, d.tdims[2]);
            k = (s << shift) | olc_tissue_key(cx, cy, cz);
        }
        keys[i] = k;
        hist_add_b(sh, k, passes);
    }
    for (int o = 16; o > 0; o >>= 1) my_dead += __shfl_xor_sync(0xffffffffu, my_dead, o);
    if ((threadIdx.x & 31) == 0 && my_dead) atomicAdd(&s_dead, my_dead);
    __syncthreads();
    for (int i = threadIdx.x; i < passes * RADIX; i += blockDim.x) {
        olc_u32 v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
    if (threadIdx.x == 0 && s_dead) atomicAdd(dead_ctr, s_dead);
}

void launch_keys_batch(const BatchArgs& b, const float* x, const float* y, const float* z, const olc_u32* sim,
                       const unsigned char* dead, const olc_u32* counters, olc_u32 n_cap, olc_u32* keys,
                       olc_u32* hist, int passes, olc_u32* dead_ctr, cudaStream_t s) {
    k_keys_batch<<<grid_cap(n_cap, 256, sm_blocks(8)), 256, 0, s>>>(x, y, z, sim, dead, counters, b.sims, b.shift,
                                                                      b.sentinel, keys, hist, passes, dead_ctr);
}

// ------------------------------------------------------------------ bin table
__global__ void __launch_bounds__(256) k_bin_ranges_batch(const olc_u32* __restrict__ keys, const olc_u32* n_dev,
                                                          const OlcSimDesc* __restrict__ sims, int shift,
                                                          olc_u32 n_sims, olc_u32* __restrict__ ranges) {
    const olc_u32 n = *n_dev;
    const olc_u32 mask = (1u << shift) - 1u;
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const olc_u32 k = keys[i];
        const olc_u32 s = k >> shift;
        if (s >= n_sims) continue;  // dead rows
        const olc_u64 e = (olc_u64)sims[s].ranges_base + (k & mask);
        if (i == 0 || keys[i - 1] != k) ranges[2 * e] = i;
        if (i + 1 == n || keys[i + 1] != k) ranges[2 * e + 1] = i + 1;
    }
}

void launch_bin_ranges_batch(const BatchArgs& b, const olc_u32* keys, const olc_u32* n_dev, olc_u32 n_cap,
                             olc_u32* ranges, cudaStream_t s) {
    k_bin_ranges_batch<<<grid_cap(n_cap, 256, sm_blocks(8)), 256, 0, s>>>(keys, n_dev, b.sims, b.shift, b.n_sims,
                                                                            ranges);
}

// ------------------------------------------------------------------ contact
// k_contact with the agent's simulation supplying the bin grid, the bin-table
// base and the clamp box.
__global__ void __launch_bounds__(256) k_contact_batch(const float4* __restrict__ posr,
                                                       const uint2* __restrict__ ranges,
                                                       const olc_u32* __restrict__ sim, const olc_u32* n_dev,
                                                       const OlcSimDesc* __restrict__ sims, ContactDev c,
                                                       float* __restrict__ xo, float* __restrict__ yo,
                                                       float* __restrict__ zo) {
    const olc_u32 n = *n_dev;
    const float md = __fmul_rn(c.mobility, c.dt);
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = posr[i];
        if (p.w < 0.0f) continue;
        const OlcSimDesc& d = sims[sim[i]];
        const uint2* rg0 = ranges + d.ranges_base;
        const int cx = olc_bin_coord(p.x, d.tvs, d.tdims[0]);
        const int cy = olc_bin_coord(p.y, d.tvs, d.tdims[1]);
        const int cz = olc_bin_coord(p.z, d.tvs, d.tdims[2]);
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        const olc_u32 kx[3] = {olc_tissue_axis(cx - 1, 0), olc_tissue_axis(cx, 0), olc_tissue_axis(cx + 1, 0)};
        const olc_u32 ky[3] = {olc_tissue_axis(cy - 1, 1), olc_tissue_axis(cy, 1), olc_tissue_axis(cy + 1, 1)};
        const olc_u32 kz[3] = {olc_tissue_axis(cz - 1, 2), olc_tissue_axis(cz, 2), olc_tissue_axis(cz + 1, 2)};
        for (int dz = -1; dz <= 1; ++dz) {
            const int nz = cz + dz;
            if (nz < 0 || nz >= d.tdims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int ny = cy + dy;
                if (ny < 0 || ny >= d.tdims[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = cx + dx;
                    if (nx < 0 || nx >= d.tdims[0]) continue;
                    const uint2 rg = __ldg(rg0 + (kx[dx + 1] | ky[dy + 1] | kz[dz + 1]));
                    for (olc_u32 j = rg.x; j < rg.y; ++j) {
                        if (j == i) continue;
                        const float4 q = __ldg(posr + j);
                        if (q.w < 0.0f) continue;
                        const float ddx = __fsub_rn(p.x, q.x);
                        const float ddy = __fsub_rn(p.y, q.y);
                        const float ddz = __fsub_rn(p.z, q.z);
                        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)),
                                                   __fmul_rn(ddz, ddz));
                        const float rsum = __fadd_rn(p.w, q.w);
                        if (d2 > __fmul_rn(__fmul_rn(rsum, rsum), 1.00000095367431640625f)) continue;
                        const float dist = sqrtf(d2);
                        if (!(dist < rsum)) continue;
                        const float ov = __fsub_rn(rsum, dist);
                        const float f = __fmul_rn(__fmul_rn(c.stiffness, ov), sqrtf(ov));
                        if (dist < 1e-5f) {
                            fx = __fadd_rn(fx, i < j ? -f : f);
                        } else {
                            const float sc = __fdiv_rn(f, dist);
                            fx = __fadd_rn(fx, __fmul_rn(ddx, sc));
                            fy = __fadd_rn(fy, __fmul_rn(ddy, sc));
                            fz = __fadd_rn(fz, __fmul_rn(ddz, sc));
                        }
                    }
                }
            }
        }
        float mx = __fmul_rn(fx, md), my = __fmul_rn(fy, md), mz = __fmul_rn(fz, md);
        const float len = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(mx, mx), __fmul_rn(my, my)), __fmul_rn(mz, mz)));
        if (len > c.max_disp) {
            const float sc = __fdiv_rn(c.max_disp, len);
            mx = __fmul_rn(mx, sc);
            my = __fmul_rn(my, sc);
            mz = __fmul_rn(mz, sc);
        }
        xo[i] = fminf(fmaxf(__fadd_rn(p.x, mx), d.lo[0]), d.hi[0]);
        yo[i] = fminf(fmaxf(__fadd_rn(p.y, my), d.lo[1]), d.hi[1]);
        zo[i] = fminf(fmaxf(__fadd_rn(p.z, mz), d.lo[2]), d.hi[2]);
    }
}

void launch_contact_batch(const BatchArgs& b, const float4* posr, const olc_u32* ranges, const olc_u32* sim,
                          const olc_u32* n_dev, olc_u32 n_cap, const ContactDev& c, float* x, float* y, float* z,
                          cudaStream_t s) {
    k_contact_batch<<<grid_cap(n_cap, 256, sm_blocks(8)), 256, 0, s>>>(
        posr, reinterpret_cast<const uint2*>(ranges), sim, n_dev, b.sims, c, x, y, z);
}

// ------------------------------------------------------------------ fields
// A field tile: BT_X x BT_Y x BT_Z voxels of one simulation's grid, 128
// threads.  The FP32 substep gives each thread four consecutive x voxels of
// one row, walking the tile's planes with the z neighbours in registers;
// neighbours are read with plain loads (reads that would leave the grid
// return 0 and only ever feed face voxels, which are pinned).  16-bit fields
// take their substeps on TMA tiles (k_substep_batch_t16).
constexpr int BT_X = BATCH_TILE_X, BT_Y = BATCH_TILE_Y, BT_Z = BATCH_TILE_Z;

__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

__device__ __forceinline__ float4 update4_b(float xl, float xr, float4 c, float4 ym, float4 yp, float4 zm,
                                            float4 zp, float r, float inv_decay) {
    float4 v;
    v.x = __fadd_rn(__fadd_rn(__fadd_rn(xl, c.y), __fadd_rn(ym.x, yp.x)), __fadd_rn(zm.x, zp.x));
    v.y = __fadd_rn(__fadd_rn(__fadd_rn(c.x, c.z), __fadd_rn(ym.y, yp.y)), __fadd_rn(zm.y, zp.y));
    v.z = __fadd_rn(__fadd_rn(__fadd_rn(c.y, c.w), __fadd_rn(ym.z, yp.z)), __fadd_rn(zm.z, zp.z));
    v.w = __fadd_rn(__fadd_rn(__fadd_rn(c.z, xr), __fadd_rn(ym.w, yp.w)), __fadd_rn(zm.w, zp.w));
    v.x = fmaxf(__fmul_rn(__fadd_rn(c.x, __fmul_rn(r, __fsub_rn(v.x, __fmul_rn(6.0f, c.x)))), inv_decay), 0.0f);
    v.y = fmaxf(__fmul_rn(__fadd_rn(c.y, __fmul_rn(r, __fsub_rn(v.y, __fmul_rn(6.0f, c.y)))), inv_decay), 0.0f);
    v.z = fmaxf(__fmul_rn(__fadd_rn(c.z, __fmul_rn(r, __fsub_rn(v.z, __fmul_rn(6.0f, c.z)))), inv_decay), 0.0f);
    v.w = fmaxf(__fmul_rn(__fadd_rn(c.w, __fmul_rn(r, __fsub_rn(v.w, __fmul_rn(6.0f, c.w)))), inv_decay), 0.0f);
    return v;
}

__global__ void __launch_bounds__(128) k_substep_batch(const uint4* __restrict__ tiles,
                                                       const OlcSimDesc* __restrict__ sims,
                                                       const FieldStep* __restrict__ steps, int field, int n_fields,
                                                       const unsigned char* __restrict__ fpar, int sub,
                                                       float* fa, float* fb) {
    const uint4 t = tiles[blockIdx.x];
    const olc_u32 k = t.x;
    const OlcSimDesc& d = sims[k];
    const FieldStep fs = steps[(size_t)k * n_fields + field];
    const int nx = d.cdims[0], ny = d.cdims[1], nz = d.cdims[2];
    const bool flip = ((fpar[(size_t)k * n_fields + field] ^ (unsigned)sub) & 1u) != 0u;
    const float* in = (flip ? fb : fa) + d.field_off;
    float* out = (flip ? fa : fb) + d.field_off;
    const int x = (int)t.y * BT_X + 4 * (threadIdx.x & 7);
    const int y = (int)t.z * BT_Y + (threadIdx.x >> 3);
    const int depth = (int)(t.w >> 16);  // the member's tile depth (8, 16 or 32 planes)
    const int z0 = (int)(t.w & 0xffffu) * depth;
    if (x >= nx || y >= ny) return;
    const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
    const bool edge_y = y == 0 || y == ny - 1;
    const bool ex0 = x == 0, ex3 = x + 3 == nx - 1;
    const float4 zero = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    size_t idx = (size_t)z0 * sz + (size_t)y * sy + x;
    float4 zm = z0 > 0 ? ld4(in + idx - sz) : zero;
    float4 c = ld4(in + idx);
    const int z1 = min(z0 + depth, nz);
    for (int zz = z0; zz < z1; ++zz, idx += sz) {
        const float4 zp = zz + 1 < nz ? ld4(in + idx + sz) : zero;
        const float4 ym = y > 0 ? ld4(in + idx - sy) : zero;
        const float4 yp = y + 1 < ny ? ld4(in + idx + sy) : zero;
        const float xl = x > 0 ? __ldg(in + idx - 1) : 0.0f;
        const float xr = x + 4 < nx ? __ldg(in + idx + 4) : 0.0f;
        float4 v = update4_b(xl, xr, c, ym, yp, zm, zp, fs.r, fs.inv_decay);
        if (edge_y || zz == 0 || zz == nz - 1) {
            v = make_float4(fs.bval, fs.bval, fs.bval, fs.bval);
        } else {
            if (ex0) v.x = fs.bval;
            if (ex3) v.w = fs.bval;
        }
        *reinterpret_cast<float4*>(out + idx) = v;
        zm = c;
        c = zp;
    }
}

void launch_substep_batch(const BatchArgs& b, const uint4* tiles, olc_u32 n_tiles, const FieldStep* steps, int field,
                          int n_fields, const unsigned char* fpar, int sub, float* fa, float* fb, cudaStream_t s) {
    if (n_tiles == 0) return;
    k_substep_batch<<<n_tiles, 128, 0, s>>>(tiles, b.sims, steps, field, n_fields, fpar, sub, fa, fb);
}

// f <- f / (1 + K dt) on interior voxels, K <- 0, per tile (as k_sink).
__global__ void __launch_bounds__(128) k_sink_batch(const uint4* __restrict__ tiles,
                                                    const OlcSimDesc* __restrict__ sims,
                                                    const FieldStep* __restrict__ steps, int field, int n_fields,
                                                    const unsigned char* __restrict__ fpar, float* fa, float* fb,
                                                    float* sink) {
    const uint4 t = tiles[blockIdx.x];
    const olc_u32 k = t.x;
    const OlcSimDesc& d = sims[k];
    const FieldStep fs = steps[(size_t)k * n_fields + field];
    if (fs.substeps == 0) return;
    const int nx = d.cdims[0], ny = d.cdims[1], nz = d.cdims[2];
    float* f = ((fpar[(size_t)k * n_fields + field] & 1u) ? fb : fa) + d.field_off;
    float* K = sink + d.field_off;
    const int x0 = (int)t.y * BT_X + 4 * (threadIdx.x & 7);
    const int y = (int)t.z * BT_Y + (threadIdx.x >> 3);
    const int z0 = (int)t.w * BT_Z;
    if (x0 >= nx || y >= ny) return;
    const int z1 = min(z0 + BT_Z, nz);
    for (int z = z0; z < z1; ++z) {
        for (int x = x0; x < x0 + 4; ++x) {
            const size_t v = ((size_t)z * ny + y) * nx + x;
            const float kv = K[v];
            if (kv != 0.0f) {
                const bool face = x == 0 || y == 0 || z == 0 || x == nx - 1 || y == ny - 1 || z == nz - 1;
                if (!face) f[v] = __fdiv_rn(f[v], __fadd_rn(1.0f, __fmul_rn(kv, fs.sink_dt)));
                K[v] = 0.0f;
            }
        }
    }
}

void launch_sink_batch(const BatchArgs& b, const uint4* tiles, olc_u32 n_tiles, const FieldStep* steps, int field,
                       int n_fields, const unsigned char* fpar, float* fa, float* fb, float* sink, cudaStream_t s) {
    if (n_tiles == 0 || !sink) return;
    k_sink_batch<<<n_tiles, 128, 0, s>>>(tiles, b.sims, steps, field, n_fields, fpar, fa, fb, sink);
}

// After a field's substeps: simulations that took an odd number of substeps
// now hold the field in the other buffer.
__global__ void k_flip_parity(const FieldStep* __restrict__ steps, int field, int n_fields, olc_u32 n_sims,
                              unsigned char* fpar) {
    for (olc_u32 k = blockIdx.x * blockDim.x + threadIdx.x; k < n_sims; k += gridDim.x * blockDim.x) {
        const size_t j = (size_t)k * n_fields + field;
        fpar[j] ^= (unsigned char)(steps[j].substeps & 1);
    }
}

void launch_flip_parity(const FieldStep* steps, int field, int n_fields, olc_u32 n_sims, unsigned char* fpar,
                        cudaStream_t s) {
    k_flip_parity<<<(n_sims + 255) / 256, 256, 0, s>>>(steps, field, n_fields, n_sims, fpar);
}

// After a chemistry rule: every member holds every field in its other buffer.
__global__ void k_flip_parity_all(int n_fields, olc_u32 n_sims, unsigned char* fpar) {
    const size_t total = (size_t)n_sims * n_fields;
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < total; j += (size_t)gridDim.x * blockDim.x)
        fpar[j] ^= (unsigned char)1;
}

void launch_flip_parity_all(int n_fields, olc_u32 n_sims, unsigned char* fpar, cudaStream_t s) {
    const size_t total = (size_t)n_sims * n_fields;
    if (total == 0) return;
    k_flip_parity_all<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(n_fields, n_sims, fpar);
}

// ------------------------------------------------------------------ 16-bit fields
// The reaction pass and the reductions on BF16 / FP16 storage
// (olc_field16.cu's arithmetic).
template <int ST, int EN>
__global__ void __launch_bounds__(128) k_react_batch16(const uint4* __restrict__ tiles,
                                                       const OlcSimDesc* __restrict__ sims,
                                                       const FieldStep* __restrict__ steps, int field, int n_fields,
                                                       const unsigned char* __restrict__ fpar, unsigned short* fa,
                                                       unsigned short* fb, float* sink, float* comp) {
    const uint4 t = tiles[blockIdx.x];
    const olc_u32 k = t.x;
    const OlcSimDesc& d = sims[k];
    const FieldStep fs = steps[(size_t)k * n_fields + field];
    if (fs.substeps == 0) return;
    const EncConst ek = {fs.bval, fs.half_b, fs.quarter_b, fs.upper_q};
    const int nx = d.cdims[0], ny = d.cdims[1], nz = d.cdims[2];
    unsigned short* f = ((fpar[(size_t)k * n_fields + field] & 1u) ? fb : fa) + d.field_off;
    float* K = sink ? sink + d.field_off : nullptr;
    float* cp = comp + d.field_off;
    const int x0 = (int)t.y * BT_X + 4 * (threadIdx.x & 7);
    const int y = (int)t.z * BT_Y + (threadIdx.x >> 3);
    const int z0 = (int)t.w * BT_Z;
    if (x0 >= nx || y >= ny) return;
    const int z1 = min(z0 + BT_Z, nz);
    // four voxels per thread with 8- and 16-byte accesses when the row and the
    // member's offset keep them aligned (batched grids have x extents that are
    // multiples of 8, so this always holds there); the arithmetic is the same
    const bool vec = ((nx & 3) == 0) && ((d.field_off & 3) == 0);
    for (int z = z0; z < z1; ++z) {
        const bool face_yz = y == 0 || z == 0 || y == ny - 1 || z == nz - 1;
        const size_t v0 = ((size_t)z * ny + y) * nx + x0;
        if (vec) {
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
            const float4 c4 = *reinterpret_cast<const float4*>(cp + v0);
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
            *reinterpret_cast<float4*>(cp + v0) = make_float4(c[0], c[1], c[2], c[3]);
            continue;
        }
        for (int x = x0; x < x0 + 4 && x < nx; ++x) {
            const size_t v = v0 + (x - x0);
            float kv = 0.0f;
            if (K) {
                kv = K[v];
                if (kv != 0.0f) K[v] = 0.0f;
            }
            if (x == 0 || x == nx - 1 || face_yz) continue;
            unsigned short h = f[v];
            float c = cp[v];
            react_voxel<ST, EN>(h, c, kv, fs, ek);
            f[v] = h;
            cp[v] = c;
        }
    }
}

template <int ST, int EN>
__global__ void __launch_bounds__(128) k_reduce_field_batch16(const uint4* __restrict__ tiles,
                                                              const OlcSimDesc* __restrict__ sims,
                                                              const FieldStep* __restrict__ steps, int field,
                                                              int n_fields, const unsigned char* __restrict__ fpar,
                                                              const unsigned short* fa, const unsigned short* fb,
                                                              const float* comp, OlcReductions* out) {
    __shared__ double s_v[3][4];
    const uint4 t = tiles[blockIdx.x];
    const olc_u32 k = t.x;
    const OlcSimDesc& d = sims[k];
    const int nx = d.cdims[0], ny = d.cdims[1], nz = d.cdims[2];
    const unsigned short* f = ((fpar[(size_t)k * n_fields + field] & 1u) ? fb : fa) + d.field_off;
    const float* cp = comp + d.field_off;
    const FieldStep& fs = steps[(size_t)k * n_fields + field];
    const EncConst ek = {fs.bval, fs.half_b, fs.quarter_b, fs.upper_q};
    const int x0 = (int)t.y * BT_X + 4 * (threadIdx.x & 7);
    const int y = (int)t.z * BT_Y + (threadIdx.x >> 3);
    const int z0 = (int)t.w * BT_Z;
    double sum = 0.0, mn = 1e300, mx = 0.0;
    if (x0 < nx && y < ny) {
        const int z1 = min(z0 + BT_Z, nz);
        for (int z = z0; z < z1; ++z)
            for (int x = x0; x < x0 + 4; ++x) {
                const size_t v = ((size_t)z * ny + y) * nx + x;
                const double val = (double)phys_with_residual<ST, EN>(f[v], cp[v], ek);
                sum += val;
                mn = fmin(mn, val);
                mx = fmax(mx, val);
            }
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
        double a = 0.0, lo = 1e300, hi = 0.0;
        for (int w = 0; w < 4; ++w) {
            a += s_v[0][w];
            lo = fmin(lo, s_v[1][w]);
            hi = fmax(hi, s_v[2][w]);
        }
        atomicAdd(&out[k].field_mass[field], a);
        atomicMin(reinterpret_cast<unsigned long long*>(&out[k].field_min[field]), (unsigned long long)__double_as_longlong(lo));
        atomicMax(reinterpret_cast<unsigned long long*>(&out[k].field_max[field]), (unsigned long long)__double_as_longlong(hi));
    }
}

void launch_react_batch16(const BatchArgs& b, int storage, int encoding, const uint4* tiles, olc_u32 n_tiles,
                          const FieldStep* steps, int field, int n_fields, const unsigned char* fpar, void* fa,
                          void* fb, float* sink, float* comp, cudaStream_t s) {
    if (n_tiles == 0) return;
    unsigned short* a = static_cast<unsigned short*>(fa);
    unsigned short* c = static_cast<unsigned short*>(fb);
    with_storage16(storage, encoding, [&](auto st, auto en) {
        k_react_batch16<BaseOf<decltype(st)::value>::value, decltype(en)::value>
            <<<n_tiles, 128, 0, s>>>(tiles, b.sims, steps, field, n_fields, fpar, a, c, sink, comp);
    });
}

void launch_reduce_field_batch16(const BatchArgs& b, int storage, int encoding, const uint4* tiles, olc_u32 n_tiles,
                                 const FieldStep* steps, int field, int n_fields, const unsigned char* fpar,
                                 const void* fa, const void* fb, const float* comp, OlcReductions* out,
                                 cudaStream_t s) {
    if (n_tiles == 0) return;
    const unsigned short* a = static_cast<const unsigned short*>(fa);
    const unsigned short* c = static_cast<const unsigned short*>(fb);
    with_storage16(storage, encoding, [&](auto st, auto en) {
        k_reduce_field_batch16<BaseOf<decltype(st)::value>::value, decltype(en)::value>
            <<<n_tiles, 128, 0, s>>>(tiles, b.sims, steps, field, n_fields, fpar, a, c, comp, out);
    });
}

// ------------------------------------------------------------------ reductions
__device__ __forceinline__ void atomic_max_nonneg_b(double* p, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_min_nonneg_b(double* p, double v) {
    atomicMin(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

// Per-simulation agent reductions (the solo k_reduce_agents per row, with the
// row's simulation choosing the output record, centre and bin width).
__global__ void __launch_bounds__(256) k_reduce_agents_batch(const float* __restrict__ x, const float* __restrict__ y,
                                                             const float* __restrict__ z, const int* __restrict__ state,
                                                             const olc_u32* __restrict__ sim,
                                                             const unsigned char* __restrict__ life,
                                                             const olc_u32* counters,
                                                             const OlcSimDesc* __restrict__ sims, OlcReductions* out) {
    const olc_u32 n = olc_total_rows(counters);
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (life[i]) continue;
        const olc_u32 s = sim[i];
        const OlcSimDesc& d = sims[s];
        OlcReductions* o = out + s;
        const float px = x[i], py = y[i], pz = z[i];
        atomicAdd(&o->n_live, 1u);
        atomicAdd(&o->sum_pos[0], (double)px);
        atomicAdd(&o->sum_pos[1], (double)py);
        atomicAdd(&o->sum_pos[2], (double)pz);
        const double dx = (double)px - (double)d.center[0], dy = (double)py - (double)d.center[1],
                     dz = (double)pz - (double)d.center[2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        atomicAdd(&o->sum_r2, r2);
        const double r = sqrt(r2);
        atomic_max_nonneg_b(&o->max_r, r);
        int b = (int)(r / (double)(d.bin_width > 0.0f ? d.bin_width : 1.0f));
        if (b >= OLC_RADIAL_BINS) b = OLC_RADIAL_BINS - 1;
        atomicAdd(&o->radial_hist[b], 1u);
        if (state) {
            const int st = state[i];
            if (st >= 0 && st < OLC_STATE_BINS) atomicAdd(&o->state_counts[st], 1u);
        }
    }
}

void launch_reduce_agents_batch(const BatchArgs& b, const ReduceArgs& a, const olc_u32* sim, const olc_u32* counters,
                                olc_u32 n_cap, OlcReductions* out, cudaStream_t s) {
    k_reduce_agents_batch<<<grid_cap(n_cap, 256, sm_blocks(4)), 256, 0, s>>>(a.x, a.y, a.z, a.state, sim, a.life,
                                                                            counters, b.sims, out);
}

// Field mass / min / max per simulation: one block per tile.
__global__ void __launch_bounds__(128) k_reduce_field_batch(const uint4* __restrict__ tiles,
                                                            const OlcSimDesc* __restrict__ sims, int field,
                                                            int n_fields, const unsigned char* __restrict__ fpar,
                                                            const float* fa, const float* fb, OlcReductions* out) {
    __shared__ double s_v[3][4];
    const uint4 t = tiles[blockIdx.x];
    const olc_u32 k = t.x;
    const OlcSimDesc& d = sims[k];
    const int nx = d.cdims[0], ny = d.cdims[1], nz = d.cdims[2];
    const float* f = ((fpar[(size_t)k * n_fields + field] & 1u) ? fb : fa) + d.field_off;
    const int x0 = (int)t.y * BT_X + 4 * (threadIdx.x & 7);
    const int y = (int)t.z * BT_Y + (threadIdx.x >> 3);
    const int z0 = (int)t.w * BT_Z;
    double sum = 0.0, mn = 1e300, mx = 0.0;
    if (x0 < nx && y < ny) {
        const int z1 = min(z0 + BT_Z, nz);
        for (int z = z0; z < z1; ++z) {
            const float4 v = ld4(f + ((size_t)z * ny + y) * nx + x0);
            sum += ((double)v.x + (double)v.y) + ((double)v.z + (double)v.w);
            mn = fmin(mn, fmin(fmin((double)v.x, (double)v.y), fmin((double)v.z, (double)v.w)));
            mx = fmax(mx, fmax(fmax((double)v.x, (double)v.y), fmax((double)v.z, (double)v.w)));
        }
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
        double a = 0.0, lo = 1e300, hi = 0.0;
        for (int w = 0; w < 4; ++w) {
            a += s_v[0][w];
            lo = fmin(lo, s_v[1][w]);
            hi = fmax(hi, s_v[2][w]);
        }
        atomicAdd(&out[k].field_mass[field], a);
        atomic_min_nonneg_b(&out[k].field_min[field], lo);
        atomic_max_nonneg_b(&out[k].field_max[field], hi);
    }
}

void launch_reduce_field_batch(const BatchArgs& b, const uint4* tiles, olc_u32 n_tiles, int field, int n_fields,
                               const unsigned char* fpar, const float* fa, const float* fb, OlcReductions* out,
                               cudaStream_t s) {
    if (n_tiles == 0) return;
    k_reduce_field_batch<<<n_tiles, 128, 0, s>>>(tiles, b.sims, field, n_fields, fpar, fa, fb, out);
}

__global__ void k_init_reductions_batch(OlcReductions* out, olc_u32 n_sims) {
    for (olc_u32 k = blockIdx.x * blockDim.x + threadIdx.x; k < n_sims; k += gridDim.x * blockDim.x)
        for (int f = 0; f < OLC_MAX_FIELDS; ++f) out[k].field_min[f] = 1e300;
}

void launch_reset_reductions_batch(OlcReductions* out, olc_u32 n_sims, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(OlcReductions) * n_sims, s);
    k_init_reductions_batch<<<(n_sims + 255) / 256, 256, 0, s>>>(out, n_sims);
}

}  // namespace olc
