// Per-step reductions and the RNG known-answer stage.
//
// Reductions restate the engine's metrics (engine/assets/shaders/tumor_sim.wgsl:248-361,
// Kernel_ClearMetrics/CollectMetrics/FinalizeMetrics) without its fixed-point
// scaling: counts are exact integers, sums are FP64, the maximum radius is
// exact.  Field masses are FP64 sums over the field grid.
#include "olc_internal.h"

namespace olc {

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ olc_u32 warp_sum_u(olc_u32 v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Non-negative doubles order like their bit patterns as unsigned 64-bit ints.
__device__ __forceinline__ void atomic_max_nonneg(double* p, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_min_nonneg(double* p, double v) {
    atomicMin(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

// The FP64 sums are deterministic: every block writes its partial sums to
// `partials`, and the last block to finish (a ticket counter, no waiting) adds
// them in block order with a fixed-shape tree.  Counts, the maximum and the
// minima are exact whatever the order, so they stay plain atomics.
__device__ __forceinline__ double block_sum_fixed(double v, double* s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum_d(v);
    if (lane == 0) s_w[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_w[w];
    __syncthreads();
    return t;  // valid in thread 0
}

// Thread 0 of each block publishes `k` partials; returns true in the last block.
__device__ __forceinline__ bool publish_partials(const double* vals, int k, double* partials, olc_u32* ticket,
                                                 bool* s_last) {
    if (threadIdx.x == 0) {
        for (int j = 0; j < k; ++j) partials[(size_t)j * gridDim.x + blockIdx.x] = vals[j];
        __threadfence();
        const olc_u32 t = atomicAdd(ticket, 1u);
        *s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (*s_last) __threadfence();
    return *s_last;
}

__global__ void __launch_bounds__(256) k_reduce_agents(ReduceArgs a, const olc_u32* counters,
                                                       OlcReductions* out, double* partials, olc_u32* ticket) {
    __shared__ olc_u32 s_hist[OLC_RADIAL_BINS];
    __shared__ olc_u32 s_state[OLC_STATE_BINS];
    __shared__ double s_sum[5][8];
    __shared__ olc_u32 s_live[8];
    __shared__ bool s_last;
    const olc_u32 n = olc_total_rows(counters);
    for (int i = threadIdx.x; i < OLC_RADIAL_BINS; i += blockDim.x) s_hist[i] = 0u;
    if (threadIdx.x < OLC_STATE_BINS) s_state[threadIdx.x] = 0u;
    __syncthreads();
    double sx = 0.0, sy = 0.0, sz = 0.0, sr2 = 0.0, mr = 0.0;
    olc_u32 live = 0;
    // per-thread state counts in registers; every row's loads are issued
    // together (the life flag does not gate the position loads), and the lanes
    // of a warp that fall into one radial bin (neighbouring rows, sorted by
    // voxel) add to it once
    olc_u32 sc[OLC_STATE_BINS];
#pragma unroll
    for (int k = 0; k < OLC_STATE_BINS; ++k) sc[k] = 0u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const olc_u32 stride = gridDim.x * blockDim.x;
    const olc_u32 first = blockIdx.x * blockDim.x + threadIdx.x;
    for (olc_u32 base = first - lane; base < n; base += stride) {
        const olc_u32 i = base + lane;
        const bool row = i < n;
        const bool dead = row ? a.life[i] != 0 : true;
        const float px = row ? a.x[i] : 0.0f, py = row ? a.y[i] : 0.0f, pz = row ? a.z[i] : 0.0f;
        const int st = (row && a.state) ? a.state[i] : -1;
        int b = -1;
        if (!dead) {
            ++live;
            sx += (double)px;
            sy += (double)py;
            sz += (double)pz;
            const double dx = (double)px - (double)a.cx, dy = (double)py - (double)a.cy,
                         dz = (double)pz - (double)a.cz;
            const double r2 = dx * dx + dy * dy + dz * dz;
            sr2 += r2;
            const double r = sqrt(r2);
            mr = fmax(mr, r);
            b = (int)(r / (double)a.bin_width);
            if (b >= OLC_RADIAL_BINS) b = OLC_RADIAL_BINS - 1;
#pragma unroll
            for (int k = 0; k < OLC_STATE_BINS; ++k) sc[k] += st == k ? 1u : 0u;
        }
        const olc_u32 peers = __match_any_sync(0xffffffffu, b);
        if (b >= 0 && lane == __ffs(peers) - 1) atomicAdd(&s_hist[b], (olc_u32)__popc(peers));
    }
#pragma unroll
    for (int k = 0; k < OLC_STATE_BINS; ++k) {
        const olc_u32 t = __reduce_add_sync(0xffffffffu, sc[k]);
        if (lane == 0 && t) atomicAdd(&s_state[k], t);
    }
    sx = warp_sum_d(sx);
    sy = warp_sum_d(sy);
    sz = warp_sum_d(sz);
    sr2 = warp_sum_d(sr2);
    mr = warp_max_d(mr);
    live = warp_sum_u(live);
    if (lane == 0) {
        s_sum[0][warp] = sx;
        s_sum[1][warp] = sy;
        s_sum[2][warp] = sz;
        s_sum[3][warp] = sr2;
        s_sum[4][warp] = mr;
        s_live[warp] = live;
    }
    __syncthreads();
    double t[4] = {0, 0, 0, 0};
    if (threadIdx.x == 0) {
        double m = 0.0;
        olc_u32 l = 0;
        for (int w = 0; w < 8; ++w) {
            for (int k = 0; k < 4; ++k) t[k] += s_sum[k][w];
            m = fmax(m, s_sum[4][w]);
            l += s_live[w];
        }
        if (l) {
            atomicAdd(&out->n_live, l);
            atomic_max_nonneg(&out->max_r, m);
        }
    }
    for (int i = threadIdx.x; i < OLC_RADIAL_BINS; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&out->radial_hist[i], s_hist[i]);
    if (threadIdx.x < OLC_STATE_BINS && s_state[threadIdx.x])
        atomicAdd(&out->state_counts[threadIdx.x], s_state[threadIdx.x]);
    if (!publish_partials(t, 4, partials, ticket, &s_last)) return;
    __shared__ double s_w[8];
    double r[4];
    for (int k = 0; k < 4; ++k) {
        double v = 0.0;
        for (olc_u32 b = threadIdx.x; b < gridDim.x; b += blockDim.x) v += __ldcg(partials + (size_t)k * gridDim.x + b);
        r[k] = block_sum_fixed(v, s_w);
    }
    if (threadIdx.x == 0) {
        out->sum_pos[0] = r[0];
        out->sum_pos[1] = r[1];
        out->sum_pos[2] = r[2];
        out->sum_r2 = r[3];
        *ticket = 0u;
    }
}

__global__ void __launch_bounds__(256) k_reduce_field(const float* __restrict__ f, size_t nvox, int slot,
                                                      OlcReductions* out, double* partials, olc_u32* ticket) {
    __shared__ double s_v[3][8];
    __shared__ bool s_last;
    double sum = 0.0, mn = 1e300, mx = 0.0;
    const size_t n4 = nvox / 4;
    const float4* f4 = reinterpret_cast<const float4*>(f);
    // four independent 16-byte loads in flight per thread and iteration (one
    // at a time left the kernel waiting on DRAM latency at half the copy
    // rate); the minimum and maximum in FP32 (exact), the sum in FP64 in a
    // fixed order
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    float lo = __int_as_float(0x7f800000), hi = 0.0f;
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n4; i += 4 * stride) {
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = __ldg(f4 + i + u * stride);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            sum += ((double)v[u].x + (double)v[u].y) + ((double)v[u].z + (double)v[u].w);
            lo = fminf(lo, fminf(fminf(v[u].x, v[u].y), fminf(v[u].z, v[u].w)));
            hi = fmaxf(hi, fmaxf(fmaxf(v[u].x, v[u].y), fmaxf(v[u].z, v[u].w)));
        }
    }
    for (; i < n4; i += stride) {
        const float4 v = __ldg(f4 + i);
        sum += ((double)v.x + (double)v.y) + ((double)v.z + (double)v.w);
        lo = fminf(lo, fminf(fminf(v.x, v.y), fminf(v.z, v.w)));
        hi = fmaxf(hi, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
    }
    mn = fmin(mn, (double)lo);
    mx = fmax(mx, (double)hi);
    if (blockIdx.x == 0) {
        for (size_t i = n4 * 4 + threadIdx.x; i < nvox; i += blockDim.x) {
            double v = (double)f[i];
            sum += v;
            mn = fmin(mn, v);
            mx = fmax(mx, v);
        }
    }
    sum = warp_sum_d(sum);
    mn = warp_min_d(mn);
    mx = warp_max_d(mx);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_v[0][warp] = sum;
        s_v[1][warp] = mn;
        s_v[2][warp] = mx;
    }
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0) {
        double a = 1e300, b = 0.0;
        for (int w = 0; w < 8; ++w) {
            t += s_v[0][w];
            a = fmin(a, s_v[1][w]);
            b = fmax(b, s_v[2][w]);
        }
        atomic_min_nonneg(&out->field_min[slot], a);
        atomic_max_nonneg(&out->field_max[slot], b);
    }
    if (!publish_partials(&t, 1, partials, ticket, &s_last)) return;
    __shared__ double s_w[8];
    double v = 0.0;
    for (olc_u32 b = threadIdx.x; b < gridDim.x; b += blockDim.x) v += __ldcg(partials + b);
    const double r = block_sum_fixed(v, s_w);
    if (threadIdx.x == 0) {
        out->field_mass[slot] = r;
        *ticket = 0u;
    }
}

void launch_reduce_agents(const ReduceArgs& a, const olc_u32* counters, olc_u32 n_cap, OlcReductions* out,
                          const RedScratch& rs, cudaStream_t s) {
    olc_u32 blocks = (n_cap + 255) / 256;
    if (blocks == 0) blocks = 1;
    if (blocks > RED_MAX_BLOCKS) blocks = RED_MAX_BLOCKS;
    k_reduce_agents<<<blocks, 256, 0, s>>>(a, counters, out, rs.partials, rs.tickets);
}

void launch_reduce_field(const float* f, size_t nvox, int slot, OlcReductions* out, const RedScratch& rs,
                         cudaStream_t s) {
    size_t blocks = (nvox / 4 + 255) / 256;
    if (blocks == 0) blocks = 1;
    if (blocks > RED_MAX_BLOCKS) blocks = RED_MAX_BLOCKS;
    k_reduce_field<<<(unsigned)blocks, 256, 0, s>>>(f, nvox, slot, out, rs.partials + (size_t)(4 + slot) * RED_MAX_BLOCKS,
                                                     rs.tickets + 1 + slot);
}

// field_min starts at +inf (all ones in the exponent) for the unsigned min.
__global__ void k_init_reductions(OlcReductions* out, int nfields) {
    if (threadIdx.x < OLC_MAX_FIELDS) out->field_min[threadIdx.x] = 1e300;
}

void launch_reset_reductions(OlcReductions* out, int nfields, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(OlcReductions), s);
    k_init_reductions<<<1, 32, 0, s>>>(out, nfields);
}

__global__ void k_rng(olc_u32* states, olc_u32 n, int draws, float* out, float* dirs) {
    olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    olc_u32 s = states[i];
    for (int k = 0; k < draws; ++k) out[(size_t)i * draws + k] = olc_next_rand(s);
    if (dirs) {
        float3 d = olc_rand_dir(s);
        dirs[3 * (size_t)i + 0] = d.x;
        dirs[3 * (size_t)i + 1] = d.y;
        dirs[3 * (size_t)i + 2] = d.z;
    }
    states[i] = s;
}

void launch_rng(olc_u32* states, olc_u32 n, int draws, float* out, float* dirs, cudaStream_t s) {
    if (n == 0) return;
    k_rng<<<(n + 255) / 256, 256, 0, s>>>(states, n, draws, out, dirs);
}

}  // namespace olc
