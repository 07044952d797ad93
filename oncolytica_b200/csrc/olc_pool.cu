// Serving pool: simulations join and leave a running batch between steps.
// No counterpart in the reference (one simulation per engine, for its whole
// life).
//
// A pool is a batch handle (olc_batch.cu) whose members occupy slots.  Rows
// of a new member are appended after every row in use, exactly where a birth
// would go; the next sort moves them into the member's key range, so the
// member's rows reach the order of its solo run's first sort.  A retired
// member's rows are flagged dead and drop out at the next sort, like rows
// that die().  Its result is first gathered (stable: device row order) into
// caller buffers.  None of these kernels waits on another block: the gather is
// count -> one-block scan -> scatter.
#include "olc_internal.h"

namespace olc {

// Rows [total, total + n) <- the staged columns; the `_sim` column gets `slot`.
// All or nothing: when the rows would pass the capacity nothing is written
// (k_pool_append_commit flags it).
__global__ void __launch_bounds__(256) k_pool_append(PoolCols cols, olc_u32 n, olc_u32 slot,
                                                     unsigned char* __restrict__ life, const olc_u32* counters,
                                                     olc_u32 capacity) {
    const olc_u32 base = olc_total_rows(counters);
    if ((olc_u64)base + n > capacity) return;
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        for (int c = 0; c < cols.ncols; ++c) {
            olc_u32* dst = static_cast<olc_u32*>(cols.dst[c]);
            dst[base + i] = c == cols.sim_col ? slot : static_cast<const olc_u32*>(cols.src[c])[i];
        }
        life[base + i] = 0;
    }
}

// Runs after k_pool_append (same stream): counts the appended rows as live.
__global__ void k_pool_append_commit(olc_u32* counters, olc_u32 n, olc_u32 capacity) {
    const olc_u32 base = olc_total_rows(counters);
    if ((olc_u64)base + n > capacity) {
        atomicOr(counters + OLC_CTR_STATUS, OLC_ST_CAPACITY);
        return;
    }
    counters[OLC_CTR_N] += n;
}

void launch_pool_append(const PoolCols& cols, olc_u32 n, olc_u32 slot, unsigned char* life, olc_u32* counters,
                        olc_u32 capacity, cudaStream_t s) {
    if (n == 0) return;
    olc_u32 blocks = (n + 255) / 256;
    if (blocks > 148u * 8u) blocks = 148u * 8u;
    k_pool_append<<<blocks, 256, 0, s>>>(cols, n, slot, life, counters, capacity);
    k_pool_append_commit<<<1, 1, 0, s>>>(counters, n, capacity);
}

// Flags every row of `slot` dead; the next sort removes them.
__global__ void __launch_bounds__(256) k_pool_retire(const olc_u32* __restrict__ sim, unsigned char* __restrict__ life,
                                                     const olc_u32* counters, olc_u32 slot) {
    const olc_u32 n = olc_total_rows(counters);
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (sim[i] == slot) life[i] = 1;
}

void launch_pool_retire(const olc_u32* sim, unsigned char* life, const olc_u32* counters, olc_u32 n_cap,
                        olc_u32 slot, cudaStream_t s) {
    olc_u32 blocks = (n_cap + 255) / 256;
    if (blocks == 0) blocks = 1;
    if (blocks > 148u * 8u) blocks = 148u * 8u;
    k_pool_retire<<<blocks, 256, 0, s>>>(sim, life, counters, slot);
}

// Zeroes the bin-table ranges of the members in the pool: chunk c covers
// entries [chunks[c].x, chunks[c].x + chunks[c].y), at most POOL_TABLE_CHUNK.
__global__ void __launch_bounds__(256) k_clear_table_chunks(const uint2* __restrict__ chunks, uint2* ranges) {
    const uint2 c = chunks[blockIdx.x];
    for (olc_u32 i = threadIdx.x; i < c.y; i += blockDim.x) ranges[(size_t)c.x + i] = make_uint2(0u, 0u);
}

void launch_clear_table_chunks(const uint2* chunks, olc_u32 n_chunks, olc_u32* ranges, cudaStream_t s) {
    if (n_chunks == 0) return;
    k_clear_table_chunks<<<n_chunks, 256, 0, s>>>(chunks, reinterpret_cast<uint2*>(ranges));
}

// ------------------------------------------------------------------ gather
// Block b owns the rows [b * chunk, (b + 1) * chunk), chunk a multiple of 256.
__device__ __forceinline__ olc_u32 gather_chunk(olc_u32 n) {
    const olc_u32 per = (n + gridDim.x - 1) / gridDim.x;
    return (per + 255u) & ~255u;
}

__device__ __forceinline__ bool gather_hit(const olc_u32* sim, const unsigned char* life, olc_u32 i, olc_u32 n,
                                           olc_u32 slot) {
    return i < n && sim[i] == slot && life[i] == 0;
}

__global__ void __launch_bounds__(256) k_gather_count(const olc_u32* __restrict__ sim,
                                                      const unsigned char* __restrict__ life, const olc_u32* counters,
                                                      olc_u32 slot, olc_u32* __restrict__ block_counts) {
    __shared__ olc_u32 s_w[8];
    const olc_u32 n = olc_total_rows(counters);
    const olc_u32 chunk = gather_chunk(n);
    const olc_u64 lo = (olc_u64)blockIdx.x * chunk;
    const olc_u64 hi = lo + chunk < n ? lo + chunk : n;
    olc_u32 c = 0;
    for (olc_u64 i = lo + threadIdx.x; i < hi; i += blockDim.x) c += gather_hit(sim, life, (olc_u32)i, n, slot);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        olc_u32 t = 0;
        for (int w = 0; w < 8; ++w) t += s_w[w];
        block_counts[blockIdx.x] = t;
    }
}

// One block of 1024 threads: exclusive scan of `blocks` (<= 1024) counts in
// place; the total goes to *count_out.
__global__ void __launch_bounds__(1024) k_gather_scan(olc_u32* block_counts, olc_u32 blocks, olc_u32* count_out) {
    __shared__ olc_u32 s_w[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const olc_u32 v = threadIdx.x < blocks ? block_counts[threadIdx.x] : 0u;
    olc_u32 x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const olc_u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
        olc_u32 w = s_w[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const olc_u32 y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_w[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const olc_u32 incl = x + (warp > 0 ? s_w[warp - 1] : 0u);
    if (threadIdx.x < blocks) block_counts[threadIdx.x] = incl - v;
    if (threadIdx.x == 1023) *count_out = incl;
}

__global__ void __launch_bounds__(256) k_gather_scatter(PoolCols cols, const olc_u32* __restrict__ sim,
                                                        const unsigned char* __restrict__ life,
                                                        const olc_u32* counters, olc_u32 slot,
                                                        const olc_u32* __restrict__ block_offsets, olc_u32 max_rows) {
    __shared__ olc_u32 s_w[8];
    __shared__ olc_u32 s_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const olc_u32 n = olc_total_rows(counters);
    const olc_u32 chunk = gather_chunk(n);
    const olc_u64 lo = (olc_u64)blockIdx.x * chunk;
    const olc_u64 hi = lo + chunk < n ? lo + chunk : n;
    olc_u32 out = block_offsets[blockIdx.x];
    for (olc_u64 t = lo; t < hi; t += 256) {
        const olc_u32 i = (olc_u32)(t + threadIdx.x);
        const bool hit = (olc_u64)i < hi && gather_hit(sim, life, i, n, slot);
        const olc_u32 ballot = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) s_w[warp] = __popc(ballot);
        __syncthreads();
        if (threadIdx.x == 0) {
            olc_u32 acc = 0;
            for (int w = 0; w < 8; ++w) {
                const olc_u32 c = s_w[w];
                s_w[w] = acc;
                acc += c;
            }
            s_total = acc;
        }
        __syncthreads();
        if (hit) {
            const olc_u32 pos = out + s_w[warp] + __popc(ballot & ((1u << lane) - 1u));
            if (pos < max_rows)
                for (int c = 0; c < cols.ncols; ++c)
                    if (cols.dst[c])
                        static_cast<olc_u32*>(cols.dst[c])[pos] = static_cast<const olc_u32*>(cols.src[c])[i];
        }
        out += s_total;
        __syncthreads();
    }
}

void launch_pool_gather(const PoolCols& cols, const olc_u32* sim, const unsigned char* life, const olc_u32* counters,
                        olc_u32 slot, olc_u32* block_counts, olc_u32* count_out, olc_u32 max_rows, cudaStream_t s) {
    k_gather_count<<<POOL_GATHER_BLOCKS, 256, 0, s>>>(sim, life, counters, slot, block_counts);
    k_gather_scan<<<1, 1024, 0, s>>>(block_counts, POOL_GATHER_BLOCKS, count_out);
    k_gather_scatter<<<POOL_GATHER_BLOCKS, 256, 0, s>>>(cols, sim, life, counters, slot, block_counts, max_rows);
}

}  // namespace olc
