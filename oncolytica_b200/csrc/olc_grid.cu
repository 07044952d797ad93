// Spatial grid: bin keys, stable LSD radix sort (onesweep), bin table, payload
// permute.  Replaces the reference's counting sort
// (framework/src/oncolytica/gpu/compiler/template.wgsl:152-343:
// Kernel_ClearVoxels, Kernel_CountAndOffset, Kernel_Scan_L0/L1/L2,
// Kernel_AddBack_L1/L0, Kernel_Scatter, Kernel_UpdateState).
//
// The reference's within-bin order comes from atomics and is unspecified;
// this sort is stable, so rows with equal keys keep their previous order and
// results are deterministic.  Dead rows carry the key die() produces in the
// reference (the largest key, voxel_table_size - 1) and sort to the tail.
#include "olc_internal.h"

#include <algorithm>

namespace olc {

BinGrid make_bin_grid(const OlcGeom& g) {
    BinGrid b;
    for (int i = 0; i < 3; ++i) b.dims[i] = g.tissue_dims[i];
    b.vs = g.tissue_voxel_size;
    b.sentinel = olc_tissue_key(g.tissue_dims[0], g.tissue_dims[1], g.tissue_dims[2]);
    return b;
}

int key_bits_for(olc_u32 max_key) {
    int bits = 1;
    while (bits < 32 && (max_key >> bits) != 0u) ++bits;
    return bits;
}

static inline unsigned grid_for(olc_u32 n, int threads, unsigned cap_blocks) {
    olc_u32 b = (n + threads - 1) / threads;
    if (b == 0) b = 1;
    return std::min<olc_u32>(b, cap_blocks);
}

// Adds `val`'s digit of every pass to the shared histograms; lanes holding
// equal digits are merged with match_any so a warp issues one atomic per
// distinct digit (keys are nearly sorted, so most lanes agree).
__device__ __forceinline__ void hist_add(olc_u32 (*sh)[RADIX], olc_u32 key, int passes) {
    const olc_u32 active = __activemask();
    const int lane = threadIdx.x & 31;
    for (int p = 0; p < passes; ++p) {
        olc_u32 d = (key >> (8 * p)) & 0xffu;
        olc_u32 peers = __match_any_sync(active, d);
        if ((peers & ((1u << lane) - 1u)) == 0u) atomicAdd(&sh[p][d], (olc_u32)__popc(peers));
    }
}

__global__ void __launch_bounds__(256) k_keys(const float* __restrict__ x, const float* __restrict__ y,
                                              const float* __restrict__ z,
                                              const unsigned char* __restrict__ dead,
                                              const olc_u32* n_dev, olc_u32 n_host,
                                              const olc_u32* counters, BinGrid g,
                                              olc_u32* __restrict__ keys, olc_u32* __restrict__ hist,
                                              int passes, olc_u32* dead_ctr) {
    __shared__ olc_u32 sh[MAX_PASSES][RADIX];
    __shared__ olc_u32 s_dead;
    // In a step the row count is live agents plus this step's children.
    const olc_u32 n = counters ? olc_total_rows(counters) : (n_dev ? *n_dev : n_host);
    if (hist) {
        for (int i = threadIdx.x; i < MAX_PASSES * RADIX; i += blockDim.x) (&sh[0][0])[i] = 0u;
    }
    if (threadIdx.x == 0) s_dead = 0u;
    __syncthreads();
    olc_u32 my_dead = 0;
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        olc_u32 k;
        if (dead && dead[i]) {
            k = g.sentinel;
            ++my_dead;
        } else {
            int cx = olc_bin_coord(x[i], g.vs, g.dims[0]);
            int cy = olc_bin_coord(y[i], g.vs, g.dims[1]);
            int cz = olc_bin_coord(z[i], g.vs, g.dims[2]);
            k = olc_tissue_key(cx, cy, cz);
        }
        keys[i] = k;
        if (hist) hist_add(sh, k, passes);
    }
    if (dead_ctr) {
        for (int o = 16; o > 0; o >>= 1) my_dead += __shfl_xor_sync(0xffffffffu, my_dead, o);
        if ((threadIdx.x & 31) == 0 && my_dead) atomicAdd(&s_dead, my_dead);
    }
    __syncthreads();
    if (hist) {
        for (int i = threadIdx.x; i < passes * RADIX; i += blockDim.x) {
            olc_u32 v = (&sh[0][0])[i];
            if (v) atomicAdd(hist + i, v);
        }
    }
    if (dead_ctr && threadIdx.x == 0 && s_dead) atomicAdd(dead_ctr, s_dead);
}

__global__ void __launch_bounds__(256) k_digit_hist(const olc_u32* __restrict__ keys, const olc_u32* n_dev,
                                                    olc_u32 n_host, olc_u32* __restrict__ hist, int passes) {
    __shared__ olc_u32 sh[MAX_PASSES][RADIX];
    const olc_u32 n = n_dev ? *n_dev : n_host;
    for (int i = threadIdx.x; i < MAX_PASSES * RADIX; i += blockDim.x) (&sh[0][0])[i] = 0u;
    __syncthreads();
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        hist_add(sh, keys[i], passes);
    __syncthreads();
    for (int i = threadIdx.x; i < passes * RADIX; i += blockDim.x) {
        olc_u32 v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// Block-wide exclusive scan of one value per thread (256 threads).
__device__ __forceinline__ olc_u32 block_excl_scan256(olc_u32 v, olc_u32* s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    olc_u32 incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        olc_u32 t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        olc_u32 w = lane < 8 ? s_w[lane] : 0u;
        olc_u32 wi = w;
        for (int o = 1; o < 8; o <<= 1) {
            olc_u32 t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < 8) s_w[lane] = wi - w;
    }
    __syncthreads();
    olc_u32 r = incl - v + s_w[warp];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(256) k_scan_hist(const olc_u32* __restrict__ hist, olc_u32* __restrict__ base,
                                                   int passes, olc_u32* tile_ctrs, olc_u32* counters,
                                                   olc_u32 capacity) {
    __shared__ olc_u32 s_w[8];
    for (int p = 0; p < passes; ++p) {
        olc_u32 v = hist[p * RADIX + threadIdx.x];
        base[p * RADIX + threadIdx.x] = block_excl_scan256(v, s_w);
    }
    if (threadIdx.x < MAX_PASSES) tile_ctrs[threadIdx.x] = 0u;
    if (counters && threadIdx.x == 0) {
        // Commit the previous step's row count and this sort's compaction.
        olc_u32 rows = olc_total_rows(counters);
        if (rows > capacity) rows = capacity;
        olc_u32 dead = counters[OLC_CTR_DEAD_TMP];
        counters[OLC_CTR_ROWS] = rows;
        counters[OLC_CTR_N] = rows - dead;
        *reinterpret_cast<unsigned long long*>(counters + OLC_CTR_AGENT_STEPS) += (unsigned long long)(rows - dead);
        counters[OLC_CTR_DEAD] = dead;
        counters[OLC_CTR_DEAD_TMP] = 0u;
        counters[OLC_CTR_FIELD_STEP] += 1u;
        for (int j = 0; j < OLC_MAX_RULE_KERNELS; ++j) {
            counters[OLC_CTR_BIRTHS + j] = 0u;
            counters[OLC_CTR_RULE_TILE + j] = 0u;
        }
    }
}

// One onesweep pass: stable partition of a tile of keys by one digit, tile
// offsets by decoupled look-back, coalesced scatter through shared memory.
// Blocks take tiles in order from a counter and loop until the rows are
// covered, so the grid need not follow the capacity; a tile's predecessors are
// always held by blocks that are already running.
template <int IPT>
__global__ void __launch_bounds__(SORT_THREADS) k_onesweep(const olc_u32* __restrict__ kin,
                                                           const olc_u32* __restrict__ vin,
                                                           olc_u32* __restrict__ kout,
                                                           olc_u32* __restrict__ vout,
                                                           const olc_u32* n_dev, olc_u32 n_host,
                                                           int shift, int bits,
                                                           const olc_u32* __restrict__ base,
                                                           olc_u32* lookback, olc_u32* tile_ctr,
                                                           olc_u32* status) {
    constexpr int TILE = SORT_THREADS * IPT;
    constexpr int WARPS = SORT_THREADS / 32;
    __shared__ olc_u32 s_keys[TILE];
    __shared__ olc_u32 s_vals[TILE];
    __shared__ olc_u32 s_whist[WARPS][RADIX];
    __shared__ olc_u32 s_off[RADIX];
    __shared__ olc_u32 s_gbase[RADIX];
    __shared__ olc_u32 s_w[8];
    __shared__ olc_u32 s_tile;

    const olc_u32 n = n_dev ? *n_dev : n_host;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
        for (int i = tid; i < WARPS * RADIX; i += SORT_THREADS) (&s_whist[0][0])[i] = 0u;
        __syncthreads();
        const olc_u32 tile = s_tile;
        if ((olc_u64)tile * TILE >= n) return;
        const olc_u32 tile_start = tile * (olc_u32)TILE;
        const olc_u32 mask = (bits >= 32) ? 0xffffffffu : ((1u << bits) - 1u);

        olc_u32 keys[IPT], vals[IPT], ranks[IPT];
        const olc_u32 wbase = tile_start + (olc_u32)warp * (32u * IPT);
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            olc_u32 idx = wbase + (olc_u32)j * 32u + (olc_u32)lane;
            if (idx < n) {
                keys[j] = kin[idx];
                vals[j] = vin ? vin[idx] : idx;
            } else {
                keys[j] = 0xffffffffu;
                vals[j] = 0u;
            }
        }
        const olc_u32 lt_mask = (1u << lane) - 1u;
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            olc_u32 idx = wbase + (olc_u32)j * 32u + (olc_u32)lane;
            bool valid = idx < n;
            olc_u32 d = valid ? ((keys[j] >> shift) & mask) : (0x100u + (olc_u32)lane);
            olc_u32 peers = __match_any_sync(0xffffffffu, d);
            olc_u32 before = __popc(peers & lt_mask);
            olc_u32 b = valid ? s_whist[warp][d] : 0u;
            __syncwarp();
            if (valid && before == 0u) s_whist[warp][d] = b + (olc_u32)__popc(peers);
            __syncwarp();
            ranks[j] = b + before;
        }
        __syncthreads();

        // thread == digit: per-warp exclusive offsets and the tile's digit count
        olc_u32 total = 0;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) {
            olc_u32 c = s_whist[w][tid];
            s_whist[w][tid] = total;
            total += c;
        }
        olc_u32 excl = olc_lookback(lookback + tid, RADIX, tile, total, status);
        olc_u32 local_off = block_excl_scan256(total, s_w);
        s_off[tid] = local_off;
        s_gbase[tid] = base[tid] + excl - local_off;
        __syncthreads();

#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            olc_u32 idx = wbase + (olc_u32)j * 32u + (olc_u32)lane;
            if (idx < n) {
                olc_u32 d = (keys[j] >> shift) & mask;
                olc_u32 pos = s_off[d] + s_whist[warp][d] + ranks[j];
                s_keys[pos] = keys[j];
                s_vals[pos] = vals[j];
            }
        }
        __syncthreads();
        const olc_u32 tile_n = min((olc_u32)TILE, n - tile_start);
        for (olc_u32 i = tid; i < tile_n; i += SORT_THREADS) {
            olc_u32 k = s_keys[i];
            olc_u32 d = (k >> shift) & mask;
            olc_u32 o = s_gbase[d] + i;
            // Offsets are exact unless a look-back wait gave up (status flagged);
            // the bound keeps even that case inside the output.
            if (o < n) {
                kout[o] = k;
                vout[o] = s_vals[i];
            }
        }
        __syncthreads();  // shared tiles are reused by the block's next tile
    }
}

__global__ void __launch_bounds__(256) k_bin_ranges(const olc_u32* __restrict__ keys, const olc_u32* n_dev,
                                                    olc_u32 n_host, olc_u32 n_bins,
                                                    olc_u32* __restrict__ ranges) {
    const olc_u32 n = n_dev ? *n_dev : n_host;
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        olc_u32 k = keys[i];
        if (k >= n_bins) continue;
        if (i == 0 || keys[i - 1] != k) ranges[2u * k] = i;
        if (i + 1 == n || keys[i + 1] != k) ranges[2u * k + 1u] = i + 1;
    }
}

// Gathers every agent column by the sorted row index; live rows only (dead
// rows sit at the tail).  Also commits the live count as the row count.
__global__ void __launch_bounds__(256) k_permute(const olc_u32* __restrict__ idx, olc_u32* counters,
                                                 PermuteArgs a) {
    const olc_u32 n = counters[OLC_CTR_N];
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const olc_u32 s = idx[i];
        if (a.life) a.life[i] = 0;  // every row that survives the sort is alive; rules only set flags
        for (int c = 0; c < a.ncols; ++c)
            reinterpret_cast<olc_u32*>(a.dst[c])[i] = reinterpret_cast<const olc_u32*>(a.src[c])[s];
        if (a.write_posr) {
            float px = reinterpret_cast<const float*>(a.src[0])[s];
            float py = reinterpret_cast<const float*>(a.src[1])[s];
            float pz = reinterpret_cast<const float*>(a.src[2])[s];
            float r = a.radius_col >= 0 ? reinterpret_cast<const float*>(a.src[a.radius_col])[s]
                                        : a.radius_const;
            a.posr[i] = make_float4(px, py, pz, r);
        }
    }
}

// ------------------------------------------------------------------ launchers
static unsigned sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return (unsigned)n;
}

void launch_keys(const float* x, const float* y, const float* z, const unsigned char* dead,
                 const olc_u32* n_dev, olc_u32 n_host, const olc_u32* counters, olc_u32 n_cap,
                 const BinGrid& g, olc_u32* keys, olc_u32* hist, int passes, olc_u32* dead_ctr,
                 cudaStream_t s) {
    unsigned blocks = grid_for(n_cap, 256, sm_count() * 8);
    k_keys<<<blocks, 256, 0, s>>>(x, y, z, dead, n_dev, n_host, counters, g, keys, hist, passes,
                                  dead_ctr);
}

void launch_digit_hist(const olc_u32* keys, const olc_u32* n_dev, olc_u32 n_host, olc_u32 n_cap,
                       olc_u32* hist, int passes, cudaStream_t s) {
    unsigned blocks = grid_for(n_cap, 256, sm_count() * 8);
    k_digit_hist<<<blocks, 256, 0, s>>>(keys, n_dev, n_host, hist, passes);
}

void launch_scan_hist(const olc_u32* hist, olc_u32* base, int passes, olc_u32* tile_ctrs,
                      olc_u32* counters, olc_u32 capacity, cudaStream_t s) {
    k_scan_hist<<<1, 256, 0, s>>>(hist, base, passes, tile_ctrs, counters, capacity);
}

void launch_onesweep(const olc_u32* kin, const olc_u32* vin, olc_u32* kout, olc_u32* vout,
                     const olc_u32* n_dev, olc_u32 n_host, olc_u32 n_cap, int shift, int bits,
                     const olc_u32* base, olc_u32* lookback, olc_u32* tile_ctr, olc_u32* status,
                     cudaStream_t s) {
    unsigned tiles = (n_cap + SORT_TILE - 1) / SORT_TILE;
    if (tiles == 0) tiles = 1;
    if (tiles > sm_count() * 8) tiles = sm_count() * 8;
    k_onesweep<SORT_IPT><<<tiles, SORT_THREADS, 0, s>>>(kin, vin, kout, vout, n_dev, n_host, shift, bits,
                                                         base, lookback, tile_ctr, status);
}

static size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

static size_t lookback_words_for(olc_u32 n, int passes) {
    size_t tiles = (n + SORT_TILE - 1) / SORT_TILE;
    if (tiles == 0) tiles = 1;
    return (size_t)passes * tiles * RADIX;
}

size_t sort_scratch_bytes(olc_u32 n, int key_bits) {
    int passes = (key_bits + 7) / 8;
    size_t b = 0;
    b += align256(MAX_PASSES * RADIX * 4);  // hist
    b += align256(MAX_PASSES * RADIX * 4);  // base
    b += align256(MAX_PASSES * 4);          // tile counters
    b += align256(4);                       // status
    b += align256(lookback_words_for(n, passes) * 4);
    b += align256((size_t)n * 4) * 2;       // alternate keys / values
    return b;
}

bool carve_sort_scratch(void* base, size_t bytes, olc_u32 n_cap, int key_bits, SortScratch* out) {
    if (key_bits < 1 || key_bits > 32) return false;
    if (bytes < sort_scratch_bytes(n_cap, key_bits)) return false;
    if (((uintptr_t)base & 255u) != 0) return false;
    int passes = (key_bits + 7) / 8;
    char* p = static_cast<char*>(base);
    out->hist = reinterpret_cast<olc_u32*>(p); p += align256(MAX_PASSES * RADIX * 4);
    out->base = reinterpret_cast<olc_u32*>(p); p += align256(MAX_PASSES * RADIX * 4);
    out->tile_ctr = reinterpret_cast<olc_u32*>(p); p += align256(MAX_PASSES * 4);
    out->status = reinterpret_cast<olc_u32*>(p); p += align256(4);
    out->lookback_words = lookback_words_for(n_cap, passes);
    out->lookback = reinterpret_cast<olc_u32*>(p); p += align256(out->lookback_words * 4);
    out->kalt = reinterpret_cast<olc_u32*>(p); p += align256((size_t)n_cap * 4);
    out->valt = reinterpret_cast<olc_u32*>(p);
    return true;
}

// Zeroes the look-back words of the tiles rows [0, *n_dev) occupy in every
// pass (the work follows the rows in use, not the capacity).
__global__ void __launch_bounds__(256) k_clear_lookback(uint4* lookback, const olc_u32* n_dev, int passes,
                                                        size_t tiles_cap) {
    const size_t used = ((size_t)*n_dev + SORT_TILE - 1) / SORT_TILE;
    const size_t vecs = used * (RADIX / 4), stride = tiles_cap * (RADIX / 4);
    for (int p = 0; p < passes; ++p)
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vecs; i += (size_t)gridDim.x * blockDim.x)
            lookback[p * stride + i] = make_uint4(0u, 0u, 0u, 0u);
}

void run_sort(const olc_u32* kin, const olc_u32* vin, olc_u32* kout, olc_u32* vout, const olc_u32* n_dev,
              olc_u32 n_host, olc_u32 n_cap, int key_bits, const SortScratch& sc, bool hist_ready,
              olc_u32* counters, olc_u32 capacity, cudaStream_t s) {
    const int passes = (key_bits + 7) / 8;
    const size_t tiles = (n_cap + SORT_TILE - 1) / SORT_TILE ? (n_cap + SORT_TILE - 1) / SORT_TILE : 1;
    // with the row count on the device (committed by the scan below), only the
    // tiles in use are cleared
    const bool rows_on_device = counters && n_dev;
    if (!rows_on_device) cudaMemsetAsync(sc.lookback, 0, (size_t)passes * tiles * RADIX * 4, s);
    if (!hist_ready) {
        cudaMemsetAsync(sc.hist, 0, MAX_PASSES * RADIX * 4, s);
        launch_digit_hist(kin, n_dev, n_host, n_cap, sc.hist, passes, s);
    }
    launch_scan_hist(sc.hist, sc.base, passes, counters ? counters + OLC_CTR_SORT_TILE : sc.tile_ctr,
                     counters, capacity, s);
    if (rows_on_device)
        k_clear_lookback<<<sm_count() * 4, 256, 0, s>>>(reinterpret_cast<uint4*>(sc.lookback), n_dev, passes, tiles);
    const olc_u32* ck = kin;
    const olc_u32* cv = vin;
    for (int p = 0; p < passes; ++p) {
        const bool to_out = ((passes - p) & 1) == 1;
        olc_u32* dk = to_out ? kout : sc.kalt;
        olc_u32* dv = to_out ? vout : sc.valt;
        int bits = std::min(8, key_bits - 8 * p);
        launch_onesweep(ck, cv, dk, dv, n_dev, n_host, n_cap, 8 * p, bits, sc.base + p * RADIX,
                        sc.lookback + (size_t)p * tiles * RADIX,
                        (counters ? counters + OLC_CTR_SORT_TILE : sc.tile_ctr) + p,
                        counters ? counters + OLC_CTR_STATUS : sc.status, s);
        ck = dk;
        cv = dv;
    }
}

void launch_bin_ranges(const olc_u32* keys, const olc_u32* n_dev, olc_u32 n_host, olc_u32 n_cap,
                       olc_u32 n_bins, olc_u32* ranges, cudaStream_t s) {
    unsigned blocks = grid_for(n_cap, 256, sm_count() * 8);
    k_bin_ranges<<<blocks, 256, 0, s>>>(keys, n_dev, n_host, n_bins, ranges);
}

void launch_permute(const olc_u32* idx, olc_u32* counters, olc_u32 n_cap, const PermuteArgs& a,
                    cudaStream_t s) {
    unsigned blocks = grid_for(n_cap, 256, sm_count() * 8);
    k_permute<<<blocks, 256, 0, s>>>(idx, counters, a);
}

}  // namespace olc
