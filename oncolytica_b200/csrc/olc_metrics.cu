// The engine's metrics set on the device.
//
// Restates Kernel_CollectMetrics / Kernel_FinalizeMetrics
// (engine/assets/shaders/tumor_sim.wgsl:255-361): per live agent, necrotic
// agents are counted and skipped; the others are counted as proliferating or
// quiescent (and as cancer stem cells), their offsets from the domain centre,
// squared radius, energy, O2 and glucose samples and speed are summed, the
// largest radius is kept, and agents in hypoxic voxels or crowded bins are
// counted.  The engine's fixed-point i32 accumulators become exact counts and
// FP64 sums (block partials summed in a fixed order by the last block, which
// also evaluates FinalizeMetrics' formulas).
#include "olc_internal.h"

namespace olc {

namespace {

constexpr int EM_SUMS = 8;  // dx, dy, dz, r^2, energy, o2, glucose, speed
constexpr int EM_COUNTS = 6;  // prolif, quiesc, necrotic, csc, hypoxic, crowded

__device__ __forceinline__ double em_warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ olc_u32 em_warp_sum_u(olc_u32 v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float em_sample(const void* f, int type, float b, olc_u32 v) {
    return olc_field_value(f, type, b, v);
}

__global__ void __launch_bounds__(256) k_engine_metrics(EngineMetricArgs a, const olc_u32* counters,
                                                        EngineMetricAcc* acc, double* partials) {
    __shared__ double s_sum[EM_SUMS][8];
    __shared__ double s_max[8];
    __shared__ olc_u32 s_cnt[EM_COUNTS][8];
    __shared__ bool s_last;
    const olc_u32 n = olc_total_rows(counters);
    double sum[EM_SUMS];
    for (int k = 0; k < EM_SUMS; ++k) sum[k] = 0.0;
    double mr = 0.0;
    olc_u32 cnt[EM_COUNTS] = {0, 0, 0, 0, 0, 0};
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (a.life[i]) continue;
        const int st = a.state ? a.state[i] : 1;
        if (st == 0) continue;  // STATE_DELETED
        if (st == 3) {          // STATE_NECROTIC
            ++cnt[2];
            continue;
        }
        if (st == 1)
            ++cnt[0];
        else
            ++cnt[1];
        if (a.csc && a.csc[i] != 0) ++cnt[3];
        const float px = a.x[i], py = a.y[i], pz = a.z[i];
        const double dx = (double)px - (double)a.cx, dy = (double)py - (double)a.cy, dz = (double)pz - (double)a.cz;
        const double r2 = dx * dx + dy * dy + dz * dz;
        sum[0] += dx;
        sum[1] += dy;
        sum[2] += dz;
        sum[3] += r2;
        mr = fmax(mr, sqrt(r2));
        if (a.energy) sum[4] += (double)a.energy[i];
        if (a.f0 || a.f1) {
            const int cx = olc_bin_coord(px, a.cvs, a.cdims[0]);
            const int cy = olc_bin_coord(py, a.cvs, a.cdims[1]);
            const int cz = olc_bin_coord(pz, a.cvs, a.cdims[2]);
            const olc_u32 v = ((olc_u32)cz * (olc_u32)a.cdims[1] + (olc_u32)cy) * (olc_u32)a.cdims[0] + (olc_u32)cx;
            if (a.f0) {
                const float o2 = em_sample(a.f0, a.f0_type, a.f0_b, v);
                sum[5] += (double)o2;
                if (o2 < a.hypoxia) ++cnt[4];
            }
            if (a.f1) sum[6] += (double)em_sample(a.f1, a.f1_type, a.f1_b, v);
        }
        if (a.speed_x) {
            const double vx = a.speed_x[i], vy = a.speed_y[i], vz = a.speed_z[i];
            sum[7] += sqrt(vx * vx + vy * vy + vz * vz);
        }
        if (a.ranges) {
            const int tx = olc_bin_coord(px, a.tvs, a.tdims[0]);
            const int ty = olc_bin_coord(py, a.tvs, a.tdims[1]);
            const int tz = olc_bin_coord(pz, a.tvs, a.tdims[2]);
            const uint2 rg = a.ranges[olc_tissue_key(tx, ty, tz)];
            if ((int)(rg.y - rg.x) > a.crowd) ++cnt[5];
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < EM_SUMS; ++k) sum[k] = em_warp_sum(sum[k]);
    for (int o = 16; o > 0; o >>= 1) mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    for (int k = 0; k < EM_COUNTS; ++k) cnt[k] = em_warp_sum_u(cnt[k]);
    if (lane == 0) {
        for (int k = 0; k < EM_SUMS; ++k) s_sum[k][warp] = sum[k];
        s_max[warp] = mr;
        for (int k = 0; k < EM_COUNTS; ++k) s_cnt[k][warp] = cnt[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < 8; ++w) m = fmax(m, s_max[w]);
        atomicMax(reinterpret_cast<unsigned long long*>(&acc->max_r), (unsigned long long)__double_as_longlong(m));
        for (int k = 0; k < EM_COUNTS; ++k) {
            olc_u32 c = 0;
            for (int w = 0; w < 8; ++w) c += s_cnt[k][w];
            if (c) atomicAdd(&acc->counts[k], c);
        }
        // block partials, summed over the warps in order
        for (int k = 0; k < EM_SUMS; ++k) {
            double t = 0.0;
            for (int w = 0; w < 8; ++w) t += s_sum[k][w];
            partials[(size_t)k * gridDim.x + blockIdx.x] = t;
        }
        __threadfence();
        s_last = atomicAdd(&acc->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x != 0) return;
    // the last block: partials in block order, then FinalizeMetrics
    double tot[EM_SUMS];
    for (int k = 0; k < EM_SUMS; ++k) {
        double t = 0.0;
        for (olc_u32 b = 0; b < gridDim.x; ++b) t += __ldcg(partials + (size_t)k * gridDim.x + b);
        tot[k] = t;
    }
    const olc_u32* c = const_cast<const olc_u32*>(acc->counts);
    const double n_prolif = (double)__ldcg(c + 0), n_quiesc = (double)__ldcg(c + 1), n_necr = (double)__ldcg(c + 2);
    const double n_csc = (double)__ldcg(c + 3), n_hyp = (double)__ldcg(c + 4), n_crowd = (double)__ldcg(c + 5);
    const double n_live = n_prolif + n_quiesc, n_total = n_live + n_necr;
    const double f_live = fmax(n_live, 1.0), f_total = fmax(n_total, 1.0);
    const double r_inv = __longlong_as_double((long long)__ldcg(reinterpret_cast<const unsigned long long*>(&acc->max_r)));
    const double r_necr = n_necr > 0.0 ? 0.5 * pow(n_necr / 0.65, 0.333333) : 0.0;
    double* o = acc->out;
    o[0] = n_live;
    o[1] = n_prolif;
    o[2] = n_quiesc;
    o[3] = n_necr;
    o[4] = n_prolif / f_live;
    o[5] = n_quiesc / f_live;
    o[6] = n_necr / f_total;
    o[7] = n_hyp / f_live;
    o[8] = n_csc;
    o[9] = n_csc / f_live;
    o[10] = (double)a.cx + tot[0] / f_live;
    o[11] = (double)a.cy + tot[1] / f_live;
    o[12] = (double)a.cz + tot[2] / f_live;
    o[13] = sqrt(tot[3] / f_live);
    o[14] = r_inv;
    o[15] = r_necr;
    o[16] = fmax(r_inv - r_necr, 0.0);
    o[17] = tot[4] / f_live;
    o[18] = tot[5] / f_live;
    o[19] = tot[6] / f_live;
    o[20] = tot[7] / f_live;
    o[21] = n_crowd / f_live;
    o[22] = a.step;
    acc->ticket = 0u;
}

}  // namespace

void launch_engine_metrics(const EngineMetricArgs& a, const olc_u32* counters, olc_u32 n_cap, EngineMetricAcc* acc,
                           double* partials, cudaStream_t s) {
    olc_u32 blocks = (n_cap + 255) / 256;
    if (blocks == 0) blocks = 1;
    if (blocks > EM_MAX_BLOCKS) blocks = EM_MAX_BLOCKS;
    cudaMemsetAsync(acc, 0, sizeof(EngineMetricAcc), s);
    k_engine_metrics<<<blocks, 256, 0, s>>>(a, counters, acc, partials);
}

}  // namespace olc
