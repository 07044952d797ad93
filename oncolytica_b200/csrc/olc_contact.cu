// Contact mechanics over the Moore neighbourhood of each agent's bin.
//
// Reference force law: engine/assets/shaders/tumor_sim.wgsl:505-628
// (Kernel_Interaction): for dist < r_i + r_j the repulsion
// k * overlap * sqrt(overlap) acts along n_ij = (p_i - p_j) / dist.
// The reference integrates a damped velocity and draws a random jitter for
// coincident points; this path is overdamped (displacement = mobility * F * dt,
// capped at max_disp, then clamped into the domain, :606-625) and pushes
// coincident points apart along x in index order, so it needs no RNG draw.
// Neighbours come from the sorted bin table (27 bins, out-of-range bins
// skipped, self skipped) in the order of the reference's MooreOffsets
// (framework/src/oncolytica/gpu/compiler/template.wgsl:11-21): x fastest,
// then y, then z; within a bin by sorted row.  The force sum follows that
// order with separately rounded operations.
#include "olc_internal.h"


namespace olc {

// One thread per agent, grid-stride.  The force sum runs over the Moore bins
// in the order above and the rows of each bin ascending.
__global__ void __launch_bounds__(256) k_contact(const float4* __restrict__ posr, const uint2* __restrict__ ranges,
                                                 const olc_u32* n_dev, olc_u32 n_host, ContactDev c,
                                                 float* __restrict__ xo, float* __restrict__ yo,
                                                 float* __restrict__ zo) {
    const olc_u32 n = n_dev ? *n_dev : n_host;
    const float md = __fmul_rn(c.mobility, c.dt);
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = posr[i];
        if (p.w < 0.0f) continue;  // dead this step: no move, no force
        const int cx = olc_bin_coord(p.x, c.tvs, c.tdims[0]);
        const int cy = olc_bin_coord(p.y, c.tvs, c.tdims[1]);
        const int cz = olc_bin_coord(p.z, c.tvs, c.tdims[2]);
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        const olc_u32 kx[3] = {olc_tissue_axis(cx - 1, 0), olc_tissue_axis(cx, 0), olc_tissue_axis(cx + 1, 0)};
        const olc_u32 ky[3] = {olc_tissue_axis(cy - 1, 1), olc_tissue_axis(cy, 1), olc_tissue_axis(cy + 1, 1)};
        const olc_u32 kz[3] = {olc_tissue_axis(cz - 1, 2), olc_tissue_axis(cz, 2), olc_tissue_axis(cz + 1, 2)};
        for (int dz = -1; dz <= 1; ++dz) {
            const int nz = cz + dz;
            if (nz < 0 || nz >= c.tdims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int ny = cy + dy;
                if (ny < 0 || ny >= c.tdims[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = cx + dx;
                    if (nx < 0 || nx >= c.tdims[0]) continue;
                    const uint2 rg = __ldg(ranges + (kx[dx + 1] | ky[dy + 1] | kz[dz + 1]));
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
                        // d2 > rsum^2 (1 + 2^-20) implies sqrt(d2) >= rsum exactly, so the
                        // exact test below would reject the pair: skip the sqrt.
                        if (d2 > __fmul_rn(__fmul_rn(rsum, rsum), 1.00000095367431640625f)) continue;
                        const float dist = sqrtf(d2);
                        if (!(dist < rsum)) continue;
                        const float ov = __fsub_rn(rsum, dist);
                        const float f = __fmul_rn(__fmul_rn(c.stiffness, ov), sqrtf(ov));
                        if (dist < 1e-5f) {
                            fx = __fadd_rn(fx, i < j ? -f : f);
                        } else {
                            const float s = __fdiv_rn(f, dist);
                            fx = __fadd_rn(fx, __fmul_rn(ddx, s));
                            fy = __fadd_rn(fy, __fmul_rn(ddy, s));
                            fz = __fadd_rn(fz, __fmul_rn(ddz, s));
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
        xo[i] = fminf(fmaxf(__fadd_rn(p.x, mx), c.lo[0]), c.hi[0]);
        yo[i] = fminf(fmaxf(__fadd_rn(p.y, my), c.lo[1]), c.hi[1]);
        zo[i] = fminf(fmaxf(__fadd_rn(p.z, mz), c.lo[2]), c.hi[2]);
    }
}

// Field value at (x, y, z) of a chemistry grid in any storage (type word and
// boundary value as olc_field_value takes them).
__device__ __forceinline__ float motion_field(const void* f, int type, float b, const int* dims, int x, int y,
                                              int z) {
    const olc_u32 v = ((olc_u32)z * (olc_u32)dims[1] + (olc_u32)y) * (olc_u32)dims[0] + (olc_u32)x;
    return olc_field_value(f, type, b, v);
}

// Central-difference gradient 0.5 (f(v + e) - f(v - e)) per axis, the
// neighbours clamped into the grid.
__device__ __forceinline__ float3 motion_grad(const void* f, int type, float b, const int* d, int x, int y, int z) {
    const int xm = x > 0 ? x - 1 : 0, xp = x < d[0] - 1 ? x + 1 : d[0] - 1;
    const int ym = y > 0 ? y - 1 : 0, yp = y < d[1] - 1 ? y + 1 : d[1] - 1;
    const int zm = z > 0 ? z - 1 : 0, zp = z < d[2] - 1 ? z + 1 : d[2] - 1;
    return make_float3(
        __fmul_rn(0.5f, __fsub_rn(motion_field(f, type, b, d, xp, y, z), motion_field(f, type, b, d, xm, y, z))),
        __fmul_rn(0.5f, __fsub_rn(motion_field(f, type, b, d, x, yp, z), motion_field(f, type, b, d, x, ym, z))),
        __fmul_rn(0.5f, __fsub_rn(motion_field(f, type, b, d, x, y, zp), motion_field(f, type, b, d, x, y, zm))));
}

// The engine's full pair law (tumor_sim.wgsl:505-628) over the same
// neighbour walk and summation order as k_contact:
//   repulsion  dist < r_i + r_j: k * ov^(3/2) along n_ij, k scaled by
//              necrotic_factor when either agent is necrotic (state 3);
//   adhesion   r_i + r_j <= dist < r_i + r_j + range, neither necrotic:
//              -adh_k * 0.5 (1 + cos(3.14159 gap / range)) along n_ij;
// then either the overdamped move of k_contact, or the engine's damped
// velocity: v += (F - damping v) dt (damping doubled for a necrotic agent),
// |v| capped at max_speed, p += v dt, clamped into the domain.  Coincident
// points are pushed apart along x in index order, as in k_contact (the engine
// draws a random direction instead).
__global__ void __launch_bounds__(256) k_contact_mech(const float4* __restrict__ posr,
                                                      const uint2* __restrict__ ranges, const olc_u32* n_dev,
                                                      olc_u32 n_host, ContactDev c, MechDev m,
                                                      float* __restrict__ xo, float* __restrict__ yo,
                                                      float* __restrict__ zo) {
    const olc_u32 n = n_dev ? *n_dev : n_host;
    const bool adh = m.adh_k != 0.0f && m.adh_range > 0.0f;
    const float k_nec = __fmul_rn(c.stiffness, m.necrotic_factor);
    for (olc_u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = posr[i];
        if (p.w < 0.0f) continue;
        const bool nec_i = m.state && m.state[i] == 3;
        const int cx = olc_bin_coord(p.x, c.tvs, c.tdims[0]);
        const int cy = olc_bin_coord(p.y, c.tvs, c.tdims[1]);
        const int cz = olc_bin_coord(p.z, c.tvs, c.tdims[2]);
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        const olc_u32 kx[3] = {olc_tissue_axis(cx - 1, 0), olc_tissue_axis(cx, 0), olc_tissue_axis(cx + 1, 0)};
        const olc_u32 ky[3] = {olc_tissue_axis(cy - 1, 1), olc_tissue_axis(cy, 1), olc_tissue_axis(cy + 1, 1)};
        const olc_u32 kz[3] = {olc_tissue_axis(cz - 1, 2), olc_tissue_axis(cz, 2), olc_tissue_axis(cz + 1, 2)};
        for (int dz = -1; dz <= 1; ++dz) {
            const int nz = cz + dz;
            if (nz < 0 || nz >= c.tdims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int ny = cy + dy;
                if (ny < 0 || ny >= c.tdims[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = cx + dx;
                    if (nx < 0 || nx >= c.tdims[0]) continue;
                    const uint2 rg = __ldg(ranges + (kx[dx + 1] | ky[dy + 1] | kz[dz + 1]));
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
                        const float reach = adh ? __fadd_rn(rsum, m.adh_range) : rsum;
                        // as in k_contact: beyond reach^2 (1 + 2^-20) the exact tests below fail
                        if (d2 > __fmul_rn(__fmul_rn(reach, reach), 1.00000095367431640625f)) continue;
                        const float dist = sqrtf(d2);
                        if (!(dist < reach)) continue;
                        const bool nec = nec_i || (m.state && __ldg(m.state + j) == 3);
                        if (dist < rsum) {
                            const float ov = __fsub_rn(rsum, dist);
                            const float f = __fmul_rn(__fmul_rn(nec ? k_nec : c.stiffness, ov), sqrtf(ov));
                            if (dist < 1e-5f) {
                                fx = __fadd_rn(fx, i < j ? -f : f);
                            } else {
                                const float s = __fdiv_rn(f, dist);
                                fx = __fadd_rn(fx, __fmul_rn(ddx, s));
                                fy = __fadd_rn(fy, __fmul_rn(ddy, s));
                                fz = __fadd_rn(fz, __fmul_rn(ddz, s));
                            }
                        } else if (!nec) {
                            const float gap = __fsub_rn(dist, rsum);
                            const float fall =
                                __fmul_rn(0.5f, __fadd_rn(1.0f, cosf(__fdiv_rn(__fmul_rn(3.14159f, gap), m.adh_range))));
                            const float s = __fdiv_rn(__fmul_rn(m.adh_k, fall), dist);
                            fx = __fsub_rn(fx, __fmul_rn(ddx, s));
                            fy = __fsub_rn(fy, __fmul_rn(ddy, s));
                            fz = __fsub_rn(fz, __fmul_rn(ddz, s));
                        }
                    }
                }
            }
        }
        // active motion of a non-necrotic agent (tumor_sim.wgsl:584-604):
        // F += chemo_force (grad O2 chemo_o2 + grad glucose chemo_glu), then
        // F += rand_dir move_prob impulse
        if (!nec_i && (m.f0 || m.f1 || m.rng)) {
            int sp = m.species ? m.species[i] : 0;
            sp = sp < 0 ? 0 : (sp >= m.n_species ? m.n_species - 1 : sp);
            if (m.f0 || m.f1) {
                const int vx = olc_bin_coord(p.x, m.cvs, m.cdims[0]);
                const int vy = olc_bin_coord(p.y, m.cvs, m.cdims[1]);
                const int vz = olc_bin_coord(p.z, m.cvs, m.cdims[2]);
                float3 g0 = make_float3(0.0f, 0.0f, 0.0f), g1 = g0;
                if (m.f0) g0 = motion_grad(m.f0, m.f0_type, m.f0_b, m.cdims, vx, vy, vz);
                if (m.f1) g1 = motion_grad(m.f1, m.f1_type, m.f1_b, m.cdims, vx, vy, vz);
                const float co2 = m.sp_o2[sp], cglu = m.sp_glu[sp];
                fx = __fadd_rn(fx, __fmul_rn(__fadd_rn(__fmul_rn(g0.x, co2), __fmul_rn(g1.x, cglu)), m.chemo_force));
                fy = __fadd_rn(fy, __fmul_rn(__fadd_rn(__fmul_rn(g0.y, co2), __fmul_rn(g1.y, cglu)), m.chemo_force));
                fz = __fadd_rn(fz, __fmul_rn(__fadd_rn(__fmul_rn(g0.z, co2), __fmul_rn(g1.z, cglu)), m.chemo_force));
            }
            if (m.rng) {
                olc_u32 st = m.rng[i];
                const float3 r = olc_rand_dir(st);
                m.rng[i] = st;
                const float mv = m.sp_move[sp];
                fx = __fadd_rn(fx, __fmul_rn(__fmul_rn(r.x, mv), m.impulse));
                fy = __fadd_rn(fy, __fmul_rn(__fmul_rn(r.y, mv), m.impulse));
                fz = __fadd_rn(fz, __fmul_rn(__fmul_rn(r.z, mv), m.impulse));
            }
        }
        float mx, my, mz;
        if (!m.vx) {
            const float md = __fmul_rn(c.mobility, c.dt);
            mx = __fmul_rn(fx, md);
            my = __fmul_rn(fy, md);
            mz = __fmul_rn(fz, md);
            const float len =
                sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(mx, mx), __fmul_rn(my, my)), __fmul_rn(mz, mz)));
            if (len > c.max_disp) {
                const float sc = __fdiv_rn(c.max_disp, len);
                mx = __fmul_rn(mx, sc);
                my = __fmul_rn(my, sc);
                mz = __fmul_rn(mz, sc);
            }
        } else {
            const float damp = nec_i ? __fmul_rn(m.damping, 2.0f) : m.damping;
            float vx = m.vx[i], vy = m.vy[i], vz = m.vz[i];
            vx = __fadd_rn(vx, __fmul_rn(__fsub_rn(fx, __fmul_rn(vx, damp)), c.dt));
            vy = __fadd_rn(vy, __fmul_rn(__fsub_rn(fy, __fmul_rn(vy, damp)), c.dt));
            vz = __fadd_rn(vz, __fmul_rn(__fsub_rn(fz, __fmul_rn(vz, damp)), c.dt));
            const float speed =
                sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz)));
            if (speed > m.max_speed) {
                vx = __fmul_rn(__fdiv_rn(vx, speed), m.max_speed);
                vy = __fmul_rn(__fdiv_rn(vy, speed), m.max_speed);
                vz = __fmul_rn(__fdiv_rn(vz, speed), m.max_speed);
            }
            m.vx[i] = vx;
            m.vy[i] = vy;
            m.vz[i] = vz;
            mx = __fmul_rn(vx, c.dt);
            my = __fmul_rn(vy, c.dt);
            mz = __fmul_rn(vz, c.dt);
        }
        xo[i] = fminf(fmaxf(__fadd_rn(p.x, mx), c.lo[0]), c.hi[0]);
        yo[i] = fminf(fmaxf(__fadd_rn(p.y, my), c.lo[1]), c.hi[1]);
        zo[i] = fminf(fmaxf(__fadd_rn(p.z, mz), c.lo[2]), c.hi[2]);
    }
}

void launch_contact_mech(const float4* posr, const olc_u32* ranges, const olc_u32* n_dev, olc_u32 n_host,
                         olc_u32 n_cap, const ContactDev& c, const MechDev& m, float* x, float* y, float* z,
                         cudaStream_t s) {
    olc_u32 blocks = (n_cap + 255) / 256;
    if (blocks == 0) blocks = 1;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_contact_mech<<<blocks, 256, 0, s>>>(posr, reinterpret_cast<const uint2*>(ranges), n_dev, n_host, c, m, x, y,
                                          z);
}

// The same sum as k_contact with one flat loop over each agent's candidates:
// a thread first lists its non-empty Moore bins (in order) in its own column
// of shared memory, then walks rows bin after bin, so the lanes of a warp stay
// converged until each has run out of candidates (the nested loops run every
// bin as long as the fullest lane's), and it requests the next candidate's
// record before using the current one (the pass waits on L2 latency).  Same
// candidates, order and arithmetic.
// One candidate of the flat walk: the pair law of k_contact, summed into f.
__device__ __forceinline__ void contact_pair(const float4& p, const float4& q, olc_u32 i, olc_u32 j,
                                             const ContactDev& c, float& fx, float& fy, float& fz) {
    if (j == i || q.w < 0.0f) return;
    const float ddx = __fsub_rn(p.x, q.x);
    const float ddy = __fsub_rn(p.y, q.y);
    const float ddz = __fsub_rn(p.z, q.z);
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)), __fmul_rn(ddz, ddz));
    const float rsum = __fadd_rn(p.w, q.w);
    if (d2 > __fmul_rn(__fmul_rn(rsum, rsum), 1.00000095367431640625f)) return;
    const float dist = sqrtf(d2);
    if (!(dist < rsum)) return;
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

constexpr int CF_THREADS = 128;
__global__ void __launch_bounds__(CF_THREADS) k_contact_flat(const float4* __restrict__ posr,
                                                            const uint2* __restrict__ ranges, const olc_u32* n_dev,
                                                            olc_u32 n_host, ContactDev c, float* __restrict__ xo,
                                                            float* __restrict__ yo, float* __restrict__ zo) {
    __shared__ uint2 s_bins[27][CF_THREADS];
    const olc_u32 n = n_dev ? *n_dev : n_host;
    const float md = __fmul_rn(c.mobility, c.dt);
    const int t = threadIdx.x;
    for (olc_u32 base = blockIdx.x * CF_THREADS; base < n; base += gridDim.x * CF_THREADS) {
        const olc_u32 i = base + t;
        if (i >= n) continue;
        const float4 p = posr[i];
        if (p.w < 0.0f) continue;  // dead this step: no move, no force
        const int cx = olc_bin_coord(p.x, c.tvs, c.tdims[0]);
        const int cy = olc_bin_coord(p.y, c.tvs, c.tdims[1]);
        const int cz = olc_bin_coord(p.z, c.tvs, c.tdims[2]);
        // per-axis key terms of the neighbour coordinates (olc_tissue_axis)
        olc_u32 kx[3], ky[3], kz[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            kx[d] = olc_tissue_axis(cx + d - 1, 0);
            ky[d] = olc_tissue_axis(cy + d - 1, 1);
            kz[d] = olc_tissue_axis(cz + d - 1, 2);
        }
        int nb = 0;
        for (int dz = -1; dz <= 1; ++dz) {
            const int nz = cz + dz;
            if (nz < 0 || nz >= c.tdims[2]) continue;
            for (int dy = -1; dy <= 1; ++dy) {
                const int ny = cy + dy;
                if (ny < 0 || ny >= c.tdims[1]) continue;
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nx = cx + dx;
                    if (nx < 0 || nx >= c.tdims[0]) continue;
                    const uint2 rg = __ldg(ranges + (kx[dx + 1] | ky[dy + 1] | kz[dz + 1]));
                    if (rg.y > rg.x) s_bins[nb++][t] = rg;
                }
            }
        }
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        // the next candidate's record is requested before this one is used
        int b = 0;
        olc_u32 j = 0, end = 0;
        float4 q = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        if (nb > 0) {
            const uint2 r = s_bins[0][t];
            j = r.x;
            end = r.y;
            q = __ldg(posr + j);
        }
        while (b < nb) {
            olc_u32 jn = j + 1, en = end;
            int bn = b;
            if (jn == en) {
                if (++bn < nb) {
                    const uint2 r = s_bins[bn][t];
                    jn = r.x;
                    en = r.y;
                }
            }
            const float4 qn = bn < nb ? __ldg(posr + jn) : q;
            contact_pair(p, q, i, j, c, fx, fy, fz);
            j = jn;
            end = en;
            b = bn;
            q = qn;
        }
        float mx = __fmul_rn(fx, md), my = __fmul_rn(fy, md), mz = __fmul_rn(fz, md);
        const float len = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(mx, mx), __fmul_rn(my, my)), __fmul_rn(mz, mz)));
        if (len > c.max_disp) {
            const float sc = __fdiv_rn(c.max_disp, len);
            mx = __fmul_rn(mx, sc);
            my = __fmul_rn(my, sc);
            mz = __fmul_rn(mz, sc);
        }
        xo[i] = fminf(fmaxf(__fadd_rn(p.x, mx), c.lo[0]), c.hi[0]);
        yo[i] = fminf(fmaxf(__fadd_rn(p.y, my), c.lo[1]), c.hi[1]);
        zo[i] = fminf(fmaxf(__fadd_rn(p.z, mz), c.lo[2]), c.hi[2]);
    }
}

// The two walks (olc.h OLC_CONTACT_*): bit-identical, chosen per handle by
// measurement (OlcTuning.contact_variant).  On the 1 M-agent scale workload
// the flat walk took 0.92 ms per step over 200 steps against 1.04 for the
// nested loops; sparser or denser populations can order them the other way.
void launch_contact(const float4* posr, const olc_u32* ranges, const olc_u32* n_dev, olc_u32 n_host,
                    olc_u32 n_cap, const ContactDev& c, float* x, float* y, float* z, cudaStream_t s, int variant,
                    olc_u32 n_table) {
    if (variant != OLC_CONTACT_NESTED) {
        olc_u32 blocks = (n_cap + CF_THREADS - 1) / CF_THREADS;
        if (blocks == 0) blocks = 1;
        if (blocks > 148 * 16) blocks = 148 * 16;
        k_contact_flat<<<blocks, CF_THREADS, 0, s>>>(posr, reinterpret_cast<const uint2*>(ranges), n_dev, n_host, c,
                                                      x, y, z);
        return;
    }
    olc_u32 blocks = (n_cap + 255) / 256;
    if (blocks == 0) blocks = 1;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_contact<<<blocks, 256, 0, s>>>(posr, reinterpret_cast<const uint2*>(ranges), n_dev, n_host, c, x, y, z);
}

}  // namespace olc
