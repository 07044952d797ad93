/*
 * olc_oracle.h — CPU oracle for the Oncolytica step (TEST INFRASTRUCTURE).
 *
 * This is a plain C restatement of the reference's algorithm for the per-step
 * hot path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it, as the checker; the product (oncolytica_b200) never does.
 *
 * Pinning: Morton keys are checked against the reference's own
 * framework/src/oncolytica/core/runtime/_geometry.py (golden fixtures made by
 * tests/golden/make_golden.py); the sort contract against the reference test
 * framework/tests/test_gpu.py:17-61 (same inputs, per-key id sets); the RNG
 * against a restatement of template.wgsl:75-82 in tests.  Diffusion, reaction,
 * contact force and the tumour rule have no reference test or golden output:
 * for those, parity is pinned only by this restatement of
 * engine/assets/shaders/tumor_sim.wgsl: their parity is unpinned by the
 * reference itself.
 *
 * Floating point: compile with -ffp-contract=off so a*b+c rounds twice, as the
 * CUDA kernels do (they use __fmul_rn/__fadd_rn and --fmad=false).
 */
#ifndef OLC_ORACLE_H
#define OLC_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* template.wgsl:75-82 */
float orc_next_rand(uint32_t* state);
/* template.wgsl:84-98 */
void orc_rand_dir(uint32_t* state, float out[3]);
/* the build's seeding of agent RNG states (MurmurHash3 fmix32 of seed*golden + i, forced odd) */
uint32_t orc_seed_rng(uint32_t seed, uint32_t index);
void orc_rng_batch(uint32_t* states, uint32_t n, int draws, float* out, float* dirs);

/* template.wgsl:100-132, _geometry.py:14-47 */
uint32_t orc_interleave9(uint32_t v);
uint32_t orc_chem_key(int cx, int cy, int cz);
uint32_t orc_tissue_key(int cx, int cy, int cz);
int orc_bin_coord(float p, float vs, int dim);
void orc_keys(const float* x, const float* y, const float* z, const uint8_t* dead, uint32_t n,
              const int32_t dims[3], float vs, uint32_t* keys);

/* stable sort of (key, value) by key; vin == NULL means 0..n-1 */
void orc_sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, uint32_t n);
void orc_bin_ranges(const uint32_t* keys, uint32_t n, uint32_t n_bins, uint32_t* ranges);

/* tumor_sim.wgsl:387-446: sink then S substeps; result in f. Returns 0 or -1 when unstable. */
int orc_diffuse(float* f, float* tmp, float* sink, const int32_t dims[3], float dx, float dt, float D,
                float decay, float boundary, int substeps, int nthreads);
int orc_diffuse_pinned(float* f, float* tmp, float* sink, const int32_t dims[3], float dx, float dt, float D,
                       float decay, float boundary, int substeps, const uint32_t* pins, uint32_t n_pins,
                       float pin_value, int nthreads);
/* The storage roundings of the 16-bit fields, element-wise: storage 1/2
 * round to nearest even (BF16 / FP16), 3/4 stochastically with rnd[i]'s bits
 * (BF16: low 16, FP16: low 13), 5 = FP16 toward zero.  For tests. */
void orc_round16(const float* in, uint16_t* out, size_t n, int storage, const uint32_t* rnd);

int orc_diffuse16(uint16_t* f, uint16_t* tmp, float* sink, float* comp, const int32_t dims[3], float dx, float dt,
                  float D, float decay, float boundary, int substeps, int storage, uint32_t step, int field,
                  int nthreads);
/* The same with an element encoding (0 value, 1 deficit, 2 three offsets;
 * olc.h OLC_ENC_*), and the encodings' conversions: orc_encode16 rounds field
 * values to nearest into encoded elements, orc_decode16 returns field values
 * (plus the residuals, in the encoded domain, when comp is not NULL). */
int orc_diffuse16e(uint16_t* f, uint16_t* tmp, float* sink, float* comp, const int32_t dims[3], float dx, float dt,
                   float D, float decay, float boundary, int substeps, int storage, int encoding, uint32_t step,
                   int field, int nthreads);
void orc_encode16(const float* f, uint16_t* out, size_t n, int storage, int encoding, float boundary);
void orc_decode16(const uint16_t* h, const float* comp, float* out, size_t n, int storage, int encoding,
                  float boundary);
int orc_diffuse_f64(double* f, double* tmp, const float* sink, const int32_t dims[3], double dx, double dt, double D,
                    double decay, double boundary, int substeps, int split, int nthreads);

/* tumor_sim.wgsl:505-628 force law, overdamped; see oncolytica_b200/csrc/olc_contact.cu */
void orc_contact(const float* posr, const uint32_t* ranges, uint32_t n, const int32_t tdims[3], float tvs,
                 float stiffness, float mobility, float max_disp, float dt, const float lo[3], const float hi[3],
                 float* x, float* y, float* z, int nthreads);
/* Contact with the engine's extras (engine/assets/shaders/tumor_sim.wgsl:505-628,
 * Kernel_Interaction): necrotic repulsion factor (state 3), cosine adhesion
 * between non-necrotic agents, and, with vx != NULL, damped velocity
 * integration with a speed cap; otherwise the overdamped move of orc_contact. */
void orc_contact_mech(const float* posr, const uint32_t* ranges, uint32_t n, const int32_t tdims[3], float tvs,
                      float stiffness, float mobility, float max_disp, float dt, const float lo[3], const float hi[3],
                      const int32_t* state, float necrotic_factor, float adh_k, float adh_range, float* vx,
                      float* vy, float* vz, float damping, float max_speed, float* xo, float* yo, float* zo,
                      int nthreads);

/* orc_contact_mech plus the engine's active motion of non-necrotic agents
 * (tumor_sim.wgsl:584-604): chemotaxis up the clamped central-difference
 * gradients of o2 / glu (x-fastest grids of cdims, voxel cvs) and random
 * motility from rng (advanced in place); per-species coefficients selected by
 * species (clamped; NULL = record 0).  n_species = 0 turns both off. */
void orc_contact_motion(const float* posr, const uint32_t* ranges, uint32_t n, const int32_t tdims[3], float tvs,
                        float stiffness, float mobility, float max_disp, float dt, const float lo[3],
                        const float hi[3], const int32_t* state, float necrotic_factor, float adh_k,
                        float adh_range, float* vx, float* vy, float* vz, float damping, float max_speed,
                        const int32_t* species, uint32_t* rng, const float* o2, const float* glu,
                        const int32_t* cdims, float cvs, float chemo_force, float impulse, int n_species,
                        const float* sp_o2, const float* sp_glu, const float* sp_move, float* xo, float* yo,
                        float* zo, int nthreads);

/* ---------------------------------------------------------------------------
 * Tumour-spheroid workload (the built-in benchmark model, restated from its
 * DSL source in oncolytica_b200/workloads.py).  Columns: x y z radius volume
 * state rng.  Fields: o2 (+ drug when has_drug).
 */
typedef struct {
    uint32_t cap, n;          /* capacity, live rows */
    float *x, *y, *z, *radius, *volume;
    int32_t* state;
    uint32_t* rng;
    /* second buffer used by the permute */
    float *x2, *y2, *z2, *radius2, *volume2;
    int32_t* state2;
    uint32_t* rng2;
    uint8_t* dead;
    int32_t tdims[3];
    float tvs;
    int32_t cdims[3];
    float cvs;
    float lo[3], hi[3];
    float *o2, *o2_tmp, *o2_sink;
    float *drug, *drug_tmp;
    int has_drug;
    /* params */
    float dt, growth, v_div, o2_necrotic, o2_quiescent, uptake, death_k;
    float D_o2, D_drug, decay_drug, bnd_o2, bnd_drug;
    int S_o2, S_drug;
    float stiffness, mobility, max_disp, margin;
    /* counters of the last step */
    uint32_t births, deaths;
} OrcTumour;

/* one step: fields, sort/compaction, rule, contact. nthreads <= 0: all. */
int orc_tumour_step(OrcTumour* t, int nthreads);
/* the parts separately (the CPU baseline times them apart) */
int orc_tumour_fields(OrcTumour* t, int nthreads);
int orc_tumour_agents(OrcTumour* t, int nthreads);
size_t orc_tumour_sizeof(void);

#ifdef __cplusplus
}
#endif
#endif
