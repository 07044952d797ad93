/*
 * olc.h — C ABI of libolc.so, the B200 (sm_100a) implementation of one
 * Oncolytica simulation step.
 *
 * The reference's boundary for this path is the backend protocol
 * ISimulationBackend (framework/src/oncolytica/core/runtime/_backend.py:7-36):
 *   compile(sim), run_step(collect_metrics), sync_to_host(), sync_to_device(),
 *   get_metrics().
 * Its GPU implementation (framework/src/oncolytica/gpu/runtime/_gpu_backend.py)
 * drives wgpu directly.  Here the Python backend class
 * oncolytica_b200.backend.CudaBackend implements that protocol and calls the
 * entry points below through ctypes; any other host language binds the same
 * symbols (ctypes here; cgo, JNI or any C FFI elsewhere).
 *
 * Conventions
 *   - Every entry point returns an int status: OLC_OK (0) or an OLC_ERR_* code.
 *     A per-handle message is available from olc_last_error(); stateless entry
 *     points report through olc_last_error(NULL).  No C++ exception crosses
 *     the ABI.
 *   - Pointers named *_dev are device pointers owned by the caller (the Python
 *     backend allocates them with torch).  The library borrows them and never
 *     frees them.  The library owns only its scratch (sort temporaries,
 *     histograms, look-back words, bin table, status word), sized in
 *     olc_create() and released by olc_destroy().
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Calls on one handle must not run concurrently.
 *   - Device-side non-fatal conditions (capacity overflow, a bounded wait that
 *     gave up) set bits in a status word that olc_read_counters() returns.
 */
#ifndef OLC_H
#define OLC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OLC_OK            0
#define OLC_ERR_ARG       1
#define OLC_ERR_NVRTC     2
#define OLC_ERR_CUDA      3
#define OLC_ERR_CAPACITY  4
#define OLC_ERR_TIMEOUT   5
#define OLC_ERR_STATE     6

/* Status-word bits (OlcCounters.status). */
#define OLC_STATUS_CAPACITY     0x1u  /* births dropped: agent capacity reached */
#define OLC_STATUS_TIMEOUT      0x2u  /* a bounded device wait gave up          */
#define OLC_STATUS_MULTI_DIVIDE 0x4u  /* a rule called divide() twice in a call  */

#define OLC_MAX_AGENT_FIELDS 64  /* 4-byte SoA columns per agent (vec3 = 3)   */
#define OLC_MAX_FIELDS       8   /* diffusing chemistry fields                 */
#define OLC_MAX_RULES        16  /* compiled rule kernels                      */
#define OLC_RADIAL_BINS      64  /* radial histogram of live agents            */
#define OLC_STATE_BINS       8   /* histogram of the designated state column   */

typedef struct OlcSim OlcSim;

/* Geometry.  The bin grid is the reference's tissue grid
 * (framework/src/oncolytica/core/runtime/_engine.py:71-82): agents are binned
 * by trunc(pos / tissue_voxel_size) and keyed by the hierarchical Morton key of
 * framework/src/oncolytica/gpu/compiler/template.wgsl:100-132.  The chemistry
 * grid holds the diffusing fields, row-major with x fastest; it may be decoupled
 * from the bin grid (engine/assets/shaders/tumor_sim.wgsl:219-236 does the
 * same). */
typedef struct {
    int32_t tissue_dims[3];
    float   tissue_voxel_size;
    int32_t chem_dims[3];
    float   chem_voxel_size;
    float   domain_lo[3];       /* agent positions are clamped into          */
    float   domain_hi[3];       /* [lo + margin, hi - margin] by mechanics    */
} OlcGeom;

typedef struct {
    uint32_t max_agents;        /* capacity of every agent column            */
    uint32_t n_agent_fields;    /* bound 4-byte columns (pos.x/y/z are 0,1,2) */
    uint32_t n_fields;          /* chemistry fields                           */
    int32_t  state_field;       /* column holding an i32 state, or -1         */
    float    radial_bin_width;  /* width of the radial histogram bins         */
    float    center[3];         /* origin of radial statistics                */
    float    dt;                /* step length (fields and contact)           */
} OlcCaps;

/* One diffusing field: explicit 7-point FTCS substeps with Dirichlet outer
 * faces (engine/assets/shaders/tumor_sim.wgsl:414-446) and an implicit
 * first-order sink (tumor_sim.wgsl:387-412). */
typedef struct {
    float   diffusion;          /* D, length^2 / time                        */
    float   decay;              /* lambda, 1 / time (applied every substep)   */
    float   boundary;           /* value pinned on the outer faces            */
    int32_t substeps;           /* S >= 1, D*dt/S/dx^2 <= 1/6 is checked;
                                   0 = static field (read by rules only)       */
    int32_t has_sink;           /* rules deposit uptake rates into this field */
    int32_t storage;            /* OLC_FIELD_F32 (default), OLC_FIELD_BF16 or
                                   OLC_FIELD_F16: element type of the buffers */
    int32_t encoding;           /* OLC_ENC_*: what a 16-bit element holds
                                   (0 for FP32 storage)                       */
} OlcDiffusion;

/* Field storage types (OlcDiffusion.storage).  16-bit storage halves the
 * stencil's bytes: each substep reads 16-bit values, updates in FP32 and
 * rounds to nearest even; uptake and decay are applied once per step in FP32
 * with the rounding residual kept in a caller-provided FP32 compensation
 * buffer (olc_bind_field_ex).  No counterpart in the reference (FP32 textures). */
#define OLC_FIELD_F32     0
#define OLC_FIELD_BF16    1
#define OLC_FIELD_F16     2
/* BF16 whose substeps round stochastically instead of to nearest: a voxel's
 * result rounds up with probability equal to the discarded fraction, using
 * hash bits of (voxel, step, substep, field), so runs are reproducible.  With
 * 8 mantissa bits, round-to-nearest loses the small per-substep diffusion
 * increments (the field stalls); stochastic rounding keeps them in
 * expectation. */
#define OLC_FIELD_BF16_SR 3
/* OLC_FIELD_F16_SR: FP16 storage whose substeps round stochastically (13
 * random bits added below the kept mantissa, then rounding toward zero; same
 * hash bits as OLC_FIELD_BF16_SR).  Unbiased rounding with FP16's 11-bit
 * significand keeps the accumulated field error near 1e-3 of FP64. */
#define OLC_FIELD_F16_SR  4

/* Encodings of 16-bit field elements (OlcDiffusion.encoding).  Values of an
 * encoded field stay within [0, boundary] (substep results are clamped to it;
 * the reference's engine clamps its fields to [0, 1]).  With b = boundary:
 *   OLC_ENC_VALUE    the element is the value f (any range; results >= 0).
 *   OLC_ENC_DEFICIT  the element is b - f.  Near the boundary value, where a
 *                    field like O2 spends its run, the short mantissa then
 *                    resolves the small deficit instead of a number near b.
 *                    The 7-point update is linear and the faces hold b, so the
 *                    substeps run on the deficits unchanged (decay adds the
 *                    constant b (1 - 1/(1 + lambda dt_sub))).
 *   OLC_ENC_OFFSET3  the element is f - o, o in {0, b/2, b} the offset nearest
 *                    f, with o and the sign in the two top bits (bit 15 the
 *                    sign, bit 14, free in both formats for magnitudes below
 *                    2, set for o = b/2 with f >= b/2 and for o = b): every
 *                    value is held to within b/4 of an offset, four times the
 *                    resolution of OLC_ENC_VALUE near b; for fields spread
 *                    over [0, b] (a decaying drug).  Needs 0 < b <= 4.
 * The FP32 residual of 16-bit storage is kept in the encoded domain (the
 * deficit for OLC_ENC_DEFICIT, the value otherwise). */
#define OLC_ENC_VALUE     0
#define OLC_ENC_DEFICIT   1
#define OLC_ENC_OFFSET3   2

/* Kernel shapes and variants of a handle (olc_set_tuning).  Every choice
 * gives the same bits; oncolytica_b200.autotune measures them on the
 * caller's workload and sets the fastest.  No counterpart in the reference
 * (its dispatches are fixed 256-wide: _gpu_backend.py:134-136). */
#define OLC_CONTACT_FLAT   0  /* one flat walk over each agent's listed non-empty Moore bins */
#define OLC_CONTACT_NESTED 1  /* nested loops over the 27 Moore bins                       */
typedef struct {
    int32_t stencil_tile_y;   /* FP32 TMA substep tile: rows (8 or 16) ...             */
    int32_t stencil_tile_z;   /* ... and planes; (y, z) in {(8,8), (16,8), (8,16), (16,4)} */
    int32_t contact_variant;  /* OLC_CONTACT_FLAT or OLC_CONTACT_NESTED */
    int32_t batch_tile_depth; /* planes per tile of the batched FP32 substep: 8, 16 or
                                 32 (members without their own, olc_set_batch_tile_depths) */
    int32_t stencil_pair_threads; /* two FP32 substeps per pass (temporal blocking) with
                                     CTAs of 128, 256, 512 or 1024 threads where the field's
                                     rows fit one TMA box (x extent <= 256); 0 = one
                                     substep per pass */
    int32_t stencil_pair_planes;  /* planes per CTA of the two-substep pass; 0 = as few
                                     as keep the whole grid resident in one wave */
    int32_t stencil_l2_keep_pct;  /* one-substep passes over an FP32 field read and write
                                     the first pct % of its planes with L2 evict_last
                                     and the rest with evict_first, so that slab of both
                                     buffers stays in L2 from substep to substep; 0 =
                                     no eviction hints (0..100) */
} OlcTuning;

/* Sets / reads a handle's kernel shapes and variants (OlcTuning; defaults
 * (8, 8), OLC_CONTACT_FLAT, 16, 0, 0, 0).  Every choice gives the same bits.  Rebuilds
 * what depends on them (tensor maps, tile lists) and drops captured graphs;
 * waits for the device. */
int olc_set_tuning(OlcSim* sim, const OlcTuning* tuning);
int olc_get_tuning(const OlcSim* sim, OlcTuning* out);
/* Batch handles: the batched FP32 substep tile depth of each member (n =
 * members; 0 = the handle's batch_tile_depth), so each grid size can take the
 * depth measured fastest for it. */
int olc_set_batch_tile_depths(OlcSim* sim, const int32_t* depths, uint32_t n);

/* Hertz-like contact repulsion (engine/assets/shaders/tumor_sim.wgsl:505-628):
 * for d < r_i + r_j, F += k * delta^(3/2) * (p_i - p_j)/d with
 * delta = r_i + r_j - d; overdamped displacement mobility * F * dt, capped at
 * max_disp, then clamped into the domain. */
typedef struct {
    int32_t enabled;
    int32_t radius_field;       /* agent column holding the radius, or -1    */
    float   radius_const;       /* radius when radius_field < 0               */
    float   stiffness;
    float   mobility;
    float   max_disp;
    float   margin;
} OlcContact;

/* The rest of the engine's pair law and integrator (Kernel_Interaction,
 * engine/assets/shaders/tumor_sim.wgsl:505-628), on top of OlcContact:
 *   - repulsion scaled by necrotic_factor (engine: 0.3) when either agent is
 *     necrotic (state 3 in state_field);
 *   - adhesion between non-necrotic agents whose gap g = d - (r_i + r_j) is in
 *     [0, adhesion_range): force adhesion_stiffness * 0.5 (1 + cos(3.14159 g /
 *     adhesion_range)) towards the neighbour;
 *   - with velocity_field >= 0 (three f32 columns holding a vec3), the
 *     engine's damped velocity instead of the overdamped move:
 *     v += (F - damping v) dt (damping doubled for a necrotic agent), |v|
 *     capped at max_speed (engine: 0.8 x bin size), p += v dt, then the domain
 *     clamp of OlcContact.margin.
 * Summation order and coincident points are as OlcContact's.  Not used by the
 * benchmark configurations; solo handles only. */
#define OLC_MAX_SPECIES 8  /* records of the species table (the engine's MAX_SPECIES) */

/* Per-species active motion (the engine's SpeciesParam chemoTaxisO2,
 * chemoTaxisGlu, baseMoveProb). */
typedef struct {
    float chemotaxis_o2;
    float chemotaxis_glucose;
    float move_prob;
    float pad;
} OlcSpecies;

typedef struct {
    int32_t state_field;        /* i32 column, or -1 (nobody necrotic)        */
    float   necrotic_factor;
    float   adhesion_stiffness; /* 0: no adhesion                             */
    float   adhesion_range;
    int32_t velocity_field;     /* first of three f32 columns, or -1          */
    float   damping;
    float   max_speed;
    int32_t enabled;            /* 0: plain OlcContact                        */
    /* Active motion of non-necrotic agents (tumor_sim.wgsl:584-604), added to
     * the contact force: chemotaxis (chemo_force x the species' coefficients
     * x the central-difference gradient of the O2 and glucose fields at the
     * agent's voxel, neighbours clamped to the grid) and random motility
     * (move_prob x motility_impulse x a random direction drawn from the
     * agent's RNG column, two draws per agent and step). */
    int32_t species_field;      /* i32 column selecting the record (clamped), or -1: record 0 */
    int32_t rng_field;          /* u32 RNG column for motility, or -1: none   */
    int32_t o2_field;           /* chemistry field for chemotaxis, or -1      */
    int32_t glucose_field;      /* second chemotactic field, or -1            */
    float   chemo_force;        /* engine CHEMO_FORCE: 2.0                    */
    float   motility_impulse;   /* engine VELOCITY_IMPULSE: 0.4               */
    int32_t n_species;          /* records used; 0 turns active motion off    */
    int32_t pad2;
    OlcSpecies species[OLC_MAX_SPECIES];
} OlcMechanics;

typedef struct {
    uint32_t n_agents;          /* agents entering the next step              */
    uint32_t n_total;           /* rows in use incl. this step's dead         */
    uint32_t births;            /* births in the last step                    */
    uint32_t deaths;            /* agents removed by the last sort            */
    uint32_t status;            /* OLC_STATUS_* bits (sticky)                 */
    uint32_t pad;
    uint64_t steps;             /* steps run on this handle                   */
    uint64_t agent_steps;       /* sum over steps of live agents at the rule  */
} OlcCounters;

/* Stage timing of the steps run since profiling was enabled (CUDA events
 * recorded on the step's stream around each stage). */
typedef struct {
    uint32_t steps;
    uint32_t substep_launches;  /* 7-point substep kernels                    */
    uint64_t kernel_launches;   /* all kernels this library launched          */
    double   ms_sink;
    double   ms_substeps;
    double   ms_grid;           /* keys, sort, bin table, permute             */
    double   ms_rules;
    double   ms_contact;
    double   ms_collect;        /* reductions and metric rules                */
} OlcProfile;

/* Per-step reductions (engine metrics, tumor_sim.wgsl:248-361, restated as
 * exact integer counts and FP64 sums). */
typedef struct {
    uint32_t n_live;
    uint32_t state_counts[OLC_STATE_BINS];
    uint32_t radial_hist[OLC_RADIAL_BINS];
    uint32_t pad;
    double   sum_pos[3];
    double   sum_r2;            /* sum |p - center|^2                         */
    double   max_r;
    double   field_mass[OLC_MAX_FIELDS];   /* FP64 sum over the field grid   */
    double   field_min[OLC_MAX_FIELDS];
    double   field_max[OLC_MAX_FIELDS];
} OlcReductions;

/* ------------------------------------------------------------------ handle */

/* Replaces GpuBackend.compile()'s buffer/pipeline creation
 * (framework/src/oncolytica/gpu/runtime/_gpu_backend.py:79-104). */
int olc_create(const OlcGeom* geom, const OlcCaps* caps, OlcSim** out);
int olc_destroy(OlcSim* sim);
const char* olc_last_error(const OlcSim* sim);
const char* olc_version(void);

/* Binds agent column `index` (4-byte elements, capacity max_agents) as a
 * ping-pong pair.  Replaces the Cells_In/Cells_Out AoS buffers
 * (framework/src/oncolytica/gpu/runtime/_device_manager.py:76-119). */
int olc_bind_agent_column(OlcSim* sim, int index, void* a_dev, void* b_dev);

/* Binds chemistry field `index` (float, chem_dims voxels) as a ping-pong pair
 * plus an optional sink buffer (NULL when the field has no sink).  Replaces
 * Chem_In/Chem_Out (_device_manager.py:76-119). */
int olc_bind_field(OlcSim* sim, int index, float* a_dev, float* b_dev, float* sink_dev,
                   const OlcDiffusion* spec);

/* olc_bind_field for any storage type: a_dev, b_dev hold 4-byte (FP32) or
 * 2-byte (BF16/FP16) elements; comp_dev is an FP32 buffer, one element per
 * voxel, zeroed by the caller, that carries each voxel's rounding residual of
 * the per-step reaction (required for 16-bit storage, ignored for FP32).  No
 * counterpart in the reference. */
int olc_bind_field_ex(OlcSim* sim, int index, void* a_dev, void* b_dev, float* sink_dev, float* comp_dev,
                      const OlcDiffusion* spec);

int olc_set_contact(OlcSim* sim, const OlcContact* spec);
int olc_set_mechanics(OlcSim* sim, const OlcMechanics* spec);

/* Binds the tissue grid for tissue_at(): `n_cols` 4-byte columns, each with
 * voxel_table_size entries indexed by the tissue (Morton) key, `stride_bytes`
 * apart starting at cols_dev.  Replaces Tissue_In
 * (framework/src/oncolytica/gpu/compiler/translator/_expr_translator.py:243-250
 * reads it by Morton key; the reference host packs it row-major,
 * _gpu_backend.py:365-367 — here the host packs it by key). */
int olc_bind_tissue(OlcSim* sim, const void* cols_dev, int n_cols, size_t stride_bytes);

/* Pinned voxels of an FP32 field: after every substep the voxels idx_dev[0..n)
 * (x-fastest indices, a caller-owned device array) hold `value` — the engine's
 * vessel mask (engine/assets/shaders/tumor_sim.wgsl:366-380 marks voxels inside
 * the vessel cylinder, and every diffusion pass stores them as 1.0, :430-433).
 * n = 0 removes the pins.  Solo handles. */
int olc_set_pinned(OlcSim* sim, int index, const uint32_t* idx_dev, uint32_t n, float value);

/* Tissue grid that tissue rules update: two buffers laid out as in
 * olc_bind_tissue; a tissue rule reads the current one and writes the other
 * (the reference's Tissue_In / Tissue_Out,
 * framework/src/oncolytica/gpu/runtime/_gpu_backend.py:130-133).
 * olc_current_tissue tells which holds the state (0 = a, 1 = b). */
int olc_bind_tissue_pair(OlcSim* sim, void* a_dev, void* b_dev, int n_cols, size_t stride_bytes);
int olc_current_tissue(const OlcSim* sim, int* tissue_buf);

/* Iterations of each kernel of the last olc_set_rule_source (chemistry rules'
 * @chemistry_rule(iterations=k); 1 for the others). */
int olc_set_rule_iterations(OlcSim* sim, const int* iterations, int n);

/* Compiles CUDA C emitted by the rule translator with NVRTC for sm_100a
 * (replaces WGSLCompiler.compile + create_shader_module,
 * framework/src/oncolytica/gpu/compiler/_compiler.py:233-352).  `kinds[i]` is
 * 0 for a cell rule, 1 for a metric rule, 2 for a tissue rule (one thread per
 * tissue voxel, tissue buffers flipped after it) and 3 for a chemistry rule
 * (one thread per chemistry voxel, FP32 fields only, every field's buffers
 * flipped after each iteration).  Per step, tissue rules and then chemistry
 * rules run after the sort (their .cells loops see the sorted agents) and
 * before the cell rules.  `include_dir` holds
 * olc_device.cuh and olc_rule_rt.cuh. */
int olc_set_rule_source(OlcSim* sim, const char* cuda_src, const char* const* kernels,
                        const int* kinds, int n, const char* include_dir);

/* Compiles `cuda_src` with NVRTC for sm_100a without loading it (needs no
 * GPU); on failure the compiler log is copied into `log` (NUL-terminated). */
int olc_nvrtc_check(const char* cuda_src, const char* include_dir, char* log, size_t log_size);

/* Uploads the Params blob (replaces pack_uniforms, _device_manager.py:180-204;
 * unlike the reference, later calls do reach the device). */
int olc_set_params(OlcSim* sim, const void* blob, size_t bytes, void* stream);

/* Sets the agent count after the host wrote agent columns into the current
 * buffer (replaces sync_to_device, _gpu_backend.py:353-371). */
int olc_set_agent_count(OlcSim* sim, uint32_t n, void* stream);

/* Step counters of a handle, for checkpoints: a state written back with
 * olc_set_agent_count plus these counters continues bit for bit as the run it
 * was taken from (the reference has no resume; its bundle export,
 * framework/src/oncolytica/gpu/runtime/_gpu_backend.py:303-334, saves the
 * buffers only). */
typedef struct {
    uint64_t steps;             /* steps run (the engine metrics' step)        */
    uint64_t agent_steps;       /* sum over steps of live agents at the rule   */
    uint32_t field_step;        /* grid stages run: salts stochastic rounding  */
    uint32_t status;            /* OLC_STATUS_* bits                           */
} OlcStepState;
int olc_get_step_state(OlcSim* sim, OlcStepState* out, void* stream);
int olc_set_step_state(OlcSim* sim, const OlcStepState* in, void* stream);

/* Which of the pair (0 = a, 1 = b) currently holds agent / field state. */
int olc_current_buffers(const OlcSim* sim, int* agent_buf, int* field_buf);

/* Runs `nsteps` steps (replaces GpuBackend.run_step,
 * framework/src/oncolytica/gpu/runtime/_gpu_backend.py:113-171).  Stage order:
 * fields (sink, substeps) -> keys + stable radix sort + compaction + bin table ->
 * cell rules -> contact -> reductions/metric rules (when collect != 0).
 * No host synchronisation inside. */
int olc_step(OlcSim* sim, int nsteps, int collect, void* stream);

/* Enables (1) or disables (0) running olc_step through CUDA graphs of whole
 * steps; no counterpart in the reference (its step is a fixed list of wgpu
 * compute passes).  Results are identical to eager steps.  A graph is cached
 * per buffer-parity state at step start and captured the second time that
 * state is met; every binding call (columns, fields, tissue, contact, rules,
 * a params blob that grows, metrics size) drops the cache.  Steps taken while
 * profiling is on run eagerly. */
int olc_set_graphs(OlcSim* sim, int enable);

/* Synchronises `stream` and copies the counters. */
int olc_read_counters(OlcSim* sim, OlcCounters* out, void* stream);

/* Enables (1) or disables (0) stage timing; enabling clears what was
 * recorded.  olc_read_profile synchronises and sums the recorded steps. */
int olc_set_profiling(OlcSim* sim, int enable);
int olc_read_profile(OlcSim* sim, OlcProfile* out);

/* The engine's metrics set: Kernel_ClearMetrics / Kernel_CollectMetrics /
 * Kernel_FinalizeMetrics (engine/assets/shaders/tumor_sim.wgsl:248-361) and
 * the 23 values of MetricIndex (engine/src/sim/readback.rs:25-50), in that
 * order: total live, proliferating, quiescent, necrotic, their fractions, the
 * hypoxic fraction, CSC count and fraction, centroid x/y/z, radius of
 * gyration, invasive radius, necrotic radius, rim thickness, mean energy,
 * mean O2, mean glucose (second field), mean speed, crowded fraction, step.
 * Counts are exact integers and sums FP64 (the engine accumulates fixed-point
 * i32: r*r, 10*delta, 1000*field, 100*r for the maximum); the last block sums
 * the block partials in a fixed order, so repeated calls give the same bits.
 * Fields are sampled at the agent's nearest voxel (chemistry_at's rule; the
 * engine samples trilinearly through a texture unit).  A live agent is one
 * whose life flag is 0 and whose state is not 0 (STATE_DELETED); state 3 is
 * necrotic, 1 proliferating, any other quiescent; with state_field < 0 every
 * live agent counts as proliferating. */
#define OLC_ENGINE_METRICS 23
typedef struct {
    int32_t state_field;        /* i32 agent column, or -1                    */
    int32_t energy_field;       /* f32 agent column, or -1 (mean energy 0)   */
    int32_t speed_field;        /* first of three f32 columns (a vec3) whose
                                   length is the speed, or -1                */
    int32_t csc_field;          /* i32 column, nonzero marks a cancer stem
                                   cell (the engine's species table: no
                                   symmetric division), or -1                */
    int32_t o2_field;           /* chemistry field sampled as O2, or -1      */
    int32_t glucose_field;      /* chemistry field sampled as glucose, or -1 */
    float   hypoxia_threshold;  /* HYPOXIA_METRIC_THR (0.1)                   */
    int32_t crowd_threshold;    /* CROWD_THRESHOLD (12): agents in the bin    */
    float   center[3];          /* DomainCenter                               */
    float   pad;
} OlcEngineMetricsSpec;

/* Computes the engine metrics of the current state on `stream` (one kernel)
 * and copies the 23 values to out[0..22] (synchronises the stream). */
int olc_engine_metrics(OlcSim* sim, const OlcEngineMetricsSpec* spec, double* out, void* stream);

/* Copies the last step's reductions / metric-rule accumulators to host memory
 * (replaces the MetricsBuffer readback, _gpu_backend.py:166-169). */
int olc_read_reductions(OlcSim* sim, OlcReductions* out, void* stream);
int olc_read_user_metrics(OlcSim* sim, void* out, size_t bytes, void* stream);

/* Readback without waiting (solo handles; replaces the same readbacks of the
 * reference, _gpu_backend.py:166-169, for callers that queue the next step
 * before reading this one's results).  olc_queue_readback queues, on
 * `stream`, copies of the counter block and of the metric accumulators into
 * one of 4 pinned host slots and returns a ticket; olc_take_readback waits
 * for that ticket's copies only and returns the first `bytes` of the
 * accumulators and the counters (either output may be NULL / 0 bytes).  The
 * 4 slots rotate: a ticket is taken before 4 later ones are queued, or its
 * take fails with OLC_ERR_STATE.  olc_set_params likewise rotates over 4
 * pinned staging slots and so waits for no earlier copy but the one 4
 * uploads back. */
int olc_queue_readback(OlcSim* sim, void* stream, uint64_t* ticket);
int olc_take_readback(OlcSim* sim, uint64_t ticket, void* metrics_out, size_t bytes, OlcCounters* counters);

/* Copies the life flags of rows [0, rows) (0 alive, 1 died this step) to host
 * memory; sync_to_host drops dead rows as the reference's sort does
 * (template.wgsl:152-159). */
int olc_read_life(OlcSim* sim, uint8_t* out, uint32_t rows, void* stream);
int olc_set_user_metrics_size(OlcSim* sim, size_t bytes);

/* ------------------------------------------------------------- batched mode
 * Many independent simulations of one model in one handle, advanced by one
 * launch per stage (no counterpart in the reference, which runs one
 * simulation per engine).  The model is translated with a `_sim` column (the
 * simulation index of each row, u32) after `_rng_state`; agent columns are
 * shared by all simulations.  Each field buffer holds the simulations' grids
 * back to back (olc_batch_field_offsets); each simulation's grid must have an
 * x extent that is a multiple of 4.  Every simulation reproduces its solo run
 * bit for bit (same keys, sort order, rule decisions, contact and stencil
 * arithmetic); per-simulation FP64 reduction sums are exact up to order.
 * olc_bind_agent_column, olc_set_contact (its margin applies to every
 * simulation's domain), olc_set_rule_source, olc_set_user_metrics_size (bytes
 * per simulation), olc_set_agent_count (all rows), olc_step, olc_read_counters,
 * olc_read_life, olc_set_graphs, olc_set_profiling and olc_current_buffers
 * (agent buffer) work on batch handles too; olc_bind_field, olc_set_params,
 * olc_read_reductions and olc_bind_tissue do not. */
int olc_create_batch(const OlcGeom* geoms, int n_sims, const OlcCaps* caps, OlcSim** out);

/* n_sims + 1 voxel offsets: simulation k's grid is [offsets[k], offsets[k+1])
 * of every field buffer (x fastest). */
int olc_batch_field_offsets(const OlcSim* sim, uint64_t* offsets);

/* Binds field `index` for every simulation; specs[k] is simulation k's
 * diffusion (its own substep count; 0 = static; one storage type for all
 * members).  comp is the FP32 residual buffer of 16-bit storage (as in
 * olc_bind_field_ex), NULL for FP32. */
int olc_bind_field_batch(OlcSim* sim, int index, void* a, void* b, float* sink, float* comp,
                         const OlcDiffusion* specs);

/* n_sims Params blobs of `stride` bytes each, back to back. */
int olc_set_params_batch(OlcSim* sim, const void* blob, size_t stride, void* stream);

/* Which buffer (0 = a, 1 = b) holds each simulation's field: n_sims x
 * n_fields bytes, simulation-major. */
int olc_read_field_parity(OlcSim* sim, uint8_t* out, void* stream);

/* Last collected step's reductions / metric accumulators of every simulation. */
int olc_read_reductions_batch(OlcSim* sim, OlcReductions* out, void* stream);
int olc_read_user_metrics_batch(OlcSim* sim, void* out, size_t bytes_per_sim, void* stream);

/* ------------------------------------------------------------- serving pool
 * A batch handle whose members join and leave between steps (no counterpart
 * in the reference).  Members occupy slots [0, max_slots); each holds one
 * range of the bin-table arena and one range of the field arena (the same
 * voxel range in every field buffer), taken at admission and returned at
 * retirement, so admission is decided by free device memory.  A member
 * reproduces its solo run bit for bit from the step it joins (its rows are
 * appended where births go and sorted into place by the next step; its
 * stochastic-rounding salt counts its own steps).  All calls on a pool are
 * stream-ordered on the caller's stream: use one stream for every call.
 * olc_bind_agent_column, olc_set_contact, olc_set_rule_source,
 * olc_set_user_metrics_size (bytes per slot), olc_step, olc_read_counters,
 * olc_set_graphs, olc_read_reductions_batch and olc_read_user_metrics_batch
 * (max_slots records) work on pools; the batch calls that bind or upload all
 * members at once do not. */
typedef struct {
    uint32_t max_slots;           /* members resident at once */
    int32_t max_tissue_dims[3];   /* largest bin grid of any member (sets the sort-key split) */
    uint64_t table_entries;       /* bin-table arena, 8-byte entries */
    uint64_t field_voxels;        /* field arena: voxels of every field buffer */
} OlcPoolConfig;

typedef struct {
    uint32_t slots_used, max_slots;
    uint64_t table_used, table_entries, table_largest_free;
    uint64_t field_used, field_voxels, field_largest_free;
} OlcPoolUsage;

int olc_create_pool(const OlcPoolConfig* cfg, const OlcCaps* caps, OlcSim** out);

/* Field `index` of every member: a and b hold cfg.field_voxels elements of the
 * storage type (OLC_FIELD_*), sink (FP32, or NULL when no rule deposits into
 * the field) and comp (FP32, 16-bit storage only) as many.  encoding
 * (OLC_ENC_*, 16-bit storage only) and, for an encoded field, its boundary
 * value are the same for every member (olc_pool_admit checks them). */
int olc_bind_field_pool(OlcSim* sim, int index, void* a, void* b, float* sink, float* comp, int storage,
                        int encoding, float boundary);

/* Admits one simulation: geometry, specs[n_fields] (specs[f].storage must
 * match the bound storage) and its Params blob (every member's blob has the
 * same size).  On success *slot and *field_off (first voxel of its grids in
 * every field buffer) are set; the caller then writes the initial grids into
 * buffer a at field_off and adds the agents.  The member's sink, residual,
 * field parity, metric and reduction records are cleared.  OLC_ERR_CAPACITY
 * (nothing changed) when no slot, table range or field range is free. */
int olc_pool_admit(OlcSim* sim, const OlcGeom* geom, const OlcDiffusion* specs, const void* params,
                   size_t params_bytes, int32_t* slot, uint64_t* field_off, void* stream);

/* Appends n agent rows of `slot`: cols_dev[c] holds n 4-byte elements of
 * agent column c (the `_sim` column's pointer is ignored; it is written with
 * the slot).  Rows past the handle's capacity are not written and set
 * OLC_STATUS_CAPACITY. */
int olc_pool_add_agents(OlcSim* sim, int32_t slot, void* const* cols_dev, uint32_t n, void* stream);

/* Copies the live rows of `slot` in device order into dst_dev[c] (NULL
 * columns skipped; at most max_rows rows) and writes the slot's live-row
 * count to *count_dev (device word; a count above max_rows means rows were
 * left out).  The result of a member is read this way before retiring it. */
int olc_pool_gather(OlcSim* sim, int32_t slot, void* const* dst_dev, uint32_t max_rows, uint32_t* count_dev,
                    void* stream);

/* Async copies of the slot's last collected reductions and metric
 * accumulators into host memory (pinned, for the copy to stay async). */
int olc_pool_copy_results(OlcSim* sim, int32_t slot, OlcReductions* red_host, void* metrics_host, void* stream);

/* Frees the slot: its rows are flagged dead (the next step's sort drops
 * them) and its arena ranges are returned. */
int olc_pool_retire(OlcSim* sim, int32_t slot, void* stream);

int olc_pool_usage(const OlcSim* sim, OlcPoolUsage* out);

/* The pool's range allocator on its own, for callers that plan admissions
 * (and for tests): best fit over [0, capacity), merged on release. */
typedef struct OlcArena OlcArena;
int olc_arena_create(uint64_t capacity, OlcArena** out);
int olc_arena_alloc(OlcArena* arena, uint64_t n, uint64_t align, uint64_t* offset);
int olc_arena_release(OlcArena* arena, uint64_t offset, uint64_t n);
int olc_arena_stats(const OlcArena* arena, uint64_t* used, uint64_t* largest_free, uint64_t* free_ranges);
int olc_arena_destroy(OlcArena* arena);

/* ---------------------------------------------------- stateless stages */
/* These run one stage on caller buffers; the parity tests call them. */

/* RNG known answers: for each of n states, `draws` xorshift32 draws
 * (template.wgsl:75-82) written to out_dev[i*draws + k]; the final state is
 * written back.  When dirs_dev != NULL, one _rand_dir (template.wgsl:84-98)
 * per state follows and is stored as xyz triples. */
int olc_stage_rng(uint32_t* states_dev, uint32_t n, int draws, float* out_dev,
                  float* dirs_dev, void* stream);

/* Bin keys (template.wgsl:174-186, Kernel_CountAndOffset's key): keys_dev[i] =
 * tissue_key(clamp(trunc(pos / vs))); agents with dead_dev[i] != 0 get the
 * sentinel tissue_key(tissue_dims) = voxel_table_size - 1 (the key that die()
 * produces, framework/src/oncolytica/gpu/compiler/translator/_stmt_translator.py:431-440).
 * dead_dev may be NULL. */
int olc_stage_keys(const float* x_dev, const float* y_dev, const float* z_dev,
                   const uint8_t* dead_dev, uint32_t n, const OlcGeom* geom,
                   uint32_t* keys_dev, void* stream);

/* Stable LSD radix sort of (key, value) pairs on the low `key_bits` bits
 * (onesweep: one upfront digit histogram, then one decoupled-look-back pass
 * per 8-bit digit).  Replaces the counting sort of template.wgsl:165-343.
 * vals_in_dev == NULL means values 0..n-1.  Scratch is caller memory of at
 * least olc_sort_scratch_bytes(n, key_bits) bytes, 256-byte aligned.  The
 * sort's status word is the uint32 at byte olc_sort_status_offset() of the
 * scratch (cleared by each call): OLC_STATUS_TIMEOUT there means a bounded
 * look-back wait gave up and that call's output is unreliable. */
size_t olc_sort_scratch_bytes(uint32_t n, int key_bits);
size_t olc_sort_status_offset(void);
int olc_stage_sort_pairs(const uint32_t* keys_in_dev, const uint32_t* vals_in_dev,
                         uint32_t* keys_out_dev, uint32_t* vals_out_dev, uint32_t n,
                         int key_bits, void* scratch_dev, size_t scratch_bytes, void* stream);

/* The same stable sort for callers that cannot allocate device memory (a
 * process whose HBM is owned by an allocator it does not expose, or a caller
 * that must not pay cudaMalloc's implicit synchronisation): no scratch
 * argument.  The temporary memory is a file-scope device array of this library
 * (about 9.4 MB, held by every GPU that loads it until exit), so n is limited
 * to 1,048,576 keys (larger n: OLC_ERR_CAPACITY).  All calls share the array:
 * calls whose work overlaps on the GPU race and must be serialised.  Each
 * call outside stream capture looks up the array's address on the current
 * device (a device reset between calls is followed); a call on a capturing
 * stream reuses the address the last uncaptured call found, so make one call
 * on a device before capturing.  Has no counterpart in the reference. */
int olc_stage_sort_pairs_noalloc(const uint32_t* keys_in_dev, const uint32_t* vals_in_dev,
                                 uint32_t* keys_out_dev, uint32_t* vals_out_dev, uint32_t n,
                                 int key_bits, void* stream);
/* The status word of the last olc_stage_sort_pairs_noalloc call on the
 * current device, read after `stream` finishes (the call waits for it):
 * OLC_STATUS_TIMEOUT means a bounded look-back wait gave up and that sort's
 * output is unreliable (possibly unsorted or with gaps).  Allocates nothing. */
int olc_sort_noalloc_status(uint32_t* status_out, void* stream);

/* Self-test of the bounded device waits: runs one look-back walk whose
 * predecessor tile is never published (olc_lookback, as in the sort and the
 * births) and one TMA-style mbarrier wait whose transaction is never issued
 * (the wait of the stencil kernels), each with `limit` polls (1..65536), and
 * returns out[0] = the look-back's status bits, out[1] = the mbarrier wait's
 * status bits (both OLC_STATUS_TIMEOUT when the waits gave up as designed),
 * out[2] = the prefix the walk returned (0).  Waits for `stream`; uses a
 * file-scope device array (allocates nothing).  No counterpart in the
 * reference. */
int olc_selftest_bounded_waits(uint32_t limit, uint32_t out[3], void* stream);

/* Bin table from sorted keys: ranges_dev[2k] = first index of key k,
 * ranges_dev[2k+1] = one past the last (both 0 when empty); keys >= n_bins are
 * ignored.  Replaces VoxelTable.startIndex/count (template.wgsl:42-45). */
int olc_stage_bin_ranges(const uint32_t* sorted_keys_dev, uint32_t n, uint32_t n_bins,
                         uint32_t* ranges_dev, void* stream);

/* One step of one field: sink f <- f / (1 + K dt) then S substeps, result in
 * f_dev (tmp_dev is a same-sized temporary; sink_dev may be NULL and is zeroed
 * after use). */
int olc_stage_diffuse(float* f_dev, float* tmp_dev, float* sink_dev, const int32_t dims[3],
                      float dx, float dt, const OlcDiffusion* spec, void* stream);

/* olc_stage_diffuse with the stencil choices of an OlcTuning (tile, and two
 * substeps per pass); every choice gives the same result.  NULL = defaults. */
int olc_stage_diffuse_tuned(float* f_dev, float* tmp_dev, float* sink_dev, const int32_t dims[3],
                            float dx, float dt, const OlcDiffusion* spec, const OlcTuning* tuning,
                            void* stream);

/* olc_stage_diffuse with pinned voxels (olc_set_pinned's rule). */
int olc_stage_diffuse_pinned(float* f_dev, float* tmp_dev, float* sink_dev, const int32_t dims[3], float dx,
                             float dt, const OlcDiffusion* spec, const uint32_t* idx_dev, uint32_t n, float value,
                             void* stream);

/* One step of one 16-bit field (reaction with compensation, then S
 * substeps), result in f_dev; f_dev, tmp_dev hold BF16/FP16 elements, comp_dev
 * the FP32 residuals; `step` and `field` salt stochastic rounding (the step
 * loop of a handle uses its step count and the field's index). */
int olc_stage_diffuse16(void* f_dev, void* tmp_dev, float* sink_dev, float* comp_dev, const int32_t dims[3],
                        float dx, float dt, const OlcDiffusion* spec, uint32_t step, int field, void* stream);

/* Contact pass over n sorted agents: posr_dev holds (x, y, z, radius) with
 * radius < 0 marking a dead agent; writes the new positions. */
int olc_stage_contact(const float* posr_dev, const uint32_t* ranges_dev, uint32_t n,
                      const OlcGeom* geom, const OlcContact* spec, float dt,
                      float* x_dev, float* y_dev, float* z_dev, void* stream);

/* olc_stage_contact with a chosen walk (OLC_CONTACT_*); every walk gives the
 * same positions.  ranges_dev must cover every bin of the tissue grid. */
int olc_stage_contact_tuned(const float* posr_dev, const uint32_t* ranges_dev, uint32_t n, const OlcGeom* geom,
                            const OlcContact* spec, float dt, int32_t contact_variant, float* x_dev,
                            float* y_dev, float* z_dev, void* stream);

/* The contact pass with OlcMechanics: state_dev (i32 per sorted row) may be
 * NULL; vx/vy/vz_dev (f32 per sorted row, updated in place) are used when
 * mech->velocity_field >= 0 and must then be non-NULL. */
int olc_stage_contact_mech(const float* posr_dev, const uint32_t* ranges_dev, uint32_t n,
                           const OlcGeom* geom, const OlcContact* spec, const OlcMechanics* mech,
                           const int32_t* state_dev, float* vx_dev, float* vy_dev, float* vz_dev, float dt,
                           float* x_dev, float* y_dev, float* z_dev, void* stream);

/* The same with active motion: species_dev (i32 per row) and rng_dev (u32 per
 * row, advanced in place) may be NULL; o2_dev / glucose_dev are FP32 fields of
 * geom->chem_dims (x fastest), or NULL.  mech's column indices are ignored
 * here: presence of a pointer turns the term on. */
int olc_stage_contact_motion(const float* posr_dev, const uint32_t* ranges_dev, uint32_t n,
                             const OlcGeom* geom, const OlcContact* spec, const OlcMechanics* mech,
                             const int32_t* state_dev, float* vx_dev, float* vy_dev, float* vz_dev,
                             const int32_t* species_dev, uint32_t* rng_dev, const float* o2_dev,
                             const float* glucose_dev, float dt, float* x_dev, float* y_dev, float* z_dev,
                             void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OLC_H */
