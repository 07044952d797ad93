// libolc.so: simulation handle, NVRTC rule compilation, step orchestration and
// the C ABI declared in include/olc.h.
//
// One step (replaces GpuBackend.run_step,
// framework/src/oncolytica/gpu/runtime/_gpu_backend.py:113-171):
//   1. fields: implicit sink, then S explicit substeps per field
//   2. grid: keys (+ digit histograms, dead count) -> onesweep passes ->
//      bin table -> payload permute into the other agent buffer
//      (compaction: dead rows sort to the tail and are dropped)
//   3. cell rules (NVRTC kernels), In -> Out with a buffer flip per rule
//   4. contact pass, in place on the current positions
//   5. reductions and metric rules when collect != 0
// Everything is enqueued on one stream; no host synchronisation.
#include "olc_internal.h"
#include "olc_arena.h"

#include <nvrtc.h>

#include <map>
#include <mutex>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace olc {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
const char* get_error() { return g_err.c_str(); }
int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return OLC_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return OLC_ERR_CUDA;
}

}  // namespace olc

using namespace olc;

#define OLC_PROF_EVENTS 7
// pinned host slots of the params upload ring and of the readback ring
constexpr int HOST_SLOTS = 4;

struct StepGraph {
    int key = 0;  // (agent buffer << 16) | (tissue buffer << 12) | (field parity mask << 1) | collect
    int agent_after = 0;
    int field_after = 0;
    int tissue_after = 0;
    uint64_t launches = 0;
    cudaGraphExec_t exec = nullptr;
};

struct OlcSim {
    OlcGeom geom;
    OlcCaps caps;
    BinGrid bins;
    int key_bits = 0;
    olc_u32 n_table = 0;  // bin table entries = sentinel + 1

    void* col[2][OLC_MAX_AGENT_COLS] = {};
    int agent_cur = 0;

    float* field[2][OLC_MAX_FIELDS] = {};
    float* sink[OLC_MAX_FIELDS] = {};
    OlcDiffusion fspec[OLC_MAX_FIELDS] = {};
    FieldStep fstep[OLC_MAX_FIELDS] = {};
    int field_cur[OLC_MAX_FIELDS] = {};
    bool field_bound[OLC_MAX_FIELDS] = {};
    FieldMaps fmaps[OLC_MAX_FIELDS];           // TMA descriptors of both buffers
    OlcTuning tuning = {8, 8, OLC_CONTACT_FLAT, 16, 0, 0, 0};  // kernel shapes and variants (olc_set_tuning)
    std::vector<int> member_depth;                    // batched FP32 tile depth per member (0: tuning's)
    FieldMaps16 fmaps16[OLC_MAX_FIELDS];       // the same for 16-bit storage
    float* comp[OLC_MAX_FIELDS] = {};          // 16-bit storage: reaction residual per voxel (FP32)
    Pins pins[OLC_MAX_FIELDS] = {};            // voxels held at a value after every substep

    OlcContact contact = {};
    ContactDev contact_dev = {};
    OlcMechanics mech = {};  // engine force-law extras (mech.enabled)

    const unsigned char* tissue = nullptr;  // borrowed tissue columns (Morton-indexed), the current buffer
    unsigned char* tissue_buf[2] = {};      // tissue rules: both buffers (olc_bind_tissue_pair)
    int tissue_cur = 0;
    int tissue_cols = 0;
    size_t tissue_stride = 0;

    // library-owned device memory
    olc_u32* counters = nullptr;
    unsigned char* life = nullptr;
    olc_u32* keys_in = nullptr;
    olc_u32* keys = nullptr;
    olc_u32* vals = nullptr;
    void* sort_mem = nullptr;
    SortScratch sc = {};
    olc_u32* ranges = nullptr;
    float4* posr = nullptr;
    olc_u32* birth_lb = nullptr;
    olc_u32 rule_tiles = 0;
    unsigned char* params_dev = nullptr;
    size_t params_cap = 0;
    unsigned char* params_host = nullptr;  // pinned staging
    OlcReductions* red_dev = nullptr;
    RedScratch red_scratch = {};
    OlcReductions* red_host = nullptr;     // pinned
    void* metrics_dev = nullptr;
    size_t metrics_bytes = 0;
    olc_u32* ctr_host_words = nullptr;     // pinned copy of the counter block
    // solo handles: params uploads rotate over HOST_SLOTS pinned staging
    // slots of params_cap bytes, each reused once the copy that last read it
    // has run (param_ev), so an upload never waits for the stream
    cudaEvent_t param_ev[HOST_SLOTS] = {};
    olc_u64 param_seq = 0;
    // queued readbacks (olc_queue_readback): slot k of rb_host holds the
    // counter block then the metric accumulators of ticket rb_ticket[k]
    unsigned char* rb_host = nullptr;      // pinned, HOST_SLOTS x rb_stride
    size_t rb_stride = 0;
    cudaEvent_t rb_ev[HOST_SLOTS] = {};
    olc_u64 rb_ticket[HOST_SLOTS] = {};
    olc_u64 rb_steps[HOST_SLOTS] = {};
    olc_u64 rb_next = 1;
    EngineMetricAcc* em_acc = nullptr;     // engine metrics (allocated on first use)
    double* em_partials = nullptr;
    EngineMetricAcc* em_host = nullptr;    // pinned

    cudaLibrary_t module = nullptr;
    std::vector<cudaKernel_t> funcs;
    std::vector<int> kinds;
    std::vector<int> iters;  // per kernel: chemistry-rule iterations (1 otherwise)
    int n_cell_rules = 0;

    uint64_t steps = 0;
    uint64_t total_launches = 0;
    std::string err;

    // stage profiling
    bool profiling = false;
    int prof_step = 0;
    uint64_t prof_launches = 0;
    uint32_t prof_substeps = 0;
    std::vector<std::array<cudaEvent_t, OLC_PROF_EVENTS>> events;

    // batched mode (n_sims > 0): many simulations of one model in one handle
    olc_u32 n_sims = 0;
    std::vector<OlcGeom> geoms;
    std::vector<OlcSimDesc> desc_host;
    OlcSimDesc* desc_dev = nullptr;
    BatchArgs bargs = {};
    std::vector<unsigned long long> field_off;        // n_sims + 1 voxel offsets into every field buffer
    void** cols_dev = nullptr;                        // agent column tables: [2][OLC_MAX_AGENT_COLS]
    bool cols_dirty = true;
    unsigned char* fpar_dev = nullptr;                // field buffer parity per (simulation, field)
    FieldStep* bsteps_dev = nullptr;                  // per (simulation, field)
    std::vector<FieldStep> bsteps_host;
    uint4* btiles_all = nullptr;                      // every field tile, simulation order
    olc_u32 n_btiles = 0;
    uint4* btiles_field[OLC_MAX_FIELDS] = {};         // per field, by substep count (descending), substep tiles
    std::vector<CUtensorMap> bmaps_host;              // [(simulation * n_fields + field) * 2 + buffer]
    CUtensorMap* bmaps_dev = nullptr;
    std::vector<olc_u32> btile_count[OLC_MAX_FIELDS];  // [s] = tiles of simulations taking > s substeps
    OlcReductions* red_batch_dev = nullptr;
    OlcReductions* red_batch_host = nullptr;          // pinned
    size_t params_stride = 0;

    // serving pool (pool == true): a batch whose members join and leave
    // between steps; n_sims is the slot count
    bool pool = false;
    RangeArena table_arena, field_arena;
    std::vector<unsigned char> slot_used;
    std::vector<olc_u64> slot_table_off, slot_table_n, slot_field_off, slot_field_n;
    olc_u32 slots_used = 0;
    bool pool_dirty = false;                          // records / tiles changed since the last upload
    uint64_t pool_steps = 0;                          // steps run on the pool
    std::vector<unsigned char> params_all;            // host copy of every slot's Params
    unsigned char* stage_host[2] = {};                // pinned upload staging, alternating
    size_t stage_cap[2] = {};
    cudaEvent_t stage_ev[2] = {};
    int stage_i = 0;
    size_t tiles_cap = 0;                             // tiles held by btiles_all / btiles_field[f]
    olc_u32* gather_counts = nullptr;                 // POOL_GATHER_BLOCKS words
    uint2* table_chunks = nullptr;                    // bin-table ranges of the members, cleared each step
    olc_u32 n_table_chunks = 0;
    size_t table_chunks_cap = 0;

    // CUDA graphs of whole steps, keyed by the buffer parities at step start
    bool use_graphs = false;
    cudaStream_t capture_stream = nullptr;
    std::vector<StepGraph> graphs;
    std::vector<int> graph_seen;
};

namespace {

int fail(OlcSim* s, int code, const std::string& msg) {
    if (s) s->err = msg;
    set_error(msg);
    return code;
}

int check(OlcSim* s, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return OLC_OK;
    return fail(s, OLC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define OLC_TRY(expr)                 \
    do {                              \
        int _rc = (expr);             \
        if (_rc != OLC_OK) return _rc; \
    } while (0)

template <typename T>
int dev_alloc(OlcSim* s, T** p, size_t bytes, const char* what) {
    if (bytes == 0) bytes = 256;
    return check(s, cudaMalloc(reinterpret_cast<void**>(p), bytes), what);
}

bool geom_ok(const OlcGeom& g, std::string* err) {
    for (int i = 0; i < 3; ++i) {
        if (g.tissue_dims[i] <= 0 || g.tissue_dims[i] > 240 || (g.tissue_dims[i] & 1)) {
            *err = "tissue_dims must be even and in [2, 240] (reference limit, _engine.py:84-96)";
            return false;
        }
        if (g.chem_dims[i] < 0) {
            *err = "chem_dims must be >= 0";
            return false;
        }
    }
    if (!(g.tissue_voxel_size > 0.0f)) {
        *err = "tissue_voxel_size must be > 0";
        return false;
    }
    return true;
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Initialises the runtime on the current device (the primary context that
// torch shares).
int ensure_context(OlcSim* s) { return check(s, cudaFree(nullptr), "cudaFree(0)"); }

OlcRuleParams make_rule_params(OlcSim* s, int rule_index, int in_buf) {
    OlcRuleParams P;
    std::memset(&P, 0, sizeof(P));
    for (olc_u32 c = 0; c < s->caps.n_agent_fields; ++c) {
        P.in[c] = s->col[in_buf][c];
        P.out[c] = s->col[1 - in_buf][c];
    }
    for (olc_u32 f = 0; f < s->caps.n_fields; ++f) {
        P.field[f] = s->field[s->field_cur[f]][f];
        P.field_type[f] = field_type_word(s->fstep[f]);
        P.field_bval[f] = s->fstep[f].bval;
        P.sink[f] = s->sink[f];
    }
    P.ranges = s->ranges;
    P.life = s->life;
    P.posr = s->contact.enabled ? s->posr : nullptr;
    P.counters = s->counters;
    P.birth_lb = s->birth_lb + (size_t)rule_index * s->rule_tiles;
    P.params = s->params_dev;
    P.metrics = s->metrics_dev;
    P.tissue = s->tissue_cols > 0 ? s->tissue : nullptr;
    P.n_tissue_cols = s->tissue_cols;
    P.tissue_stride = (olc_u32)s->tissue_stride;
    for (int i = 0; i < 3; ++i) {
        P.tdims[i] = s->geom.tissue_dims[i];
        P.cdims[i] = s->geom.chem_dims[i];
    }
    P.tvs = s->geom.tissue_voxel_size;
    P.cvs = s->geom.chem_voxel_size;
    P.capacity = s->caps.max_agents;
    P.n_cols = s->caps.n_agent_fields;
    P.radius_col = s->contact.radius_field;
    P.radius_const = s->contact.radius_const;
    P.rule_index = rule_index;
    if (s->n_sims) {
        P.sims = s->desc_dev;
        P.cols_in = s->cols_dev + (size_t)in_buf * OLC_MAX_AGENT_COLS;
        P.cols_out = s->cols_dev + (size_t)(1 - in_buf) * OLC_MAX_AGENT_COLS;
        for (olc_u32 f = 0; f < s->caps.n_fields; ++f) {
            P.field[f] = s->field[0][f];
            P.field_alt[f] = s->field[1][f];
            P.field_type[f] = field_type_word(s->fstep[f]);
            P.field_bval[f] = s->fstep[f].bval;
        }
        P.fpar = s->fpar_dev;
        P.n_fields = (int)s->caps.n_fields;
        P.sim_col = (int)s->caps.n_agent_fields - 1;
        P.vtiles = s->btiles_all;
        P.n_vtiles = (olc_u32)s->n_btiles;
        P.vtile[0] = BATCH_TILE_X;
        P.vtile[1] = BATCH_TILE_Y;
        P.vtile[2] = BATCH_TILE_Z;
        P.tissue = nullptr;
        P.n_tissue_cols = 0;
    }
    return P;
}

// Active-motion inputs of the engine's force law from a handle's current buffers.
void fill_motion(OlcSim* s, const OlcMechanics& mech, int cc, MechDev* m) {
    if (mech.n_species < 1) return;  // no species table: no active motion
    m->species = mech.species_field >= 0 ? static_cast<const int*>(s->col[cc][mech.species_field]) : nullptr;
    m->rng = mech.rng_field >= 0 ? static_cast<olc_u32*>(s->col[cc][mech.rng_field]) : nullptr;
    m->f0 = mech.o2_field >= 0 ? s->field[s->field_cur[mech.o2_field]][mech.o2_field] : nullptr;
    m->f1 = mech.glucose_field >= 0 ? s->field[s->field_cur[mech.glucose_field]][mech.glucose_field] : nullptr;
    m->f0_type = mech.o2_field >= 0 ? field_type_word(s->fstep[mech.o2_field]) : 0;
    m->f1_type = mech.glucose_field >= 0 ? field_type_word(s->fstep[mech.glucose_field]) : 0;
    m->f0_b = mech.o2_field >= 0 ? s->fstep[mech.o2_field].bval : 0.0f;
    m->f1_b = mech.glucose_field >= 0 ? s->fstep[mech.glucose_field].bval : 0.0f;
    for (int i = 0; i < 3; ++i) m->cdims[i] = s->geom.chem_dims[i];
    m->cvs = s->geom.chem_voxel_size;
    m->chemo_force = mech.chemo_force;
    m->impulse = mech.motility_impulse;
    m->n_species = mech.n_species < 1 ? 1 : (mech.n_species > OLC_MAX_SPECIES ? OLC_MAX_SPECIES : mech.n_species);
    for (int k = 0; k < OLC_MAX_SPECIES; ++k) {
        m->sp_o2[k] = mech.species[k].chemotaxis_o2;
        m->sp_glu[k] = mech.species[k].chemotaxis_glucose;
        m->sp_move[k] = mech.species[k].move_prob;
    }
}

int launch_rule(OlcSim* s, int k, const OlcRuleParams& P, cudaStream_t st, olc_u32 units = 0) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (units == 0) units = s->caps.max_agents;
    olc_u32 blocks = (units + OLC_RULE_THREADS - 1) / OLC_RULE_THREADS;
    if (blocks == 0) blocks = 1;
    const olc_u32 cap_blocks = (olc_u32)sms * 8u;
    if (blocks > cap_blocks) blocks = cap_blocks;
    void* args[] = {const_cast<OlcRuleParams*>(&P)};
    return check(s, cudaLaunchKernel(reinterpret_cast<const void*>(s->funcs[k]), dim3(blocks), dim3(OLC_RULE_THREADS),
                                     args, 0, st),
                 "cudaLaunchKernel(rule)");
}

// Records stage event `k` of the current profiled step.
void mark(OlcSim* s, int k, cudaStream_t st) {
    if (!s->profiling) return;
    cudaEventRecord(s->events[s->prof_step][k], st);
}

int step_once(OlcSim* s, int collect, cudaStream_t st) {
    const olc_u32 cap = s->caps.max_agents;
    if (s->profiling) {
        if ((size_t)s->prof_step >= s->events.size()) {
            std::array<cudaEvent_t, OLC_PROF_EVENTS> ev;
            for (auto& e : ev) OLC_TRY(check(s, cudaEventCreate(&e), "cudaEventCreate"));
            s->events.push_back(ev);
        }
    }
    uint64_t launches = 0;
    uint32_t substeps = 0;
    mark(s, 0, st);
    // 1. fields: implicit sinks, then the substeps of every field
    for (olc_u32 f = 0; f < s->caps.n_fields; ++f) {
        if (!s->field_bound[f] || s->fstep[f].substeps == 0) continue;
        if (s->fstep[f].storage != OLC_FIELD_F32) {
            // 16-bit storage: uptake and the step's decay, compensated, every step
            launch_react16(s->field[s->field_cur[f]][f], s->sink[f], s->comp[f], s->fstep[f], st);
            ++launches;
            continue;
        }
        if (!s->sink[f]) continue;
        launch_sink(s->field[s->field_cur[f]][f], s->sink[f], s->fstep[f], st);
        ++launches;
    }
    mark(s, 1, st);
    for (olc_u32 f = 0; f < s->caps.n_fields; ++f) {
        if (!s->field_bound[f] || s->fstep[f].substeps == 0) continue;  // unbound or static
        int cur = s->field_cur[f];
        if (s->fstep[f].storage != OLC_FIELD_F32) {
            void* res = run_substeps16(s->field[cur][f], s->field[1 - cur][f], s->fmaps16[f], cur, s->fstep[f],
                                       s->counters + OLC_CTR_STATUS, s->counters + OLC_CTR_FIELD_STEP, 0u, (int)f, st);
            s->field_cur[f] = (res == s->field[cur][f]) ? cur : 1 - cur;
            substeps += (uint32_t)s->fstep[f].substeps;
            launches += (uint64_t)s->fstep[f].substeps;
            continue;
        }
        float* a = s->field[cur][f];
        float* b = s->field[1 - cur][f];
        const bool tma_path = s->fmaps[f].ok;
        const Pins* pins = s->pins[f].n ? &s->pins[f] : nullptr;
        float* res = tma_path ? run_substeps_tma(a, b, s->fmaps[f], cur, s->fstep[f], s->counters + OLC_CTR_STATUS, st,
                                                 pins)
                              : run_substeps(a, b, s->fstep[f], st, pins);
        s->field_cur[f] = (res == a) ? cur : 1 - cur;
        substeps += (uint32_t)s->fstep[f].substeps;
        launches += (uint64_t)(tma_path ? substep_launches(s->fmaps[f], s->fstep[f], pins)
                                        : (pins ? 2 * s->fstep[f].substeps : s->fstep[f].substeps));
    }
    mark(s, 2, st);
    // 2. grid + compaction
    const int passes = (s->key_bits + 7) / 8;
    const int ac = s->agent_cur;
    OLC_TRY(check(s, cudaMemsetAsync(s->sc.hist, 0, MAX_PASSES * RADIX * 4, st), "memset hist"));
    launch_keys(static_cast<const float*>(s->col[ac][0]), static_cast<const float*>(s->col[ac][1]),
                static_cast<const float*>(s->col[ac][2]), s->life, nullptr, 0, s->counters, cap, s->bins,
                s->keys_in, s->sc.hist, passes, s->counters + OLC_CTR_DEAD_TMP, st);
    run_sort(s->keys_in, nullptr, s->keys, s->vals, s->counters + OLC_CTR_ROWS, 0, cap, s->key_bits, s->sc,
             true, s->counters, cap, st);
    OLC_TRY(check(s, cudaMemsetAsync(s->ranges, 0, (size_t)s->n_table * 8, st), "memset ranges"));
    launch_bin_ranges(s->keys, s->counters + OLC_CTR_ROWS, 0, cap, s->bins.sentinel, s->ranges, st);
    PermuteArgs pa;
    std::memset(&pa, 0, sizeof(pa));
    pa.ncols = (int)s->caps.n_agent_fields;
    for (int c = 0; c < pa.ncols; ++c) {
        pa.src[c] = s->col[ac][c];
        pa.dst[c] = s->col[1 - ac][c];
    }
    pa.radius_col = s->contact.radius_field;
    pa.radius_const = s->contact.radius_const;
    pa.write_posr = (s->contact.enabled && s->n_cell_rules == 0) ? 1 : 0;
    pa.posr = s->posr;
    pa.life = s->life;
    launch_permute(s->vals, s->counters, cap, pa, st);
    s->agent_cur = 1 - ac;
    launches += 4 + (uint64_t)passes;  // keys, scan, passes, bin table, permute
    // 3a. tissue rules, then chemistry rules (one thread per voxel; each reads
    // the state before it and writes the other buffer)
    for (size_t k = 0; k < s->funcs.size(); ++k) {
        if (s->kinds[k] != 2) continue;
        if (!s->tissue_buf[0] || !s->tissue_buf[1])
            return fail(s, OLC_ERR_STATE, "tissue rule: bind the tissue grid with olc_bind_tissue_pair");
        OlcRuleParams P = make_rule_params(s, 0, s->agent_cur);
        P.tissue = s->tissue_buf[s->tissue_cur];
        P.tissue_out = s->tissue_buf[1 - s->tissue_cur];
        const olc_u32 nv = (olc_u32)s->geom.tissue_dims[0] * s->geom.tissue_dims[1] * s->geom.tissue_dims[2];
        OLC_TRY(launch_rule(s, (int)k, P, st, nv));
        s->tissue_cur = 1 - s->tissue_cur;
        s->tissue = s->tissue_buf[s->tissue_cur];
        ++launches;
    }
    for (size_t k = 0; k < s->funcs.size(); ++k) {
        if (s->kinds[k] != 3) continue;
        for (olc_u32 f = 0; f < s->caps.n_fields; ++f)
            if (!s->field_bound[f] || s->fstep[f].storage != OLC_FIELD_F32)
                return fail(s, OLC_ERR_STATE, "chemistry rule: every chemistry field must be bound with FP32 storage");
        const olc_u32 nv = (olc_u32)s->geom.chem_dims[0] * s->geom.chem_dims[1] * s->geom.chem_dims[2];
        for (int it = 0; it < s->iters[k]; ++it) {
            OlcRuleParams P = make_rule_params(s, 0, s->agent_cur);
            for (olc_u32 f = 0; f < s->caps.n_fields; ++f) P.field_out[f] = s->field[1 - s->field_cur[f]][f];
            OLC_TRY(launch_rule(s, (int)k, P, st, nv));
            for (olc_u32 f = 0; f < s->caps.n_fields; ++f) s->field_cur[f] = 1 - s->field_cur[f];
            ++launches;
        }
    }
    mark(s, 3, st);
    // 3. cell rules
    if (s->n_cell_rules > 0) {
        OLC_TRY(check(s, cudaMemsetAsync(s->birth_lb, 0, (size_t)s->n_cell_rules * s->rule_tiles * 4, st),
                      "memset birth look-back"));
    }
    int cell_idx = 0;
    for (size_t k = 0; k < s->funcs.size(); ++k) {
        if (s->kinds[k] != 0) continue;
        OlcRuleParams P = make_rule_params(s, cell_idx, s->agent_cur);
        OLC_TRY(launch_rule(s, (int)k, P, st));
        s->agent_cur = 1 - s->agent_cur;
        ++cell_idx;
        ++launches;
    }
    mark(s, 4, st);
    // 4. contact
    const int cc = s->agent_cur;
    if (s->contact.enabled && s->mech.enabled) {
        MechDev m = {};
        m.state = s->mech.state_field >= 0 ? static_cast<const int*>(s->col[cc][s->mech.state_field]) : nullptr;
        m.necrotic_factor = s->mech.necrotic_factor;
        m.adh_k = s->mech.adhesion_stiffness;
        m.adh_range = s->mech.adhesion_range;
        if (s->mech.velocity_field >= 0) {
            m.vx = static_cast<float*>(s->col[cc][s->mech.velocity_field]);
            m.vy = static_cast<float*>(s->col[cc][s->mech.velocity_field + 1]);
            m.vz = static_cast<float*>(s->col[cc][s->mech.velocity_field + 2]);
        }
        m.damping = s->mech.damping;
        m.max_speed = s->mech.max_speed;
        fill_motion(s, s->mech, cc, &m);
        launch_contact_mech(s->posr, s->ranges, s->counters + OLC_CTR_N, 0, cap, s->contact_dev, m,
                            static_cast<float*>(s->col[cc][0]), static_cast<float*>(s->col[cc][1]),
                            static_cast<float*>(s->col[cc][2]), st);
        ++launches;
    } else if (s->contact.enabled) {
        launch_contact(s->posr, s->ranges, s->counters + OLC_CTR_N, 0, cap, s->contact_dev,
                       static_cast<float*>(s->col[cc][0]), static_cast<float*>(s->col[cc][1]),
                       static_cast<float*>(s->col[cc][2]), st, s->tuning.contact_variant, s->n_table);
        ++launches;
    }
    mark(s, 5, st);
    // 5. reductions + metric rules
    if (collect) {
        launch_reset_reductions(s->red_dev, (int)s->caps.n_fields, st);
        launches += 2;
        ReduceArgs ra;
        ra.x = static_cast<const float*>(s->col[cc][0]);
        ra.y = static_cast<const float*>(s->col[cc][1]);
        ra.z = static_cast<const float*>(s->col[cc][2]);
        ra.state = s->caps.state_field >= 0 ? static_cast<const int*>(s->col[cc][s->caps.state_field]) : nullptr;
        ra.life = s->life;
        ra.cx = s->caps.center[0];
        ra.cy = s->caps.center[1];
        ra.cz = s->caps.center[2];
        ra.bin_width = s->caps.radial_bin_width > 0.0f ? s->caps.radial_bin_width : 1.0f;
        launch_reduce_agents(ra, s->counters, cap, s->red_dev, s->red_scratch, st);
        for (olc_u32 f = 0; f < s->caps.n_fields; ++f) {
            if (!s->field_bound[f]) continue;
            const size_t nvox = (size_t)s->geom.chem_dims[0] * s->geom.chem_dims[1] * s->geom.chem_dims[2];
            if (s->fstep[f].storage != OLC_FIELD_F32) {
                FieldStep fsr = s->fstep[f];
                for (int i = 0; i < 3; ++i) fsr.dims[i] = s->geom.chem_dims[i];
                launch_reduce_field16(s->field[s->field_cur[f]][f], s->comp[f], fsr, (int)f, s->red_dev,
                                      s->red_scratch, st);
            } else {
                launch_reduce_field(s->field[s->field_cur[f]][f], nvox, (int)f, s->red_dev, s->red_scratch, st);
            }
            ++launches;
        }
        if (s->metrics_dev && s->metrics_bytes) {
            OLC_TRY(check(s, cudaMemsetAsync(s->metrics_dev, 0, s->metrics_bytes, st), "memset metrics"));
        }
        for (size_t k = 0; k < s->funcs.size(); ++k) {
            if (s->kinds[k] != 1) continue;
            OlcRuleParams P = make_rule_params(s, 0, cc);
            OLC_TRY(launch_rule(s, (int)k, P, st));
            ++launches;
        }
    }
    mark(s, 6, st);
    if (s->profiling) {
        s->prof_step++;
        s->prof_launches += launches;
        s->prof_substeps += substeps;
    }
    s->total_launches += launches;
    s->steps++;
    return check(s, cudaGetLastError(), "step launch");
}

// One step of a batch: the stages of step_once over every simulation at once
// (olc_batch.cu holds the kernels and the layout).
int step_once_batch(OlcSim* s, int collect, cudaStream_t st) {
    const olc_u32 cap = s->caps.max_agents;
    const olc_u32 F = s->caps.n_fields;
    if (s->cols_dirty) {
        void* tab[2 * OLC_MAX_AGENT_COLS] = {};
        for (int b = 0; b < 2; ++b)
            for (olc_u32 c = 0; c < s->caps.n_agent_fields; ++c) tab[b * OLC_MAX_AGENT_COLS + c] = s->col[b][c];
        OLC_TRY(check(s, cudaMemcpy(s->cols_dev, tab, sizeof(tab), cudaMemcpyHostToDevice), "column tables"));
        s->cols_dirty = false;
    }
    if (s->profiling && (size_t)s->prof_step >= s->events.size()) {
        std::array<cudaEvent_t, OLC_PROF_EVENTS> ev;
        for (auto& e : ev) OLC_TRY(check(s, cudaEventCreate(&e), "cudaEventCreate"));
        s->events.push_back(ev);
    }
    uint64_t launches = 0;
    uint32_t substeps = 0;
    const BatchArgs& B = s->bargs;
    mark(s, 0, st);
    // 1. fields: sinks, then every field's substeps over the simulations that take them
    for (olc_u32 f = 0; f < F; ++f) {
        if (!s->field_bound[f]) continue;
        const int stor = s->fstep[f].storage;
        if (stor != OLC_FIELD_F32) {
            launch_react_batch16(B, stor, s->fstep[f].encoding, s->btiles_all, s->n_btiles, s->bsteps_dev, (int)f,
                                 (int)F, s->fpar_dev, s->field[0][f], s->field[1][f], s->sink[f], s->comp[f], st);
            ++launches;
            continue;
        }
        if (!s->sink[f]) continue;
        launch_sink_batch(B, s->btiles_all, s->n_btiles, s->bsteps_dev, (int)f, (int)F, s->fpar_dev, s->field[0][f],
                          s->field[1][f], s->sink[f], st);
        ++launches;
    }
    mark(s, 1, st);
    for (olc_u32 f = 0; f < F; ++f) {
        if (!s->field_bound[f]) continue;
        const std::vector<olc_u32>& cnt = s->btile_count[f];
        const int stor = s->fstep[f].storage;
        for (size_t sub = 0; sub < cnt.size(); ++sub) {
            if (stor != OLC_FIELD_F32)
                launch_substep_batch_t16(B, stor, s->fstep[f].encoding, s->btiles_field[f], cnt[sub], s->bsteps_dev,
                                         s->bmaps_dev, (int)f,
                                         (int)F, s->fpar_dev, (int)sub, s->field[0][f], s->field[1][f],
                                         s->counters + OLC_CTR_FIELD_STEP, s->counters + OLC_CTR_STATUS, st);
            else
                launch_substep_batch(B, s->btiles_field[f], cnt[sub], s->bsteps_dev, (int)f, (int)F, s->fpar_dev,
                                     (int)sub, s->field[0][f], s->field[1][f], st);
            ++launches;
        }
        substeps += (uint32_t)cnt.size();
        launch_flip_parity(s->bsteps_dev, (int)f, (int)F, s->n_sims, s->fpar_dev, st);
        ++launches;
    }
    mark(s, 2, st);
    // 2. grid + compaction
    const int passes = (s->key_bits + 7) / 8;
    const int ac = s->agent_cur;
    const int sim_col = (int)s->caps.n_agent_fields - 1;
    OLC_TRY(check(s, cudaMemsetAsync(s->sc.hist, 0, MAX_PASSES * RADIX * 4, st), "memset hist"));
    launch_keys_batch(B, static_cast<const float*>(s->col[ac][0]), static_cast<const float*>(s->col[ac][1]),
                      static_cast<const float*>(s->col[ac][2]), static_cast<const olc_u32*>(s->col[ac][sim_col]),
                      s->life, s->counters, cap, s->keys_in, s->sc.hist, passes, s->counters + OLC_CTR_DEAD_TMP, st);
    run_sort(s->keys_in, nullptr, s->keys, s->vals, s->counters + OLC_CTR_ROWS, 0, cap, s->key_bits, s->sc, true,
             s->counters, cap, st);
    if (s->pool) {
        launch_clear_table_chunks(s->table_chunks, s->n_table_chunks, s->ranges, st);
    } else {
        OLC_TRY(check(s, cudaMemsetAsync(s->ranges, 0, (size_t)s->n_table * 8, st), "memset ranges"));
    }
    launch_bin_ranges_batch(B, s->keys, s->counters + OLC_CTR_ROWS, cap, s->ranges, st);
    PermuteArgs pa;
    std::memset(&pa, 0, sizeof(pa));
    pa.ncols = (int)s->caps.n_agent_fields;
    for (int c = 0; c < pa.ncols; ++c) {
        pa.src[c] = s->col[ac][c];
        pa.dst[c] = s->col[1 - ac][c];
    }
    pa.radius_col = s->contact.radius_field;
    pa.radius_const = s->contact.radius_const;
    pa.write_posr = (s->contact.enabled && s->n_cell_rules == 0) ? 1 : 0;
    pa.posr = s->posr;
    pa.life = s->life;
    launch_permute(s->vals, s->counters, cap, pa, st);
    s->agent_cur = 1 - ac;
    launches += 4 + (uint64_t)passes;
    // 3a. chemistry rules over every member (a CTA per field tile), each
    // iteration writing the members' other buffers, whose parity then flips
    for (size_t k = 0; k < s->funcs.size(); ++k) {
        if (s->kinds[k] != 3) continue;
        for (olc_u32 f = 0; f < F; ++f)
            if (!s->field_bound[f] || s->fstep[f].storage != OLC_FIELD_F32)
                return fail(s, OLC_ERR_STATE, "chemistry rule: every chemistry field must be bound with FP32 storage");
        for (int it = 0; it < s->iters[k]; ++it) {
            const OlcRuleParams P = make_rule_params(s, 0, s->agent_cur);
            OLC_TRY(launch_rule(s, (int)k, P, st, (olc_u32)s->n_btiles * (BATCH_TILE_X * BATCH_TILE_Y * BATCH_TILE_Z)));
            launch_flip_parity_all((int)F, s->n_sims, s->fpar_dev, st);
            launches += 2;
        }
    }
    mark(s, 3, st);
    // 3. cell rules
    if (s->n_cell_rules > 0) {
        OLC_TRY(check(s, cudaMemsetAsync(s->birth_lb, 0, (size_t)s->n_cell_rules * s->rule_tiles * 4, st),
                      "memset birth look-back"));
    }
    int cell_idx = 0;
    for (size_t k = 0; k < s->funcs.size(); ++k) {
        if (s->kinds[k] != 0) continue;
        OlcRuleParams P = make_rule_params(s, cell_idx, s->agent_cur);
        OLC_TRY(launch_rule(s, (int)k, P, st));
        s->agent_cur = 1 - s->agent_cur;
        ++cell_idx;
        ++launches;
    }
    mark(s, 4, st);
    // 4. contact
    const int cc = s->agent_cur;
    if (s->contact.enabled) {
        launch_contact_batch(B, s->posr, s->ranges, static_cast<const olc_u32*>(s->col[cc][sim_col]),
                             s->counters + OLC_CTR_N, cap, s->contact_dev, static_cast<float*>(s->col[cc][0]),
                             static_cast<float*>(s->col[cc][1]), static_cast<float*>(s->col[cc][2]), st);
        ++launches;
    }
    mark(s, 5, st);
    // 5. per-simulation reductions + metric rules
    if (collect) {
        launch_reset_reductions_batch(s->red_batch_dev, s->n_sims, st);
        ReduceArgs ra;
        ra.x = static_cast<const float*>(s->col[cc][0]);
        ra.y = static_cast<const float*>(s->col[cc][1]);
        ra.z = static_cast<const float*>(s->col[cc][2]);
        ra.state = s->caps.state_field >= 0 ? static_cast<const int*>(s->col[cc][s->caps.state_field]) : nullptr;
        ra.life = s->life;
        ra.cx = ra.cy = ra.cz = 0.0f;
        ra.bin_width = 1.0f;
        launch_reduce_agents_batch(B, ra, static_cast<const olc_u32*>(s->col[cc][sim_col]), s->counters, cap,
                                   s->red_batch_dev, st);
        launches += 3;
        for (olc_u32 f = 0; f < F; ++f) {
            if (!s->field_bound[f]) continue;
            if (s->fstep[f].storage != OLC_FIELD_F32)
                launch_reduce_field_batch16(B, s->fstep[f].storage, s->fstep[f].encoding, s->btiles_all,
                                            s->n_btiles, s->bsteps_dev, (int)f, (int)F, s->fpar_dev, s->field[0][f],
                                            s->field[1][f], s->comp[f], s->red_batch_dev, st);
            else
                launch_reduce_field_batch(B, s->btiles_all, s->n_btiles, (int)f, (int)F, s->fpar_dev, s->field[0][f],
                                          s->field[1][f], s->red_batch_dev, st);
            ++launches;
        }
        if (s->metrics_dev && s->metrics_bytes) {
            OLC_TRY(check(s, cudaMemsetAsync(s->metrics_dev, 0, s->metrics_bytes * s->n_sims, st), "memset metrics"));
        }
        for (size_t k = 0; k < s->funcs.size(); ++k) {
            if (s->kinds[k] != 1) continue;
            OlcRuleParams P = make_rule_params(s, 0, cc);
            OLC_TRY(launch_rule(s, (int)k, P, st));
            ++launches;
        }
    }
    mark(s, 6, st);
    if (s->profiling) {
        s->prof_step++;
        s->prof_launches += launches;
        s->prof_substeps += substeps;
    }
    s->total_launches += launches;
    s->steps++;
    return check(s, cudaGetLastError(), "batch step launch");
}

int step_any(OlcSim* s, int collect, cudaStream_t st) {
    return s->n_sims ? step_once_batch(s, collect, st) : step_once(s, collect, st);
}

int upload_desc(OlcSim* s) {
    return check(s, cudaMemcpy(s->desc_dev, s->desc_host.data(), sizeof(OlcSimDesc) * s->n_sims,
                               cudaMemcpyHostToDevice),
                 "upload simulation records");
}

int field_mask(const OlcSim* s) {
    int m = 0;
    for (int f = 0; f < OLC_MAX_FIELDS; ++f) m |= (s->field_cur[f] & 1) << f;
    return m;
}

void set_field_mask(OlcSim* s, int m) {
    for (int f = 0; f < OLC_MAX_FIELDS; ++f) s->field_cur[f] = (m >> f) & 1;
}

void drop_graphs(OlcSim* s) {
    if (!s->graphs.empty()) {
        cudaDeviceSynchronize();
        for (auto& g : s->graphs) cudaGraphExecDestroy(g.exec);
        s->graphs.clear();
    }
    s->graph_seen.clear();
}

// Without the device synchronisation: an executable graph destroyed while in
// flight is released when it completes.  For membership changes of a pool,
// whose buffers stay allocated.
void drop_graphs_nosync(OlcSim* s) {
    for (auto& g : s->graphs) cudaGraphExecDestroy(g.exec);
    s->graphs.clear();
    s->graph_seen.clear();
}

// One step through a cached CUDA graph.  A step's launches depend only on the
// bindings and on the buffer parities at its start (agent buffer, one bit per
// field) plus `collect`, so graphs are cached by that state; the parity pattern
// repeats with period <= 2, so only a few graphs ever exist.  The first step
// from a given state runs eagerly (which also loads every kernel it uses); the
// second captures it.  Capture runs on the handle's own stream (the legacy
// default stream cannot be captured); the graph is launched on the caller's.
int step_graph(OlcSim* s, int collect, cudaStream_t st) {
    const int ac = s->agent_cur, fm = field_mask(s), tc = s->tissue_cur;
    const int key = (ac << 16) | (tc << 12) | (fm << 1) | collect;
    StepGraph* g = nullptr;
    for (auto& e : s->graphs)
        if (e.key == key) g = &e;
    if (!g) {
        bool seen = false;
        for (int k : s->graph_seen) seen |= (k == key);
        if (!seen) {
            s->graph_seen.push_back(key);
            return step_any(s, collect, st);
        }
        if (!s->capture_stream)
            OLC_TRY(check(s, cudaStreamCreateWithFlags(&s->capture_stream, cudaStreamNonBlocking), "capture stream"));
        const uint64_t steps0 = s->steps, launches0 = s->total_launches;
        OLC_TRY(check(s, cudaStreamBeginCapture(s->capture_stream, cudaStreamCaptureModeThreadLocal), "begin capture"));
        const int rc = step_any(s, collect, s->capture_stream);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(s->capture_stream, &graph);
        StepGraph ng;
        ng.key = key;
        ng.agent_after = s->agent_cur;
        ng.field_after = field_mask(s);
        ng.tissue_after = s->tissue_cur;
        ng.launches = s->total_launches - launches0;
        // nothing ran yet: restore the state the graph starts from
        s->steps = steps0;
        s->total_launches = launches0;
        s->agent_cur = ac;
        set_field_mask(s, fm);
        s->tissue_cur = tc;
        if (s->tissue_buf[tc]) s->tissue = s->tissue_buf[tc];
        if (rc != OLC_OK || e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            return rc != OLC_OK ? rc : check(s, e, "end capture");
        }
        e = cudaGraphInstantiate(&ng.exec, graph, 0);
        cudaGraphDestroy(graph);
        OLC_TRY(check(s, e, "graph instantiate"));
        s->graphs.push_back(ng);
        g = &s->graphs.back();
    }
    OLC_TRY(check(s, cudaGraphLaunch(g->exec, st), "graph launch"));
    s->agent_cur = g->agent_after;
    set_field_mask(s, g->field_after);
    s->tissue_cur = g->tissue_after;
    if (s->tissue_buf[s->tissue_cur]) s->tissue = s->tissue_buf[s->tissue_cur];
    s->total_launches += g->launches;
    s->steps++;
    return OLC_OK;
}

// ------------------------------------------------------------------ serving pool
// Field tiles of one member (slot, tile x, tile y, tile z), x fastest.
void pool_tiles(const OlcGeom& g, olc_u32 slot, std::vector<uint4>* out) {
    const int tx = (g.chem_dims[0] + BATCH_TILE_X - 1) / BATCH_TILE_X;
    const int ty = (g.chem_dims[1] + BATCH_TILE_Y - 1) / BATCH_TILE_Y;
    const int tz = (g.chem_dims[2] + BATCH_TILE_Z - 1) / BATCH_TILE_Z;
    for (int z = 0; z < tz; ++z)
        for (int y = 0; y < ty; ++y)
            for (int x = 0; x < tx; ++x) out->push_back(make_uint4(slot, (unsigned)x, (unsigned)y, (unsigned)z));
}

// Substep tiles of one member for the substep kernel of `storage`.  FP32
// tiles are 32 x 16 x depth (depth 8, 16 or 32: the member's tile depth); the
// entry's w word holds the z-tile index in its low half and the depth in its
// high half.
void substep_tiles(const OlcGeom& g, olc_u32 k, int storage, int depth, std::vector<uint4>* out) {
    const bool f32 = storage == OLC_FIELD_F32;
    const int TX = f32 ? BATCH_TILE_X : BATCH_T16_TX, TY = f32 ? BATCH_TILE_Y : BATCH_T16_TY;
    const int TZ = f32 ? depth : BATCH_T16_TZ;
    const int tx = (g.chem_dims[0] + TX - 1) / TX, ty = (g.chem_dims[1] + TY - 1) / TY;
    const int tz = (g.chem_dims[2] + TZ - 1) / TZ;
    for (int z = 0; z < tz; ++z)
        for (int y = 0; y < ty; ++y)
            for (int x = 0; x < tx; ++x)
                out->push_back(make_uint4(k, (unsigned)x, (unsigned)y, f32 ? ((unsigned)z | ((unsigned)depth << 16))
                                                                           : (unsigned)z));
}

// The batched FP32 substep tile depth of member k.
int member_tile_depth(const OlcSim* s, olc_u32 k) {
    const int d = k < s->member_depth.size() ? s->member_depth[k] : 0;
    return d > 0 ? d : s->tuning.batch_tile_depth;
}

// Tensor maps of member k's grid of field f in buffers a and b (its voxels
// from field_off on), for the batched substep kernels.
bool member_maps(OlcSim* s, olc_u32 k, int f, void* a, void* b, olc_u64 field_off, const OlcGeom& g, int storage) {
    const int elem = storage == OLC_FIELD_F32 ? 4 : 2;
    cuuint32_t box[3];
    batch_substep_box(storage, box);
    CUtensorMap* m = &s->bmaps_host[((size_t)k * s->caps.n_fields + f) * 2];
    return encode_map_elems(&m[0], static_cast<char*>(a) + field_off * elem, g.chem_dims, box, elem) &&
           encode_map_elems(&m[1], static_cast<char*>(b) + field_off * elem, g.chem_dims, box, elem);
}

int pool_grow_tiles(OlcSim* s, size_t need, cudaStream_t st) {
    if (need <= s->tiles_cap) return OLC_OK;
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync before tile-list growth"));
    const size_t cap = std::max<size_t>(need + need / 2, 4096);
    cudaFree(s->btiles_all);
    s->btiles_all = nullptr;
    OLC_TRY(dev_alloc(s, &s->btiles_all, cap * sizeof(uint4), "field tiles"));
    for (olc_u32 f = 0; f < s->caps.n_fields; ++f) {
        cudaFree(s->btiles_field[f]);
        s->btiles_field[f] = nullptr;
        OLC_TRY(dev_alloc(s, &s->btiles_field[f], cap * sizeof(uint4), "field tiles"));
    }
    s->tiles_cap = cap;
    return OLC_OK;
}

// Uploads the member records, field steps, Params and tile lists of the
// current membership (stream-ordered before the next step's kernels) through
// one of two pinned staging buffers.
int pool_commit(OlcSim* s, cudaStream_t st) {
    const olc_u32 F = s->caps.n_fields;
    std::vector<uint4> all;
    std::vector<uint2> chunks;
    std::vector<std::vector<uint4>> per_slot(s->n_sims);
    for (olc_u32 k = 0; k < s->n_sims; ++k) {
        if (!s->slot_used[k]) continue;
        pool_tiles(s->geoms[k], k, &per_slot[k]);
        all.insert(all.end(), per_slot[k].begin(), per_slot[k].end());
        for (olc_u64 e = 0; e < s->slot_table_n[k]; e += POOL_TABLE_CHUNK)
            chunks.push_back(make_uint2((unsigned)(s->slot_table_off[k] + e),
                                        (unsigned)std::min<olc_u64>(POOL_TABLE_CHUNK, s->slot_table_n[k] - e)));
    }
    if (chunks.size() > s->table_chunks_cap) return fail(s, OLC_ERR_STATE, "pool: bin-table chunk list overflow");
    std::vector<uint4> fl[OLC_MAX_FIELDS];
    std::vector<olc_u32> counts[OLC_MAX_FIELDS];
    for (olc_u32 f = 0; f < F; ++f) {
        if (!s->field_bound[f]) continue;
        std::vector<std::pair<int, olc_u32>> order;  // (substeps, slot), most substeps first, slots ascending
        for (olc_u32 k = 0; k < s->n_sims; ++k)
            if (s->slot_used[k]) order.push_back({s->bsteps_host[(size_t)k * F + f].substeps, k});
        std::stable_sort(order.begin(), order.end(), [](const std::pair<int, olc_u32>& x,
                                                        const std::pair<int, olc_u32>& y) { return x.first > y.first; });
        std::vector<int> steps_of;
        std::vector<uint4> mt;
        for (const auto& o : order) {
            mt.clear();
            substep_tiles(s->geoms[o.second], o.second, s->fstep[f].storage, member_tile_depth(s, o.second), &mt);
            fl[f].insert(fl[f].end(), mt.begin(), mt.end());
            steps_of.insert(steps_of.end(), mt.size(), o.first);
        }
        const int max_s = order.empty() ? 0 : order.front().first;
        counts[f].assign(max_s, 0u);
        olc_u32 c = (olc_u32)fl[f].size();
        for (int sub = 0; sub < max_s; ++sub) {  // tiles of members taking more than `sub` substeps
            while (c > 0 && steps_of[c - 1] <= sub) --c;
            counts[f][sub] = c;
        }
    }
    size_t need = std::max<size_t>(all.size(), 1);
    for (olc_u32 f = 0; f < F; ++f) need = std::max(need, fl[f].size());
    OLC_TRY(pool_grow_tiles(s, need, st));
    auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
    const size_t n_desc = sizeof(OlcSimDesc) * s->n_sims;
    const size_t n_steps = sizeof(FieldStep) * s->bsteps_host.size();
    const size_t n_params = s->params_all.size();
    const size_t n_maps = sizeof(CUtensorMap) * s->bmaps_host.size();
    size_t off = 0;
    const size_t o_desc = off;
    off = al(off + n_desc);
    const size_t o_steps = off;
    off = al(off + n_steps);
    const size_t o_params = off;
    off = al(off + n_params);
    const size_t o_all = off;
    off = al(off + all.size() * sizeof(uint4));
    const size_t o_chunks = off;
    off = al(off + chunks.size() * sizeof(uint2));
    const size_t o_maps = off;
    off = al(off + n_maps);
    size_t o_f[OLC_MAX_FIELDS] = {};
    for (olc_u32 f = 0; f < F; ++f) {
        o_f[f] = off;
        off = al(off + fl[f].size() * sizeof(uint4));
    }
    const int i = s->stage_i;
    if (s->stage_ev[i]) OLC_TRY(check(s, cudaEventSynchronize(s->stage_ev[i]), "staging reuse"));
    if (s->stage_cap[i] < off) {
        if (s->stage_host[i]) cudaFreeHost(s->stage_host[i]);
        s->stage_host[i] = nullptr;
        s->stage_cap[i] = 0;
        const size_t cap = off + off / 2;
        OLC_TRY(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->stage_host[i]), cap), "pinned staging"));
        s->stage_cap[i] = cap;
    }
    unsigned char* h = s->stage_host[i];
    std::memcpy(h + o_desc, s->desc_host.data(), n_desc);
    std::memcpy(h + o_steps, s->bsteps_host.data(), n_steps);
    if (n_params) std::memcpy(h + o_params, s->params_all.data(), n_params);
    if (!all.empty()) std::memcpy(h + o_all, all.data(), all.size() * sizeof(uint4));
    if (!chunks.empty()) std::memcpy(h + o_chunks, chunks.data(), chunks.size() * sizeof(uint2));
    if (n_maps) std::memcpy(h + o_maps, s->bmaps_host.data(), n_maps);
    for (olc_u32 f = 0; f < F; ++f)
        if (!fl[f].empty()) std::memcpy(h + o_f[f], fl[f].data(), fl[f].size() * sizeof(uint4));
    auto up = [&](void* dst, size_t o, size_t n, const char* what) {
        return n ? check(s, cudaMemcpyAsync(dst, h + o, n, cudaMemcpyHostToDevice, st), what) : OLC_OK;
    };
    OLC_TRY(up(s->desc_dev, o_desc, n_desc, "upload member records"));
    OLC_TRY(up(s->bsteps_dev, o_steps, n_steps, "upload field steps"));
    OLC_TRY(up(s->params_dev, o_params, n_params, "upload params"));
    OLC_TRY(up(s->btiles_all, o_all, all.size() * sizeof(uint4), "upload field tiles"));
    OLC_TRY(up(s->table_chunks, o_chunks, chunks.size() * sizeof(uint2), "upload bin-table chunks"));
    OLC_TRY(up(s->bmaps_dev, o_maps, n_maps, "upload tensor maps"));
    for (olc_u32 f = 0; f < F; ++f)
        if (s->field_bound[f]) OLC_TRY(up(s->btiles_field[f], o_f[f], fl[f].size() * sizeof(uint4), "upload tiles"));
    if (!s->stage_ev[i])
        OLC_TRY(check(s, cudaEventCreateWithFlags(&s->stage_ev[i], cudaEventDisableTiming), "staging event"));
    OLC_TRY(check(s, cudaEventRecord(s->stage_ev[i], st), "staging event"));
    s->stage_i ^= 1;
    s->n_btiles = (olc_u32)all.size();
    s->n_table_chunks = (olc_u32)chunks.size();
    for (olc_u32 f = 0; f < F; ++f) s->btile_count[f] = counts[f];
    drop_graphs_nosync(s);
    s->pool_dirty = false;
    return OLC_OK;
}

}  // namespace

extern "C" {

const char* olc_version(void) { return "oncolytica_b200 libolc 0.1 (sm_100a)"; }

const char* olc_last_error(const OlcSim* sim) {
    if (sim) return sim->err.c_str();
    return get_error();
}

}  // extern "C"

namespace {

bool caps_ok(const OlcCaps* caps, const char* who, std::string* err) {
    if (caps->max_agents == 0 || caps->max_agents > (1u << 30)) {
        *err = std::string(who) + ": max_agents must be in [1, 2^30]";
        return false;
    }
    if (caps->n_agent_fields < 3 || caps->n_agent_fields > OLC_MAX_AGENT_FIELDS) {
        *err = std::string(who) + ": n_agent_fields must be in [3, 64] (pos.x/y/z first)";
        return false;
    }
    if (caps->n_fields > OLC_MAX_FIELDS) {
        *err = std::string(who) + ": too many fields";
        return false;
    }
    if (caps->state_field >= (int)caps->n_agent_fields) {
        *err = std::string(who) + ": state_field out of range";
        return false;
    }
    return true;
}

// Allocates the library-owned buffers of a handle whose geometry fields
// (geom, caps, bins, key_bits, n_table) are set.
int alloc_common(OlcSim* s) {
    const olc_u32 cap = s->caps.max_agents;
    int rc = OLC_OK;
    auto A = [&](int r) {
        if (rc == OLC_OK) rc = r;
    };
    A(ensure_context(s));
    A(dev_alloc(s, &s->counters, OLC_CTR_WORDS * 4, "counters"));
    A(dev_alloc(s, &s->life, cap, "life"));
    A(dev_alloc(s, &s->keys_in, (size_t)cap * 4, "keys_in"));
    A(dev_alloc(s, &s->keys, (size_t)cap * 4, "keys"));
    A(dev_alloc(s, &s->vals, (size_t)cap * 4, "vals"));
    const size_t sbytes = sort_scratch_bytes(cap, s->key_bits);
    A(dev_alloc(s, &s->sort_mem, sbytes, "sort scratch"));
    A(dev_alloc(s, &s->ranges, (size_t)s->n_table * 8, "bin table"));
    A(dev_alloc(s, &s->posr, (size_t)cap * sizeof(float4), "posr"));
    s->rule_tiles = (cap + OLC_RULE_THREADS - 1) / OLC_RULE_THREADS;
    A(dev_alloc(s, &s->birth_lb, (size_t)OLC_MAX_RULES * s->rule_tiles * 4, "birth look-back"));
    A(dev_alloc(s, &s->red_dev, sizeof(OlcReductions), "reductions"));
    A(dev_alloc(s, &s->red_scratch.partials, RED_PARTIALS * sizeof(double), "reduction partials"));
    A(dev_alloc(s, &s->red_scratch.tickets, RED_TICKETS * sizeof(olc_u32), "reduction tickets"));
    A(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->red_host), sizeof(OlcReductions)), "pinned reductions"));
    A(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->ctr_host_words), OLC_CTR_WORDS * 4), "pinned counters"));
    if (rc == OLC_OK && !carve_sort_scratch(s->sort_mem, sbytes, cap, s->key_bits, &s->sc))
        rc = fail(s, OLC_ERR_STATE, "sort scratch layout");
    if (rc == OLC_OK) {
        A(check(s, cudaMemset(s->counters, 0, OLC_CTR_WORDS * 4), "memset counters"));
        A(check(s, cudaMemset(s->life, 0, cap), "memset life"));
        A(check(s, cudaMemset(s->red_dev, 0, sizeof(OlcReductions)), "memset reductions"));
        A(check(s, cudaMemset(s->red_scratch.tickets, 0, RED_TICKETS * sizeof(olc_u32)), "memset tickets"));
    }
    return rc;
}

}  // namespace

extern "C" {

int olc_create(const OlcGeom* geom, const OlcCaps* caps, OlcSim** out) {
    if (!geom || !caps || !out) return fail(nullptr, OLC_ERR_ARG, "olc_create: null argument");
    std::string err;
    if (!geom_ok(*geom, &err)) return fail(nullptr, OLC_ERR_ARG, "olc_create: " + err);
    if (!caps_ok(caps, "olc_create", &err)) return fail(nullptr, OLC_ERR_ARG, err);
    OlcSim* s = new OlcSim();
    s->geom = *geom;
    s->caps = *caps;
    s->bins = make_bin_grid(*geom);
    s->key_bits = key_bits_for(s->bins.sentinel);
    s->n_table = s->bins.sentinel + 1u;
    const int rc = alloc_common(s);
    if (rc != OLC_OK) {
        std::string msg = s->err;
        olc_destroy(s);
        return fail(nullptr, rc, msg);
    }
    *out = s;
    return OLC_OK;
}

int olc_create_batch(const OlcGeom* geoms, int n_sims, const OlcCaps* caps, OlcSim** out) {
    if (!geoms || !caps || !out || n_sims < 1) return fail(nullptr, OLC_ERR_ARG, "olc_create_batch: bad arguments");
    std::string err;
    if (!caps_ok(caps, "olc_create_batch", &err)) return fail(nullptr, OLC_ERR_ARG, err);
    int shift = 1;
    olc_u64 n_table = 0, voxels = 0;
    for (int k = 0; k < n_sims; ++k) {
        if (!geom_ok(geoms[k], &err))
            return fail(nullptr, OLC_ERR_ARG, "olc_create_batch: simulation " + std::to_string(k) + ": " + err);
        const olc_u32 top = olc_tissue_key(geoms[k].tissue_dims[0], geoms[k].tissue_dims[1], geoms[k].tissue_dims[2]);
        shift = std::max(shift, key_bits_for(top));
        n_table += (olc_u64)top + 1u;
        voxels += (olc_u64)geoms[k].chem_dims[0] * geoms[k].chem_dims[1] * geoms[k].chem_dims[2];
    }
    if (shift + key_bits_for((olc_u32)n_sims) > 32)
        return fail(nullptr, OLC_ERR_ARG, "olc_create_batch: simulation index and bin key exceed 32 key bits");
    if (n_table >= (1ull << 31)) return fail(nullptr, OLC_ERR_ARG, "olc_create_batch: bin tables too large");
    OlcSim* s = new OlcSim();
    s->geom = geoms[0];
    s->caps = *caps;
    s->n_sims = (olc_u32)n_sims;
    s->geoms.assign(geoms, geoms + n_sims);
    s->bins = make_bin_grid(geoms[0]);
    s->bargs.shift = shift;
    s->bargs.n_sims = (olc_u32)n_sims;
    s->bargs.sentinel = (olc_u32)n_sims << shift;
    s->key_bits = key_bits_for(s->bargs.sentinel);
    s->n_table = (olc_u32)n_table;
    // per-simulation records, bin-table bases, field offsets, field tiles
    s->desc_host.resize(n_sims);
    s->field_off.assign(n_sims + 1, 0ull);
    std::vector<uint4> tiles;
    olc_u64 base = 0;
    for (int k = 0; k < n_sims; ++k) {
        const OlcGeom& g = geoms[k];
        OlcSimDesc& d = s->desc_host[k];
        std::memset(&d, 0, sizeof(d));
        for (int i = 0; i < 3; ++i) {
            d.tdims[i] = g.tissue_dims[i];
            d.cdims[i] = g.chem_dims[i];
            d.lo[i] = g.domain_lo[i];
            d.hi[i] = g.domain_hi[i];
            d.center[i] = 0.5f * (g.domain_lo[i] + g.domain_hi[i]);
        }
        d.tvs = g.tissue_voxel_size;
        d.cvs = g.chem_voxel_size;
        d.bin_width = caps->radial_bin_width > 0.0f ? caps->radial_bin_width : 1.0f;
        d.ranges_base = (olc_u32)base;
        base += (olc_u64)olc_tissue_key(g.tissue_dims[0], g.tissue_dims[1], g.tissue_dims[2]) + 1u;
        d.field_off = s->field_off[k];
        s->field_off[k + 1] = s->field_off[k] + (olc_u64)g.chem_dims[0] * g.chem_dims[1] * g.chem_dims[2];
        const int tx = (g.chem_dims[0] + BATCH_TILE_X - 1) / BATCH_TILE_X;
        const int ty = (g.chem_dims[1] + BATCH_TILE_Y - 1) / BATCH_TILE_Y;
        const int tz = (g.chem_dims[2] + BATCH_TILE_Z - 1) / BATCH_TILE_Z;
        for (int z = 0; z < tz; ++z)
            for (int y = 0; y < ty; ++y)
                for (int x = 0; x < tx; ++x) tiles.push_back(make_uint4((unsigned)k, (unsigned)x, (unsigned)y, (unsigned)z));
    }
    s->n_btiles = (olc_u32)tiles.size();
    s->bsteps_host.assign((size_t)n_sims * std::max<olc_u32>(1u, caps->n_fields), FieldStep{});
    int rc = alloc_common(s);
    auto A = [&](int r) {
        if (rc == OLC_OK) rc = r;
    };
    A(dev_alloc(s, &s->desc_dev, sizeof(OlcSimDesc) * n_sims, "simulation records"));
    A(dev_alloc(s, &s->cols_dev, sizeof(void*) * 2 * OLC_MAX_AGENT_COLS, "column tables"));
    A(dev_alloc(s, &s->fpar_dev, (size_t)n_sims * OLC_MAX_FIELDS, "field parity"));
    A(dev_alloc(s, &s->bsteps_dev, sizeof(FieldStep) * s->bsteps_host.size(), "field steps"));
    A(dev_alloc(s, &s->btiles_all, sizeof(uint4) * tiles.size(), "field tiles"));
    A(dev_alloc(s, &s->red_batch_dev, sizeof(OlcReductions) * n_sims, "batch reductions"));
    s->bmaps_host.assign((size_t)n_sims * std::max<olc_u32>(1u, caps->n_fields) * 2, CUtensorMap{});
    A(dev_alloc(s, &s->bmaps_dev, sizeof(CUtensorMap) * s->bmaps_host.size(), "tensor maps"));
    A(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->red_batch_host), sizeof(OlcReductions) * n_sims),
            "pinned batch reductions"));
    if (rc == OLC_OK) {
        A(check(s, cudaMemcpy(s->desc_dev, s->desc_host.data(), sizeof(OlcSimDesc) * n_sims, cudaMemcpyHostToDevice),
                "upload simulation records"));
        A(check(s, cudaMemcpy(s->btiles_all, tiles.data(), sizeof(uint4) * tiles.size(), cudaMemcpyHostToDevice),
                "upload field tiles"));
        A(check(s, cudaMemset(s->fpar_dev, 0, (size_t)n_sims * OLC_MAX_FIELDS), "memset field parity"));
        A(check(s, cudaMemset(s->bsteps_dev, 0, sizeof(FieldStep) * s->bsteps_host.size()), "memset field steps"));
        A(check(s, cudaMemset(s->red_batch_dev, 0, sizeof(OlcReductions) * n_sims), "memset batch reductions"));
    }
    s->bargs.sims = s->desc_dev;
    if (rc != OLC_OK) {
        std::string msg = s->err;
        olc_destroy(s);
        return fail(nullptr, rc, msg);
    }
    *out = s;
    return OLC_OK;
}

int olc_batch_field_offsets(const OlcSim* s, uint64_t* offsets) {
    if (!s || !offsets) return fail(nullptr, OLC_ERR_ARG, "olc_batch_field_offsets: null argument");
    if (!s->n_sims || s->pool)
        return fail(const_cast<OlcSim*>(s), OLC_ERR_STATE, "olc_batch_field_offsets: not a batch handle");
    for (olc_u32 k = 0; k <= s->n_sims; ++k) offsets[k] = s->field_off[k];
    return OLC_OK;
}

int olc_destroy(OlcSim* s) {
    if (!s) return OLC_OK;
    cudaDeviceSynchronize();
    drop_graphs(s);
    if (s->capture_stream) cudaStreamDestroy(s->capture_stream);
    if (s->module) cudaLibraryUnload(s->module);
    for (auto& ev : s->events)
        for (auto e : ev) cudaEventDestroy(e);
    cudaFree(s->counters);
    cudaFree(s->life);
    cudaFree(s->keys_in);
    cudaFree(s->keys);
    cudaFree(s->vals);
    cudaFree(s->sort_mem);
    cudaFree(s->ranges);
    cudaFree(s->posr);
    cudaFree(s->birth_lb);
    cudaFree(s->params_dev);
    cudaFree(s->red_dev);
    cudaFree(s->red_scratch.partials);
    cudaFree(s->red_scratch.tickets);
    cudaFree(s->desc_dev);
    cudaFree(s->cols_dev);
    cudaFree(s->fpar_dev);
    cudaFree(s->bsteps_dev);
    cudaFree(s->btiles_all);
    for (int f = 0; f < OLC_MAX_FIELDS; ++f) cudaFree(s->btiles_field[f]);
    cudaFree(s->red_batch_dev);
    if (s->red_batch_host) cudaFreeHost(s->red_batch_host);
    cudaFree(s->gather_counts);
    cudaFree(s->bmaps_dev);
    cudaFree(s->table_chunks);
    for (int i = 0; i < 2; ++i) {
        if (s->stage_host[i]) cudaFreeHost(s->stage_host[i]);
        if (s->stage_ev[i]) cudaEventDestroy(s->stage_ev[i]);
    }
    cudaFree(s->metrics_dev);
    if (s->params_host) cudaFreeHost(s->params_host);
    if (s->rb_host) cudaFreeHost(s->rb_host);
    for (int i = 0; i < HOST_SLOTS; ++i) {
        if (s->param_ev[i]) cudaEventDestroy(s->param_ev[i]);
        if (s->rb_ev[i]) cudaEventDestroy(s->rb_ev[i]);
    }
    if (s->red_host) cudaFreeHost(s->red_host);
    if (s->ctr_host_words) cudaFreeHost(s->ctr_host_words);
    cudaFree(s->em_acc);
    cudaFree(s->em_partials);
    if (s->em_host) cudaFreeHost(s->em_host);
    delete s;
    return OLC_OK;
}

int olc_bind_agent_column(OlcSim* s, int index, void* a, void* b) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (index < 0 || index >= (int)s->caps.n_agent_fields || !a || !b)
        return fail(s, OLC_ERR_ARG, "olc_bind_agent_column: bad index or null buffer");
    drop_graphs(s);
    s->col[0][index] = a;
    s->col[1][index] = b;
    s->cols_dirty = true;
    return OLC_OK;
}

int olc_bind_field(OlcSim* s, int index, float* a, float* b, float* sink, const OlcDiffusion* spec) {
    if (spec && spec->storage != OLC_FIELD_F32)
        return fail(s, OLC_ERR_ARG, "olc_bind_field: 16-bit storage needs olc_bind_field_ex (compensation buffer)");
    return olc_bind_field_ex(s, index, a, b, sink, nullptr, spec);
}

int olc_bind_field_ex(OlcSim* s, int index, void* a_, void* b_, float* sink, float* comp, const OlcDiffusion* spec) {
    float* a = static_cast<float*>(a_);
    float* b = static_cast<float*>(b_);
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (index < 0 || index >= (int)s->caps.n_fields || !a || !b || !spec)
        return fail(s, OLC_ERR_ARG, "olc_bind_field: bad index or null argument");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_bind_field: batch handle (use olc_bind_field_batch)");
    std::string err;
    FieldStep fs = {};
    if (spec->substeps != 0 &&
        !make_field_step(*spec, s->geom.chem_dims, s->geom.chem_voxel_size, s->caps.dt, &fs, &err))
        return fail(s, OLC_ERR_ARG, "olc_bind_field: " + err);
    if (spec->substeps == 0) {
        if (spec->storage < OLC_FIELD_F32 || spec->storage > OLC_FIELD_F16_SR)
            return fail(s, OLC_ERR_ARG, "olc_bind_field: bad storage type");
        if (spec->encoding < OLC_ENC_VALUE || spec->encoding > OLC_ENC_OFFSET3 ||
            (spec->encoding != OLC_ENC_VALUE && spec->storage == OLC_FIELD_F32))
            return fail(s, OLC_ERR_ARG, "olc_bind_field: bad encoding (encodings apply to 16-bit storage only)");
        fs.storage = spec->storage;
        fs.encoding = spec->encoding;
        fs.bval = spec->boundary;
    }
    if (spec->has_sink && !sink) return fail(s, OLC_ERR_ARG, "olc_bind_field: has_sink without a sink buffer");
    const bool half = fs.storage != OLC_FIELD_F32;
    if (half && spec->substeps != 0 && !comp)
        return fail(s, OLC_ERR_ARG, "olc_bind_field_ex: 16-bit storage needs a compensation buffer");
    drop_graphs(s);
    s->field[0][index] = a;
    s->field[1][index] = b;
    s->fmaps[index].ok = false;
    s->fmaps16[index].ok = false;
    if (spec->substeps > 0 && !half)
        make_field_maps(&s->fmaps[index], a, b, s->geom.chem_dims, s->tuning.stencil_tile_y, s->tuning.stencil_tile_z,
                        s->tuning.stencil_pair_threads, s->tuning.stencil_pair_planes, s->tuning.stencil_l2_keep_pct);
    if (spec->substeps > 0 && half && !make_field_maps16(&s->fmaps16[index], a, b, s->geom.chem_dims))
        return fail(s, OLC_ERR_ARG, "olc_bind_field_ex: TMA descriptors of the 16-bit field failed (16-byte aligned "
                                    "buffers, x extent a multiple of 8)");
    s->comp[index] = half ? comp : nullptr;
    s->sink[index] = spec->has_sink ? sink : nullptr;
    s->fspec[index] = *spec;
    s->fstep[index] = fs;
    s->field_cur[index] = 0;
    s->field_bound[index] = true;
    return OLC_OK;
}

int olc_bind_tissue(OlcSim* s, const void* cols, int n_cols, size_t stride_bytes) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (n_cols < 0 || (n_cols > 0 && (!cols || stride_bytes < (size_t)s->n_table * 4)))
        return fail(s, OLC_ERR_ARG, "olc_bind_tissue: columns must hold voxel_table_size entries");
    if (s->n_sims && n_cols > 0) return fail(s, OLC_ERR_STATE, "olc_bind_tissue: tissue grids are not bound in batched mode");
    drop_graphs(s);
    s->tissue = static_cast<const unsigned char*>(cols);
    s->tissue_buf[0] = s->tissue_buf[1] = nullptr;
    s->tissue_cur = 0;
    s->tissue_cols = n_cols;
    s->tissue_stride = stride_bytes;
    return OLC_OK;
}

int olc_set_pinned(OlcSim* s, int index, const uint32_t* idx_dev, uint32_t n, float value) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_set_pinned: solo handles only");
    if (index < 0 || index >= (int)s->caps.n_fields || !s->field_bound[index])
        return fail(s, OLC_ERR_ARG, "olc_set_pinned: field not bound");
    if (n && !idx_dev) return fail(s, OLC_ERR_ARG, "olc_set_pinned: null index list");
    if (n && s->fstep[index].storage != OLC_FIELD_F32)
        return fail(s, OLC_ERR_ARG, "olc_set_pinned: FP32 fields only");
    drop_graphs(s);
    s->pins[index].idx = idx_dev;
    s->pins[index].n = n;
    s->pins[index].value = value;
    return OLC_OK;
}

int olc_bind_tissue_pair(OlcSim* s, void* a, void* b, int n_cols, size_t stride_bytes) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (n_cols <= 0 || !a || !b || stride_bytes < (size_t)s->n_table * 4)
        return fail(s, OLC_ERR_ARG, "olc_bind_tissue_pair: two buffers of columns with voxel_table_size entries");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_bind_tissue_pair: tissue grids are not bound in batched mode");
    drop_graphs(s);
    s->tissue_buf[0] = static_cast<unsigned char*>(a);
    s->tissue_buf[1] = static_cast<unsigned char*>(b);
    s->tissue_cur = 0;
    s->tissue = s->tissue_buf[0];
    s->tissue_cols = n_cols;
    s->tissue_stride = stride_bytes;
    return OLC_OK;
}

int olc_current_tissue(const OlcSim* s, int* tissue_buf) {
    if (!s || !tissue_buf) return fail(nullptr, OLC_ERR_ARG, "olc_current_tissue: null argument");
    *tissue_buf = s->tissue_cur;
    return OLC_OK;
}

int olc_set_rule_iterations(OlcSim* s, const int* iters, int n) {
    if (!s || (n > 0 && !iters)) return fail(s, OLC_ERR_ARG, "olc_set_rule_iterations: null argument");
    if (n != (int)s->funcs.size()) return fail(s, OLC_ERR_ARG, "olc_set_rule_iterations: one count per kernel");
    for (int i = 0; i < n; ++i)
        if (iters[i] < 0) return fail(s, OLC_ERR_ARG, "olc_set_rule_iterations: negative count");
    drop_graphs(s);
    s->iters.assign(iters, iters + n);
    return OLC_OK;
}

int olc_set_mechanics(OlcSim* s, const OlcMechanics* m) {
    if (!s || !m) return fail(s, OLC_ERR_ARG, "olc_set_mechanics: null argument");
    if (s->n_sims && m->enabled) return fail(s, OLC_ERR_STATE, "olc_set_mechanics: solo handles only");
    const int nc = (int)s->caps.n_agent_fields;
    if (m->enabled) {
        if (m->state_field >= nc || m->velocity_field + 3 > nc)
            return fail(s, OLC_ERR_ARG, "olc_set_mechanics: column out of range");
        if (m->adhesion_stiffness != 0.0f && !(m->adhesion_range > 0.0f))
            return fail(s, OLC_ERR_ARG, "olc_set_mechanics: adhesion needs adhesion_range > 0");
        if (m->velocity_field >= 0 && !(m->max_speed > 0.0f))
            return fail(s, OLC_ERR_ARG, "olc_set_mechanics: velocity integration needs max_speed > 0");
        if (m->n_species < 0 || m->n_species > OLC_MAX_SPECIES)
            return fail(s, OLC_ERR_ARG, "olc_set_mechanics: n_species must be in [0, OLC_MAX_SPECIES]");
        if (m->n_species > 0) {
            if (m->species_field >= nc || m->rng_field >= nc)
                return fail(s, OLC_ERR_ARG, "olc_set_mechanics: species or RNG column out of range");
            for (int f : {m->o2_field, m->glucose_field})
                if (f >= (int)s->caps.n_fields || (f >= 0 && !s->field_bound[f]))
                    return fail(s, OLC_ERR_ARG, "olc_set_mechanics: chemotactic field not bound");
        }
    }
    drop_graphs(s);
    s->mech = *m;
    return OLC_OK;
}

int olc_set_contact(OlcSim* s, const OlcContact* c) {
    if (!s || !c) return fail(s, OLC_ERR_ARG, "olc_set_contact: null argument");
    if (c->enabled && (c->radius_field >= (int)s->caps.n_agent_fields))
        return fail(s, OLC_ERR_ARG, "olc_set_contact: radius_field out of range");
    drop_graphs(s);
    s->contact = *c;
    ContactDev& d = s->contact_dev;
    for (int i = 0; i < 3; ++i) {
        d.tdims[i] = s->geom.tissue_dims[i];
        d.lo[i] = s->geom.domain_lo[i] + c->margin;
        d.hi[i] = s->geom.domain_hi[i] - c->margin;
    }
    d.tvs = s->geom.tissue_voxel_size;
    d.stiffness = c->stiffness;
    d.mobility = c->mobility;
    d.max_disp = c->max_disp;
    d.dt = s->caps.dt;
    if (s->n_sims) {
        for (olc_u32 k = 0; k < s->n_sims; ++k)
            for (int i = 0; i < 3; ++i) {
                s->desc_host[k].lo[i] = s->geoms[k].domain_lo[i] + c->margin;
                s->desc_host[k].hi[i] = s->geoms[k].domain_hi[i] - c->margin;
            }
        if (s->pool) {
            s->pool_dirty = true;
            return OLC_OK;
        }
        return upload_desc(s);
    }
    return OLC_OK;
}

static int nvrtc_compile(const char* src, const char* include_dir, std::vector<char>* cubin, std::string* log) {
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src, "olc_rules.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        *log = "nvrtcCreateProgram failed";
        return OLC_ERR_NVRTC;
    }
    std::string inc = std::string("-I") + (include_dir ? include_dir : ".");
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=false", "-lineinfo",
                          "--device-as-default-execution-space", inc.c_str()};
    nvrtcResult r = nvrtcCompileProgram(prog, (int)(sizeof(opts) / sizeof(opts[0])), opts);
    size_t log_size = 0;
    nvrtcGetProgramLogSize(prog, &log_size);
    log->assign(log_size, '\0');
    if (log_size > 1) nvrtcGetProgramLog(prog, &(*log)[0]);
    if (r != NVRTC_SUCCESS) {
        *log = std::string("NVRTC: ") + nvrtcGetErrorString(r) + "\n" + *log;
        nvrtcDestroyProgram(&prog);
        return OLC_ERR_NVRTC;
    }
    if (cubin) {
        size_t cubin_size = 0;
        nvrtcGetCUBINSize(prog, &cubin_size);
        cubin->resize(cubin_size);
        nvrtcGetCUBIN(prog, cubin->data());
    }
    nvrtcDestroyProgram(&prog);
    return OLC_OK;
}

int olc_nvrtc_check(const char* src, const char* include_dir, char* log, size_t log_size) {
    if (!src) return fail(nullptr, OLC_ERR_ARG, "olc_nvrtc_check: null source");
    std::string msg;
    int rc = nvrtc_compile(src, include_dir, nullptr, &msg);
    if (log && log_size) {
        size_t k = msg.size() < log_size - 1 ? msg.size() : log_size - 1;
        std::memcpy(log, msg.data(), k);
        log[k] = '\0';
    }
    if (rc != OLC_OK) set_error(msg);
    return rc;
}

int olc_set_rule_source(OlcSim* s, const char* src, const char* const* kernels, const int* kinds, int n,
                        const char* include_dir) {
    if (!s || !src || (n > 0 && (!kernels || !kinds)) || n < 0 || n > OLC_MAX_RULES)
        return fail(s, OLC_ERR_ARG, "olc_set_rule_source: bad arguments");
    int ncell = 0;
    for (int i = 0; i < n; ++i) {
        if (kinds[i] < 0 || kinds[i] > 3) return fail(s, OLC_ERR_ARG, "olc_set_rule_source: kind must be 0..3");
        if (kinds[i] == 2 && s->n_sims)
            return fail(s, OLC_ERR_STATE, "olc_set_rule_source: tissue rules need a solo handle");
        ncell += kinds[i] == 0;
    }
    OLC_TRY(ensure_context(s));
    // Compiled modules are cached in the process by their source and include
    // directory (the runtime headers there do not change while it runs), so
    // engines of one model compile once; each handle still loads its own copy.
    static std::mutex cache_mu;
    static std::map<std::string, std::vector<char>> cache;
    std::string key = std::string(include_dir ? include_dir : "") + '\n' + src;
    std::vector<char> cubin;
    {
        std::lock_guard<std::mutex> lk(cache_mu);
        auto it = cache.find(key);
        if (it != cache.end()) cubin = it->second;
    }
    if (cubin.empty()) {
        std::string log;
        if (nvrtc_compile(src, include_dir, &cubin, &log) != OLC_OK) return fail(s, OLC_ERR_NVRTC, log);
        std::lock_guard<std::mutex> lk(cache_mu);
        if (cache.size() >= 64) cache.clear();
        cache.emplace(std::move(key), cubin);
    }
    drop_graphs(s);
    if (s->module) {
        cudaDeviceSynchronize();
        cudaLibraryUnload(s->module);
        s->module = nullptr;
    }
    s->funcs.clear();
    s->kinds.clear();
    s->iters.clear();
    OLC_TRY(check(s, cudaLibraryLoadData(&s->module, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0),
                  "cudaLibraryLoadData"));
    for (int i = 0; i < n; ++i) {
        cudaKernel_t fn;
        OLC_TRY(check(s, cudaLibraryGetKernel(&fn, s->module, kernels[i]), kernels[i]));
        s->funcs.push_back(fn);
        s->kinds.push_back(kinds[i]);
        s->iters.push_back(1);
    }
    s->n_cell_rules = ncell;
    return OLC_OK;
}

int olc_set_params(OlcSim* s, const void* blob, size_t bytes, void* stream) {
    if (!s || (bytes && !blob)) return fail(s, OLC_ERR_ARG, "olc_set_params: bad arguments");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_set_params: batch handle (use olc_set_params_batch)");
    if (bytes == 0) return OLC_OK;
    cudaStream_t st = as_stream(stream);
    if (bytes > s->params_cap) {
        drop_graphs(s);
        OLC_TRY(check(s, cudaStreamSynchronize(st), "sync before params reallocation"));
        cudaFree(s->params_dev);
        if (s->params_host) cudaFreeHost(s->params_host);
        s->params_dev = nullptr;
        s->params_host = nullptr;
        size_t cap = (bytes + 255) & ~size_t(255);
        OLC_TRY(dev_alloc(s, &s->params_dev, cap, "params"));
        OLC_TRY(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->params_host), cap * HOST_SLOTS),
                      "pinned params"));
        s->params_cap = cap;
    }
    // the slot's previous copy was queued HOST_SLOTS uploads ago: wait for it
    // (normally long done) instead of for the whole stream
    const int slot = (int)(s->param_seq % HOST_SLOTS);
    if (s->param_ev[slot]) OLC_TRY(check(s, cudaEventSynchronize(s->param_ev[slot]), "params staging reuse"));
    else OLC_TRY(check(s, cudaEventCreateWithFlags(&s->param_ev[slot], cudaEventDisableTiming), "params event"));
    unsigned char* h = s->params_host + (size_t)slot * s->params_cap;
    std::memcpy(h, blob, bytes);
    OLC_TRY(check(s, cudaMemcpyAsync(s->params_dev, h, bytes, cudaMemcpyHostToDevice, st), "params upload"));
    OLC_TRY(check(s, cudaEventRecord(s->param_ev[slot], st), "params event"));
    s->param_seq++;
    return OLC_OK;
}

int olc_set_user_metrics_size(OlcSim* s, size_t bytes) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    drop_graphs(s);
    cudaFree(s->metrics_dev);
    s->metrics_dev = nullptr;
    s->metrics_bytes = bytes;
    const size_t copies = s->n_sims ? s->n_sims : 1;  // one accumulator block per simulation
    if (bytes) {
        OLC_TRY(dev_alloc(s, &s->metrics_dev, bytes * copies, "metrics"));
        OLC_TRY(check(s, cudaMemset(s->metrics_dev, 0, bytes * copies), "memset metrics"));
    }
    if (s->n_sims) {
        for (olc_u32 k = 0; k < s->n_sims; ++k) s->desc_host[k].metrics_off = (olc_u32)(k * bytes);
        if (s->pool) {
            s->pool_dirty = true;
            return OLC_OK;
        }
        return upload_desc(s);
    }
    return OLC_OK;
}

int olc_set_agent_count(OlcSim* s, uint32_t n, void* stream) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (s->pool) return fail(s, OLC_ERR_STATE, "olc_set_agent_count: pools add rows with olc_pool_add_agents");
    if (n > s->caps.max_agents) return fail(s, OLC_ERR_CAPACITY, "olc_set_agent_count: n exceeds max_agents");
    for (olc_u32 c = 0; c < s->caps.n_agent_fields; ++c)
        if (!s->col[0][c]) return fail(s, OLC_ERR_STATE, "olc_set_agent_count: agent column not bound");
    cudaStream_t st = as_stream(stream);
    olc_u32 words[OLC_CTR_WORDS];
    std::memset(words, 0, sizeof(words));
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync"));
    OLC_TRY(check(s, cudaMemcpy(words, s->counters, sizeof(words), cudaMemcpyDeviceToHost), "read counters"));
    const olc_u32 status = words[OLC_CTR_STATUS];
    const olc_u32 as_lo = words[OLC_CTR_AGENT_STEPS], as_hi = words[OLC_CTR_AGENT_STEPS + 1];
    const olc_u32 fstep = words[OLC_CTR_FIELD_STEP];
    std::memset(words, 0, sizeof(words));
    words[OLC_CTR_FIELD_STEP] = fstep;
    words[OLC_CTR_N] = n;
    words[OLC_CTR_ROWS] = n;
    words[OLC_CTR_STATUS] = status;
    words[OLC_CTR_AGENT_STEPS] = as_lo;
    words[OLC_CTR_AGENT_STEPS + 1] = as_hi;
    OLC_TRY(check(s, cudaMemcpy(s->counters, words, sizeof(words), cudaMemcpyHostToDevice), "write counters"));
    OLC_TRY(check(s, cudaMemset(s->life, 0, s->caps.max_agents), "memset life"));
    return OLC_OK;
}

int olc_get_step_state(OlcSim* s, OlcStepState* out, void* stream) {
    if (!s || !out) return fail(s, OLC_ERR_ARG, "olc_get_step_state: null argument");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_get_step_state: batch handle");
    cudaStream_t st = as_stream(stream);
    OLC_TRY(check(s, cudaMemcpyAsync(s->ctr_host_words, s->counters, OLC_CTR_WORDS * 4, cudaMemcpyDeviceToHost, st),
                  "counters readback"));
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync"));
    const olc_u32* w = s->ctr_host_words;
    out->steps = s->steps;
    out->agent_steps = (uint64_t)w[OLC_CTR_AGENT_STEPS] | ((uint64_t)w[OLC_CTR_AGENT_STEPS + 1] << 32);
    out->field_step = w[OLC_CTR_FIELD_STEP];
    out->status = w[OLC_CTR_STATUS];
    return OLC_OK;
}

int olc_set_step_state(OlcSim* s, const OlcStepState* in, void* stream) {
    if (!s || !in) return fail(s, OLC_ERR_ARG, "olc_set_step_state: null argument");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_set_step_state: batch handle");
    cudaStream_t st = as_stream(stream);
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync"));
    olc_u32 w[OLC_CTR_WORDS];
    OLC_TRY(check(s, cudaMemcpy(w, s->counters, sizeof(w), cudaMemcpyDeviceToHost), "read counters"));
    w[OLC_CTR_AGENT_STEPS] = (olc_u32)(in->agent_steps & 0xffffffffu);
    w[OLC_CTR_AGENT_STEPS + 1] = (olc_u32)(in->agent_steps >> 32);
    w[OLC_CTR_FIELD_STEP] = in->field_step;
    w[OLC_CTR_STATUS] = in->status;
    OLC_TRY(check(s, cudaMemcpy(s->counters, w, sizeof(w), cudaMemcpyHostToDevice), "write counters"));
    s->steps = in->steps;  // host count only; kernels read the device counters
    return OLC_OK;
}

int olc_current_buffers(const OlcSim* s, int* agent_buf, int* field_buf) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (agent_buf) *agent_buf = s->agent_cur;
    if (field_buf) {
        int m = 0;
        for (int f = 0; f < OLC_MAX_FIELDS; ++f) m |= (s->field_cur[f] & 1) << f;
        *field_buf = m;
    }
    return OLC_OK;
}

int olc_set_graphs(OlcSim* s, int enable) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    drop_graphs(s);
    s->use_graphs = enable != 0;
    return OLC_OK;
}

int olc_step(OlcSim* s, int nsteps, int collect, void* stream) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (nsteps < 0) return fail(s, OLC_ERR_ARG, "olc_step: nsteps < 0");
    for (olc_u32 c = 0; c < s->caps.n_agent_fields; ++c)
        if (!s->col[0][c]) return fail(s, OLC_ERR_STATE, "olc_step: agent column not bound");
    cudaStream_t st = as_stream(stream);
    for (int i = 0; i < nsteps; ++i) {
        const int c = (collect && i == nsteps - 1) ? 1 : 0;
        if (s->pool) {
            if (s->pool_dirty) OLC_TRY(pool_commit(s, st));
            s->pool_steps++;
        }
        if (s->use_graphs && !s->profiling) {
            OLC_TRY(step_graph(s, c, st));
        } else {
            OLC_TRY(step_any(s, c, st));
        }
    }
    return OLC_OK;
}

// OlcCounters from a copy of the device counter block.
static void counters_from_words(const olc_u32* w, uint64_t steps, OlcCounters* out) {
    olc_u32 births = 0;
    for (int j = 0; j < OLC_MAX_RULE_KERNELS; ++j) births += w[OLC_CTR_BIRTHS + j];
    out->n_agents = w[OLC_CTR_N] + births;
    out->n_total = w[OLC_CTR_N] + births;
    out->births = births;
    out->deaths = w[OLC_CTR_DEAD];
    out->status = w[OLC_CTR_STATUS];
    out->pad = 0;
    out->steps = steps;
    out->agent_steps = (uint64_t)w[OLC_CTR_AGENT_STEPS] | ((uint64_t)w[OLC_CTR_AGENT_STEPS + 1] << 32);
}

int olc_read_counters(OlcSim* s, OlcCounters* out, void* stream) {
    if (!s || !out) return fail(s, OLC_ERR_ARG, "olc_read_counters: null argument");
    cudaStream_t st = as_stream(stream);
    OLC_TRY(check(s, cudaMemcpyAsync(s->ctr_host_words, s->counters, OLC_CTR_WORDS * 4, cudaMemcpyDeviceToHost, st),
                  "counters readback"));
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync"));
    counters_from_words(s->ctr_host_words, s->steps, out);
    return OLC_OK;
}

int olc_queue_readback(OlcSim* s, void* stream, uint64_t* ticket) {
    if (!s || !ticket) return fail(s, OLC_ERR_ARG, "olc_queue_readback: null argument");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_queue_readback: batch handle");
    cudaStream_t st = as_stream(stream);
    const size_t ctr_bytes = OLC_CTR_WORDS * 4;
    const size_t stride = (ctr_bytes + s->metrics_bytes + 63) & ~size_t(63);
    if (stride != s->rb_stride) {
        // metric size changed: every queued copy lands before the ring goes
        for (int i = 0; i < HOST_SLOTS; ++i) {
            if (s->rb_ev[i]) OLC_TRY(check(s, cudaEventSynchronize(s->rb_ev[i]), "readback reuse"));
            s->rb_ticket[i] = 0;
        }
        if (s->rb_host) cudaFreeHost(s->rb_host);
        s->rb_host = nullptr;
        s->rb_stride = 0;
        OLC_TRY(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->rb_host), stride * HOST_SLOTS), "pinned readback"));
        s->rb_stride = stride;
    }
    const int slot = (int)(s->rb_next % HOST_SLOTS);
    if (s->rb_ev[slot]) OLC_TRY(check(s, cudaEventSynchronize(s->rb_ev[slot]), "readback reuse"));
    else OLC_TRY(check(s, cudaEventCreateWithFlags(&s->rb_ev[slot], cudaEventDisableTiming), "readback event"));
    unsigned char* h = s->rb_host + (size_t)slot * s->rb_stride;
    s->rb_ticket[slot] = 0;
    OLC_TRY(check(s, cudaMemcpyAsync(h, s->counters, ctr_bytes, cudaMemcpyDeviceToHost, st), "counters readback"));
    if (s->metrics_bytes)
        OLC_TRY(check(s, cudaMemcpyAsync(h + ctr_bytes, s->metrics_dev, s->metrics_bytes, cudaMemcpyDeviceToHost, st),
                      "metrics readback"));
    OLC_TRY(check(s, cudaEventRecord(s->rb_ev[slot], st), "readback event"));
    s->rb_ticket[slot] = s->rb_next;
    s->rb_steps[slot] = s->steps;
    *ticket = s->rb_next++;
    return OLC_OK;
}

int olc_take_readback(OlcSim* s, uint64_t ticket, void* metrics_out, size_t bytes, OlcCounters* counters) {
    if (!s || (bytes && !metrics_out)) return fail(s, OLC_ERR_ARG, "olc_take_readback: bad arguments");
    if (bytes > s->metrics_bytes) return fail(s, OLC_ERR_ARG, "olc_take_readback: more bytes than allocated");
    const int slot = (int)(ticket % HOST_SLOTS);
    if (ticket == 0 || s->rb_ticket[slot] != ticket)
        return fail(s, OLC_ERR_STATE, "olc_take_readback: unknown ticket, or its slot was reused by a later one");
    OLC_TRY(check(s, cudaEventSynchronize(s->rb_ev[slot]), "readback wait"));
    const unsigned char* h = s->rb_host + (size_t)slot * s->rb_stride;
    if (bytes) std::memcpy(metrics_out, h + OLC_CTR_WORDS * 4, bytes);
    if (counters) counters_from_words(reinterpret_cast<const olc_u32*>(h), s->rb_steps[slot], counters);
    return OLC_OK;
}

int olc_set_profiling(OlcSim* s, int enable) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    OLC_TRY(check(s, cudaDeviceSynchronize(), "sync"));
    s->profiling = enable != 0;
    s->prof_step = 0;
    s->prof_launches = 0;
    s->prof_substeps = 0;
    return OLC_OK;
}

int olc_read_profile(OlcSim* s, OlcProfile* out) {
    if (!s || !out) return fail(s, OLC_ERR_ARG, "olc_read_profile: null argument");
    std::memset(out, 0, sizeof(*out));
    double* slots[6] = {&out->ms_sink, &out->ms_substeps, &out->ms_grid, &out->ms_rules, &out->ms_contact,
                        &out->ms_collect};
    for (int i = 0; i < s->prof_step; ++i) {
        OLC_TRY(check(s, cudaEventSynchronize(s->events[i][OLC_PROF_EVENTS - 1]), "event sync"));
        for (int k = 0; k < 6; ++k) {
            float ms = 0.0f;
            OLC_TRY(check(s, cudaEventElapsedTime(&ms, s->events[i][k], s->events[i][k + 1]), "elapsed"));
            *slots[k] += ms;
        }
    }
    out->steps = (uint32_t)s->prof_step;
    out->substep_launches = s->prof_substeps;
    out->kernel_launches = s->prof_launches;
    return OLC_OK;
}

int olc_read_life(OlcSim* s, uint8_t* out, uint32_t rows, void* stream) {
    if (!s || (rows && !out)) return fail(s, OLC_ERR_ARG, "olc_read_life: bad arguments");
    if (rows > s->caps.max_agents) return fail(s, OLC_ERR_ARG, "olc_read_life: rows exceed max_agents");
    if (!rows) return OLC_OK;
    cudaStream_t st = as_stream(stream);
    OLC_TRY(check(s, cudaMemcpyAsync(out, s->life, rows, cudaMemcpyDeviceToHost, st), "life readback"));
    return check(s, cudaStreamSynchronize(st), "sync");
}

int olc_read_reductions(OlcSim* s, OlcReductions* out, void* stream) {
    if (!s || !out) return fail(s, OLC_ERR_ARG, "olc_read_reductions: null argument");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_read_reductions: batch handle (use olc_read_reductions_batch)");
    cudaStream_t st = as_stream(stream);
    OLC_TRY(check(s, cudaMemcpyAsync(s->red_host, s->red_dev, sizeof(OlcReductions), cudaMemcpyDeviceToHost, st),
                  "reductions readback"));
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync"));
    std::memcpy(out, s->red_host, sizeof(OlcReductions));
    return OLC_OK;
}

int olc_engine_metrics(OlcSim* s, const OlcEngineMetricsSpec* spec, double* out, void* stream) {
    if (!s || !spec || !out) return fail(s, OLC_ERR_ARG, "olc_engine_metrics: null argument");
    if (s->n_sims) return fail(s, OLC_ERR_STATE, "olc_engine_metrics: batch handle");
    const int ncol = (int)s->caps.n_agent_fields;
    auto col_ok = [&](int c, int width) { return c < 0 || (c + width <= ncol); };
    if (!col_ok(spec->state_field, 1) || !col_ok(spec->energy_field, 1) || !col_ok(spec->speed_field, 3) ||
        !col_ok(spec->csc_field, 1))
        return fail(s, OLC_ERR_ARG, "olc_engine_metrics: agent column out of range");
    for (int f : {spec->o2_field, spec->glucose_field})
        if (f >= (int)s->caps.n_fields || (f >= 0 && !s->field_bound[f]))
            return fail(s, OLC_ERR_ARG, "olc_engine_metrics: field not bound");
    if (!s->col[0][0]) return fail(s, OLC_ERR_STATE, "olc_engine_metrics: agent columns not bound");
    cudaStream_t st = as_stream(stream);
    if (!s->em_acc) {
        OLC_TRY(dev_alloc(s, &s->em_acc, sizeof(EngineMetricAcc), "engine metrics"));
        OLC_TRY(dev_alloc(s, &s->em_partials, sizeof(double) * EM_PARTIALS, "engine metric partials"));
        OLC_TRY(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->em_host), sizeof(EngineMetricAcc)),
                      "pinned engine metrics"));
    }
    const int cc = s->agent_cur;
    auto colp = [&](int c) { return c < 0 ? nullptr : s->col[cc][c]; };
    EngineMetricArgs a = {};
    a.x = static_cast<const float*>(s->col[cc][0]);
    a.y = static_cast<const float*>(s->col[cc][1]);
    a.z = static_cast<const float*>(s->col[cc][2]);
    a.life = s->life;
    a.state = static_cast<const int*>(colp(spec->state_field));
    a.csc = static_cast<const int*>(colp(spec->csc_field));
    a.energy = static_cast<const float*>(colp(spec->energy_field));
    if (spec->speed_field >= 0) {
        a.speed_x = static_cast<const float*>(colp(spec->speed_field));
        a.speed_y = static_cast<const float*>(colp(spec->speed_field + 1));
        a.speed_z = static_cast<const float*>(colp(spec->speed_field + 2));
    }
    if (spec->o2_field >= 0) {
        a.f0 = s->field[s->field_cur[spec->o2_field]][spec->o2_field];
        a.f0_type = field_type_word(s->fstep[spec->o2_field]);
        a.f0_b = s->fstep[spec->o2_field].bval;
    }
    if (spec->glucose_field >= 0) {
        a.f1 = s->field[s->field_cur[spec->glucose_field]][spec->glucose_field];
        a.f1_type = field_type_word(s->fstep[spec->glucose_field]);
        a.f1_b = s->fstep[spec->glucose_field].bval;
    }
    for (int i = 0; i < 3; ++i) {
        a.cdims[i] = s->geom.chem_dims[i];
        a.tdims[i] = s->bins.dims[i];
    }
    a.cvs = s->geom.chem_voxel_size;
    a.tvs = s->bins.vs;
    // the bin table holds the ranges of the last sort; before any step it is empty
    a.ranges = s->steps ? reinterpret_cast<const uint2*>(s->ranges) : nullptr;
    a.cx = spec->center[0];
    a.cy = spec->center[1];
    a.cz = spec->center[2];
    a.hypoxia = spec->hypoxia_threshold;
    a.crowd = spec->crowd_threshold;
    a.step = (double)s->steps;
    launch_engine_metrics(a, s->counters, s->caps.max_agents, s->em_acc, s->em_partials, st);
    OLC_TRY(check(s, cudaGetLastError(), "engine metrics launch"));
    OLC_TRY(check(s, cudaMemcpyAsync(s->em_host, s->em_acc, sizeof(EngineMetricAcc), cudaMemcpyDeviceToHost, st),
                  "engine metrics readback"));
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync"));
    std::memcpy(out, s->em_host->out, sizeof(double) * OLC_ENGINE_METRICS);
    return OLC_OK;
}

int olc_read_user_metrics(OlcSim* s, void* out, size_t bytes, void* stream) {
    if (!s || (bytes && !out)) return fail(s, OLC_ERR_ARG, "olc_read_user_metrics: bad arguments");
    if (bytes > s->metrics_bytes) return fail(s, OLC_ERR_ARG, "olc_read_user_metrics: more bytes than allocated");
    if (!bytes) return OLC_OK;
    cudaStream_t st = as_stream(stream);
    OLC_TRY(check(s, cudaMemcpyAsync(out, s->metrics_dev, bytes, cudaMemcpyDeviceToHost, st), "metrics readback"));
    return check(s, cudaStreamSynchronize(st), "sync");
}

// ------------------------------------------------------------------ batched mode

// The substep tile list of field `index` of a batch handle: members taking the
// most substeps first (stable), so substep s launches a prefix of the list;
// btile_count[index][s] is that prefix's length.
static int build_batch_field_tiles(OlcSim* s, int index) {
    const olc_u32 F = s->caps.n_fields;
    std::vector<std::pair<int, olc_u32>> order;  // (substeps, simulation)
    for (olc_u32 k = 0; k < s->n_sims; ++k) order.push_back({s->bsteps_host[(size_t)k * F + index].substeps, k});
    std::stable_sort(order.begin(), order.end(),
                     [](const std::pair<int, olc_u32>& x, const std::pair<int, olc_u32>& y) { return x.first > y.first; });
    std::vector<uint4> tiles, mt;
    std::vector<int> tile_steps;
    for (const auto& o : order) {
        mt.clear();
        substep_tiles(s->geoms[o.second], o.second, s->fstep[index].storage, member_tile_depth(s, o.second), &mt);
        tiles.insert(tiles.end(), mt.begin(), mt.end());
        tile_steps.insert(tile_steps.end(), mt.size(), o.first);
    }
    const int max_s = order.empty() ? 0 : order.front().first;
    std::vector<olc_u32> count(max_s, 0u);
    for (int sub = 0; sub < max_s; ++sub) {
        olc_u32 c = 0;
        while (c < tiles.size() && tile_steps[c] > sub) ++c;
        count[sub] = c;
    }
    cudaFree(s->btiles_field[index]);
    s->btiles_field[index] = nullptr;
    OLC_TRY(dev_alloc(s, &s->btiles_field[index], sizeof(uint4) * std::max<size_t>(1, tiles.size()), "field tiles"));
    if (!tiles.empty())
        OLC_TRY(check(s, cudaMemcpy(s->btiles_field[index], tiles.data(), sizeof(uint4) * tiles.size(),
                                    cudaMemcpyHostToDevice),
                      "upload field tiles"));
    s->btile_count[index] = count;
    return OLC_OK;
}

int olc_bind_field_batch(OlcSim* s, int index, void* a_, void* b_, float* sink, float* comp,
                         const OlcDiffusion* specs) {
    float* a = static_cast<float*>(a_);
    float* b = static_cast<float*>(b_);
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (!s->n_sims || s->pool) return fail(s, OLC_ERR_STATE, "olc_bind_field_batch: not a batch handle");
    if (index < 0 || index >= (int)s->caps.n_fields || !a || !b || !specs)
        return fail(s, OLC_ERR_ARG, "olc_bind_field_batch: bad index or null argument");
    const olc_u32 F = s->caps.n_fields;
    const int storage = specs[0].storage;
    const int encoding = specs[0].encoding;
    for (olc_u32 k = 0; k < s->n_sims; ++k) {
        if (specs[k].storage != storage)
            return fail(s, OLC_ERR_ARG, "olc_bind_field_batch: every member stores a field with the same type");
        // rules read an encoded field through one boundary value per handle
        if (specs[k].encoding != encoding ||
            (encoding != OLC_ENC_VALUE && specs[k].boundary != specs[0].boundary))
            return fail(s, OLC_ERR_ARG,
                        "olc_bind_field_batch: every member encodes a field the same way (encoding and, when "
                        "encoded, boundary value)");
    }
    if (storage != OLC_FIELD_F32 && !comp)
        return fail(s, OLC_ERR_ARG, "olc_bind_field_batch: 16-bit storage needs a compensation buffer");
    bool any_sink = false;
    for (olc_u32 k = 0; k < s->n_sims; ++k) {
        const OlcDiffusion& spec = specs[k];
        const OlcGeom& g = s->geoms[k];
        if (g.chem_dims[0] % (storage == OLC_FIELD_F32 ? 4 : 8) != 0)
            return fail(s, OLC_ERR_ARG, "olc_bind_field_batch: simulation " + std::to_string(k) +
                                            ": field x extent must be a multiple of 4 (8 for 16-bit storage)");
        FieldStep fs = {};
        std::string err;
        if (spec.substeps != 0 && !make_field_step(spec, g.chem_dims, g.chem_voxel_size, s->caps.dt, &fs, &err))
            return fail(s, OLC_ERR_ARG, "olc_bind_field_batch: simulation " + std::to_string(k) + ": " + err);
        if (spec.substeps == 0) {
            for (int i = 0; i < 3; ++i) fs.dims[i] = g.chem_dims[i];
            fs.substeps = 0;
            fs.storage = storage;
            fs.encoding = encoding;
            fs.bval = spec.boundary;
        }
        any_sink = any_sink || (spec.has_sink && spec.substeps != 0);
        s->bsteps_host[(size_t)k * F + index] = fs;
    }
    if (any_sink && !sink) return fail(s, OLC_ERR_ARG, "olc_bind_field_batch: has_sink without a sink buffer");
    drop_graphs(s);
    // each member's tensor maps (16-bit storage)
    for (olc_u32 k = 0; k < s->n_sims; ++k)
        if (storage != OLC_FIELD_F32 && specs[k].substeps != 0 &&
            !member_maps(s, k, index, a, b, s->field_off[k], s->geoms[k], storage))
            return fail(s, OLC_ERR_ARG, "olc_bind_field_batch: simulation " + std::to_string(k) +
                                            ": tensor maps of its grid failed (16-byte aligned grids)");
    OLC_TRY(check(s, cudaMemcpy(s->bmaps_dev, s->bmaps_host.data(), sizeof(CUtensorMap) * s->bmaps_host.size(),
                                cudaMemcpyHostToDevice),
                  "upload tensor maps"));
    s->fstep[index].storage = storage;
    OLC_TRY(build_batch_field_tiles(s, index));
    OLC_TRY(check(s, cudaMemcpy(s->bsteps_dev, s->bsteps_host.data(), sizeof(FieldStep) * s->bsteps_host.size(),
                                cudaMemcpyHostToDevice),
                  "upload field steps"));
    // every simulation's grid starts in buffer a
    std::vector<unsigned char> par((size_t)s->n_sims * OLC_MAX_FIELDS);
    OLC_TRY(check(s, cudaMemcpy(par.data(), s->fpar_dev, par.size(), cudaMemcpyDeviceToHost), "read field parity"));
    for (olc_u32 k = 0; k < s->n_sims; ++k) par[(size_t)k * F + index] = 0;
    OLC_TRY(check(s, cudaMemcpy(s->fpar_dev, par.data(), par.size(), cudaMemcpyHostToDevice), "write field parity"));
    s->field[0][index] = a;
    s->field[1][index] = b;
    s->sink[index] = any_sink ? sink : nullptr;
    s->comp[index] = storage != OLC_FIELD_F32 ? comp : nullptr;
    s->fstep[index].storage = storage;
    s->fstep[index].encoding = encoding;
    s->fstep[index].bval = specs[0].boundary;
    s->fspec[index] = specs[0];
    s->field_cur[index] = 0;
    s->field_bound[index] = true;
    return OLC_OK;
}

int olc_read_field_parity(OlcSim* s, uint8_t* out, void* stream) {
    if (!s || !out) return fail(s, OLC_ERR_ARG, "olc_read_field_parity: null argument");
    if (!s->n_sims) return fail(s, OLC_ERR_STATE, "olc_read_field_parity: not a batch handle");
    cudaStream_t st = as_stream(stream);
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync"));
    std::vector<unsigned char> par((size_t)s->n_sims * OLC_MAX_FIELDS);
    OLC_TRY(check(s, cudaMemcpy(par.data(), s->fpar_dev, par.size(), cudaMemcpyDeviceToHost), "read field parity"));
    const olc_u32 F = s->caps.n_fields;
    for (olc_u32 k = 0; k < s->n_sims; ++k)
        for (olc_u32 f = 0; f < F; ++f) out[(size_t)k * F + f] = par[(size_t)k * F + f];
    return OLC_OK;
}

int olc_set_params_batch(OlcSim* s, const void* blob, size_t stride, void* stream) {
    if (!s || !blob || stride == 0) return fail(s, OLC_ERR_ARG, "olc_set_params_batch: bad arguments");
    if (!s->n_sims || s->pool) return fail(s, OLC_ERR_STATE, "olc_set_params_batch: not a batch handle");
    cudaStream_t st = as_stream(stream);
    const size_t bytes = stride * s->n_sims;
    if (bytes > s->params_cap || stride != s->params_stride) {
        drop_graphs(s);
        OLC_TRY(check(s, cudaStreamSynchronize(st), "sync before params upload"));
        if (bytes > s->params_cap) {
            cudaFree(s->params_dev);
            if (s->params_host) cudaFreeHost(s->params_host);
            s->params_dev = nullptr;
            s->params_host = nullptr;
            const size_t cap = (bytes + 255) & ~size_t(255);
            OLC_TRY(dev_alloc(s, &s->params_dev, cap, "params"));
            OLC_TRY(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->params_host), cap), "pinned params"));
            s->params_cap = cap;
        }
        s->params_stride = stride;
        for (olc_u32 k = 0; k < s->n_sims; ++k) s->desc_host[k].params_off = (olc_u32)(k * stride);
        OLC_TRY(upload_desc(s));
    } else {
        OLC_TRY(check(s, cudaStreamSynchronize(st), "sync before params upload"));
    }
    std::memcpy(s->params_host, blob, bytes);
    return check(s, cudaMemcpyAsync(s->params_dev, s->params_host, bytes, cudaMemcpyHostToDevice, st),
                 "params upload");
}

int olc_read_reductions_batch(OlcSim* s, OlcReductions* out, void* stream) {
    if (!s || !out) return fail(s, OLC_ERR_ARG, "olc_read_reductions_batch: null argument");
    if (!s->n_sims) return fail(s, OLC_ERR_STATE, "olc_read_reductions_batch: not a batch handle");
    cudaStream_t st = as_stream(stream);
    const size_t bytes = sizeof(OlcReductions) * s->n_sims;
    OLC_TRY(check(s, cudaMemcpyAsync(s->red_batch_host, s->red_batch_dev, bytes, cudaMemcpyDeviceToHost, st),
                  "reductions readback"));
    OLC_TRY(check(s, cudaStreamSynchronize(st), "sync"));
    std::memcpy(out, s->red_batch_host, bytes);
    return OLC_OK;
}

int olc_read_user_metrics_batch(OlcSim* s, void* out, size_t bytes_per_sim, void* stream) {
    if (!s || !out) return fail(s, OLC_ERR_ARG, "olc_read_user_metrics_batch: null argument");
    if (!s->n_sims) return fail(s, OLC_ERR_STATE, "olc_read_user_metrics_batch: not a batch handle");
    if (bytes_per_sim != s->metrics_bytes)
        return fail(s, OLC_ERR_ARG, "olc_read_user_metrics_batch: bytes_per_sim must equal the metrics size");
    if (!bytes_per_sim) return OLC_OK;
    cudaStream_t st = as_stream(stream);
    OLC_TRY(check(s, cudaMemcpyAsync(out, s->metrics_dev, bytes_per_sim * s->n_sims, cudaMemcpyDeviceToHost, st),
                  "metrics readback"));
    return check(s, cudaStreamSynchronize(st), "sync");
}

// ------------------------------------------------------------------ serving pool

int olc_create_pool(const OlcPoolConfig* cfg, const OlcCaps* caps, OlcSim** out) {
    if (!cfg || !caps || !out) return fail(nullptr, OLC_ERR_ARG, "olc_create_pool: null argument");
    std::string err;
    if (!caps_ok(caps, "olc_create_pool", &err)) return fail(nullptr, OLC_ERR_ARG, err);
    if (cfg->max_slots < 1 || cfg->max_slots > (1u << 20))
        return fail(nullptr, OLC_ERR_ARG, "olc_create_pool: max_slots must be in [1, 2^20]");
    OlcGeom gmax = {};
    for (int i = 0; i < 3; ++i) gmax.tissue_dims[i] = cfg->max_tissue_dims[i];
    gmax.tissue_voxel_size = 1.0f;
    if (!geom_ok(gmax, &err)) return fail(nullptr, OLC_ERR_ARG, "olc_create_pool: max_tissue_dims: " + err);
    const olc_u32 top = olc_tissue_key(gmax.tissue_dims[0], gmax.tissue_dims[1], gmax.tissue_dims[2]);
    const int shift = std::max(1, key_bits_for(top));
    if (shift + key_bits_for(cfg->max_slots) > 32)
        return fail(nullptr, OLC_ERR_ARG, "olc_create_pool: slot index and bin key exceed 32 key bits");
    if (cfg->table_entries == 0 || cfg->table_entries >= (1ull << 31))
        return fail(nullptr, OLC_ERR_ARG, "olc_create_pool: table_entries must be in [1, 2^31)");
    if (caps->n_fields && cfg->field_voxels == 0)
        return fail(nullptr, OLC_ERR_ARG, "olc_create_pool: field_voxels must be > 0 with fields");
    OlcSim* s = new OlcSim();
    const olc_u32 n = cfg->max_slots;
    s->pool = true;
    s->caps = *caps;
    s->geom = gmax;
    s->n_sims = n;
    s->geoms.assign(n, OlcGeom{});
    s->bins = make_bin_grid(gmax);
    s->bargs.shift = shift;
    s->bargs.n_sims = n;
    s->bargs.sentinel = n << shift;
    s->key_bits = key_bits_for(s->bargs.sentinel);
    s->n_table = (olc_u32)cfg->table_entries;
    s->desc_host.assign(n, OlcSimDesc{});
    s->bsteps_host.assign((size_t)n * std::max<olc_u32>(1u, caps->n_fields), FieldStep{});
    s->slot_used.assign(n, 0);
    s->slot_table_off.assign(n, 0);
    s->slot_table_n.assign(n, 0);
    s->slot_field_off.assign(n, 0);
    s->slot_field_n.assign(n, 0);
    s->table_arena.reset(cfg->table_entries);
    s->field_arena.reset(cfg->field_voxels);
    int rc = alloc_common(s);
    auto A = [&](int r) {
        if (rc == OLC_OK) rc = r;
    };
    A(dev_alloc(s, &s->desc_dev, sizeof(OlcSimDesc) * n, "member records"));
    A(dev_alloc(s, &s->cols_dev, sizeof(void*) * 2 * OLC_MAX_AGENT_COLS, "column tables"));
    A(dev_alloc(s, &s->fpar_dev, (size_t)n * OLC_MAX_FIELDS, "field parity"));
    A(dev_alloc(s, &s->bsteps_dev, sizeof(FieldStep) * s->bsteps_host.size(), "field steps"));
    A(dev_alloc(s, &s->red_batch_dev, sizeof(OlcReductions) * n, "pool reductions"));
    s->bmaps_host.assign((size_t)n * std::max<olc_u32>(1u, caps->n_fields) * 2, CUtensorMap{});
    A(dev_alloc(s, &s->bmaps_dev, sizeof(CUtensorMap) * s->bmaps_host.size(), "tensor maps"));
    A(dev_alloc(s, &s->gather_counts, POOL_GATHER_BLOCKS * sizeof(olc_u32), "gather counts"));
    // each member's range splits into at most n / CHUNK + 1 chunks
    s->table_chunks_cap = (size_t)(cfg->table_entries / POOL_TABLE_CHUNK) + n + 1;
    A(dev_alloc(s, &s->table_chunks, s->table_chunks_cap * sizeof(uint2), "bin-table chunks"));
    A(check(s, cudaMallocHost(reinterpret_cast<void**>(&s->red_batch_host), sizeof(OlcReductions) * n),
            "pinned pool reductions"));
    if (rc == OLC_OK) {
        A(check(s, cudaMemset(s->desc_dev, 0, sizeof(OlcSimDesc) * n), "memset member records"));
        A(check(s, cudaMemset(s->fpar_dev, 0, (size_t)n * OLC_MAX_FIELDS), "memset field parity"));
        A(check(s, cudaMemset(s->bsteps_dev, 0, sizeof(FieldStep) * s->bsteps_host.size()), "memset field steps"));
        A(check(s, cudaMemset(s->red_batch_dev, 0, sizeof(OlcReductions) * n), "memset pool reductions"));
    }
    s->bargs.sims = s->desc_dev;
    s->pool_dirty = true;
    if (rc != OLC_OK) {
        std::string msg = s->err;
        olc_destroy(s);
        return fail(nullptr, rc, msg);
    }
    *out = s;
    return OLC_OK;
}

int olc_bind_field_pool(OlcSim* s, int index, void* a, void* b, float* sink, float* comp, int storage, int encoding,
                        float boundary) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (!s->pool) return fail(s, OLC_ERR_STATE, "olc_bind_field_pool: not a pool");
    if (index < 0 || index >= (int)s->caps.n_fields || !a || !b)
        return fail(s, OLC_ERR_ARG, "olc_bind_field_pool: bad index or null buffer");
    if (storage < OLC_FIELD_F32 || storage > OLC_FIELD_F16_SR)
        return fail(s, OLC_ERR_ARG, "olc_bind_field_pool: bad storage type");
    if (storage != OLC_FIELD_F32 && !comp)
        return fail(s, OLC_ERR_ARG, "olc_bind_field_pool: 16-bit storage needs a compensation buffer");
    if (encoding < OLC_ENC_VALUE || encoding > OLC_ENC_OFFSET3 || (encoding != OLC_ENC_VALUE && storage == OLC_FIELD_F32))
        return fail(s, OLC_ERR_ARG, "olc_bind_field_pool: bad encoding (encodings apply to 16-bit storage only)");
    if (s->slots_used) return fail(s, OLC_ERR_STATE, "olc_bind_field_pool: bind fields before admitting members");
    drop_graphs(s);
    s->field[0][index] = static_cast<float*>(a);
    s->field[1][index] = static_cast<float*>(b);
    s->sink[index] = sink;
    s->comp[index] = storage != OLC_FIELD_F32 ? comp : nullptr;
    s->fstep[index] = FieldStep{};
    s->fstep[index].storage = storage;
    s->fstep[index].encoding = encoding;
    s->fstep[index].bval = boundary;
    s->field_cur[index] = 0;
    s->field_bound[index] = true;
    s->pool_dirty = true;
    return OLC_OK;
}

int olc_pool_admit(OlcSim* s, const OlcGeom* geom, const OlcDiffusion* specs, const void* params,
                   size_t params_bytes, int32_t* slot_out, uint64_t* field_off_out, void* stream) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (!s->pool) return fail(s, OLC_ERR_STATE, "olc_pool_admit: not a pool");
    if (!geom || !slot_out || !field_off_out || (s->caps.n_fields && !specs) || (params_bytes && !params))
        return fail(s, OLC_ERR_ARG, "olc_pool_admit: null argument");
    std::string err;
    if (!geom_ok(*geom, &err)) return fail(s, OLC_ERR_ARG, "olc_pool_admit: " + err);
    const olc_u32 top = olc_tissue_key(geom->tissue_dims[0], geom->tissue_dims[1], geom->tissue_dims[2]);
    if (top >> s->bargs.shift) return fail(s, OLC_ERR_ARG, "olc_pool_admit: bin grid larger than max_tissue_dims");
    const olc_u32 F = s->caps.n_fields;
    const olc_u64 nvox = (olc_u64)geom->chem_dims[0] * geom->chem_dims[1] * geom->chem_dims[2];
    FieldStep fs[OLC_MAX_FIELDS] = {};
    for (olc_u32 f = 0; f < F; ++f) {
        if (!s->field_bound[f]) return fail(s, OLC_ERR_STATE, "olc_pool_admit: bind every field before admitting");
        const int storage = s->fstep[f].storage;
        if (specs[f].storage != storage)
            return fail(s, OLC_ERR_ARG, "olc_pool_admit: field " + std::to_string(f) + " storage differs from the pool's");
        if (specs[f].encoding != s->fstep[f].encoding ||
            (specs[f].encoding != OLC_ENC_VALUE && specs[f].boundary != s->fstep[f].bval))
            return fail(s, OLC_ERR_ARG, "olc_pool_admit: field " + std::to_string(f) +
                                            " encoding (or an encoded field's boundary value) differs from the pool's");
        if (nvox == 0 || geom->chem_dims[0] % (storage == OLC_FIELD_F32 ? 4 : 8) != 0)
            return fail(s, OLC_ERR_ARG, "olc_pool_admit: field x extent must be a multiple of 4 (8 for 16-bit storage)");
        if (specs[f].substeps != 0) {
            if (!make_field_step(specs[f], geom->chem_dims, geom->chem_voxel_size, s->caps.dt, &fs[f], &err))
                return fail(s, OLC_ERR_ARG, "olc_pool_admit: field " + std::to_string(f) + ": " + err);
        } else {
            for (int i = 0; i < 3; ++i) fs[f].dims[i] = geom->chem_dims[i];
            fs[f].storage = storage;
            fs[f].encoding = s->fstep[f].encoding;
            fs[f].bval = specs[f].boundary;
        }
    }
    if (params_bytes && s->params_stride && params_bytes != s->params_stride)
        return fail(s, OLC_ERR_ARG, "olc_pool_admit: every member's Params blob has the same size");
    cudaStream_t st = as_stream(stream);
    if (params_bytes && !s->params_stride) {
        const size_t bytes = params_bytes * s->n_sims;
        const size_t cap = (bytes + 255) & ~size_t(255);
        OLC_TRY(dev_alloc(s, &s->params_dev, cap, "params"));
        s->params_cap = cap;
        s->params_stride = params_bytes;
        s->params_all.assign(bytes, 0);
    }
    olc_u32 slot = 0;
    while (slot < s->n_sims && s->slot_used[slot]) ++slot;
    if (slot == s->n_sims) return fail(s, OLC_ERR_CAPACITY, "olc_pool_admit: no free slot");
    const olc_u64 t_off = s->table_arena.alloc((olc_u64)top + 1u);
    if (t_off == RangeArena::NONE) return fail(s, OLC_ERR_CAPACITY, "olc_pool_admit: bin-table arena full");
    olc_u64 f_off = 0;
    if (F) {
        f_off = s->field_arena.alloc(nvox, 32);  // 128-byte aligned grids
        if (f_off == RangeArena::NONE) {
            s->table_arena.release(t_off, (olc_u64)top + 1u);
            return fail(s, OLC_ERR_CAPACITY, "olc_pool_admit: field arena full");
        }
    }
    for (olc_u32 f = 0; f < F; ++f)
        if (fs[f].storage != OLC_FIELD_F32 && fs[f].substeps != 0 &&
            !member_maps(s, slot, (int)f, s->field[0][f], s->field[1][f], f_off, *geom, fs[f].storage)) {
            s->table_arena.release(t_off, (olc_u64)top + 1u);
            s->field_arena.release(f_off, nvox);
            return fail(s, OLC_ERR_ARG, "olc_pool_admit: tensor maps of the member's grid failed");
        }
    OlcSimDesc& d = s->desc_host[slot];
    std::memset(&d, 0, sizeof(d));
    for (int i = 0; i < 3; ++i) {
        d.tdims[i] = geom->tissue_dims[i];
        d.cdims[i] = geom->chem_dims[i];
        d.lo[i] = geom->domain_lo[i] + s->contact.margin;
        d.hi[i] = geom->domain_hi[i] - s->contact.margin;
        d.center[i] = 0.5f * (geom->domain_lo[i] + geom->domain_hi[i]);
    }
    d.tvs = geom->tissue_voxel_size;
    d.cvs = geom->chem_voxel_size;
    d.bin_width = s->caps.radial_bin_width > 0.0f ? s->caps.radial_bin_width : 1.0f;
    d.ranges_base = (olc_u32)t_off;
    d.params_off = (olc_u32)(slot * s->params_stride);
    d.metrics_off = (olc_u32)(slot * s->metrics_bytes);
    d.step_base = (olc_u32)s->pool_steps;
    d.field_off = f_off;
    s->geoms[slot] = *geom;
    for (olc_u32 f = 0; f < F; ++f) s->bsteps_host[(size_t)slot * F + f] = fs[f];
    if (params_bytes) std::memcpy(s->params_all.data() + (size_t)slot * s->params_stride, params, params_bytes);
    // clear the member's per-slot device records and field side buffers
    int rc = OLC_OK;
    auto A = [&](int r) {
        if (rc == OLC_OK) rc = r;
    };
    if (F) A(check(s, cudaMemsetAsync(s->fpar_dev + (size_t)slot * F, 0, F, st), "clear field parity"));
    if (s->metrics_dev && s->metrics_bytes)
        A(check(s, cudaMemsetAsync(static_cast<unsigned char*>(s->metrics_dev) + (size_t)slot * s->metrics_bytes, 0,
                                   s->metrics_bytes, st),
                "clear metrics"));
    launch_reset_reductions_batch(s->red_batch_dev + slot, 1u, st);
    for (olc_u32 f = 0; f < F; ++f) {
        if (s->sink[f]) A(check(s, cudaMemsetAsync(s->sink[f] + f_off, 0, nvox * 4, st), "clear sink"));
        if (s->comp[f]) A(check(s, cudaMemsetAsync(s->comp[f] + f_off, 0, nvox * 4, st), "clear residuals"));
    }
    A(check(s, cudaGetLastError(), "olc_pool_admit"));
    if (rc != OLC_OK) {
        s->table_arena.release(t_off, (olc_u64)top + 1u);
        if (F) s->field_arena.release(f_off, nvox);
        return rc;
    }
    s->slot_used[slot] = 1;
    s->slot_table_off[slot] = t_off;
    s->slot_table_n[slot] = (olc_u64)top + 1u;
    s->slot_field_off[slot] = f_off;
    s->slot_field_n[slot] = F ? nvox : 0;
    s->slots_used++;
    s->pool_dirty = true;
    *slot_out = (int32_t)slot;
    *field_off_out = f_off;
    return OLC_OK;
}

static bool pool_slot_ok(OlcSim* s, int32_t slot, const char* who) {
    if (!s->pool) {
        fail(s, OLC_ERR_STATE, std::string(who) + ": not a pool");
        return false;
    }
    if (slot < 0 || (olc_u32)slot >= s->n_sims || !s->slot_used[slot]) {
        fail(s, OLC_ERR_ARG, std::string(who) + ": slot not in use");
        return false;
    }
    return true;
}

int olc_pool_add_agents(OlcSim* s, int32_t slot, void* const* cols_dev, uint32_t n, void* stream) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (!pool_slot_ok(s, slot, "olc_pool_add_agents")) return s->pool ? OLC_ERR_ARG : OLC_ERR_STATE;
    if (n == 0) return OLC_OK;
    const int sim_col = (int)s->caps.n_agent_fields - 1;
    PoolCols pc;
    std::memset(&pc, 0, sizeof(pc));
    pc.ncols = (int)s->caps.n_agent_fields;
    pc.sim_col = sim_col;
    for (int c = 0; c < pc.ncols; ++c) {
        if (!s->col[s->agent_cur][c]) return fail(s, OLC_ERR_STATE, "olc_pool_add_agents: agent column not bound");
        if (c != sim_col && (!cols_dev || !cols_dev[c]))
            return fail(s, OLC_ERR_ARG, "olc_pool_add_agents: null source column");
        pc.src[c] = c == sim_col ? nullptr : cols_dev[c];
        pc.dst[c] = s->col[s->agent_cur][c];
    }
    cudaStream_t st = as_stream(stream);
    launch_pool_append(pc, n, (olc_u32)slot, s->life, s->counters, s->caps.max_agents, st);
    return check(s, cudaGetLastError(), "olc_pool_add_agents");
}

int olc_pool_gather(OlcSim* s, int32_t slot, void* const* dst_dev, uint32_t max_rows, uint32_t* count_dev,
                    void* stream) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (!pool_slot_ok(s, slot, "olc_pool_gather")) return s->pool ? OLC_ERR_ARG : OLC_ERR_STATE;
    if (!dst_dev || !count_dev) return fail(s, OLC_ERR_ARG, "olc_pool_gather: null argument");
    const int sim_col = (int)s->caps.n_agent_fields - 1;
    PoolCols pc;
    std::memset(&pc, 0, sizeof(pc));
    pc.ncols = (int)s->caps.n_agent_fields;
    pc.sim_col = sim_col;
    for (int c = 0; c < pc.ncols; ++c) {
        pc.src[c] = s->col[s->agent_cur][c];
        pc.dst[c] = c == sim_col ? nullptr : dst_dev[c];
    }
    cudaStream_t st = as_stream(stream);
    launch_pool_gather(pc, static_cast<const olc_u32*>(s->col[s->agent_cur][sim_col]), s->life, s->counters,
                       (olc_u32)slot, s->gather_counts, count_dev, max_rows, st);
    return check(s, cudaGetLastError(), "olc_pool_gather");
}

int olc_pool_copy_results(OlcSim* s, int32_t slot, OlcReductions* red_host, void* metrics_host, void* stream) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (!pool_slot_ok(s, slot, "olc_pool_copy_results")) return s->pool ? OLC_ERR_ARG : OLC_ERR_STATE;
    cudaStream_t st = as_stream(stream);
    if (red_host)
        OLC_TRY(check(s, cudaMemcpyAsync(red_host, s->red_batch_dev + slot, sizeof(OlcReductions),
                                         cudaMemcpyDeviceToHost, st),
                      "reductions readback"));
    if (metrics_host && s->metrics_dev && s->metrics_bytes)
        OLC_TRY(check(s, cudaMemcpyAsync(metrics_host,
                                         static_cast<unsigned char*>(s->metrics_dev) + (size_t)slot * s->metrics_bytes,
                                         s->metrics_bytes, cudaMemcpyDeviceToHost, st),
                      "metrics readback"));
    return OLC_OK;
}

int olc_pool_retire(OlcSim* s, int32_t slot, void* stream) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (!pool_slot_ok(s, slot, "olc_pool_retire")) return s->pool ? OLC_ERR_ARG : OLC_ERR_STATE;
    const int sim_col = (int)s->caps.n_agent_fields - 1;
    const void* simc = s->col[s->agent_cur][sim_col];
    if (simc)
        launch_pool_retire(static_cast<const olc_u32*>(simc), s->life, s->counters, s->caps.max_agents,
                           (olc_u32)slot, as_stream(stream));
    s->table_arena.release(s->slot_table_off[slot], s->slot_table_n[slot]);
    if (s->slot_field_n[slot]) s->field_arena.release(s->slot_field_off[slot], s->slot_field_n[slot]);
    const olc_u32 F = s->caps.n_fields;
    for (olc_u32 f = 0; f < F; ++f) s->bsteps_host[(size_t)slot * F + f] = FieldStep{};
    std::memset(&s->desc_host[slot], 0, sizeof(OlcSimDesc));
    s->slot_used[slot] = 0;
    s->slot_table_n[slot] = s->slot_field_n[slot] = 0;
    s->slots_used--;
    s->pool_dirty = true;
    return check(s, cudaGetLastError(), "olc_pool_retire");
}

int olc_pool_usage(const OlcSim* s, OlcPoolUsage* out) {
    if (!s || !out) return fail(nullptr, OLC_ERR_ARG, "olc_pool_usage: null argument");
    if (!s->pool) return fail(const_cast<OlcSim*>(s), OLC_ERR_STATE, "olc_pool_usage: not a pool");
    out->slots_used = s->slots_used;
    out->max_slots = s->n_sims;
    out->table_used = s->table_arena.used();
    out->table_entries = s->table_arena.capacity();
    out->table_largest_free = s->table_arena.largest_free();
    out->field_used = s->field_arena.used();
    out->field_voxels = s->field_arena.capacity();
    out->field_largest_free = s->field_arena.largest_free();
    return OLC_OK;
}

}  // extern "C"

struct OlcArena {
    olc::RangeArena a;
};

extern "C" {

int olc_arena_create(uint64_t capacity, OlcArena** out) {
    if (!out || capacity == 0) return fail(nullptr, OLC_ERR_ARG, "olc_arena_create: bad arguments");
    *out = new OlcArena();
    (*out)->a.reset(capacity);
    return OLC_OK;
}

int olc_arena_alloc(OlcArena* arena, uint64_t n, uint64_t align, uint64_t* offset) {
    if (!arena || !offset || n == 0 || align == 0 || (align & (align - 1)))
        return fail(nullptr, OLC_ERR_ARG, "olc_arena_alloc: bad arguments (n > 0, align a power of two)");
    const uint64_t off = arena->a.alloc(n, align);
    if (off == RangeArena::NONE) return fail(nullptr, OLC_ERR_CAPACITY, "olc_arena_alloc: no free range fits");
    *offset = off;
    return OLC_OK;
}

int olc_arena_release(OlcArena* arena, uint64_t offset, uint64_t n) {
    if (!arena) return fail(nullptr, OLC_ERR_ARG, "olc_arena_release: null arena");
    if (!arena->a.release(offset, n)) return fail(nullptr, OLC_ERR_ARG, "olc_arena_release: range not allocated");
    return OLC_OK;
}

int olc_arena_stats(const OlcArena* arena, uint64_t* used, uint64_t* largest_free, uint64_t* free_ranges) {
    if (!arena) return fail(nullptr, OLC_ERR_ARG, "olc_arena_stats: null arena");
    if (used) *used = arena->a.used();
    if (largest_free) *largest_free = arena->a.largest_free();
    if (free_ranges) *free_ranges = arena->a.free_ranges();
    return OLC_OK;
}

int olc_arena_destroy(OlcArena* arena) {
    delete arena;
    return OLC_OK;
}

// ------------------------------------------------------------------ stages

int olc_stage_rng(uint32_t* states, uint32_t n, int draws, float* out, float* dirs, void* stream) {
    if (n && (!states || (draws > 0 && !out))) return fail(nullptr, OLC_ERR_ARG, "olc_stage_rng: null buffer");
    if (draws < 0) return fail(nullptr, OLC_ERR_ARG, "olc_stage_rng: draws < 0");
    launch_rng(states, n, draws, out, dirs, as_stream(stream));
    return cuda_status(cudaGetLastError(), "olc_stage_rng");
}

int olc_stage_keys(const float* x, const float* y, const float* z, const uint8_t* dead, uint32_t n,
                   const OlcGeom* geom, uint32_t* keys, void* stream) {
    if (!geom || (n && (!x || !y || !z || !keys))) return fail(nullptr, OLC_ERR_ARG, "olc_stage_keys: null argument");
    std::string err;
    if (!geom_ok(*geom, &err)) return fail(nullptr, OLC_ERR_ARG, "olc_stage_keys: " + err);
    if (n == 0) return OLC_OK;
    BinGrid g = make_bin_grid(*geom);
    launch_keys(x, y, z, dead, nullptr, n, nullptr, n, g, keys, nullptr, 0, nullptr, as_stream(stream));
    return cuda_status(cudaGetLastError(), "olc_stage_keys");
}

size_t olc_sort_scratch_bytes(uint32_t n, int key_bits) {
    if (key_bits < 1 || key_bits > 32) return 0;
    return sort_scratch_bytes(n, key_bits);
}

size_t olc_sort_status_offset(void) {
    // carve_sort_scratch's layout: the status word follows the histograms,
    // the scanned bases and the tile counters, whatever n and key_bits are
    SortScratch sc;
    alignas(256) static unsigned char probe[16384];
    carve_sort_scratch(probe, sizeof(probe), 1, 8, &sc);
    return (size_t)(reinterpret_cast<unsigned char*>(sc.status) - probe);
}

int olc_stage_sort_pairs(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, uint32_t n,
                         int key_bits, void* scratch, size_t bytes, void* stream) {
    if (key_bits < 1 || key_bits > 32) return fail(nullptr, OLC_ERR_ARG, "olc_stage_sort_pairs: key_bits in [1, 32]");
    if (n == 0) return OLC_OK;
    if (!kin || !kout || !vout || !scratch)
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_sort_pairs: null buffer");
    if (n > (1u << 30)) return fail(nullptr, OLC_ERR_ARG, "olc_stage_sort_pairs: n > 2^30");
    SortScratch sc;
    if (!carve_sort_scratch(scratch, bytes, n, key_bits, &sc))
        return fail(nullptr, OLC_ERR_ARG,
                    "olc_stage_sort_pairs: scratch too small or not 256-byte aligned (need " +
                        std::to_string(sort_scratch_bytes(n, key_bits)) + " bytes)");
    cudaStream_t st = as_stream(stream);
    cudaMemsetAsync(sc.status, 0, 4, st);
    run_sort(kin, vin, kout, vout, nullptr, n, n, key_bits, sc, false, nullptr, 0, st);
    return cuda_status(cudaGetLastError(), "olc_stage_sort_pairs");
}

int olc_stage_bin_ranges(const uint32_t* keys, uint32_t n, uint32_t n_bins, uint32_t* ranges, void* stream) {
    if (n_bins == 0 || !ranges || (n && !keys)) return fail(nullptr, OLC_ERR_ARG, "olc_stage_bin_ranges: bad arguments");
    cudaStream_t st = as_stream(stream);
    cudaMemsetAsync(ranges, 0, (size_t)n_bins * 8, st);
    if (n) launch_bin_ranges(keys, nullptr, n, n, n_bins, ranges, st);
    return cuda_status(cudaGetLastError(), "olc_stage_bin_ranges");
}

static int stage_diffuse(float* f, float* tmp, float* sink, const int32_t dims[3], float dx, float dt,
                         const OlcDiffusion* spec, const OlcTuning* t, void* stream, const char* who) {
    if (!f || !tmp || !dims || !spec) return fail(nullptr, OLC_ERR_ARG, std::string(who) + ": null argument");
    if (spec->storage != OLC_FIELD_F32)
        return fail(nullptr, OLC_ERR_ARG, std::string(who) + ": FP32 storage only (olc_stage_diffuse16 for 16-bit)");
    std::string err;
    FieldStep fs;
    if (!make_field_step(*spec, dims, dx, dt, &fs, &err)) return fail(nullptr, OLC_ERR_ARG, std::string(who) + ": " + err);
    const OlcTuning def = {8, 8, OLC_CONTACT_FLAT, 16, 0, 0, 0};
    if (!t) t = &def;
    if (!stencil_tile_known(t->stencil_tile_y, t->stencil_tile_z) || !pair_threads_known(t->stencil_pair_threads) ||
        t->stencil_pair_planes < 0 || t->stencil_pair_planes > 4096 || t->stencil_l2_keep_pct < 0 ||
        t->stencil_l2_keep_pct > 100)
        return fail(nullptr, OLC_ERR_ARG, std::string(who) + ": unknown stencil tile or pair shape");
    cudaStream_t st = as_stream(stream);
    FieldMaps maps;
    olc_u32* status = stage_status_word();
    float* res;
    if (status && make_field_maps(&maps, f, tmp, dims, t->stencil_tile_y, t->stencil_tile_z, t->stencil_pair_threads,
                                  t->stencil_pair_planes, t->stencil_l2_keep_pct)) {
        launch_sink(f, spec->has_sink ? sink : nullptr, fs, st);
        res = run_substeps_tma(f, tmp, maps, 0, fs, status, st);
    } else {
        res = run_field_step(f, tmp, spec->has_sink ? sink : nullptr, fs, st);
    }
    if (res != f) {
        const size_t bytes = (size_t)dims[0] * dims[1] * dims[2] * 4;
        cudaMemcpyAsync(f, res, bytes, cudaMemcpyDeviceToDevice, st);
    }
    return cuda_status(cudaGetLastError(), who);
}

int olc_stage_diffuse(float* f, float* tmp, float* sink, const int32_t dims[3], float dx, float dt,
                      const OlcDiffusion* spec, void* stream) {
    return stage_diffuse(f, tmp, sink, dims, dx, dt, spec, nullptr, stream, "olc_stage_diffuse");
}

int olc_stage_diffuse_tuned(float* f, float* tmp, float* sink, const int32_t dims[3], float dx, float dt,
                            const OlcDiffusion* spec, const OlcTuning* tuning, void* stream) {
    return stage_diffuse(f, tmp, sink, dims, dx, dt, spec, tuning, stream, "olc_stage_diffuse_tuned");
}

int olc_stage_diffuse_pinned(float* f, float* tmp, float* sink, const int32_t dims[3], float dx, float dt,
                             const OlcDiffusion* spec, const uint32_t* idx, uint32_t n, float value, void* stream) {
    if (!f || !tmp || !dims || !spec || (n && !idx))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_diffuse_pinned: null argument");
    if (spec->storage != OLC_FIELD_F32) return fail(nullptr, OLC_ERR_ARG, "olc_stage_diffuse_pinned: FP32 only");
    std::string err;
    FieldStep fs;
    if (!make_field_step(*spec, dims, dx, dt, &fs, &err))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_diffuse_pinned: " + err);
    cudaStream_t st = as_stream(stream);
    Pins pins = {idx, n, value};
    FieldMaps maps;
    olc_u32* status = stage_status_word();
    float* res;
    if (status && make_field_maps(&maps, f, tmp, dims)) {
        launch_sink(f, spec->has_sink ? sink : nullptr, fs, st);
        res = run_substeps_tma(f, tmp, maps, 0, fs, status, st, &pins);
    } else {
        res = run_field_step(f, tmp, spec->has_sink ? sink : nullptr, fs, st, &pins);
    }
    if (res != f) {
        const size_t bytes = (size_t)dims[0] * dims[1] * dims[2] * 4;
        cudaMemcpyAsync(f, res, bytes, cudaMemcpyDeviceToDevice, st);
    }
    return cuda_status(cudaGetLastError(), "olc_stage_diffuse_pinned");
}

int olc_stage_diffuse16(void* f, void* tmp, float* sink, float* comp, const int32_t dims[3], float dx, float dt,
                        const OlcDiffusion* spec, uint32_t step, int field, void* stream) {
    if (!f || !tmp || !comp || !dims || !spec)
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_diffuse16: null argument");
    if (spec->storage < OLC_FIELD_BF16 || spec->storage > OLC_FIELD_F16_SR)
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_diffuse16: storage must be BF16, FP16 or BF16_SR");
    std::string err;
    FieldStep fs;
    if (!make_field_step(*spec, dims, dx, dt, &fs, &err))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_diffuse16: " + err);
    cudaStream_t st = as_stream(stream);
    olc_u32* status = stage_status_word();
    FieldMaps16 maps;
    if (!status || !make_field_maps16(&maps, f, tmp, dims))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_diffuse16: TMA descriptors failed (16-byte aligned buffers)");
    launch_react16(f, spec->has_sink ? sink : nullptr, comp, fs, st);
    void* res = run_substeps16(f, tmp, maps, 0, fs, status, nullptr, step, field, st);
    if (res != f) {
        const size_t bytes = (size_t)dims[0] * dims[1] * dims[2] * 2;
        cudaMemcpyAsync(f, res, bytes, cudaMemcpyDeviceToDevice, st);
    }
    return cuda_status(cudaGetLastError(), "olc_stage_diffuse16");
}

static int stage_contact(const float* posr, const uint32_t* ranges, uint32_t n, const OlcGeom* geom,
                         const OlcContact* spec, float dt, int variant, float* x, float* y, float* z, void* stream,
                         const char* who) {
    if (!geom || !spec || (n && (!posr || !ranges || !x || !y || !z)))
        return fail(nullptr, OLC_ERR_ARG, std::string(who) + ": null argument");
    if (variant != OLC_CONTACT_FLAT && variant != OLC_CONTACT_NESTED)
        return fail(nullptr, OLC_ERR_ARG, std::string(who) + ": contact_variant must be an OLC_CONTACT_* value");
    std::string err;
    if (!geom_ok(*geom, &err)) return fail(nullptr, OLC_ERR_ARG, std::string(who) + ": " + err);
    if (n == 0) return OLC_OK;
    ContactDev d;
    for (int i = 0; i < 3; ++i) {
        d.tdims[i] = geom->tissue_dims[i];
        d.lo[i] = geom->domain_lo[i] + spec->margin;
        d.hi[i] = geom->domain_hi[i] - spec->margin;
    }
    d.tvs = geom->tissue_voxel_size;
    d.stiffness = spec->stiffness;
    d.mobility = spec->mobility;
    d.max_disp = spec->max_disp;
    d.dt = dt;
    launch_contact(reinterpret_cast<const float4*>(posr), ranges, nullptr, n, n, d, x, y, z, as_stream(stream),
                   variant);
    return cuda_status(cudaGetLastError(), who);
}

int olc_stage_contact(const float* posr, const uint32_t* ranges, uint32_t n, const OlcGeom* geom,
                      const OlcContact* spec, float dt, float* x, float* y, float* z, void* stream) {
    return stage_contact(posr, ranges, n, geom, spec, dt, OLC_CONTACT_FLAT, x, y, z, stream, "olc_stage_contact");
}

int olc_stage_contact_tuned(const float* posr, const uint32_t* ranges, uint32_t n, const OlcGeom* geom,
                            const OlcContact* spec, float dt, int32_t contact_variant, float* x, float* y, float* z,
                            void* stream) {
    return stage_contact(posr, ranges, n, geom, spec, dt, contact_variant, x, y, z, stream,
                         "olc_stage_contact_tuned");
}

int olc_stage_contact_mech(const float* posr, const uint32_t* ranges, uint32_t n, const OlcGeom* geom,
                           const OlcContact* spec, const OlcMechanics* mech, const int32_t* state, float* vx,
                           float* vy, float* vz, float dt, float* x, float* y, float* z, void* stream) {
    if (!geom || !spec || !mech || (n && (!posr || !ranges || !x || !y || !z)))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_mech: null argument");
    if (mech->velocity_field >= 0 && n && (!vx || !vy || !vz))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_mech: velocity columns missing");
    if (mech->adhesion_stiffness != 0.0f && !(mech->adhesion_range > 0.0f))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_mech: adhesion needs adhesion_range > 0");
    std::string err;
    if (!geom_ok(*geom, &err)) return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_mech: " + err);
    if (n == 0) return OLC_OK;
    ContactDev d;
    for (int i = 0; i < 3; ++i) {
        d.tdims[i] = geom->tissue_dims[i];
        d.lo[i] = geom->domain_lo[i] + spec->margin;
        d.hi[i] = geom->domain_hi[i] - spec->margin;
    }
    d.tvs = geom->tissue_voxel_size;
    d.stiffness = spec->stiffness;
    d.mobility = spec->mobility;
    d.max_disp = spec->max_disp;
    d.dt = dt;
    MechDev m = {};
    m.state = state;
    m.necrotic_factor = mech->necrotic_factor;
    m.adh_k = mech->adhesion_stiffness;
    m.adh_range = mech->adhesion_range;
    if (mech->velocity_field >= 0) {
        m.vx = vx;
        m.vy = vy;
        m.vz = vz;
    }
    m.damping = mech->damping;
    m.max_speed = mech->max_speed;
    launch_contact_mech(reinterpret_cast<const float4*>(posr), ranges, nullptr, n, n, d, m, x, y, z,
                        as_stream(stream));
    return cuda_status(cudaGetLastError(), "olc_stage_contact_mech");
}

int olc_stage_contact_motion(const float* posr, const uint32_t* ranges, uint32_t n, const OlcGeom* geom,
                             const OlcContact* spec, const OlcMechanics* mech, const int32_t* state, float* vx,
                             float* vy, float* vz, const int32_t* species, uint32_t* rng, const float* o2,
                             const float* glucose, float dt, float* x, float* y, float* z, void* stream) {
    if (!geom || !spec || !mech || (n && (!posr || !ranges || !x || !y || !z)))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_motion: null argument");
    if (mech->velocity_field >= 0 && n && (!vx || !vy || !vz))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_motion: velocity columns missing");
    if (mech->adhesion_stiffness != 0.0f && !(mech->adhesion_range > 0.0f))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_motion: adhesion needs adhesion_range > 0");
    if (mech->n_species < 0 || mech->n_species > OLC_MAX_SPECIES)
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_motion: n_species out of range");
    std::string err;
    if (!geom_ok(*geom, &err)) return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_motion: " + err);
    if ((o2 || glucose) && (geom->chem_dims[0] < 1 || geom->chem_dims[1] < 1 || geom->chem_dims[2] < 1))
        return fail(nullptr, OLC_ERR_ARG, "olc_stage_contact_motion: chemotaxis needs chem_dims");
    if (n == 0) return OLC_OK;
    ContactDev d;
    for (int i = 0; i < 3; ++i) {
        d.tdims[i] = geom->tissue_dims[i];
        d.lo[i] = geom->domain_lo[i] + spec->margin;
        d.hi[i] = geom->domain_hi[i] - spec->margin;
    }
    d.tvs = geom->tissue_voxel_size;
    d.stiffness = spec->stiffness;
    d.mobility = spec->mobility;
    d.max_disp = spec->max_disp;
    d.dt = dt;
    MechDev m = {};
    m.state = state;
    m.necrotic_factor = mech->necrotic_factor;
    m.adh_k = mech->adhesion_stiffness;
    m.adh_range = mech->adhesion_range;
    if (mech->velocity_field >= 0) {
        m.vx = vx;
        m.vy = vy;
        m.vz = vz;
    }
    m.damping = mech->damping;
    m.max_speed = mech->max_speed;
    m.species = species;
    m.rng = rng;
    m.f0 = o2;
    m.f1 = glucose;
    for (int i = 0; i < 3; ++i) m.cdims[i] = geom->chem_dims[i];
    m.cvs = geom->chem_voxel_size;
    m.chemo_force = mech->chemo_force;
    m.impulse = mech->motility_impulse;
    m.n_species = mech->n_species < 1 ? 1 : mech->n_species;
    for (int k = 0; k < OLC_MAX_SPECIES; ++k) {
        m.sp_o2[k] = mech->species[k].chemotaxis_o2;
        m.sp_glu[k] = mech->species[k].chemotaxis_glucose;
        m.sp_move[k] = mech->species[k].move_prob;
    }
    launch_contact_mech(reinterpret_cast<const float4*>(posr), ranges, nullptr, n, n, d, m, x, y, z,
                        as_stream(stream));
    return cuda_status(cudaGetLastError(), "olc_stage_contact_motion");
}

}  // extern "C"

// ------------------------------------------------------------------ tuning
int olc_set_tuning(OlcSim* s, const OlcTuning* t) {
    if (!s || !t) return fail(s, OLC_ERR_ARG, "olc_set_tuning: null argument");
    if (!stencil_tile_known(t->stencil_tile_y, t->stencil_tile_z))
        return fail(s, OLC_ERR_ARG, "olc_set_tuning: stencil tile (" + std::to_string(t->stencil_tile_y) + ", " +
                                        std::to_string(t->stencil_tile_z) +
                                        ") is not one of (8,8), (16,8), (8,16), (16,4)");
    if (t->contact_variant != OLC_CONTACT_FLAT && t->contact_variant != OLC_CONTACT_NESTED)
        return fail(s, OLC_ERR_ARG, "olc_set_tuning: contact_variant must be an OLC_CONTACT_* value");
    if (t->batch_tile_depth != 8 && t->batch_tile_depth != 16 && t->batch_tile_depth != 32)
        return fail(s, OLC_ERR_ARG, "olc_set_tuning: batch_tile_depth must be 8, 16 or 32");
    if (!pair_threads_known(t->stencil_pair_threads) || t->stencil_pair_planes < 0 || t->stencil_pair_planes > 4096)
        return fail(s, OLC_ERR_ARG, "olc_set_tuning: stencil_pair_threads must be 0, 128, 256, 512 or 1024 and "
                                    "stencil_pair_planes in [0, 4096]");
    if (t->stencil_l2_keep_pct < 0 || t->stencil_l2_keep_pct > 100)
        return fail(s, OLC_ERR_ARG, "olc_set_tuning: stencil_l2_keep_pct must be in [0, 100]");
    OLC_TRY(check(s, cudaDeviceSynchronize(), "sync"));
    drop_graphs(s);
    const bool depth_changed = t->batch_tile_depth != s->tuning.batch_tile_depth;
    s->tuning = *t;
    // solo handles: the FP32 fields' tensor maps for the new tile
    if (!s->n_sims) {
        for (olc_u32 f = 0; f < s->caps.n_fields; ++f) {
            if (!s->field_bound[f] || s->fstep[f].storage != OLC_FIELD_F32 || s->fstep[f].substeps == 0) continue;
            make_field_maps(&s->fmaps[f], s->field[0][f], s->field[1][f], s->geom.chem_dims, t->stencil_tile_y,
                            t->stencil_tile_z, t->stencil_pair_threads, t->stencil_pair_planes,
                            t->stencil_l2_keep_pct);
        }
    } else if (depth_changed && !s->pool) {
        for (olc_u32 f = 0; f < s->caps.n_fields; ++f)
            if (s->field_bound[f] && s->fstep[f].storage == OLC_FIELD_F32) OLC_TRY(build_batch_field_tiles(s, (int)f));
    } else if (depth_changed) {
        s->pool_dirty = true;
    }
    return OLC_OK;
}

int olc_get_tuning(const OlcSim* s, OlcTuning* out) {
    if (!s || !out) return fail(nullptr, OLC_ERR_ARG, "olc_get_tuning: null argument");
    *out = s->tuning;
    return OLC_OK;
}

int olc_set_batch_tile_depths(OlcSim* s, const int32_t* depths, uint32_t n) {
    if (!s) return fail(nullptr, OLC_ERR_ARG, "null handle");
    if (!s->n_sims || s->pool) return fail(s, OLC_ERR_STATE, "olc_set_batch_tile_depths: not a batch handle");
    if (n != s->n_sims || !depths) return fail(s, OLC_ERR_ARG, "olc_set_batch_tile_depths: one depth per member");
    for (uint32_t k = 0; k < n; ++k)
        if (depths[k] != 0 && depths[k] != 8 && depths[k] != 16 && depths[k] != 32)
            return fail(s, OLC_ERR_ARG, "olc_set_batch_tile_depths: depths must be 0 (the handle's), 8, 16 or 32");
    OLC_TRY(check(s, cudaDeviceSynchronize(), "sync"));
    drop_graphs(s);
    s->member_depth.assign(depths, depths + n);
    for (olc_u32 f = 0; f < s->caps.n_fields; ++f)
        if (s->field_bound[f] && s->fstep[f].storage == OLC_FIELD_F32) OLC_TRY(build_batch_field_tiles(s, (int)f));
    return OLC_OK;
}
