// Host-side declarations shared by the translation units of libolc.so.
#pragma once
#include <cuda.h>  // CUtensorMap type; no driver-library link (entry points via the runtime)
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <string>

#include "olc_device.cuh"
#include "olc_rule_rt.cuh"
#include "../../include/olc.h"

namespace olc {

constexpr int RADIX = 256;
constexpr int SORT_THREADS = 256;
constexpr int SORT_IPT = 16;
constexpr int SORT_TILE = SORT_THREADS * SORT_IPT;
constexpr int MAX_PASSES = 4;

// Geometry of the bin grid as the kernels see it.
struct BinGrid {
    int dims[3];
    float vs;
    olc_u32 sentinel;  // tissue_key(dims): key of dead rows, voxel_table_size - 1
};

BinGrid make_bin_grid(const OlcGeom& g);
int key_bits_for(olc_u32 max_key);

// Thread-local error message for stateless entry points.
void set_error(const std::string& msg);
const char* get_error();
int cuda_status(cudaError_t e, const char* what);

// ------------------------------------------------------------------ grid
// Keys of rows [0, n) (n = n_dev ? *n_dev : n_host); dead rows get the
// sentinel.  When hist != null the 8-bit digit histograms of `passes` passes
// are accumulated into hist (passes x 256 words) and dead rows are counted
// into dead_ctr.
// With counters != null the row count is olc_total_rows(counters).
void launch_keys(const float* x, const float* y, const float* z, const unsigned char* dead,
                 const olc_u32* n_dev, olc_u32 n_host, const olc_u32* counters, olc_u32 n_cap,
                 const BinGrid& g, olc_u32* keys, olc_u32* hist, int passes, olc_u32* dead_ctr,
                 cudaStream_t s);

void launch_digit_hist(const olc_u32* keys, const olc_u32* n_dev, olc_u32 n_host, olc_u32 n_cap,
                       olc_u32* hist, int passes, cudaStream_t s);

// Exclusive scan of each pass's histogram into base; zeroes the pass tile
// counters.  With counters != null also commits the step's compaction:
// N <- rows - dead, DEAD <- dead, births and rule tile counters reset.
void launch_scan_hist(const olc_u32* hist, olc_u32* base, int passes, olc_u32* tile_ctrs,
                      olc_u32* counters, olc_u32 capacity, cudaStream_t s);

void launch_onesweep(const olc_u32* kin, const olc_u32* vin, olc_u32* kout, olc_u32* vout,
                     const olc_u32* n_dev, olc_u32 n_host, olc_u32 n_cap, int shift, int bits,
                     const olc_u32* base, olc_u32* lookback, olc_u32* tile_ctr, olc_u32* status,
                     cudaStream_t s);

size_t sort_scratch_bytes(olc_u32 n, int key_bits);

// Full sort on caller scratch (n rows; n_dev optional).  keys/vals in may
// alias nothing in scratch; the result lands in kout/vout.  When `keys_ready`
// the histogram in scratch was already accumulated by launch_keys.
struct SortScratch {
    olc_u32* hist;      // MAX_PASSES x 256
    olc_u32* base;      // MAX_PASSES x 256
    olc_u32* tile_ctr;  // MAX_PASSES
    olc_u32* status;    // 1
    olc_u32* lookback;  // passes x tiles x 256
    olc_u32* kalt;      // n
    olc_u32* valt;      // n
    size_t lookback_words;
};
bool carve_sort_scratch(void* base, size_t bytes, olc_u32 n_cap, int key_bits, SortScratch* out);
void run_sort(const olc_u32* kin, const olc_u32* vin, olc_u32* kout, olc_u32* vout,
              const olc_u32* n_dev, olc_u32 n_host, olc_u32 n_cap, int key_bits,
              const SortScratch& sc, bool hist_ready, olc_u32* counters, olc_u32 capacity,
              cudaStream_t s);

void launch_bin_ranges(const olc_u32* keys, const olc_u32* n_dev, olc_u32 n_host, olc_u32 n_cap,
                       olc_u32 n_bins, olc_u32* ranges, cudaStream_t s);

struct PermuteArgs {
    const void* src[OLC_MAX_AGENT_COLS];
    void* dst[OLC_MAX_AGENT_COLS];
    int ncols;
    int radius_col;
    float radius_const;
    int write_posr;
    float4* posr;
    unsigned char* life;
};
void launch_permute(const olc_u32* idx, olc_u32* counters, olc_u32 n_cap, const PermuteArgs& a,
                    cudaStream_t s);

// ------------------------------------------------------------------ field
struct FieldStep {
    int dims[3];
    float r;           // D * dt_sub / dx^2
    float inv_decay;   // 1 / (1 + lambda * dt_sub) (FP32 storage; 1 for 16-bit storage)
    float bval;
    float sink_dt;     // dt of the implicit sink
    int substeps;
    int storage;       // OLC_FIELD_F32 / OLC_FIELD_BF16 / OLC_FIELD_F16
    float decay_step;  // 16-bit storage: (1 + lambda dt/S)^-S, applied once per step by the reaction
    // 16-bit encodings (OLC_ENC_*): constants in FP32, computed once on the host
    int encoding;
    float dec_sub;     // b * (1 - inv_decay): a deficit substep adds it after the decay factor
    float dec_step;    // b * (1 - decay_step): a deficit reaction adds it after decay_step
    float half_b;      // b / 2: the middle offset of OLC_ENC_OFFSET3
    float quarter_b;   // b / 4: below it OLC_ENC_OFFSET3 uses offset 0
    float upper_q;     // b - b / 4: above it OLC_ENC_OFFSET3 uses offset b
};
bool make_field_step(const OlcDiffusion& d, const int dims[3], float dx, float dt, FieldStep* out,
                     std::string* err);
// The type word device code reads a field by: storage | (encoding << 8).
inline int field_type_word(const FieldStep& fs) { return fs.storage | (fs.encoding << 8); }
void launch_sink(float* f, float* sink, const FieldStep& fs, cudaStream_t s);
// Voxels held at a value after every substep (x-fastest indices, device memory).
struct Pins {
    const olc_u32* idx;
    olc_u32 n;
    float value;
};
void launch_pins(float* f, const Pins* pins, cudaStream_t s);
void launch_substep(const float* in, float* out, const FieldStep& fs, cudaStream_t s);
// Runs sink + S substeps starting from a; returns the buffer holding the result.
float* run_field_step(float* a, float* b, float* sink, const FieldStep& fs, cudaStream_t s,
                      const Pins* pins = nullptr);
// The S substeps alone.
float* run_substeps(float* a, float* b, const FieldStep& fs, cudaStream_t s, const Pins* pins = nullptr);
// TMA tile path (x extent must be a multiple of 4): tensor maps of both
// buffers for the single-substep kernel and for the T-substep temporal block.
struct FieldMaps {
    bool ok = false;
    int VY = 8, VZ = 8;  // tile of k_substep_x4: rows and planes (a compiled shape)
    CUtensorMap vec[2];
    // two substeps per pass (k_substep_pair): threads per CTA (0: off), output
    // rows per CTA, planes per CTA (0: as many as fill one wave of CTAs)
    int pair_nt = 0, pair_ty = 0, pair_zl = 0;
    CUtensorMap pair[2];
    int keep = 0;  // planes [0, keep) kept L2-resident across substeps by eviction hints (0: none)
};
// The TMA tensor maps of a FP32 field's two buffers for the (tile_y, tile_z)
// tile; false when the tile is not compiled in or the field cannot be mapped
// (the plain kernel runs then).
bool make_field_maps(FieldMaps* m, float* a, float* b, const int dims[3], int tile_y = 8, int tile_z = 8,
                     int pair_threads = 0, int pair_planes = 0, int keep_pct = 0);
// k_substep_pair's output rows per CTA of nt threads on a field (0: it does
// not apply), and whether nt is a compiled CTA size (0 included: off).
int pair_rows(int nt, const int dims[3]);
bool pair_threads_known(int nt);
// Kernel launches of run_substeps_tma for one field step.
int substep_launches(const FieldMaps& m, const FieldStep& fs, const Pins* pins);
bool stencil_tile_known(int tile_y, int tile_z);
// Runs fs.substeps substeps starting from a (buffer index a_index of m).
float* run_substeps_tma(float* a, float* b, const FieldMaps& m, int a_index, const FieldStep& fs, olc_u32* status,
                        cudaStream_t s, const Pins* pins = nullptr);
bool encode_map_elems(CUtensorMap* map, void* base, const int dims[3], const cuuint32_t box[3], int elem_bytes);

// 16-bit field storage (olc_field16.cu): fields stored as BF16 or FP16,
// every update computed in FP32.  Per step: one reaction pass (uptake and the
// step's decay, with the FP32 rounding residual of each voxel kept in `comp`
// and added back the next step, i.e. Kahan-compensated), then S diffusion
// substeps that round each result to the storage type.
struct FieldMaps16 {
    bool ok = false;
    CUtensorMap map[2];
};
bool make_field_maps16(FieldMaps16* m, void* a, void* b, const int dims[3]);
void launch_react16(void* f, float* sink, float* comp, const FieldStep& fs, cudaStream_t s);
// Runs fs.substeps substeps from buffer a_index of (a, b); returns the buffer holding the result.
// step_ctr (device, else step_host) and field salt stochastic rounding.
void* run_substeps16(void* a, void* b, const FieldMaps16& m, int a_index, const FieldStep& fs, olc_u32* status,
                     const olc_u32* step_ctr, olc_u32 step_host, int field, cudaStream_t s);

olc_u32* stage_status_word();

// ------------------------------------------------------------------ contact
struct ContactDev {
    int tdims[3];
    float tvs;
    float stiffness, mobility, max_disp, dt;
    float lo[3], hi[3];
};
void launch_contact(const float4* posr, const olc_u32* ranges, const olc_u32* n_dev, olc_u32 n_host,
                    olc_u32 n_cap, const ContactDev& c, float* x, float* y, float* z, cudaStream_t s,
                    int variant = OLC_CONTACT_FLAT, olc_u32 n_table = 0);
// The rest of the engine's force law (OlcMechanics): necrotic repulsion
// factor, adhesion, damped velocity integration.
struct MechDev {
    const int* state;        // null: no agent is necrotic
    float necrotic_factor;
    float adh_k, adh_range;  // adh_k == 0: no adhesion
    float* vx;               // null: overdamped (ContactDev.mobility, max_disp)
    float* vy;
    float* vz;
    float damping, max_speed;
    // active motion (non-necrotic agents): chemotaxis up the field gradients
    // and random motility from the agent's RNG
    const int* species;      // null: record 0
    olc_u32* rng;            // null: no motility
    const void* f0;          // O2 (current buffer), or null
    const void* f1;          // glucose, or null
    int f0_type, f1_type;    // field type words (field_type_word)
    float f0_b, f1_b;        // their boundary values (the encodings' b)
    int cdims[3];
    float cvs;
    float chemo_force, impulse;
    int n_species;
    float sp_o2[OLC_MAX_SPECIES], sp_glu[OLC_MAX_SPECIES], sp_move[OLC_MAX_SPECIES];
};
void launch_contact_mech(const float4* posr, const olc_u32* ranges, const olc_u32* n_dev, olc_u32 n_host,
                         olc_u32 n_cap, const ContactDev& c, const MechDev& m, float* x, float* y, float* z,
                         cudaStream_t s);

// ------------------------------------------------------------------ reductions
struct ReduceArgs {
    const float* x;
    const float* y;
    const float* z;
    const int* state;       // may be null
    const unsigned char* life;
    float cx, cy, cz;
    float bin_width;
};
// Block partials of the FP64 sums (4 agent sums, then one per field, each
// RED_MAX_BLOCKS long) and one ticket per reduction kernel (zero at rest).
constexpr olc_u32 RED_MAX_BLOCKS = 148 * 4;
constexpr size_t RED_PARTIALS = (size_t)(4 + OLC_MAX_FIELDS) * RED_MAX_BLOCKS;
constexpr int RED_TICKETS = 1 + OLC_MAX_FIELDS;
struct RedScratch {
    double* partials;
    olc_u32* tickets;
};
void launch_reduce_agents(const ReduceArgs& a, const olc_u32* counters, olc_u32 n_cap,
                          OlcReductions* out_dev, const RedScratch& rs, cudaStream_t s);
void launch_reduce_field(const float* f, size_t nvox, int slot, OlcReductions* out_dev, const RedScratch& rs,
                         cudaStream_t s);
void launch_reset_reductions(OlcReductions* out_dev, int nfields, cudaStream_t s);
void launch_reduce_field16(const void* f, const float* comp, const FieldStep& fs, int slot, OlcReductions* out,
                           const RedScratch& rs, cudaStream_t s);

// ------------------------------------------------------------------ engine metrics
// Inputs of k_engine_metrics (olc_metrics.cu): current agent columns (optional
// ones null), the current buffers of the sampled fields, and the bin table.
struct EngineMetricArgs {
    const float* x;
    const float* y;
    const float* z;
    const unsigned char* life;
    const int* state;
    const int* csc;
    const float* energy;
    const float* speed_x;
    const float* speed_y;
    const float* speed_z;
    const void* f0;
    const void* f1;
    int f0_type, f1_type;  // field type words (field_type_word)
    float f0_b, f1_b;
    int cdims[3];
    float cvs;
    const uint2* ranges;
    int tdims[3];
    float tvs;
    float cx, cy, cz;
    float hypoxia;
    int crowd;
    double step;
};
// Device accumulators; `out` receives the 23 finalized values.
struct EngineMetricAcc {
    olc_u32 counts[6];
    olc_u32 ticket;
    olc_u32 pad;
    double max_r;
    double out[OLC_ENGINE_METRICS];
};
constexpr olc_u32 EM_MAX_BLOCKS = 148 * 4;
constexpr size_t EM_PARTIALS = 8 * (size_t)EM_MAX_BLOCKS;  // doubles
void launch_engine_metrics(const EngineMetricArgs& a, const olc_u32* counters, olc_u32 n_cap, EngineMetricAcc* acc,
                           double* partials, cudaStream_t s);

void launch_rng(olc_u32* states, olc_u32 n, int draws, float* out, float* dirs, cudaStream_t s);

// ------------------------------------------------------------------ batched mode (olc_batch.cu)
struct BatchArgs {
    const OlcSimDesc* sims;  // device, n_sims records
    int shift;               // sort key = (simulation << shift) | bin key
    olc_u32 sentinel;        // key of dead rows: n_sims << shift
    olc_u32 n_sims;
};
void launch_keys_batch(const BatchArgs& b, const float* x, const float* y, const float* z, const olc_u32* sim,
                       const unsigned char* dead, const olc_u32* counters, olc_u32 n_cap, olc_u32* keys,
                       olc_u32* hist, int passes, olc_u32* dead_ctr, cudaStream_t s);
void launch_bin_ranges_batch(const BatchArgs& b, const olc_u32* keys, const olc_u32* n_dev, olc_u32 n_cap,
                             olc_u32* ranges, cudaStream_t s);
void launch_contact_batch(const BatchArgs& b, const float4* posr, const olc_u32* ranges, const olc_u32* sim,
                          const olc_u32* n_dev, olc_u32 n_cap, const ContactDev& c, float* x, float* y, float* z,
                          cudaStream_t s);
// Field tiles: uint4 (simulation, tile x, tile y, tile z) of BATCH_TILE_X x
// BATCH_TILE_Y x BATCH_TILE_Z voxels.
constexpr int BATCH_TILE_X = 32, BATCH_TILE_Y = 16, BATCH_TILE_Z = 16;
// Substeps of a batch: FP32 fields on BATCH_TILE tiles with plain loads
// (olc_batch.cu); 16-bit fields on TMA tiles of k_substep16's 64 x 16 x 8
// geometry (olc_field16.cu), each member's grid read through its tensor maps
// (maps[2 * (member * n_fields + field) + buffer], box from batch_substep_box).
constexpr int BATCH_T16_TX = 64, BATCH_T16_TY = 16, BATCH_T16_TZ = 8;
void batch_substep_box(int storage, cuuint32_t box[3]);
void launch_substep_batch(const BatchArgs& b, const uint4* tiles, olc_u32 n_tiles, const FieldStep* steps, int field,
                          int n_fields, const unsigned char* fpar, int sub, float* fa, float* fb, cudaStream_t s);
void launch_substep_batch_t16(const BatchArgs& b, int storage, int encoding, const uint4* tiles, olc_u32 n_tiles,
                              const FieldStep* steps, const CUtensorMap* maps, int field, int n_fields,
                              const unsigned char* fpar, int sub, void* fa, void* fb, const olc_u32* step_ctr,
                              olc_u32* status, cudaStream_t s);
void launch_sink_batch(const BatchArgs& b, const uint4* tiles, olc_u32 n_tiles, const FieldStep* steps, int field,
                       int n_fields, const unsigned char* fpar, float* fa, float* fb, float* sink, cudaStream_t s);
void launch_flip_parity_all(int n_fields, olc_u32 n_sims, unsigned char* fpar, cudaStream_t s);
void launch_flip_parity(const FieldStep* steps, int field, int n_fields, olc_u32 n_sims, unsigned char* fpar,
                        cudaStream_t s);
void launch_reduce_agents_batch(const BatchArgs& b, const ReduceArgs& a, const olc_u32* sim, const olc_u32* counters,
                                olc_u32 n_cap, OlcReductions* out, cudaStream_t s);
void launch_reduce_field_batch(const BatchArgs& b, const uint4* tiles, olc_u32 n_tiles, int field, int n_fields,
                               const unsigned char* fpar, const float* fa, const float* fb, OlcReductions* out,
                               cudaStream_t s);
void launch_reset_reductions_batch(OlcReductions* out, olc_u32 n_sims, cudaStream_t s);
void launch_react_batch16(const BatchArgs& b, int storage, int encoding, const uint4* tiles, olc_u32 n_tiles,
                          const FieldStep* steps, int field, int n_fields, const unsigned char* fpar, void* fa,
                          void* fb, float* sink, float* comp, cudaStream_t s);
void launch_reduce_field_batch16(const BatchArgs& b, int storage, int encoding, const uint4* tiles, olc_u32 n_tiles,
                                 const FieldStep* steps, int field, int n_fields, const unsigned char* fpar,
                                 const void* fa, const void* fb, const float* comp, OlcReductions* out,
                                 cudaStream_t s);

// ------------------------------------------------------------------ serving pool (olc_pool.cu)
// Column pointer sets of the row kernels; every column holds 4-byte elements.
struct PoolCols {
    const void* src[OLC_MAX_AGENT_COLS];
    void* dst[OLC_MAX_AGENT_COLS];  // gather: null columns are skipped
    int ncols;
    int sim_col;                    // append: this column is written with the slot
};
constexpr olc_u32 POOL_GATHER_BLOCKS = 592;  // 4 per SM; the scan takes <= 1024 block counts
constexpr olc_u32 POOL_TABLE_CHUNK = 8192;    // bin-table entries cleared per block
void launch_clear_table_chunks(const uint2* chunks, olc_u32 n_chunks, olc_u32* ranges, cudaStream_t s);
void launch_pool_append(const PoolCols& cols, olc_u32 n, olc_u32 slot, unsigned char* life, olc_u32* counters,
                        olc_u32 capacity, cudaStream_t s);
void launch_pool_retire(const olc_u32* sim, unsigned char* life, const olc_u32* counters, olc_u32 n_cap,
                        olc_u32 slot, cudaStream_t s);
void launch_pool_gather(const PoolCols& cols, const olc_u32* sim, const unsigned char* life, const olc_u32* counters,
                        olc_u32 slot, olc_u32* block_counts, olc_u32* count_out, olc_u32 max_rows, cudaStream_t s);

}  // namespace olc
