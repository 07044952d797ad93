"""ctypes binding of libolc.so (include/olc.h).

The library is the only implementation of the step: there is no CPU path.  If
it cannot be loaded, every entry point raises ``OlcError``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libolc.so")
CSRC_DIR = os.path.join(HERE, "csrc")

OLC_OK = 0
OLC_ERR_ARG = 1
OLC_ERR_NVRTC = 2
OLC_ERR_CUDA = 3
OLC_ERR_CAPACITY = 4
OLC_ERR_TIMEOUT = 5
OLC_ERR_STATE = 6

OLC_STATUS_CAPACITY = 0x1
OLC_STATUS_TIMEOUT = 0x2
OLC_STATUS_MULTI_DIVIDE = 0x4

OLC_ENC_VALUE = 0
OLC_ENC_DEFICIT = 1
OLC_ENC_OFFSET3 = 2

OLC_MAX_AGENT_FIELDS = 64
OLC_MAX_FIELDS = 8
OLC_MAX_RULES = 16
OLC_RADIAL_BINS = 64
OLC_STATE_BINS = 8
# pinned host slots of olc_queue_readback / olc_take_readback
READBACK_SLOTS = 4

# Every symbol include/olc.h declares (the loader checks each one).
EXPORTS = (
    "olc_create", "olc_destroy", "olc_last_error", "olc_version",
    "olc_bind_agent_column", "olc_bind_field", "olc_set_contact", "olc_set_rule_source",
    "olc_set_params", "olc_set_agent_count", "olc_current_buffers", "olc_step", "olc_set_graphs",
    "olc_read_counters", "olc_read_reductions", "olc_read_user_metrics",
    "olc_set_user_metrics_size", "olc_read_life", "olc_nvrtc_check", "olc_bind_tissue",
    "olc_set_profiling", "olc_read_profile", "olc_stage_sort_pairs_noalloc",
    "olc_stage_rng", "olc_stage_keys", "olc_sort_scratch_bytes", "olc_stage_sort_pairs",
    "olc_stage_bin_ranges", "olc_stage_diffuse", "olc_stage_contact",
    "olc_create_batch", "olc_batch_field_offsets", "olc_bind_field_batch", "olc_set_params_batch",
    "olc_read_field_parity", "olc_read_reductions_batch", "olc_read_user_metrics_batch",
    "olc_bind_field_ex", "olc_stage_diffuse16",
    "olc_create_pool", "olc_bind_field_pool", "olc_pool_admit", "olc_pool_add_agents", "olc_pool_gather",
    "olc_pool_copy_results", "olc_pool_retire", "olc_pool_usage",
    "olc_arena_create", "olc_arena_alloc", "olc_arena_release", "olc_arena_stats", "olc_arena_destroy",
    "olc_engine_metrics", "olc_get_step_state", "olc_set_step_state", "olc_set_mechanics",
    "olc_stage_contact_mech", "olc_stage_contact_motion", "olc_bind_tissue_pair", "olc_current_tissue", "olc_set_rule_iterations",
    "olc_set_pinned", "olc_stage_diffuse_pinned", "olc_sort_noalloc_status", "olc_sort_status_offset",
    "olc_selftest_bounded_waits", "olc_set_tuning", "olc_get_tuning", "olc_set_batch_tile_depths",
    "olc_stage_diffuse_tuned", "olc_stage_contact_tuned", "olc_queue_readback", "olc_take_readback",
)


class OlcError(RuntimeError):
    """A libolc entry point returned an error status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"libolc error {code}: {message}")
        self.code = code


_STATUS_NAMES = ((OLC_STATUS_CAPACITY, "capacity (children dropped: max_agents reached)"),
                 (OLC_STATUS_TIMEOUT, "timeout (a bounded device wait gave up: results of that step are unreliable)"),
                 (OLC_STATUS_MULTI_DIVIDE, "multi_divide (a rule called divide() twice in one call)"))


def status_names(bits: int) -> str:
    """The OLC_STATUS_* bits of a device status word, by name."""
    names = [n for b, n in _STATUS_NAMES if bits & b]
    rest = bits & ~sum(b for b, _ in _STATUS_NAMES)
    if rest:
        names.append(f"unknown bits {rest:#x}")
    return ", ".join(names) or "clean"


class DeviceStatusError(OlcError):
    """The device status word of a handle gained bits: a capacity overflow
    (children dropped), a bounded wait that gave up, or a second divide() in
    one rule call.  Raised by the host after the steps that set them; the
    error code follows the first bit (OLC_ERR_CAPACITY, OLC_ERR_TIMEOUT,
    OLC_ERR_STATE)."""

    def __init__(self, bits: int, new_bits: int, where: str):
        code = (OLC_ERR_TIMEOUT if new_bits & OLC_STATUS_TIMEOUT else
                OLC_ERR_CAPACITY if new_bits & OLC_STATUS_CAPACITY else OLC_ERR_STATE)
        super().__init__(code, f"{where}: device status {bits:#x}: {status_names(new_bits)}")
        self.status = bits
        self.new_bits = new_bits


class StatusWatch:
    """Checks a handle's sticky device status word every ``every`` steps
    (one counter read, which waits for the stream) and after every step that
    already waited for the device (metric collection).  ``policy`` "raise"
    raises DeviceStatusError when bits appear that were not reported before,
    "warn" issues a RuntimeWarning instead, "ignore" reads nothing.  Each bit
    is reported once; the word itself stays sticky (olc_read_counters)."""

    DEFAULT_EVERY = 64

    def __init__(self, read_status, where: str, every: int = DEFAULT_EVERY, policy: str = "raise"):
        self.read_status = read_status
        self.where = where
        self.every = max(1, int(every))
        self.policy = policy
        self.seen = 0
        self.since = 0

    def chunks(self, n: int):
        """Step counts to enqueue so that no chunk passes a check point."""
        n = int(n)
        while n > 0:
            k = min(n, self.every - self.since) if self.policy != "ignore" else n
            yield k
            n -= k

    def after(self, steps: int, synced: bool = False) -> None:
        self.since += int(steps)
        if self.policy == "ignore" or (self.since < self.every and not synced):
            return
        self.since = 0
        self.check()

    def check(self) -> int:
        return self.report(int(self.read_status()))

    def report(self, bits: int) -> int:
        """The check of ``check`` on a status word read elsewhere (a queued
        readback's counters)."""
        if self.policy == "ignore":
            return bits
        bits = int(bits)
        new = bits & ~self.seen
        self.seen |= bits
        if new:
            err = DeviceStatusError(bits, new, self.where)
            if self.policy == "raise":
                raise err
            if self.policy == "warn":
                import warnings

                warnings.warn(str(err), RuntimeWarning, stacklevel=3)
        return bits


class OlcGeom(C.Structure):
    _fields_ = [
        ("tissue_dims", C.c_int32 * 3),
        ("tissue_voxel_size", C.c_float),
        ("chem_dims", C.c_int32 * 3),
        ("chem_voxel_size", C.c_float),
        ("domain_lo", C.c_float * 3),
        ("domain_hi", C.c_float * 3),
    ]


class OlcCaps(C.Structure):
    _fields_ = [
        ("max_agents", C.c_uint32),
        ("n_agent_fields", C.c_uint32),
        ("n_fields", C.c_uint32),
        ("state_field", C.c_int32),
        ("radial_bin_width", C.c_float),
        ("center", C.c_float * 3),
        ("dt", C.c_float),
    ]


class OlcDiffusion(C.Structure):
    _fields_ = [
        ("diffusion", C.c_float),
        ("decay", C.c_float),
        ("boundary", C.c_float),
        ("substeps", C.c_int32),
        ("has_sink", C.c_int32),
        ("storage", C.c_int32),
        ("encoding", C.c_int32),
    ]


OLC_CONTACT_FLAT = 0
OLC_CONTACT_NESTED = 1


class OlcTuning(C.Structure):
    _fields_ = [
        ("stencil_tile_y", C.c_int32),
        ("stencil_tile_z", C.c_int32),
        ("contact_variant", C.c_int32),
        ("batch_tile_depth", C.c_int32),
        ("stencil_pair_threads", C.c_int32),
        ("stencil_pair_planes", C.c_int32),
        ("stencil_l2_keep_pct", C.c_int32),
    ]


class OlcContact(C.Structure):
    _fields_ = [
        ("enabled", C.c_int32),
        ("radius_field", C.c_int32),
        ("radius_const", C.c_float),
        ("stiffness", C.c_float),
        ("mobility", C.c_float),
        ("max_disp", C.c_float),
        ("margin", C.c_float),
    ]


class OlcCounters(C.Structure):
    _fields_ = [
        ("n_agents", C.c_uint32),
        ("n_total", C.c_uint32),
        ("births", C.c_uint32),
        ("deaths", C.c_uint32),
        ("status", C.c_uint32),
        ("pad", C.c_uint32),
        ("steps", C.c_uint64),
        ("agent_steps", C.c_uint64),
    ]


class OlcProfile(C.Structure):
    _fields_ = [
        ("steps", C.c_uint32),
        ("substep_launches", C.c_uint32),
        ("kernel_launches", C.c_uint64),
        ("ms_sink", C.c_double),
        ("ms_substeps", C.c_double),
        ("ms_grid", C.c_double),
        ("ms_rules", C.c_double),
        ("ms_contact", C.c_double),
        ("ms_collect", C.c_double),
    ]


class OlcReductions(C.Structure):
    _fields_ = [
        ("n_live", C.c_uint32),
        ("state_counts", C.c_uint32 * OLC_STATE_BINS),
        ("radial_hist", C.c_uint32 * OLC_RADIAL_BINS),
        ("pad", C.c_uint32),
        ("sum_pos", C.c_double * 3),
        ("sum_r2", C.c_double),
        ("max_r", C.c_double),
        ("field_mass", C.c_double * OLC_MAX_FIELDS),
        ("field_min", C.c_double * OLC_MAX_FIELDS),
        ("field_max", C.c_double * OLC_MAX_FIELDS),
    ]


OLC_ENGINE_METRICS = 23
# MetricIndex of engine/src/sim/readback.rs:25-50, in output order
ENGINE_METRIC_NAMES = (
    "total_live", "n_prolif", "n_quiesc", "n_necr", "frac_prolif", "frac_quiesc", "frac_necr", "frac_hypoxic",
    "csc_count", "csc_frac", "centroid_x", "centroid_y", "centroid_z", "r_gyration", "r_invasive", "r_necrotic",
    "rim_thickness", "mean_energy", "mean_o2", "mean_glu", "mean_speed", "crowd_frac", "step",
)


class OlcEngineMetricsSpec(C.Structure):
    _fields_ = [
        ("state_field", C.c_int32),
        ("energy_field", C.c_int32),
        ("speed_field", C.c_int32),
        ("csc_field", C.c_int32),
        ("o2_field", C.c_int32),
        ("glucose_field", C.c_int32),
        ("hypoxia_threshold", C.c_float),
        ("crowd_threshold", C.c_int32),
        ("center", C.c_float * 3),
        ("pad", C.c_float),
    ]


OLC_MAX_SPECIES = 8


class OlcSpecies(C.Structure):
    _fields_ = [("chemotaxis_o2", C.c_float), ("chemotaxis_glucose", C.c_float), ("move_prob", C.c_float),
                ("pad", C.c_float)]


class OlcMechanics(C.Structure):
    _fields_ = [
        ("state_field", C.c_int32),
        ("necrotic_factor", C.c_float),
        ("adhesion_stiffness", C.c_float),
        ("adhesion_range", C.c_float),
        ("velocity_field", C.c_int32),
        ("damping", C.c_float),
        ("max_speed", C.c_float),
        ("enabled", C.c_int32),
        ("species_field", C.c_int32),
        ("rng_field", C.c_int32),
        ("o2_field", C.c_int32),
        ("glucose_field", C.c_int32),
        ("chemo_force", C.c_float),
        ("motility_impulse", C.c_float),
        ("n_species", C.c_int32),
        ("pad2", C.c_int32),
        ("species", OlcSpecies * OLC_MAX_SPECIES),
    ]


class OlcStepState(C.Structure):
    _fields_ = [
        ("steps", C.c_uint64),
        ("agent_steps", C.c_uint64),
        ("field_step", C.c_uint32),
        ("status", C.c_uint32),
    ]


class OlcPoolConfig(C.Structure):
    _fields_ = [
        ("max_slots", C.c_uint32),
        ("max_tissue_dims", C.c_int32 * 3),
        ("table_entries", C.c_uint64),
        ("field_voxels", C.c_uint64),
    ]


class OlcPoolUsage(C.Structure):
    _fields_ = [
        ("slots_used", C.c_uint32),
        ("max_slots", C.c_uint32),
        ("table_used", C.c_uint64),
        ("table_entries", C.c_uint64),
        ("table_largest_free", C.c_uint64),
        ("field_used", C.c_uint64),
        ("field_voxels", C.c_uint64),
        ("field_largest_free", C.c_uint64),
    ]


_VP = C.c_void_p
_U64P = C.POINTER(C.c_uint64)
_SIGS = {
    "olc_create": (C.c_int, [C.POINTER(OlcGeom), C.POINTER(OlcCaps), C.POINTER(_VP)]),
    "olc_destroy": (C.c_int, [_VP]),
    "olc_last_error": (C.c_char_p, [_VP]),
    "olc_version": (C.c_char_p, []),
    "olc_bind_agent_column": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "olc_bind_field": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP, C.POINTER(OlcDiffusion)]),
    "olc_set_contact": (C.c_int, [_VP, C.POINTER(OlcContact)]),
    "olc_set_rule_source": (C.c_int, [_VP, C.c_char_p, C.POINTER(C.c_char_p), C.POINTER(C.c_int), C.c_int,
                                      C.c_char_p]),
    "olc_set_params": (C.c_int, [_VP, _VP, C.c_size_t, _VP]),
    "olc_set_agent_count": (C.c_int, [_VP, C.c_uint32, _VP]),
    "olc_current_buffers": (C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "olc_step": (C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    "olc_set_graphs": (C.c_int, [_VP, C.c_int]),
    "olc_read_counters": (C.c_int, [_VP, C.POINTER(OlcCounters), _VP]),
    "olc_read_reductions": (C.c_int, [_VP, C.POINTER(OlcReductions), _VP]),
    "olc_read_user_metrics": (C.c_int, [_VP, _VP, C.c_size_t, _VP]),
    "olc_queue_readback": (C.c_int, [_VP, _VP, C.POINTER(C.c_uint64)]),
    "olc_take_readback": (C.c_int, [_VP, C.c_uint64, _VP, C.c_size_t, C.POINTER(OlcCounters)]),
    "olc_create_batch": (C.c_int, [C.POINTER(OlcGeom), C.c_int, C.POINTER(OlcCaps), C.POINTER(_VP)]),
    "olc_batch_field_offsets": (C.c_int, [_VP, C.POINTER(C.c_uint64)]),
    "olc_bind_field_batch": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP, _VP, C.POINTER(OlcDiffusion)]),
    "olc_bind_field_ex": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP, _VP, C.POINTER(OlcDiffusion)]),
    "olc_stage_diffuse16": (C.c_int, [_VP, _VP, _VP, _VP, C.POINTER(C.c_int32 * 3), C.c_float, C.c_float,
                                      C.POINTER(OlcDiffusion), C.c_uint32, C.c_int, _VP]),
    "olc_set_params_batch": (C.c_int, [_VP, _VP, C.c_size_t, _VP]),
    "olc_read_field_parity": (C.c_int, [_VP, C.POINTER(C.c_uint8), _VP]),
    "olc_read_reductions_batch": (C.c_int, [_VP, C.POINTER(OlcReductions), _VP]),
    "olc_read_user_metrics_batch": (C.c_int, [_VP, _VP, C.c_size_t, _VP]),
    "olc_set_user_metrics_size": (C.c_int, [_VP, C.c_size_t]),
    "olc_read_life": (C.c_int, [_VP, _VP, C.c_uint32, _VP]),
    "olc_nvrtc_check": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]),
    "olc_bind_tissue": (C.c_int, [_VP, _VP, C.c_int, C.c_size_t]),
    "olc_set_profiling": (C.c_int, [_VP, C.c_int]),
    "olc_read_profile": (C.c_int, [_VP, C.POINTER(OlcProfile)]),
    "olc_stage_sort_pairs_noalloc": (C.c_int, [_VP, _VP, _VP, _VP, C.c_uint32, C.c_int, _VP]),
    "olc_stage_rng": (C.c_int, [_VP, C.c_uint32, C.c_int, _VP, _VP, _VP]),
    "olc_stage_keys": (C.c_int, [_VP, _VP, _VP, _VP, C.c_uint32, C.POINTER(OlcGeom), _VP, _VP]),
    "olc_sort_scratch_bytes": (C.c_size_t, [C.c_uint32, C.c_int]),
    "olc_stage_sort_pairs": (C.c_int, [_VP, _VP, _VP, _VP, C.c_uint32, C.c_int, _VP, C.c_size_t, _VP]),
    "olc_stage_bin_ranges": (C.c_int, [_VP, C.c_uint32, C.c_uint32, _VP, _VP]),
    "olc_stage_diffuse": (C.c_int, [_VP, _VP, _VP, C.POINTER(C.c_int32 * 3), C.c_float, C.c_float,
                                    C.POINTER(OlcDiffusion), _VP]),
    "olc_stage_diffuse_tuned": (C.c_int, [_VP, _VP, _VP, C.POINTER(C.c_int32 * 3), C.c_float, C.c_float,
                                          C.POINTER(OlcDiffusion), C.POINTER(OlcTuning), _VP]),
    "olc_stage_contact": (C.c_int, [_VP, _VP, C.c_uint32, C.POINTER(OlcGeom), C.POINTER(OlcContact), C.c_float,
                                    _VP, _VP, _VP, _VP]),
    "olc_stage_contact_tuned": (C.c_int, [_VP, _VP, C.c_uint32, C.POINTER(OlcGeom), C.POINTER(OlcContact),
                                          C.c_float, C.c_int32, _VP, _VP, _VP, _VP]),
    "olc_create_pool": (C.c_int, [C.POINTER(OlcPoolConfig), C.POINTER(OlcCaps), C.POINTER(_VP)]),
    "olc_bind_field_pool": (C.c_int, [_VP, C.c_int, _VP, _VP, _VP, _VP, C.c_int, C.c_int, C.c_float]),
    "olc_pool_admit": (C.c_int, [_VP, C.POINTER(OlcGeom), C.POINTER(OlcDiffusion), _VP, C.c_size_t,
                                 C.POINTER(C.c_int32), _U64P, _VP]),
    "olc_pool_add_agents": (C.c_int, [_VP, C.c_int32, C.POINTER(_VP), C.c_uint32, _VP]),
    "olc_pool_gather": (C.c_int, [_VP, C.c_int32, C.POINTER(_VP), C.c_uint32, _VP, _VP]),
    "olc_pool_copy_results": (C.c_int, [_VP, C.c_int32, _VP, _VP, _VP]),
    "olc_pool_retire": (C.c_int, [_VP, C.c_int32, _VP]),
    "olc_pool_usage": (C.c_int, [_VP, C.POINTER(OlcPoolUsage)]),
    "olc_arena_create": (C.c_int, [C.c_uint64, C.POINTER(_VP)]),
    "olc_arena_alloc": (C.c_int, [_VP, C.c_uint64, C.c_uint64, _U64P]),
    "olc_arena_release": (C.c_int, [_VP, C.c_uint64, C.c_uint64]),
    "olc_arena_stats": (C.c_int, [_VP, _U64P, _U64P, _U64P]),
    "olc_arena_destroy": (C.c_int, [_VP]),
    "olc_engine_metrics": (C.c_int, [_VP, C.POINTER(OlcEngineMetricsSpec), C.POINTER(C.c_double), _VP]),
    "olc_get_step_state": (C.c_int, [_VP, C.POINTER(OlcStepState), _VP]),
    "olc_set_mechanics": (C.c_int, [_VP, C.POINTER(OlcMechanics)]),
    "olc_bind_tissue_pair": (C.c_int, [_VP, _VP, _VP, C.c_int, C.c_size_t]),
    "olc_set_pinned": (C.c_int, [_VP, C.c_int, _VP, C.c_uint32, C.c_float]),
    "olc_stage_diffuse_pinned": (C.c_int, [_VP, _VP, _VP, C.POINTER(C.c_int32 * 3), C.c_float, C.c_float,
                                           C.POINTER(OlcDiffusion), _VP, C.c_uint32, C.c_float, _VP]),
    "olc_stage_contact_motion": (C.c_int, [_VP, _VP, C.c_uint32, C.POINTER(OlcGeom), C.POINTER(OlcContact),
                                           C.POINTER(OlcMechanics), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                                           C.c_float, _VP, _VP, _VP, _VP]),
    "olc_current_tissue": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "olc_set_rule_iterations": (C.c_int, [_VP, C.POINTER(C.c_int), C.c_int]),
    "olc_stage_contact_mech": (C.c_int, [_VP, _VP, C.c_uint32, C.POINTER(OlcGeom), C.POINTER(OlcContact),
                                         C.POINTER(OlcMechanics), _VP, _VP, _VP, _VP, C.c_float, _VP, _VP, _VP,
                                         _VP]),
    "olc_set_step_state": (C.c_int, [_VP, C.POINTER(OlcStepState), _VP]),
    "olc_sort_noalloc_status": (C.c_int, [C.POINTER(C.c_uint32), _VP]),
    "olc_sort_status_offset": (C.c_size_t, []),
    "olc_selftest_bounded_waits": (C.c_int, [C.c_uint32, C.POINTER(C.c_uint32 * 3), _VP]),
    "olc_set_tuning": (C.c_int, [_VP, C.POINTER(OlcTuning)]),
    "olc_get_tuning": (C.c_int, [_VP, C.POINTER(OlcTuning)]),
    "olc_set_batch_tile_depths": (C.c_int, [_VP, C.POINTER(C.c_int32), C.c_uint32]),
}

_lock = threading.Lock()
_lib: C.CDLL | None = None


def load(build_if_missing: bool = True) -> C.CDLL:
    """Loads libolc.so (building it with nvcc first when it is missing or stale)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing:
            from oncolytica_b200.build_lib import build
            build()
        if not os.path.exists(LIB_PATH):
            raise OlcError(OLC_ERR_STATE, f"{LIB_PATH} is missing; run python -m oncolytica_b200.build_lib")
        lib = C.CDLL(LIB_PATH)
        for name in EXPORTS:
            fn = getattr(lib, name)
            res, args = _SIGS[name]
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error(handle=None) -> str:
    msg = load().olc_last_error(handle)
    return msg.decode(errors="replace") if msg else ""


def check(rc: int, handle=None) -> None:
    if rc != OLC_OK:
        raise OlcError(rc, last_error(handle))
