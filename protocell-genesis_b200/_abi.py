"""ctypes mirror of include/soup_b200.h and the loader of the native library.

The native library (csrc/ -> libsoup_b200.so) is the product: this module only declares the C
structs and function signatures.  There is deliberately no pure-Python implementation behind any
of these calls -- if the library is missing, every entry point raises.
"""
import ctypes as C
import os

MAX_KINDS = 8
MAX_RULES = 4
ABI_VERSION = 1
NONE = 0xFFFFFFFF

STATUS = {
    0: "SOUP_OK", 1: "SOUP_E_ARG", 2: "SOUP_E_NONFINITE", 3: "SOUP_E_LIST_OVERFLOW",
    4: "SOUP_E_ES_OVERFLOW", 5: "SOUP_E_DRIFT", 6: "SOUP_E_GEOMETRY", 7: "SOUP_E_OOM",
    8: "SOUP_E_TIMEOUT", 9: "SOUP_E_CUDA", 10: "SOUP_E_STATE",
}

# debug phases (soup_debug_phase)
PHASE_REBUILD = 1
PHASE_FORCE = 2
PHASE_KICK_DRIFT = 3
PHASE_KICK_THERMO = 4
PHASE_BONDS = 5
PHASE_MAX_DRIFT = 6


class SoupConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("n", C.c_uint32),
        ("n_kinds", C.c_uint32),
        ("seed", C.c_uint32),
        ("counts", C.c_uint32 * MAX_KINDS),
        ("box", C.c_double * 3),
        ("sigma", C.c_double), ("epsilon", C.c_double), ("b_tt", C.c_double),
        ("k_fene", C.c_double), ("r_inf", C.c_double), ("k_bend", C.c_double),
        ("r_bend", C.c_double), ("wc", C.c_double), ("kT", C.c_double),
        ("gamma", C.c_double), ("dt", C.c_double),
        ("radius", C.c_double * MAX_KINDS),
        ("kind_class", C.c_uint32 * MAX_KINDS),
        ("attr_scale", (C.c_double * 4) * 4),
        ("acid_soap_scale", C.c_double),
        ("interaction_range", C.c_double),
        ("skin", C.c_double),
        ("list_range", C.c_double),
        ("rebuild_every", C.c_uint32),
        ("rebuild_on_drift", C.c_uint32),
        ("list_capacity", C.c_uint32),
        ("es_enabled", C.c_uint32),
        ("charged_kind", C.c_int32),
        ("charge_deprotonated", C.c_double),
        ("es_coeff_a", C.c_double), ("es_kappa", C.c_double), ("es_cutoff", C.c_double),
        ("es_shift_u", C.c_double), ("es_shift_f", C.c_double),
        ("es_split_radius", C.c_double),
        ("es_list_range", C.c_double),
        ("es_list_capacity", C.c_uint32),
        ("pka_intrinsic", C.c_double), ("ph", C.c_double),
        ("sweep_every", C.c_uint32),
        ("protonation_rng", C.c_uint32),
        ("rc_attr", C.c_double),
        ("n_rules", C.c_uint32),
        ("rule_kind_a", C.c_int32 * MAX_RULES), ("rule_kind_b", C.c_int32 * MAX_RULES),
        ("attempt_form", C.c_double * MAX_RULES), ("attempt_break", C.c_double * MAX_RULES),
        ("accept_form", C.c_double * MAX_RULES), ("accept_break", C.c_double * MAX_RULES),
        ("requires_catalyst", C.c_uint32 * MAX_RULES),
        ("role_a", C.c_uint32 * MAX_RULES), ("role_b", C.c_uint32 * MAX_RULES),
        ("catalyst_kind", C.c_int32),
        ("head_terminal_only", C.c_uint32), ("head_chain_capacity", C.c_uint32),
        ("max_hold_steps", C.c_uint32), ("bond_interval", C.c_uint32),
        ("wall_radius", C.c_double), ("wall_k", C.c_double),
        ("global_step", C.c_uint64),
        ("chunk_steps", C.c_uint32),
        ("cell_divisor", C.c_uint32), ("reserved", C.c_uint32 * 6),
    ]


class SoupInitState(C.Structure):
    _fields_ = [
        ("positions", C.c_void_p), ("velocities", C.c_void_p), ("bond_slots", C.c_void_p),
        ("center_link", C.c_void_p), ("center_held", C.c_void_p), ("bond_rng", C.c_void_p),
        ("thermo_rng", C.c_void_p), ("charges", C.c_void_p), ("frozen", C.c_void_p),
        ("events", C.c_void_p), ("desorb_events", C.c_void_p),
    ]


class SoupSweepResult(C.Structure):
    _fields_ = [
        ("attempts", C.c_uint32), ("accepted", C.c_uint32), ("heads", C.c_uint32),
        ("deprotonated", C.c_uint32), ("alpha", C.c_double), ("d_es_mean_kt", C.c_double),
    ]


class SoupClosureResult(C.Structure):
    _fields_ = [
        ("encapsulated_count", C.c_uint32), ("total_water", C.c_uint32),
        ("bulk_water_density", C.c_double), ("threshold_count", C.c_double),
        ("closed", C.c_uint32), ("total_empty_cells", C.c_uint32),
        ("unreached_cells", C.c_uint32), ("seed_cell", C.c_uint32),
        ("seed_dist_from_centre", C.c_double),
    ]


class SoupPairingStats(C.Structure):
    _fields_ = [
        ("heads", C.c_uint32), ("with_neighbour", C.c_uint32), ("unlike_contacts", C.c_uint32),
        ("like_contacts", C.c_uint32), ("paired", C.c_uint32), ("charged", C.c_uint32),
        ("unlike_fraction", C.c_double), ("unlike_fraction_random", C.c_double), ("paired_fraction", C.c_double),
        ("contact_radius", C.c_double), ("alpha", C.c_double),
    ]


class SoupAggregateShape(C.Structure):
    _fields_ = [("size", C.c_uint32), ("label", C.c_uint32), ("centre", C.c_double * 3), ("gyration", C.c_double * 6)]


class SoupTuneResult(C.Structure):
    _fields_ = [
        ("tpp", C.c_uint32), ("walk", C.c_uint32), ("tpp_before", C.c_uint32), ("walk_before", C.c_uint32),
        ("skin_scale", C.c_double), ("ms_per_step_before", C.c_double), ("ms_per_step_after", C.c_double),
        ("queued", C.c_uint32), ("queued_before", C.c_uint32), ("list_cells", C.c_uint32),
    ]


CHECKPOINT_BYTES_PER_PARTICLE = 64
NOALLOC_MAX_MEMBERS = 1 << 18   # SOUP_NOALLOC_MAX_MEMBERS
NOALLOC_MAX_CELLS = 1 << 18     # SOUP_NOALLOC_MAX_CELLS


class SoupCheckpointScalars(C.Structure):
    _fields_ = [
        ("global_step", C.c_uint64), ("n", C.c_uint32), ("n_rules", C.c_uint32),
        ("protonation_rng", C.c_uint32), ("desorb", C.c_uint32 * 2), ("events", C.c_uint32 * (2 * MAX_RULES)),
        ("live_box", C.c_double * 3),
    ]


class SoupInfo(C.Structure):
    _fields_ = [
        ("n", C.c_uint32), ("global_step", C.c_uint64), ("list_capacity", C.c_uint32),
        ("es_list_capacity", C.c_uint32), ("heads", C.c_uint32), ("rebuilds", C.c_uint64),
        ("sweeps", C.c_uint64), ("box", C.c_double * 3), ("max_drift", C.c_double),
    ]


LIB_NAME = "libsoup_b200.so"
_P = C.c_void_p
_SZ = C.c_size_t
_U32P = C.POINTER(C.c_uint32)

# name -> (restype, argtypes); the exported surface of include/soup_b200.h
SIGNATURES = {
    "soup_create": (C.c_int, [C.POINTER(SoupConfig), C.POINTER(SoupInitState), C.POINTER(_P)]),
    "soup_destroy": (None, [_P]),
    "soup_last_error": (C.c_char_p, [_P]),
    "soup_get_info": (C.c_int, [_P, C.POINTER(SoupInfo)]),
    "soup_fresh_state": (C.c_int, [C.POINTER(SoupConfig), _P, _P, _P, _P, _P]),
    "soup_initial_charges": (C.c_int, [C.POINTER(SoupConfig), _P, _P, _U32P]),
    "soup_step": (C.c_int, [_P, C.c_uint64]),
    "soup_relax_cold_start": (C.c_int, [_P, C.c_uint32, C.c_double, C.POINTER(C.c_double)]),
    "soup_read_pos": (C.c_int, [_P, _P, _SZ]),
    "soup_read_vel": (C.c_int, [_P, _P, _SZ]),
    "soup_read_force": (C.c_int, [_P, _P, _SZ]),
    "soup_forces": (C.c_int, [_P, _P, _SZ]),
    "soup_forces_brute": (C.c_int, [_P, _P, _SZ]),
    "soup_read_slots": (C.c_int, [_P, _P, _SZ]),
    "soup_read_center_link": (C.c_int, [_P, _P, _SZ]),
    "soup_read_center_held": (C.c_int, [_P, _P, _SZ]),
    "soup_read_charges": (C.c_int, [_P, _P, _SZ]),
    "soup_read_rng_bond": (C.c_int, [_P, _P, _SZ]),
    "soup_read_rng_thermo": (C.c_int, [_P, _P, _SZ]),
    "soup_read_frozen": (C.c_int, [_P, _P, _SZ]),
    "soup_read_events": (C.c_int, [_P, _P, _SZ]),
    "soup_read_desorb": (C.c_int, [_P, _P, _SZ]),
    "soup_nonfinite_count": (C.c_int, [_P, _U32P]),
    "soup_read_verlet": (C.c_int, [_P, _U32P, _U32P, _SZ]),
    "soup_read_es_list": (C.c_int, [_P, _U32P, _U32P, _SZ]),
    "soup_set_wait_limit": (C.c_int, [_P, C.c_uint32]),
    "soup_read_protonation_rng": (C.c_int, [_P, _U32P]),
    "soup_read_checkpoint": (C.c_int, [_P, _P, _SZ, C.POINTER(SoupCheckpointScalars)]),
    "soup_scale_box": (C.c_int, [_P, C.POINTER(C.c_double), C.c_double, _U32P, C.c_uint32]),
    "soup_aggregate_unwrap": (C.c_int, [_P, _U32P, C.c_uint32, _P]),
    "soup_local_cavity_volume": (C.c_int, [_P, _P, C.c_uint32, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "soup_box_cavity_volume": (C.c_int, [_P, _P, C.c_uint32, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "soup_cluster_labels": (C.c_int, [_P, _U32P, C.c_uint32, C.c_double, C.c_int, _U32P, C.POINTER(C.c_uint32)]),
    "soup_scale_molecules_rigid": (C.c_int, [_P, _P, C.c_uint32, _U32P, C.c_uint32, C.POINTER(C.c_double),
                                             C.POINTER(C.c_double), _P]),
    "soup_write_charges": (C.c_int, [_P, _P, _SZ]),
    "soup_set_box": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "soup_autotune": (C.c_int, [_P, C.c_uint32, C.POINTER(SoupTuneResult)]),
    "soup_apply_tuning": (C.c_int, [_P, C.POINTER(SoupTuneResult)]),
    "soup_prepare_graphs": (C.c_int, [_P]),
    "soup_write_state": (C.c_int, [_P, C.POINTER(SoupInitState)]),
    "soup_protonation_sweep": (C.c_int, [_P, C.POINTER(SoupSweepResult)]),
    "soup_closure": (C.c_int, [_P, _U32P, C.c_uint32, _U32P, C.c_uint32, C.POINTER(C.c_double),
                               C.c_double, C.c_double, C.c_double, C.POINTER(SoupClosureResult)]),
    "soup_closure_in_parcel": (C.c_int, [_P, _U32P, C.c_uint32, _U32P, C.c_uint32, C.POINTER(C.c_double),
                                         C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_double,
                                         C.POINTER(SoupClosureResult)]),
    "soup_amphiphile_labels": (C.c_int, [_P, _U32P, _U32P]),
    "soup_aggregate_labels": (C.c_int, [_P, _U32P, C.c_uint32, C.c_double, _U32P, _U32P]),
    "soup_pairing_stats": (C.c_int, [_P, C.c_double, C.POINTER(SoupPairingStats)]),
    "soup_density_profile_z": (C.c_int, [_P, C.c_uint32, C.c_uint32, _U32P, _U32P, _U32P]),
    "soup_get_diff_params": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "soup_set_diff_params": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "soup_diff_forward": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P]),
    "soup_diff_forward_strided": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, _P]),
    "soup_diff_backward": (C.c_int, [_P, _P, C.POINTER(C.c_double), _P, _P]),
    "soup_aggregate_shapes": (C.c_int, [_P, _U32P, _U32P, C.c_uint32, C.c_uint32, C.POINTER(SoupAggregateShape),
                                        _U32P]),
    "soup_aggregate_labels_noalloc": (C.c_int, [_P, _U32P, C.c_uint32, C.c_double, _U32P, _U32P]),
    "soup_batch_create": (C.c_int, [C.POINTER(SoupConfig), C.POINTER(SoupInitState), C.c_uint32,
                                    C.POINTER(_P)]),
    "soup_batch_step": (C.c_int, [_P, C.c_uint64]),
    "soup_batch_replica": (_P, [_P, C.c_uint32]),
    "soup_batch_last_error": (C.c_char_p, [_P]),
    "soup_batch_destroy": (None, [_P]),
    "soup_debug_phase": (C.c_int, [_P, C.c_int]),
    "soup_stream": (_P, [_P]),
    "soup_profile": (C.c_int, [_P, C.c_int]),
    "soup_kernel_time": (C.c_int, [_P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "soup_launch_count": (C.c_uint64, [_P]),
}

# soup_kernel_time groups
DIFF_NPARAM = 9

K_FORCE, K_ES_FAR, K_LIST, K_SORT, K_KICK_DRIFT, K_KICK_THERMO, K_BONDS, K_SWEEP = range(8)
K_NAMES = ["force", "es_far", "list", "sort", "kick_drift", "kick_thermo", "bonds", "sweep"]


def library_path() -> str:
    here = os.path.dirname(os.path.abspath(__file__))
    return os.path.join(here, LIB_NAME)


_lib = None


def lib():
    """Load libsoup_b200.so (built in-tree by csrc/build.py).  Raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(
            f"{LIB_NAME} not found at {path}: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
        )
    handle = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    _lib = handle
    return handle


class SoupError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.code = STATUS.get(status, str(status))
