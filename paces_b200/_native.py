"""ctypes binding of libpaces_b200.so (the C ABI declared in include/paces_b200.h).

The library is built in-tree by `paces_b200.build`.  There is no fallback: if the
shared library is missing or cannot be loaded, importing this module raises.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpaces_b200.so")

PACES_OK = 0
STATUS_NAMES = {
    0: "ok",
    1: "capacity exceeded",
    2: "lookup miss",
    3: "non-finite amplitudes",
    4: "device wait timed out",
    5: "bad argument",
    6: "CUDA error",
    7: "norm explosion",
    8: "tie shuffle would touch more than 90% of the states",
}
ERR_CAPACITY = 1
ERR_LOOKUP = 2
ERR_NONFINITE = 3
ERR_TIMEOUT = 4
ERR_SHUFFLE = 8

C128 = 0
C64 = 1
MAX_SITES = 128
MAX_LANCZOS_ORDER = 63
BATCH_SINGLE_CAP = 1 << 25  # PACES_BATCH_SINGLE_CAP
OBS_NORM, OBS_ENERGY, OBS_SITES = 1, 2, 4
WEIGHT_NONE, WEIGHT_COHERENCE, WEIGHT_NORM, WEIGHT_HAM_ONES = 0, 1, 2, 3


class ModelDesc(ctypes.Structure):
    _fields_ = [
        ("nchain", ctypes.c_int32),
        ("periodic", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("max_ho_dims", ctypes.POINTER(ctypes.c_int32)),
        ("eps_sys", ctypes.c_double),
        ("hbar_omega", ctypes.c_double),
        ("delta_eps", ctypes.c_double),
        ("J", ctypes.c_double),
        ("g", ctypes.c_double),
        ("site_eps", ctypes.POINTER(ctypes.c_double)),
        ("geo_dim", ctypes.c_int32),
        ("hopping2", ctypes.c_int32),
        ("J2", ctypes.c_double),
    ]


class Basis(ctypes.Structure):
    _fields_ = [("keys", ctypes.c_void_p), ("blk", ctypes.c_void_p), ("cap", ctypes.c_int64)]


class HMat(ctypes.Structure):
    _fields_ = [("nbr", ctypes.c_void_p), ("meta", ctypes.c_void_p), ("cap", ctypes.c_int64),
                ("xnbr", ctypes.c_void_p)]


class StepParams(ctypes.Structure):
    _fields_ = [
        ("maxstates", ctypes.c_int64),
        ("enlarge_steps", ctypes.c_int32),
        ("evolve", ctypes.c_int32),
        ("dt", ctypes.c_double),
        ("m_star", ctypes.c_int32),
        ("diagnostics", ctypes.c_int32),
        ("tol", ctypes.c_double),
        ("shuffle", ctypes.c_int32),
        ("renormalize", ctypes.c_int32),
        ("shuffle_seed", ctypes.c_uint64),
        ("step_index", ctypes.c_uint64),
        ("explosion_cutoff", ctypes.c_double),
        ("proposal", ctypes.c_int32),
        ("proposal_threshold", ctypes.c_float),
        ("proposal_params", ctypes.c_void_p),
        ("weighting", ctypes.c_int32),
        ("reserved0", ctypes.c_int32),
        ("tau", ctypes.c_double),
        ("old_h", ctypes.c_void_p),
        ("lanczos_order", ctypes.c_int32),
        ("reserved1", ctypes.c_int32),
        ("krylov", ctypes.c_void_p),
        ("krylov_bytes", ctypes.c_size_t),
        ("basis_ready", ctypes.c_void_p),
    ]


class StepRecord(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("n_select", ctypes.c_int32),
        ("n_enlarged", ctypes.c_int32),
        ("n_states", ctypes.c_int32),
        ("converged", ctypes.c_int32),
        ("final_m", ctypes.c_int32),
        ("ceiling_hits", ctypes.c_int32),
        ("n_tied", ctypes.c_int32),
        ("n_candidates", ctypes.c_int32),
        ("n_candidates_kept", ctypes.c_int32),
        ("c1_plus_c2", ctypes.c_double),
        ("term_ratio", ctypes.c_double),
        ("post_adapt_norm", ctypes.c_double),
        ("post_adapt_energy_re", ctypes.c_double),
        ("post_adapt_energy_im", ctypes.c_double),
        ("norm", ctypes.c_double),
        ("energy_re", ctypes.c_double),
        ("energy_im", ctypes.c_double),
        ("n_exc", ctypes.c_double * MAX_SITES),
        ("n_pho", ctypes.c_double * MAX_SITES),
    ]


class ExpmInfo(ctypes.Structure):
    _fields_ = [("converged", ctypes.c_int32), ("final_m", ctypes.c_int32),
                ("c1_plus_c2", ctypes.c_double), ("term_ratio", ctypes.c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("merge_stride", ctypes.c_int32),
        ("taylor_blocks_per_sm", ctypes.c_int32),
        ("merge_stride_min", ctypes.c_int32),
        ("merge_stride_max", ctypes.c_int32),
        ("taylor_blocks_per_sm_max", ctypes.c_int32),
        ("taylor_variant", ctypes.c_int32),
        ("assemble_stride", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 1),
    ]


class BatchItem(ctypes.Structure):
    _fields_ = [
        ("ctx", ctypes.c_void_p),
        ("old_basis", ctypes.POINTER(Basis)),
        ("old_psi", ctypes.c_void_p),
        ("new_basis", ctypes.POINTER(Basis)),
        ("new_psi", ctypes.c_void_p),
        ("h", ctypes.POINTER(HMat)),
        ("params", ctypes.POINTER(StepParams)),
        ("record", ctypes.c_void_p),
        ("workspace", ctypes.c_void_p),
        ("workspace_bytes", ctypes.c_size_t),
    ]


MAX_BATCH = 128

# entry point name -> (argtypes); every entry point returns int (status) unless listed in _RESTYPES
_P = ctypes.c_void_p
_SIGNATURES = {
    "paces_create": [ctypes.POINTER(ModelDesc), ctypes.POINTER(ctypes.c_void_p)],
    "paces_destroy": [_P],
    "paces_last_error": [_P],
    "paces_key_words": [_P],
    "paces_ref_words": [_P],
    "paces_key_layout": [_P, _P, _P, _P],
    "paces_version": [],
    "paces_hop_channels": [_P],
    "paces_workspace_bytes": [_P, ctypes.c_int64, ctypes.POINTER(ctypes.c_size_t)],
    "paces_read_status": [_P, _P, ctypes.POINTER(ctypes.c_int32)],
    "paces_keys_from_ref": [_P, _P, ctypes.c_int64, ctypes.c_int32, _P, _P, _P],
    "paces_keys_to_ref": [_P, ctypes.POINTER(Basis), ctypes.c_int32, _P, _P],
    "paces_expand": [_P, ctypes.POINTER(Basis), ctypes.POINTER(Basis), _P, ctypes.c_size_t, _P],
    "paces_assemble": [_P, ctypes.POINTER(Basis), ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, _P,
                       ctypes.c_size_t, _P],
    "paces_truncate": [_P, ctypes.POINTER(Basis), _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64,
                       ctypes.c_uint64, ctypes.POINTER(Basis), _P, ctypes.c_size_t, _P],
    "paces_truncate_weighted": [_P, ctypes.POINTER(Basis), _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64,
                                ctypes.c_uint64, ctypes.POINTER(Basis), _P, ctypes.c_size_t, _P],
    "paces_lookahead_weights": [_P, ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, ctypes.c_double, ctypes.c_int32,
                                _P, _P],
    "paces_remap": [_P, ctypes.POINTER(Basis), _P, ctypes.POINTER(Basis), _P, _P, ctypes.c_size_t, _P],
    "paces_remap_noalloc": [_P, ctypes.POINTER(Basis), _P, ctypes.POINTER(Basis), _P, _P],
    "paces_rows_lower_bound": [_P, ctypes.c_int64, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _P, _P, _P],
    "paces_rows_sort_bytes": [ctypes.c_int64],
    "paces_rows_sort_unique": [_P, ctypes.c_int64, ctypes.c_int32, _P, _P, _P, ctypes.c_size_t, _P],
    "paces_lanczos_bytes": [_P, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(ctypes.c_size_t)],
    "paces_lanczos": [_P, ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, _P, ctypes.c_double, ctypes.c_int32, _P, _P,
                      ctypes.c_size_t, _P],
    "paces_taylor": [_P, ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, _P, ctypes.c_double, ctypes.c_int32,
                     ctypes.c_double, _P, _P, ctypes.c_size_t, _P],
    "paces_observables": [_P, ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, ctypes.c_int32, _P, _P,
                          ctypes.c_size_t, _P],
    "paces_apply_h": [_P, ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, _P, _P],
    "paces_term_energies": [_P, ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, _P, _P, ctypes.c_size_t, _P],
    "paces_hnorms": [_P, ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, _P, _P, ctypes.c_size_t, _P],
    "paces_expm_scaled": [_P, ctypes.POINTER(Basis), ctypes.POINTER(HMat), _P, _P, ctypes.c_double, ctypes.c_double,
                          ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P, _P,
                          ctypes.c_size_t, _P],
    "paces_lookup": [_P, ctypes.POINTER(Basis), _P, _P, ctypes.c_int64, ctypes.c_int32, _P, _P,
                     ctypes.c_size_t, _P],
    "paces_step": [_P, ctypes.POINTER(Basis), _P, ctypes.POINTER(Basis), _P, ctypes.POINTER(HMat),
                   ctypes.POINTER(StepParams), _P, _P, ctypes.c_size_t, _P],
    "paces_set_profiling": [_P, ctypes.c_int32],
    "paces_set_test_hooks": [_P, ctypes.c_uint64, ctypes.c_int32],
    "paces_stage_times": [_P, ctypes.POINTER(ctypes.c_float)],
    "paces_kernel_launches": [_P],
    "paces_get_tuning": [_P, ctypes.POINTER(Tuning)],
    "paces_set_tuning": [_P, ctypes.POINTER(Tuning)],
    "paces_mlp_param_bytes": [],
    "paces_mlp_master_floats": [],
    "paces_selected_view": [_P, _P, ctypes.c_size_t, ctypes.POINTER(Basis), ctypes.POINTER(ctypes.c_void_p),
                            ctypes.POINTER(ctypes.c_void_p)],
    "paces_proposal_score": [_P, ctypes.POINTER(Basis), _P, _P, _P, ctypes.c_float, _P, ctypes.c_int64, _P, _P, _P],
    "paces_proposal_features": [_P, ctypes.POINTER(Basis), _P, _P, _P, _P, _P],
    "paces_proposal_labels": [_P, ctypes.POINTER(Basis), ctypes.POINTER(Basis), _P, _P],
    "paces_mlp_pack": [_P, _P, _P],
    "paces_mlp_forward": [_P, _P, ctypes.c_int64, _P, _P],
    "paces_mlp_backward": [_P, _P, _P, _P, ctypes.c_int64, ctypes.c_float, _P, _P, _P],
    "paces_mlp_adam": [_P, _P, _P, _P, ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                       _P, _P],
    "paces_batch_create": [ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)],
    "paces_batch_destroy": [_P],
    "paces_batch_step": [_P, ctypes.POINTER(BatchItem), ctypes.c_int32, _P],
    "paces_batch_last_error": [_P],
    "paces_batch_kernel_launches": [_P],
    "paces_batch_set_profiling": [_P, ctypes.c_int32],
    "paces_batch_set_test_hooks": [_P, ctypes.c_uint64, ctypes.c_int32],
    "paces_batch_stage_times": [_P, ctypes.POINTER(ctypes.c_float)],
}
_RESTYPES = {"paces_last_error": ctypes.c_char_p, "paces_rows_sort_bytes": ctypes.c_size_t, "paces_kernel_launches": ctypes.c_ulonglong,
             "paces_mlp_param_bytes": ctypes.c_size_t, "paces_mlp_master_floats": ctypes.c_int32,
             "paces_batch_last_error": ctypes.c_char_p, "paces_batch_kernel_launches": ctypes.c_ulonglong}
STAGES = ("truncate", "expand", "assemble", "remap", "diagnostics", "taylor", "observables")
BATCH_STAGES = ("front", "taylor", "back")

_lib = None


def load():
    """Load libpaces_b200.so (once).  Raises OSError if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing; build it with `python -m paces_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def exported_symbols():
    return sorted(_SIGNATURES)


class PacesError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"paces_b200: {STATUS_NAMES.get(code, code)}{': ' + msg if msg else ''}")


class CapacityError(PacesError):
    pass


def check(code, ctx=None, what=""):
    if code == PACES_OK:
        return
    msg = what
    if ctx is not None:
        detail = load().paces_last_error(ctx)
        if detail:
            msg = f"{what}: {detail.decode(errors='replace')}"
    if code == ERR_CAPACITY:
        raise CapacityError(code, msg)
    raise PacesError(code, msg)
