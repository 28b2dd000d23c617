"""ctypes binding of libfln.so, the C ABI declared in include/fln.h.

The library is built in-tree (fastlinkingnumbers_b200/lib/libfln.so) by
``fastlinkingnumbers_b200.build``. Loading fails loudly when it is missing:
there is no CPU fallback for the linking-number kernels.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libfln.so")

# fln_status
OK = 0
STATUS_NAMES = {
    0: "FLN_OK", 1: "FLN_ERR_INVALID_ARGUMENT", 2: "FLN_ERR_IO", 3: "FLN_ERR_FORMAT",
    4: "FLN_ERR_CUDA", 5: "FLN_ERR_NO_DEVICE", 6: "FLN_ERR_OUT_OF_MEMORY",
    7: "FLN_ERR_SEGMENT_TOO_SMALL", 8: "FLN_ERR_MAX_RECURSION", 9: "FLN_ERR_UNLOOPED",
    10: "FLN_ERR_NONFINITE", 11: "FLN_ERR_STACK_OVERFLOW", 12: "FLN_ERR_TIMEOUT",
    13: "FLN_ERR_INTERNAL",
}
METHOD_DIRECTSUM, METHOD_BARNESHUT = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
SEG_BSPLINE, SEG_CATMULLROM, SEG_BEZIER, SEG_POLYLINE = 0, 1, 2, 3
PAIR_FP64_RECOMPUTED, PAIR_BETA_RETRIED, PAIR_NONFINITE, PAIR_SWAPPED = 1, 2, 4, 8
PAIR_BETA_ESCALATED = 16

# Every symbol include/fln.h declares (checked by the CPU tests).
EXPORTED = [
    "fln_status_string", "fln_last_error", "fln_abi_version", "fln_default_params",
    "fln_ctx_create", "fln_ctx_destroy", "fln_ctx_stats", "fln_linking_numbers",
    "fln_linking_numbers_device", "fln_linking_numbers_direct_noalloc", "fln_direct_pair", "fln_model_create", "fln_model_destroy",
    "fln_model_load_bcc", "fln_model_save_bcc", "fln_model_set_curves", "fln_model_num_curves",
    "fln_model_num_points", "fln_model_get_curves", "fln_model_prepare",
    "fln_model_prepared_sizes", "fln_model_get_prepared", "fln_certificate_compute",
    "fln_certificate_load", "fln_certificate_destroy", "fln_certificate_save",
    "fln_certificate_text", "fln_certificate_num_curves", "fln_certificate_num_entries",
    "fln_certificate_entries", "fln_certificate_num_pairs", "fln_certificate_pairs",
    "fln_certificate_equals", "fln_certificate_export_diffs",
    "fln_learned_default_options", "fln_learned_train", "fln_learned_create", "fln_learned_destroy",
    "fln_learned_get", "fln_ctx_set_learned", "fln_learned_collect", "fln_learned_predict",
    "fln_learned_gradients", "fln_model_prepare_device", "fln_autotune", "fln_autotune_direct", "fln_learned_configure",
]


class TuneResult(C.Structure):
    _fields_ = [
        ("best_ms", C.c_double), ("default_ms", C.c_double), ("trials", C.c_int32),
        ("sample_pairs", C.c_int32), ("best_budget", C.c_int32), ("best_direct_tile", C.c_int32),
        ("best_beta", C.c_double), ("best_bucket", C.c_int32), ("best_occupancy", C.c_int32),
        ("reserved", C.c_double * 2),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}

MLP_PARAMS = 4801  # FLN_MLP_PARAMS
ABI_VERSION = 3  # FLN_ABI_VERSION: the layout of the structs below


class Params(C.Structure):
    _fields_ = [
        ("barnes_hut_init_beta", C.c_double), ("barnes_hut_beta_limit", C.c_double),
        ("epssq", C.c_double), ("target_error", C.c_double), ("error_est_scale", C.c_double),
        ("precision", C.c_int32), ("fp64_margin", C.c_double), ("near_factor", C.c_double),
        ("bh_tree", C.c_int32), ("bh_escalations", C.c_int32), ("bh_err_limit", C.c_double),
        ("bh_schedule", C.c_int32), ("host_prepare", C.c_int32), ("bh_budget", C.c_int32),
        ("bh_bucket", C.c_int32), ("bh_retry_from_roots", C.c_int32), ("bh_spill_cap", C.c_int32),
        ("bh_wait_polls", C.c_int64), ("direct_tile", C.c_int32), ("bh_occupancy", C.c_int32),
        ("bh_exact_serial", C.c_int32), ("reserved_int", C.c_int32), ("reserved_params", C.c_double * 3),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("pairs", C.c_int64), ("segment_pairs", C.c_double), ("fp64_recomputed", C.c_int64),
        ("beta_retried", C.c_int64), ("bh_far_evals", C.c_double), ("bh_leaf_evals", C.c_double),
        ("near_fp64_terms", C.c_double), ("ms_kernels", C.c_double), ("ms_total", C.c_double),
        ("ms_discretize", C.c_double), ("mean_off_integer", C.c_double),
        ("max_off_integer", C.c_double), ("discretize_rounds", C.c_int32),
        ("kernel_launches", C.c_int32), ("ms_main_kernel", C.c_double),
        ("ms_tree_build", C.c_double), ("bh_rounds", C.c_int32), ("reserved_stats", C.c_int32),
        ("bh_escalated", C.c_int64), ("bh_wait_timeouts", C.c_int64),
        ("ms_exact", C.c_double), ("bh_exact_entries", C.c_double), ("ms_retry", C.c_double),
        ("bh_front_records", C.c_int64), ("bh_retry_from_roots", C.c_int64),
        ("bh_far_reused", C.c_double), ("bh_far_subtracted", C.c_double), ("ms_traverse", C.c_double),
        ("reserved_stats2", C.c_double * 1),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class LearnedOptions(C.Structure):
    _fields_ = [
        ("s_min", C.c_double), ("sample_keep", C.c_double), ("max_samples", C.c_int64),
        ("max_terms", C.c_int64), ("epochs", C.c_int32), ("batch", C.c_int32),
        ("learning_rate", C.c_double), ("quantile", C.c_double), ("tau_quantile", C.c_double),
        ("val_fraction", C.c_double), ("min_candidates", C.c_int32), ("min_node_segments", C.c_int32),
        ("seed", C.c_uint64), ("reserved", C.c_double * 4),
    ]


class LearnedInfo(C.Structure):
    _fields_ = [
        ("recorded", C.c_int64), ("samples", C.c_int64), ("train_samples", C.c_int64),
        ("val_samples", C.c_int64), ("s_min", C.c_double), ("log10_tau", C.c_double),
        ("min_candidates", C.c_int32), ("epochs", C.c_int32), ("train_loss", C.c_double),
        ("val_loss", C.c_double), ("val_coverage", C.c_double), ("ms_collect", C.c_double),
        ("ms_train", C.c_double), ("min_node_segments", C.c_int32), ("reserved_i", C.c_int32),
        ("reserved", C.c_double * 3),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class FlnError(RuntimeError):
    """A non-OK fln_status; the reference throws std::runtime_error in the same places."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def load():
    """Loads libfln.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FlnError(13, f"{LIB_PATH} is missing; build it with "
                           "`python -m fastlinkingnumbers_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    P = C.POINTER
    L.fln_status_string.restype = C.c_char_p
    L.fln_status_string.argtypes = [C.c_int]
    L.fln_last_error.restype = C.c_char_p
    L.fln_abi_version.restype = C.c_int
    if L.fln_abi_version() != ABI_VERSION:
        raise FlnError(13, f"{LIB_PATH} has ABI version {L.fln_abi_version()}, this binding expects "
                           f"{ABI_VERSION}: rebuild it")
    L.fln_default_params.argtypes = [P(Params)]
    L.fln_ctx_create.argtypes = [C.c_int, vp, P(vp)]
    L.fln_ctx_destroy.argtypes = [vp]
    L.fln_ctx_stats.argtypes = [vp, P(Stats)]
    L.fln_linking_numbers.argtypes = [vp, vp, vp, i32, vp, i64, C.c_int, P(Params), vp, vp, vp]
    L.fln_linking_numbers_device.argtypes = [vp, vp, vp, i32, vp, i64, C.c_int, P(Params), vp, vp,
                                             vp]
    L.fln_direct_pair.argtypes = [vp, vp, i64, vp, i64, i32, P(f64)]
    L.fln_linking_numbers_direct_noalloc.argtypes = [vp, vp, i32, vp, i64, i32, vp, vp]
    L.fln_model_create.argtypes = [P(vp)]
    L.fln_model_destroy.argtypes = [vp]
    L.fln_model_load_bcc.argtypes = [vp, C.c_char_p]
    L.fln_model_save_bcc.argtypes = [vp, C.c_char_p]
    L.fln_model_set_curves.argtypes = [vp, C.c_int, i32, vp, vp]
    L.fln_model_num_curves.argtypes = [vp]
    L.fln_model_num_curves.restype = i32
    L.fln_model_num_points.argtypes = [vp]
    L.fln_model_num_points.restype = i64
    L.fln_model_get_curves.argtypes = [vp, P(i32), vp, vp]
    L.fln_model_prepare.argtypes = [vp, C.c_int, P(i32)]
    L.fln_model_prepare_device.argtypes = [vp, vp, C.c_int, P(i32)]
    L.fln_autotune.argtypes = [vp, vp, vp, i32, vp, i64, P(Params), i32, i64, P(Params), P(TuneResult)]
    L.fln_autotune_direct.argtypes = [vp, vp, vp, i32, vp, i64, P(Params), i64, P(Params), P(TuneResult)]
    L.fln_model_prepared_sizes.argtypes = [vp, P(i64), P(i64)]
    L.fln_model_get_prepared.argtypes = [vp, vp, vp, vp]
    L.fln_certificate_compute.argtypes = [vp, vp, C.c_int, C.c_int, P(Params), P(vp)]
    L.fln_certificate_load.argtypes = [C.c_char_p, P(vp)]
    L.fln_certificate_destroy.argtypes = [vp]
    L.fln_certificate_save.argtypes = [vp, C.c_char_p]
    L.fln_certificate_text.argtypes = [vp, C.c_char_p, i64]
    L.fln_certificate_text.restype = i64
    L.fln_certificate_num_curves.argtypes = [vp]
    L.fln_certificate_num_curves.restype = i32
    L.fln_certificate_num_entries.argtypes = [vp]
    L.fln_certificate_num_entries.restype = i64
    L.fln_certificate_entries.argtypes = [vp, vp]
    L.fln_certificate_num_pairs.argtypes = [vp]
    L.fln_certificate_num_pairs.restype = i64
    L.fln_certificate_pairs.argtypes = [vp, vp, vp, vp, vp]
    L.fln_certificate_equals.argtypes = [vp, vp]
    L.fln_certificate_equals.restype = C.c_int
    L.fln_certificate_export_diffs.argtypes = [vp, vp, C.c_char_p, C.c_char_p]
    L.fln_learned_default_options.argtypes = [P(LearnedOptions)]
    L.fln_learned_default_options.restype = None
    L.fln_learned_train.argtypes = [vp, vp, vp, i32, vp, i64, P(Params), P(LearnedOptions), P(vp)]
    L.fln_learned_create.argtypes = [vp, f64, f64, i32, P(vp)]
    L.fln_learned_destroy.argtypes = [vp]
    L.fln_learned_configure.argtypes = [vp, i32, i32]
    L.fln_learned_destroy.restype = None
    L.fln_learned_get.argtypes = [vp, vp, P(LearnedInfo)]
    L.fln_ctx_set_learned.argtypes = [vp, vp]
    L.fln_learned_collect.argtypes = [vp, vp, vp, i32, vp, i64, P(Params), f64, f64, i64, i64, vp, vp,
                                      vp, vp, P(i64)]
    L.fln_learned_predict.argtypes = [vp, vp, vp, i64, i32, vp]
    L.fln_learned_gradients.argtypes = [vp, vp, vp, vp, i64, f64, vp, P(f64)]
    _lib = L
    return L


def check(status: int):
    if status != OK:
        raise FlnError(status, load().fln_last_error().decode(errors="replace"))


def default_params(**overrides) -> Params:
    p = Params()
    load().fln_default_params(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p
