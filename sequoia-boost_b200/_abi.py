"""ctypes view of include/sb_gpu.h and the loader of libsb_gpu.so.

The library is built in-tree (`python -m sequoia_boost_b200.build` or
`__graft_entry__.build()`); there is no CPU fallback, so a missing or
unloadable library raises instead of degrading.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsb_gpu.so")

SB_OK = 0
SB_ERR_INVALID_ARG = 1
SB_ERR_OOM = 2
SB_ERR_CUDA = 3
SB_ERR_TIMEOUT = 4
SB_ERR_UNSUPPORTED = 5
SB_ERR_NO_DEVICE = 6
SB_ERR_DIMENSION = 7

SB_FEAT_NUMERICAL = 0
SB_FEAT_CATEGORICAL = 1
SB_OBJ_SQUARED_ERROR = 0
SB_OBJ_PSEUDOHUBER = 1
SB_OBJ_LOGISTIC = 2
SB_OBJ_SOFTMAX = 3
SB_OBJ_SOFTPROB = 4
SB_METRIC_RMSE, SB_METRIC_MAE, SB_METRIC_LOGLOSS, SB_METRIC_ERROR, SB_METRIC_MLOGLOSS, SB_METRIC_MERROR = range(6)
SB_EVAL_MAX_METRICS = 8
SB_GROW_DEPTHWISE = 0
SB_GROW_LOSSGUIDE = 1
SB_HIST_FP32 = 0
SB_HIST_FIXED = 1
SB_TREE_HIST = 0
SB_TREE_APPROX = 1


class SbGradPair(ctypes.Structure):
    _fields_ = [("grad", ctypes.c_float), ("hess", ctypes.c_float)]


class SbGradStats(ctypes.Structure):
    _fields_ = [("grad", ctypes.c_double), ("hess", ctypes.c_double)]


class SbNode(ctypes.Structure):
    _fields_ = [
        ("left", ctypes.c_int32),
        ("right", ctypes.c_int32),
        ("split_feature", ctypes.c_uint32),
        ("split_cond", ctypes.c_float),
        ("leaf_value", ctypes.c_float),
        ("sum_hess", ctypes.c_float),
        ("split_gain", ctypes.c_float),
        ("default_left", ctypes.c_uint8),
        ("is_categorical", ctypes.c_uint8),
        ("reserved", ctypes.c_uint16),
        ("cat_begin", ctypes.c_uint32),
        ("cat_end", ctypes.c_uint32),
    ]


class SbTrainParams(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("base_score", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("min_child_weight", ctypes.c_double),
        ("max_delta_step", ctypes.c_double),
        ("subsample", ctypes.c_double),
        ("colsample_bytree", ctypes.c_double),
        ("colsample_bylevel", ctypes.c_double),
        ("colsample_bynode", ctypes.c_double),
        ("lambda_", ctypes.c_double),
        ("alpha", ctypes.c_double),
        ("scale_pos_weight", ctypes.c_double),
        ("monotone", ctypes.POINTER(ctypes.c_int8)),
        ("interaction_offsets", ctypes.POINTER(ctypes.c_uint32)),
        ("interaction_features", ctypes.POINTER(ctypes.c_uint32)),
        ("objective", ctypes.c_int32),
        ("num_class", ctypes.c_int32),
        ("has_base_score", ctypes.c_int32),
        ("max_depth", ctypes.c_int32),
        ("max_leaves", ctypes.c_int32),
        ("grow_policy", ctypes.c_int32),
        ("max_bin", ctypes.c_int32),
        ("hist_precision", ctypes.c_int32),
        ("quantize_bits", ctypes.c_int32),
        ("n_monotone", ctypes.c_int32),
        ("n_interaction_groups", ctypes.c_int32),
        ("tree_method", ctypes.c_int32),
    ]


class SbModelView(ctypes.Structure):
    _fields_ = [
        ("tree_node_offset", ctypes.POINTER(ctypes.c_int64)),
        ("nodes", ctypes.POINTER(SbNode)),
        ("tree_cat_offset", ctypes.POINTER(ctypes.c_int64)),
        ("categories", ctypes.POINTER(ctypes.c_uint32)),
        ("tree_weights", ctypes.POINTER(ctypes.c_float)),
        ("n_trees", ctypes.c_int32),
        ("num_class", ctypes.c_int32),
        ("n_features", ctypes.c_int32),
        ("objective", ctypes.c_int32),
        ("base_score", ctypes.c_float),
        ("reserved", ctypes.c_int32),
    ]


class SbBoosterStats(ctypes.Structure):
    _fields_ = [
        ("rounds", ctypes.c_uint64),
        ("hist_launches", ctypes.c_uint64),
        ("hist_ms", ctypes.c_double),
        ("hist_bytes", ctypes.c_double),
        ("round_ms", ctypes.c_double),
        ("quant_err_grad", ctypes.c_double),
        ("quant_err_hess", ctypes.c_double),
        ("quant_shift_grad", ctypes.c_int32),
        ("quant_shift_hess", ctypes.c_int32),
    ]


class SbServerStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "submitted", "completed", "failed", "batches", "rows", "max_batch_requests", "memory_waits",
        "mem_bytes", "mem_peak")]



class SbJob(ctypes.Structure):
    _fields_ = [
        ("X", ctypes.POINTER(ctypes.c_float)),
        ("n_rows", ctypes.c_size_t),
        ("n_cols", ctypes.c_size_t),
        ("feature_types", ctypes.POINTER(ctypes.c_uint8)),
        ("missing", ctypes.c_float),
        ("labels", ctypes.POINTER(ctypes.c_float)),
        ("weights", ctypes.POINTER(ctypes.c_float)),
        ("base_margin", ctypes.POINTER(ctypes.c_float)),
        ("params", ctypes.POINTER(SbTrainParams)),
        ("num_boost_round", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("out", ctypes.c_void_p),
    ]


SB_REQ_MARGIN = 0
SB_REQ_CONTRIBS = 1

# name -> (restype, argtypes) of every symbol include/sb_gpu.h declares.
P = ctypes.c_void_p
SZ = ctypes.c_size_t
I32 = ctypes.c_int
F32P = ctypes.POINTER(ctypes.c_float)
U32P = ctypes.POINTER(ctypes.c_uint32)
U16P = ctypes.POINTER(ctypes.c_uint16)
U8P = ctypes.POINTER(ctypes.c_uint8)
I32P = ctypes.POINTER(ctypes.c_int32)
I64P = ctypes.POINTER(ctypes.c_int64)
SIGNATURES = {
    "sb_last_error": (ctypes.c_char_p, []),
    "sb_version": (ctypes.c_char_p, []),
    "sb_train_params_default": (None, [ctypes.POINTER(SbTrainParams)]),
    "sb_train_params_validate": (I32, [ctypes.POINTER(SbTrainParams)]),
    "sb_ctx_create": (I32, [I32, ctypes.POINTER(P)]),
    "sb_ctx_destroy": (I32, [P]),
    "sb_ctx_synchronize": (I32, [P]),
    "sb_ctx_stream": (P, [P]),
    "sb_ctx_launch_count": (ctypes.c_uint64, [P]),
    "sb_ghist_create": (I32, [P, F32P, SZ, SZ, U8P, ctypes.c_float, I32, ctypes.POINTER(P)]),
    "sb_ghist_create_device": (I32, [P, P, SZ, SZ, U8P, ctypes.c_float, I32, ctypes.POINTER(P)]),
    "sb_ghist_destroy": (I32, [P]),
    "sb_ghist_info": (I32, [P, ctypes.POINTER(SZ), ctypes.POINTER(SZ), ctypes.POINTER(SZ)]),
    "sb_ghist_layout": (I32, [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(SZ),
                              ctypes.POINTER(ctypes.c_int)]),
    "sb_ghist_codes": (I32, [P, P]),
    "sb_ghist_cuts": (I32, [P, U32P, F32P, U8P]),
    "sb_ghist_bins": (I32, [P, U16P]),
    "sb_hist_build": (I32, [P, P, U32P, SZ, ctypes.POINTER(SbGradPair), SZ, I32, I32,
                            ctypes.POINTER(SbGradStats), SZ]),
    "sb_hist_subtract": (I32, [P, ctypes.POINTER(SbGradStats), ctypes.POINTER(SbGradStats),
                               ctypes.POINTER(SbGradStats), SZ]),
    "sb_hist_build_static": (I32, [P, P, P, SZ, P, SZ, P, SZ]),  # device pointers
    "sb_objective_gradient": (I32, [P, I32, I32, ctypes.c_double, F32P, F32P, F32P, SZ,
                                    ctypes.POINTER(SbGradPair)]),
    "sb_ghist_create_weighted": (I32, [P, F32P, SZ, SZ, U8P, ctypes.c_float, I32, F32P, ctypes.POINTER(P)]),
    "sb_tree_build": (I32, [P, P, ctypes.POINTER(SbTrainParams), ctypes.POINTER(SbGradPair), SZ,
                            U32P, SZ, ctypes.c_uint64, ctypes.c_uint32, I32P, ctypes.POINTER(P)]),
    "sb_booster_create": (I32, [P, P, ctypes.POINTER(SbTrainParams), F32P, F32P, F32P,
                                ctypes.POINTER(P)]),
    "sb_booster_update": (I32, [P, I32]),
    "sb_booster_margins": (I32, [P, F32P]),
    "sb_booster_gradients": (I32, [P, ctypes.POINTER(SbGradPair)]),
    "sb_booster_row_mask": (I32, [P, ctypes.c_uint64, U8P]),
    "sb_booster_model": (I32, [P, ctypes.POINTER(P)]),
    "sb_booster_destroy": (I32, [P]),
    "sb_booster_set_graphs": (I32, [P, I32]),
    "sb_booster_set_timing": (I32, [P, I32]),
    "sb_booster_stats_get": (I32, [P, ctypes.POINTER(SbBoosterStats)]),
    "sb_booster_stats_reset": (I32, [P]),
    "sb_train_many": (I32, [P, ctypes.POINTER(SbJob), SZ, I32]),
    "sb_train": (I32, [P, F32P, SZ, SZ, U8P, ctypes.c_float, F32P, F32P, F32P,
                       ctypes.POINTER(SbTrainParams), I32, ctypes.POINTER(P)]),
    "sb_train_dart": (I32, [P, F32P, SZ, SZ, U8P, ctypes.c_float, F32P, F32P, F32P,
                            ctypes.POINTER(SbTrainParams), ctypes.c_double, ctypes.c_double, I32,
                            ctypes.POINTER(P)]),
    "sb_model_create": (I32, [P, ctypes.POINTER(SbModelView), ctypes.POINTER(P)]),
    "sb_model_destroy": (I32, [P]),
    "sb_model_export_sizes": (I32, [P, I32P, I64P, I64P]),
    "sb_model_export": (I32, [P, I64P, ctypes.POINTER(SbNode), I64P, U32P, F32P]),
    "sb_model_info": (I32, [P, F32P, I32P, I32P, I32P]),
    "sb_predict_margin": (I32, [P, F32P, SZ, SZ, ctypes.c_float, F32P, SZ, F32P]),
    "sb_predict": (I32, [P, F32P, SZ, SZ, ctypes.c_float, F32P, F32P]),
    "sb_predict_contribs": (I32, [P, F32P, SZ, SZ, ctypes.c_float, F32P]),
    "sb_booster_set_margins": (I32, [P, F32P]),
    "sb_booster_eval_add": (I32, [P, F32P, SZ, SZ, ctypes.c_float, F32P, F32P, F32P, ctypes.POINTER(I32)]),
    "sb_booster_eval": (I32, [P, I32, ctypes.POINTER(I32), ctypes.POINTER(ctypes.c_double)]),
    "sb_booster_eval_margins": (I32, [P, I32, F32P]),
    "sb_model_set_best_iteration": (I32, [P, ctypes.c_int64]),
    "sb_model_best_iteration": (I32, [P, ctypes.POINTER(ctypes.c_int64)]),
    "sb_predict_leaf": (I32, [P, F32P, SZ, SZ, ctypes.c_float, ctypes.POINTER(ctypes.c_uint32)]),
    "sb_predict_interactions": (I32, [P, F32P, SZ, SZ, ctypes.c_float, F32P]),
    "sb_server_create": (I32, [P, P, SZ, I32, ctypes.POINTER(P)]),
    "sb_server_submit": (I32, [P, I32, F32P, SZ, SZ, ctypes.c_float, F32P, ctypes.POINTER(ctypes.c_uint64)]),
    "sb_server_wait": (I32, [P, ctypes.c_uint64, I32, ctypes.POINTER(ctypes.c_double)]),
    "sb_server_stats_get": (I32, [P, ctypes.POINTER(SbServerStats)]),
    "sb_server_destroy": (I32, [P]),
}


class SbError(RuntimeError):
    """A non-zero status from the C ABI (SequoiaError analogue)."""

    def __init__(self, code, msg):
        super().__init__(f"sb error {code}: {msg}")
        self.code = code


_LIB = None


def lib():
    """Loads libsb_gpu.so once; raises if it is missing (no fallback)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run __graft_entry__.build() (there is no CPU fallback)")
        h = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = h
    return _LIB


def check(status):
    if status != SB_OK:
        raise SbError(status, lib().sb_last_error().decode(errors="replace"))


def ptr(arr, ctype):
    """Pointer to a C-contiguous numpy array (or NULL for None)."""
    if arr is None:
        return None
    assert arr.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return arr.ctypes.data_as(ctypes.POINTER(ctype))
