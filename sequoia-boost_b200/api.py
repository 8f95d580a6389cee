"""Python mirror of the reference crate's API over libsb_gpu.so (see __init__)."""
import ctypes
import math
import sys
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _abi as A

OBJECTIVES = {
    "reg:squarederror": A.SB_OBJ_SQUARED_ERROR,
    "reg:linear": A.SB_OBJ_SQUARED_ERROR,
    "reg:pseudohubererror": A.SB_OBJ_PSEUDOHUBER,
    "binary:logistic": A.SB_OBJ_LOGISTIC,
    "reg:logistic": A.SB_OBJ_LOGISTIC,
    "multi:softmax": A.SB_OBJ_SOFTMAX,
    "multi:softprob": A.SB_OBJ_SOFTPROB,
}


class Monotone:
    """config/params.rs:60-68."""
    NONE = 0
    INCREASING = 1
    DECREASING = -1


@dataclass
class TrainingParams:
    """TrainingParams with the reference's field names and defaults
    (config/params.rs:76-186). `hist_precision` ("fixed" | "fp32") and
    `quantize_bits` select this backend's histogram form. The default is the
    fixed-point form: each round's gradient pairs are rounded to integers with
    a power-of-two scale and summed exactly in int64, so two trainings with the
    same data, parameters and seed give identical models, as the reference's
    do (tests/properties.rs:40-46). "fp32" sums f32 gradients with atomics
    whose order varies from run to run."""
    seed: int = 0
    objective: str = "reg:squarederror"
    num_class: int = 0
    base_score: Optional[float] = None
    eta: float = 0.3
    gamma: float = 0.0
    max_depth: int = 6
    max_leaves: int = 0
    min_child_weight: float = 1.0
    max_delta_step: float = 0.0
    subsample: float = 1.0
    colsample_bytree: float = 1.0
    colsample_bylevel: float = 1.0
    colsample_bynode: float = 1.0
    lambda_: float = 1.0
    alpha: float = 0.0
    scale_pos_weight: float = 1.0
    grow_policy: str = "depthwise"
    tree_method: str = "hist"  # "auto" | "hist" | "approx" (params.rs TreeMethod; "exact" is not built)
    max_bin: int = 256
    monotone_constraints: List[int] = field(default_factory=list)
    interaction_constraints: List[List[int]] = field(default_factory=list)
    hist_precision: str = "fixed"
    quantize_bits: int = 0
    eval_metric: List[str] = field(default_factory=list)  # XGBoost `eval_metric` (params.rs:96-97)
    booster: str = "gbtree"  # "gbtree" | "dart" (params.rs:79; gblinear is not built)
    rate_drop: float = 0.0   # DART (params.rs:143-146)
    skip_drop: float = 0.0

    @staticmethod
    def builder():
        return _ParamsBuilder()

    def to_c(self):
        """A C struct plus the buffers it points into (keep both alive)."""
        p = A.SbTrainParams()
        A.lib().sb_train_params_default(ctypes.byref(p))
        if self.objective not in OBJECTIVES:
            raise A.SbError(A.SB_ERR_INVALID_ARG, f"unknown value `{self.objective}` for objective")
        p.seed = self.seed
        p.objective = OBJECTIVES[self.objective]
        p.num_class = self.num_class
        p.has_base_score = 0 if self.base_score is None else 1
        p.base_score = 0.0 if self.base_score is None else float(self.base_score)
        p.eta = self.eta
        p.gamma = self.gamma
        p.max_depth = self.max_depth
        p.max_leaves = self.max_leaves
        p.min_child_weight = self.min_child_weight
        p.max_delta_step = self.max_delta_step
        p.subsample = self.subsample
        p.colsample_bytree = self.colsample_bytree
        p.colsample_bylevel = self.colsample_bylevel
        p.colsample_bynode = self.colsample_bynode
        p.lambda_ = self.lambda_
        p.alpha = self.alpha
        p.scale_pos_weight = self.scale_pos_weight
        p.grow_policy = A.SB_GROW_LOSSGUIDE if self.grow_policy == "lossguide" else A.SB_GROW_DEPTHWISE
        if self.tree_method not in ("auto", "hist", "approx"):
            code = A.SB_ERR_UNSUPPORTED if self.tree_method == "exact" else A.SB_ERR_INVALID_ARG
            raise A.SbError(code, f"tree_method `{self.tree_method}` is not available (auto, hist, approx)")
        p.tree_method = A.SB_TREE_APPROX if self.tree_method == "approx" else A.SB_TREE_HIST
        p.max_bin = self.max_bin
        p.hist_precision = A.SB_HIST_FIXED if self.hist_precision == "fixed" else A.SB_HIST_FP32
        p.quantize_bits = self.quantize_bits
        keep = []
        if self.monotone_constraints:
            mono = np.asarray(self.monotone_constraints, dtype=np.int8)
            keep.append(mono)
            p.monotone = A.ptr(mono, ctypes.c_int8)
            p.n_monotone = len(mono)
        if self.interaction_constraints:
            offs = [0]
            flat = []
            for g in self.interaction_constraints:
                flat += list(g)
                offs.append(len(flat))
            o = np.asarray(offs, dtype=np.uint32)
            fl = np.asarray(flat if flat else [0], dtype=np.uint32)
            keep += [o, fl]
            p.interaction_offsets = A.ptr(o, ctypes.c_uint32)
            p.interaction_features = A.ptr(fl, ctypes.c_uint32)
            p.n_interaction_groups = len(self.interaction_constraints)
        return p, keep

    def validate(self):
        p, _keep = self.to_c()
        A.check(A.lib().sb_train_params_validate(ctypes.byref(p)))
        if self.booster not in ("gbtree", "dart"):
            raise A.SbError(A.SB_ERR_UNSUPPORTED if self.booster == "gblinear" else A.SB_ERR_INVALID_ARG,
                            f"booster `{self.booster}` is not available (gbtree, dart)")
        for name in ("rate_drop", "skip_drop"):  # params.rs:244-245
            v = getattr(self, name)
            if not (0.0 <= v <= 1.0):
                raise A.SbError(A.SB_ERR_INVALID_ARG, f"invalid parameter {name}={v}: must be in [0, 1]")
        return self


class _ParamsBuilder:
    """TrainingParamsBuilder (params.rs:264-373): chained setters."""

    def __init__(self):
        self.params = TrainingParams()

    def __getattr__(self, name):
        key = "lambda_" if name in ("lambda_", "reg_lambda") else name

        def setter(value):
            if key == "eval_metric":  # the builder appends (params.rs:342-345)
                self.params.eval_metric = list(self.params.eval_metric) + [value]
            else:
                setattr(self.params, key, value)
            return self
        return setter

    def build(self):
        return self.params.validate()

    def build_unchecked(self):
        return self.params


class _Native:
    """Owner of a native handle `h`. Its destroy call waits until every object
    created on it (a model on a context, a server on a model) has destroyed
    its own handle: the finalizers of garbage in a reference cycle run in any
    order. At interpreter exit nothing is destroyed; the driver reclaims the
    device memory with the process."""

    _deps = 0
    _released = False
    _parents = ()

    def _adopt(self, *parents):
        self._parents = tuple(p for p in parents if p is not None)
        for p in self._parents:
            p._deps += 1

    def _drop(self):
        if self._released and self._deps == 0 and getattr(self, "h", None):
            self._free()
            self.h = None
            for p in self._parents:
                p._deps -= 1
                p._drop()

    def __del__(self, _sys=sys):
        if _sys.is_finalizing():
            return
        self._released = True
        self._drop()


class Context(_Native):
    """A device context (sb_ctx): one GPU, one CUDA stream."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        A.check(A.lib().sb_ctx_create(device, ctypes.byref(h)))
        self.h = h
        self.device = device

    def synchronize(self):
        A.check(A.lib().sb_ctx_synchronize(self.h))

    def stream(self):
        return A.lib().sb_ctx_stream(self.h)

    def launch_count(self):
        return A.lib().sb_ctx_launch_count(self.h)

    def _free(self, _A=A):
        _A.lib().sb_ctx_destroy(self.h)


_DEFAULT = None


def default_context():
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Context(0)
    return _DEFAULT


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class DMatrix:
    """A dense f32 dataset with labels/weights/base margin (data/dmatrix.rs).
    Missing entries are NaN, or equal to `missing` (dmatrix.rs:10-16)."""

    def __init__(self, data, labels=None, weights=None, base_margin=None, feature_types=None,
                 missing=float("nan")):
        x = _f32(data)
        if x.ndim != 2 or x.shape[0] == 0 or x.shape[1] == 0:
            raise A.SbError(A.SB_ERR_INVALID_ARG, "empty dataset: from_dense: zero rows or columns")
        self.data = x
        self.missing = float(missing)
        self.labels = None if labels is None else _f32(labels)
        self.weights = None if weights is None else _f32(weights)
        self.base_margin = None if base_margin is None else _f32(base_margin)
        self.feature_types = feature_types
        for name, v in (("labels", self.labels), ("weights", self.weights)):
            if v is not None and v.shape[0] != x.shape[0]:
                raise A.SbError(A.SB_ERR_DIMENSION, f"dimension mismatch: {name}")

    @staticmethod
    def from_dense(data, n_rows, n_cols, missing=float("nan")):
        a = _f32(data)
        if a.size != n_rows * n_cols:
            raise A.SbError(A.SB_ERR_DIMENSION, "dimension mismatch: dense data length")
        return DMatrix(a.reshape(n_rows, n_cols), missing=missing)

    def with_labels(self, labels):
        self.labels = _f32(labels)
        return self

    def with_weights(self, weights):
        self.weights = _f32(weights)
        return self

    def with_base_margin(self, bm):
        self.base_margin = _f32(bm)
        return self

    def with_feature_types(self, types):
        self.feature_types = list(types)
        return self

    @property
    def n_rows(self):
        return self.data.shape[0]

    @property
    def n_cols(self):
        return self.data.shape[1]

    def _ftypes(self):
        if self.feature_types is None:
            return None
        return np.asarray([1 if t in (1, "c", "categorical") else 0 for t in self.feature_types],
                          dtype=np.uint8)


class GHistIndex(_Native):
    """HistCuts + GHistIndex resident on the device (sb_ghist)."""

    def __init__(self, dmat: DMatrix, max_bin=256, ctx: Context = None, device_ptr=None):
        self.ctx = ctx or default_context()
        h = ctypes.c_void_p()
        ft = dmat._ftypes() if dmat is not None else None
        A.check(A.lib().sb_ghist_create(self.ctx.h, A.ptr(dmat.data, ctypes.c_float), dmat.n_rows,
                                        dmat.n_cols, A.ptr(ft, ctypes.c_uint8), dmat.missing, max_bin,
                                        ctypes.byref(h)))
        self.h = h
        self._adopt(self.ctx)
        self._keep = ft

    @classmethod
    def from_device(cls, d_ptr, n_rows, n_cols, max_bin=256, missing=float("nan"), feature_types=None,
                    ctx: Context = None):
        self = cls.__new__(cls)
        self.ctx = ctx or default_context()
        ft = None if feature_types is None else np.asarray(feature_types, dtype=np.uint8)
        h = ctypes.c_void_p()
        A.check(A.lib().sb_ghist_create_device(self.ctx.h, ctypes.c_void_p(d_ptr), n_rows, n_cols,
                                               A.ptr(ft, ctypes.c_uint8), missing, max_bin,
                                               ctypes.byref(h)))
        self.h = h
        self._adopt(self.ctx)
        self._keep = ft
        return self

    @classmethod
    def weighted(cls, dmat: DMatrix, hessians, max_bin=256, ctx: Context = None):
        """HistCuts::from_dmatrix_weighted + GHistIndex::from_dmatrix
        (data/quantile.rs:81-122): the cuts and bins of one tree_method=approx
        round, numeric cuts at the hessian-weighted quantiles."""
        self = cls.__new__(cls)
        self.ctx = ctx or default_context()
        ft = dmat._ftypes()
        hs = _f32(hessians).reshape(-1)
        h = ctypes.c_void_p()
        A.check(A.lib().sb_ghist_create_weighted(self.ctx.h, A.ptr(dmat.data, ctypes.c_float), dmat.n_rows,
                                                 dmat.n_cols, A.ptr(ft, ctypes.c_uint8), dmat.missing, max_bin,
                                                 A.ptr(hs, ctypes.c_float), ctypes.byref(h)))
        self.h = h
        self._adopt(self.ctx)
        self._keep = ft
        return self

    def info(self):
        n, f, t = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        A.check(A.lib().sb_ghist_info(self.h, ctypes.byref(n), ctypes.byref(f), ctypes.byref(t)))
        return n.value, f.value, t.value

    @property
    def total_bins(self):
        return self.info()[2]

    def layout(self):
        """The device ELLPACK's form: {"layout": "tiled"|"lanes", "code_bytes":
        1|2, "row_stride": codes per row, "rows_per_instruction": 1..8}."""
        lay, cb, rpi = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        st = ctypes.c_size_t()
        A.check(A.lib().sb_ghist_layout(self.h, ctypes.byref(lay), ctypes.byref(cb), ctypes.byref(st),
                                        ctypes.byref(rpi)))
        return {"layout": "lanes" if lay.value == 1 else "tiled", "code_bytes": cb.value,
                "row_stride": st.value, "rows_per_instruction": rpi.value}

    def codes(self):
        """The row-major histogram codes as stored on the device: [n][row_stride]
        u8 or u16 (GHistIndex::bins, ghist.rs:117)."""
        lay = self.layout()
        n = self.info()[0]
        out = np.zeros((n, lay["row_stride"]), np.uint8 if lay["code_bytes"] == 1 else np.uint16)
        A.check(A.lib().sb_ghist_codes(self.h, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def cuts(self):
        """(feature_offset[F+1], cut_values[total_bins], is_categorical[F])."""
        n, f, t = self.info()
        off = np.zeros(f + 1, np.uint32)
        vals = np.zeros(t, np.float32)
        cat = np.zeros(f, np.uint8)
        A.check(A.lib().sb_ghist_cuts(self.h, A.ptr(off, ctypes.c_uint32), A.ptr(vals, ctypes.c_float),
                                      A.ptr(cat, ctypes.c_uint8)))
        return off, vals, cat

    def local_bins(self):
        n, f, _ = self.info()
        out = np.zeros((n, f), np.uint16)
        A.check(A.lib().sb_ghist_bins(self.h, A.ptr(out, ctypes.c_uint16)))
        return out

    def global_bins(self):
        """Global bin per entry (feature_offset[f] + local), UINT32_MAX = missing."""
        off, _, _ = self.cuts()
        lb = self.local_bins().astype(np.uint32)
        g = lb + off[:-1][None, :]
        g[lb == 0xFFFF] = 0xFFFFFFFF
        return g

    def _free(self, _A=A):
        _A.lib().sb_ghist_destroy(self.h)


def _gpair(gpair):
    g = np.ascontiguousarray(gpair, dtype=np.float32)
    if g.ndim == 1:
        g = g.reshape(-1, 2)
    return np.ascontiguousarray(g)


class GpuBackend:
    """HistogramBackend on the device (tree/hist/mod.rs:31-45)."""

    def __init__(self, precision="fp32", quantize_bits=0, ctx: Context = None):
        self.precision = A.SB_HIST_FIXED if precision == "fixed" else A.SB_HIST_FP32
        self.bits = quantize_bits
        self.ctx = ctx or default_context()

    def build(self, ghist: GHistIndex, rows, gpair, out=None):
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        g = _gpair(gpair)
        total = ghist.total_bins
        if out is None:
            out = np.zeros((total, 2), np.float64)
        A.check(A.lib().sb_hist_build(self.ctx.h, ghist.h, A.ptr(rows, ctypes.c_uint32), rows.size,
                                      g.ctypes.data_as(ctypes.POINTER(A.SbGradPair)), g.shape[0],
                                      self.precision, self.bits,
                                      out.ctypes.data_as(ctypes.POINTER(A.SbGradStats)), total))
        return out

    def subtract(self, parent, child, out=None):
        p = np.ascontiguousarray(parent, dtype=np.float64)
        c = np.ascontiguousarray(child, dtype=np.float64)
        if out is None:
            out = np.zeros_like(p)
        A.check(A.lib().sb_hist_subtract(self.ctx.h, p.ctypes.data_as(ctypes.POINTER(A.SbGradStats)),
                                         c.ctypes.data_as(ctypes.POINTER(A.SbGradStats)),
                                         out.ctypes.data_as(ctypes.POINTER(A.SbGradStats)),
                                         p.shape[0]))
        return out


NODE_DTYPE = np.dtype([
    ("left", "<i4"), ("right", "<i4"), ("split_feature", "<u4"), ("split_cond", "<f4"),
    ("leaf_value", "<f4"), ("sum_hess", "<f4"), ("split_gain", "<f4"), ("default_left", "u1"),
    ("is_categorical", "u1"), ("reserved", "<u2"), ("cat_begin", "<u4"), ("cat_end", "<u4")])
assert NODE_DTYPE.itemsize == ctypes.sizeof(A.SbNode)


class RegTree:
    """A host copy of one tree (tree/regtree.rs:74-83)."""

    def __init__(self, nodes, categories):
        self.nodes = nodes
        self.categories = categories

    def num_nodes(self):
        return len(self.nodes)

    def num_leaves(self):
        return int((self.nodes["left"] == -1).sum())


class BoostedModel(_Native):
    """The trained ensemble (learner/model.rs:34-54); arrays live on the host,
    a device copy is made on the first prediction."""

    def __init__(self, handle, ctx: Context):
        self.h = handle
        self.ctx = ctx
        self._adopt(ctx)

    @classmethod
    def from_arrays(cls, node_off, nodes, cat_off, cats, base_score, num_class, n_features,
                    objective="reg:squarederror", weights=None, ctx: Context = None):
        ctx = ctx or default_context()
        node_off = np.ascontiguousarray(node_off, np.int64)
        nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
        cat_off = np.ascontiguousarray(cat_off, np.int64)
        cats = np.ascontiguousarray(cats if len(cats) else np.zeros(1, np.uint32), np.uint32)
        v = A.SbModelView()
        v.tree_node_offset = A.ptr(node_off, ctypes.c_int64)
        v.nodes = nodes.ctypes.data_as(ctypes.POINTER(A.SbNode))
        v.tree_cat_offset = A.ptr(cat_off, ctypes.c_int64)
        v.categories = A.ptr(cats, ctypes.c_uint32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        v.tree_weights = A.ptr(w, ctypes.c_float)
        v.n_trees = len(node_off) - 1
        v.num_class = num_class
        v.n_features = n_features
        v.objective = OBJECTIVES.get(objective, objective) if isinstance(objective, str) else objective
        v.base_score = base_score
        h = ctypes.c_void_p()
        A.check(A.lib().sb_model_create(ctx.h, ctypes.byref(v), ctypes.byref(h)))
        return cls(h, ctx)

    def export(self):
        """(node_off, nodes, cat_off, cats, weights)."""
        nt, nn, nc = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        A.check(A.lib().sb_model_export_sizes(self.h, ctypes.byref(nt), ctypes.byref(nn),
                                              ctypes.byref(nc)))
        node_off = np.zeros(nt.value + 1, np.int64)
        nodes = np.zeros(nn.value, NODE_DTYPE)
        cat_off = np.zeros(nt.value + 1, np.int64)
        cats = np.zeros(max(nc.value, 1), np.uint32)
        w = np.zeros(max(nt.value, 1), np.float32)
        A.check(A.lib().sb_model_export(self.h, A.ptr(node_off, ctypes.c_int64),
                                        nodes.ctypes.data_as(ctypes.POINTER(A.SbNode)),
                                        A.ptr(cat_off, ctypes.c_int64), A.ptr(cats, ctypes.c_uint32),
                                        A.ptr(w, ctypes.c_float)))
        return node_off, nodes, cat_off, cats[:nc.value], w[:nt.value]

    def info(self):
        bs, k, f, o = ctypes.c_float(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        A.check(A.lib().sb_model_info(self.h, ctypes.byref(bs), ctypes.byref(k), ctypes.byref(f),
                                      ctypes.byref(o)))
        return bs.value, k.value, f.value, o.value

    def base_score(self):
        return self.info()[0]

    def n_outputs(self):
        k = self.info()[1]
        return k if k >= 2 else 1

    def num_trees(self):
        return len(self.export()[0]) - 1

    def trees(self):
        off, nodes, coff, cats, _ = self.export()
        return [RegTree(nodes[off[t]:off[t + 1]], cats[coff[t]:coff[t + 1]])
                for t in range(len(off) - 1)]

    def predict_margin_limited(self, d: DMatrix, ntree_limit=0):
        k = self.n_outputs()
        out = np.zeros((d.n_rows, k), np.float32)
        bm = None
        if d.base_margin is not None:
            bm = d.base_margin
            if bm.size == d.n_rows and k > 1:
                bm = np.repeat(bm.reshape(-1, 1), k, axis=1)
            bm = np.ascontiguousarray(bm.reshape(-1), np.float32)
        A.check(A.lib().sb_predict_margin(self.h, A.ptr(d.data, ctypes.c_float), d.n_rows, d.n_cols,
                                          d.missing, A.ptr(bm, ctypes.c_float), ntree_limit,
                                          A.ptr(out, ctypes.c_float)))
        return out.reshape(-1)

    def best_iteration(self):
        """Early stopping's pick, or None (model.rs:209-211)."""
        v = ctypes.c_int64()
        A.check(A.lib().sb_model_best_iteration(self.h, ctypes.byref(v)))
        return None if v.value < 0 else v.value

    def set_best_iteration(self, it):
        A.check(A.lib().sb_model_set_best_iteration(self.h, -1 if it is None else int(it)))

    def predict_margin(self, d: DMatrix):
        """predict_margin (model.rs:222-226): (best_iteration + 1) * K trees
        after early stopping, else all."""
        it = self.best_iteration()
        return self.predict_margin_limited(d, 0 if it is None else (it + 1) * self.n_outputs())

    def predict(self, d: DMatrix):
        k = self.n_outputs()
        out = np.zeros((d.n_rows, k), np.float32)
        bm = None
        if d.base_margin is not None:
            bm = np.ascontiguousarray(np.broadcast_to(d.base_margin.reshape(d.n_rows, -1),
                                                      (d.n_rows, k)).reshape(-1), np.float32)
        A.check(A.lib().sb_predict(self.h, A.ptr(d.data, ctypes.c_float), d.n_rows, d.n_cols, d.missing,
                                   A.ptr(bm, ctypes.c_float), A.ptr(out, ctypes.c_float)))
        return out.reshape(-1)

    def predict_contribs(self, d: DMatrix):
        k = self.n_outputs()
        out = np.zeros((d.n_rows, k, d.n_cols + 1), np.float32)
        A.check(A.lib().sb_predict_contribs(self.h, A.ptr(d.data, ctypes.c_float), d.n_rows, d.n_cols,
                                            d.missing, A.ptr(out, ctypes.c_float)))
        return out.reshape(-1)

    def objective_name(self):
        from .xgboost_json import OBJECTIVE_NAMES
        return OBJECTIVE_NAMES[self.info()[3]]

    def to_xgboost_json(self):
        """BoostedModel::to_xgboost_json (model.rs:435-437): the model in
        XGBoost's JSON model schema (numeric splits only, as the reference)."""
        from .xgboost_json import arrays_to_xgboost_json
        base, k, f, _ = self.info()
        off, nodes, _, _, _ = self.export()
        return arrays_to_xgboost_json(off, nodes, base, k, f, self.objective_name())

    @classmethod
    def from_xgboost_json(cls, text, ctx: Context = None):
        """BoostedModel::from_xgboost_json (model.rs:442-444)."""
        from .xgboost_json import xgboost_json_to_arrays
        off, nodes, coff, cats, base, k, f, obj = xgboost_json_to_arrays(text, NODE_DTYPE)
        return cls.from_arrays(off, nodes, coff, cats, base, k, f, objective=obj, ctx=ctx)

    def save_xgboost_json(self, path):
        with open(path, "w") as fh:
            fh.write(self.to_xgboost_json())

    @classmethod
    def load_xgboost_json(cls, path, ctx: Context = None):
        with open(path) as fh:
            return cls.from_xgboost_json(fh.read(), ctx=ctx)

    def predict_leaf(self, d: DMatrix):
        """Leaf node index per (row, tree), flat [n_rows * num_trees] u32
        (predict_leaf, model.rs:330-341)."""
        t = self.num_trees()
        out = np.zeros((d.n_rows, t), np.uint32)
        A.check(A.lib().sb_predict_leaf(self.h, A.ptr(d.data, ctypes.c_float), d.n_rows, d.n_cols, d.missing,
                                        A.ptr(out, ctypes.c_uint32)))
        return out.reshape(-1)

    def predict_interactions(self, d: DMatrix):
        """TreeSHAP interaction values, flat [n_rows][n_outputs][F+1][F+1]
        (predict_interactions, shap.rs:395-509)."""
        k = self.n_outputs()
        w = d.n_cols + 1
        out = np.zeros((d.n_rows, k, w, w), np.float32)
        A.check(A.lib().sb_predict_interactions(self.h, A.ptr(d.data, ctypes.c_float), d.n_rows, d.n_cols,
                                                d.missing, A.ptr(out, ctypes.c_float)))
        return out.reshape(-1)

    def _free(self, _A=A):
        _A.lib().sb_model_destroy(self.h)


def objective_gradient(objective, preds, labels, weights=None, num_class=0, scale_pos_weight=1.0,
                       ctx: Context = None):
    """Objective::gradient (objective/mod.rs:58-69) on the device: margins
    `preds` [n][K] -> GradPair [n][K] as an (n*K, 2) f32 array, with the code
    the boosting rounds use (sb_objective_gradient)."""
    ctx = ctx or default_context()
    if isinstance(objective, (int, np.integer)):
        code = int(objective)  # an SB_OBJ_* code
    elif objective in OBJECTIVES:
        code = OBJECTIVES[objective]
    else:
        raise A.SbError(A.SB_ERR_INVALID_ARG, f"unknown value `{objective}` for objective")
    preds = _f32(preds).reshape(-1)
    labels = _f32(labels).reshape(-1)
    w = None if weights is None else _f32(weights).reshape(-1)
    out = np.zeros((preds.size, 2), np.float32)
    A.check(A.lib().sb_objective_gradient(ctx.h, code, num_class, float(scale_pos_weight),
                                          A.ptr(preds, ctypes.c_float), A.ptr(labels, ctypes.c_float),
                                          A.ptr(w, ctypes.c_float), labels.size,
                                          out.ctypes.data_as(ctypes.POINTER(A.SbGradPair))))
    return out


def train(params: TrainingParams, dtrain: DMatrix, num_boost_round: int, ctx: Context = None):
    """learner/train.rs:107-113 (hist branch): upload, cuts, binning, rounds,
    model download — one C ABI call (sb_train)."""
    ctx = ctx or default_context()
    if dtrain.labels is None:
        raise A.SbError(A.SB_ERR_INVALID_ARG, "empty dataset: train: dtrain has no labels")
    if params.booster != "gbtree":
        params.validate()
        return _train_dart(params, dtrain, num_boost_round, ctx)
    p, keep = params.to_c()
    ft = dtrain._ftypes()
    bm = None
    k = params.num_class if params.objective.startswith("multi:") else 1
    if dtrain.base_margin is not None:
        bm = dtrain.base_margin
        if bm.size == dtrain.n_rows and k > 1:
            bm = np.repeat(bm.reshape(-1, 1), k, axis=1)
        bm = np.ascontiguousarray(bm.reshape(-1), np.float32)
    h = ctypes.c_void_p()
    A.check(A.lib().sb_train(ctx.h, A.ptr(dtrain.data, ctypes.c_float), dtrain.n_rows, dtrain.n_cols,
                             A.ptr(ft, ctypes.c_uint8), dtrain.missing,
                             A.ptr(dtrain.labels, ctypes.c_float), A.ptr(dtrain.weights, ctypes.c_float),
                             A.ptr(bm, ctypes.c_float), ctypes.byref(p), num_boost_round,
                             ctypes.byref(h)))
    del keep
    return BoostedModel(h, ctx)


METRICS = {"rmse": A.SB_METRIC_RMSE, "mae": A.SB_METRIC_MAE, "logloss": A.SB_METRIC_LOGLOSS,
           "error": A.SB_METRIC_ERROR, "mlogloss": A.SB_METRIC_MLOGLOSS, "merror": A.SB_METRIC_MERROR}
# Objective::default_metric (regression.rs:47, :83, classification.rs:93, multiclass.rs:107)
DEFAULT_METRIC = {"reg:squarederror": "rmse", "reg:linear": "rmse", "reg:pseudohubererror": "mae",
                  "binary:logistic": "logloss", "reg:logistic": "logloss", "multi:softmax": "mlogloss",
                  "multi:softprob": "mlogloss"}


def _metric_id(name):
    if name not in METRICS:
        raise A.SbError(A.SB_ERR_UNSUPPORTED, f"metric `{name}` is not computed on the device "
                                              f"(supported: {', '.join(METRICS)})")
    return METRICS[name]


@dataclass
class RoundEval:
    """One row of the evaluation history (train.rs:87-95)."""
    iteration: int
    scores: List[tuple]  # (eval set name, metric name, value)


@dataclass
class TrainResult:
    """train_with_eval's result (train.rs:97-104)."""
    model: "BoostedModel"
    history: List[RoundEval]


def train_with_eval(params: TrainingParams, dtrain: DMatrix, num_boost_round: int, evals=(),
                    early_stopping_rounds: Optional[int] = None, ctx: Context = None):
    """train_with_eval (learner/train.rs:121-140, loop :276-379): the rounds run
    on the device-resident booster, each eval set keeps its margin cache on the
    device, and only the metric values come back per round. Early stopping
    watches the last metric of the last eval set; it stops after
    `early_stopping_rounds` rounds without improvement and records the best
    round, which `predict` / `predict_margin` then use."""
    ctx = ctx or default_context()
    if dtrain.labels is None:
        raise A.SbError(A.SB_ERR_INVALID_ARG, "empty dataset: train: dtrain has no labels")
    if params.booster != "gbtree":
        params.validate()
        if evals:
            raise A.SbError(A.SB_ERR_UNSUPPORTED, "eval sets with booster=dart are not built")
        return TrainResult(_train_dart(params, dtrain, num_boost_round, ctx), [])
    names = list(params.eval_metric) or [DEFAULT_METRIC.get(params.objective, "rmse")]
    if len(names) > A.SB_EVAL_MAX_METRICS:
        raise A.SbError(A.SB_ERR_INVALID_ARG, f"at most {A.SB_EVAL_MAX_METRICS} metrics")
    for nm in names:
        _metric_id(nm)
    gh = GHistIndex(dtrain, max_bin=params.max_bin, ctx=ctx)
    k = params.num_class if params.objective.startswith("multi:") else 1
    bm = None
    if dtrain.base_margin is not None:
        bm = np.ascontiguousarray(np.broadcast_to(dtrain.base_margin.reshape(dtrain.n_rows, -1),
                                                  (dtrain.n_rows, k)).reshape(-1), np.float32)
    b = Booster(gh, params, dtrain.labels, weights=dtrain.weights, base_margin=bm, ctx=ctx)
    for d, _ in evals:
        b.add_eval(d)
    history = []
    # none of the device metrics is maximised (metric/mod.rs:15-17)
    stop = EarlyStopping(early_stopping_rounds, maximize=False)
    for rnd in range(num_boost_round):
        b.update(1)
        if not evals:
            continue
        vals = b.eval(names)
        scores = [(evals[e][1], names[j], float(vals[e, j])) for e in range(len(evals)) for j in range(len(names))]
        history.append(RoundEval(rnd, scores))
        if stop.update(rnd, scores[-1][2]):
            break
    m = b.model()
    if stop.best_iteration is not None:
        m.set_best_iteration(stop.best_iteration)
    return TrainResult(m, history)


_M64 = (1 << 64) - 1


def _mix64(z):
    """sb_mix64 of include/sb_sampling.h."""
    z = (z + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def dart_dropout(seed, rnd, existing, rate_drop, skip_drop):
    """DART's dropout set for round `rnd` over the `existing` trees
    (train.rs:397-425): skipped with probability skip_drop, else each tree
    with probability rate_drop, and at least one. The draws come from the
    SplitMix64 stream of sb_dart_key (include/sb_sampling.h), not rand 0.8."""
    s = _mix64((seed & _M64) ^ _mix64((rnd + 0x0DA27) & _M64) ^ 0x64617274)

    def nxt():
        nonlocal s
        x = _mix64(s)
        s = (s + 0x9E3779B97F4A7C15) & _M64
        return x

    def u01():
        return (nxt() >> 11) * (1.0 / 9007199254740992.0)

    if u01() < skip_drop or existing == 0:
        return []
    dropped = [i for i in range(existing) if u01() < rate_drop]
    if not dropped:
        dropped = [(nxt() * existing) >> 64]
    return dropped


def _train_dart(params, dtrain, num_boost_round, ctx):
    """dart_round (learner/train.rs:384-456) through sb_train_dart: per round,
    the margins of the ensemble minus the dropout set (dart_dropout's draws)
    are predicted on the device with the tree weights and handed to the
    booster, whose round grows the K new trees from their gradients; the new
    trees get weight 1/(k+1) and the k dropped trees are scaled by k/(k+1)."""
    p, keep = params.to_c()
    k_out = params.num_class if params.objective.startswith("multi:") else 1
    bm = None
    if dtrain.base_margin is not None:
        bm = np.ascontiguousarray(np.broadcast_to(dtrain.base_margin.reshape(dtrain.n_rows, -1),
                                                  (dtrain.n_rows, k_out)), np.float32).reshape(-1)
    ft = dtrain._ftypes()
    h = ctypes.c_void_p()
    A.check(A.lib().sb_train_dart(ctx.h, A.ptr(dtrain.data, ctypes.c_float), dtrain.n_rows, dtrain.n_cols,
                                  A.ptr(ft, ctypes.c_uint8), dtrain.missing,
                                  A.ptr(dtrain.labels, ctypes.c_float), A.ptr(dtrain.weights, ctypes.c_float),
                                  A.ptr(bm, ctypes.c_float), ctypes.byref(p), float(params.rate_drop),
                                  float(params.skip_drop), num_boost_round, ctypes.byref(h)))
    del keep
    return BoostedModel(h, ctx)


class EarlyStopping:
    """train_impl's early-stopping bookkeeping (train.rs:264-271, 350-377): the
    last metric of the last eval set must improve strictly within `patience`
    rounds; on a stop, `best_iteration` is the round of the best value."""

    def __init__(self, patience, maximize=False):
        self.patience = patience
        self.maximize = maximize
        self.best_score = -math.inf if maximize else math.inf
        self.best_round = 0
        self.since = 0
        self.best_iteration = None

    def update(self, rnd, value):
        """Records round `rnd`'s value; True when training must stop."""
        if self.patience is None:
            return False
        if (value > self.best_score) if self.maximize else (value < self.best_score):
            self.best_score, self.best_round, self.since = value, rnd, 0
            return False
        self.since += 1
        if self.since >= self.patience:
            self.best_iteration = self.best_round
            return True
        return False


def train_many(jobs, n_streams=32, ctx: Context = None):
    """Trains independent jobs together on the GPU (sb_train_many): `jobs` is
    a list of (TrainingParams, DMatrix with labels, num_boost_round). Returns
    one BoostedModel per job, each equal to what `train` gives for that job."""
    ctx = ctx or default_context()
    arr = (A.SbJob * len(jobs))()
    keep = []
    for i, (params, d, rounds) in enumerate(jobs):
        if d.labels is None:
            raise A.SbError(A.SB_ERR_INVALID_ARG, f"empty dataset: job {i} has no labels")
        p, kp = params.to_c()
        ft = d._ftypes()
        bm = None
        k = params.num_class if params.objective.startswith("multi:") else 1
        if d.base_margin is not None:
            bm = d.base_margin
            if bm.size == d.n_rows and k > 1:
                bm = np.repeat(bm.reshape(-1, 1), k, axis=1)
            bm = np.ascontiguousarray(bm.reshape(-1), np.float32)
        keep.append((p, kp, ft, bm, d))
        j = arr[i]
        j.X = A.ptr(d.data, ctypes.c_float)
        j.n_rows, j.n_cols = d.n_rows, d.n_cols
        j.feature_types = A.ptr(ft, ctypes.c_uint8)
        j.missing = d.missing
        j.labels = A.ptr(d.labels, ctypes.c_float)
        j.weights = A.ptr(d.weights, ctypes.c_float)
        j.base_margin = A.ptr(bm, ctypes.c_float)
        j.params = ctypes.pointer(p)
        j.num_boost_round = rounds
    st = A.lib().sb_train_many(ctx.h, arr, len(jobs), n_streams)
    models = [BoostedModel(ctypes.c_void_p(arr[i].out), ctx) if arr[i].out else None for i in range(len(jobs))]
    del keep
    A.check(st)
    return models


class HistTreeBuilder:
    """HistTreeBuilder::build (tree/builder/hist.rs:139-202) on the device."""

    def __init__(self, params: TrainingParams, ctx: Context = None):
        self.params = params
        self.ctx = ctx or default_context()

    def build(self, ghist: GHistIndex, gpair, row_subset, round=0, k=0, return_row_leaf=False):
        p, keep = self.params.to_c()
        g = _gpair(gpair)
        rows = np.ascontiguousarray(row_subset, np.uint32)
        n = g.shape[0]
        leaf = np.zeros(n, np.int32) if return_row_leaf else None
        h = ctypes.c_void_p()
        A.check(A.lib().sb_tree_build(self.ctx.h, ghist.h, ctypes.byref(p),
                                      g.ctypes.data_as(ctypes.POINTER(A.SbGradPair)), n,
                                      A.ptr(rows, ctypes.c_uint32), rows.size, round, k,
                                      A.ptr(leaf, ctypes.c_int32), ctypes.byref(h)))
        del keep
        m = BoostedModel(h, self.ctx)
        return (m, leaf) if return_row_leaf else m


class Booster(_Native):
    """The device-resident round loop (sb_booster): labels, margins,
    gradients and row lists stay on the GPU; `update(r)` runs r rounds."""

    def __init__(self, ghist: GHistIndex, params: TrainingParams, labels, weights=None,
                 base_margin=None, ctx: Context = None):
        self.ctx = ctx or ghist.ctx
        self.ghist = ghist
        self.params = params
        p, keep = params.to_c()
        lab = _f32(labels)
        w = None if weights is None else _f32(weights)
        bm = None if base_margin is None else _f32(base_margin)
        h = ctypes.c_void_p()
        A.check(A.lib().sb_booster_create(self.ctx.h, ghist.h, ctypes.byref(p),
                                          A.ptr(lab, ctypes.c_float), A.ptr(w, ctypes.c_float),
                                          A.ptr(bm, ctypes.c_float), ctypes.byref(h)))
        del keep
        self.h = h
        self._adopt(self.ctx, ghist)
        self.n = lab.shape[0]
        self.k = params.num_class if params.objective.startswith("multi:") else 1
        self._eval_rows = []

    def update(self, rounds=1):
        A.check(A.lib().sb_booster_update(self.h, rounds))

    def margins(self):
        out = np.zeros((self.n, self.k), np.float32)
        A.check(A.lib().sb_booster_margins(self.h, A.ptr(out, ctypes.c_float)))
        return out

    def set_margins(self, margins):
        """Replaces the margins [n][K] the next round takes its gradients from."""
        m = np.ascontiguousarray(margins, np.float32).reshape(self.n, self.k)
        A.check(A.lib().sb_booster_set_margins(self.h, A.ptr(m, ctypes.c_float)))

    def gradients(self):
        out = np.zeros((self.k, self.n, 2), np.float32)
        A.check(A.lib().sb_booster_gradients(self.h, out.ctypes.data_as(ctypes.POINTER(A.SbGradPair))))
        return out

    def row_mask(self, round_):
        out = np.zeros(self.n, np.uint8)
        A.check(A.lib().sb_booster_row_mask(self.h, round_, A.ptr(out, ctypes.c_uint8)))
        return out.astype(bool)

    def model(self):
        h = ctypes.c_void_p()
        A.check(A.lib().sb_booster_model(self.h, ctypes.byref(h)))
        return BoostedModel(h, self.ctx)

    def add_eval(self, d: DMatrix):
        """Attaches an eval set (its rows, labels, weights and margin cache go
        to the device); returns its index."""
        if d.labels is None:
            raise A.SbError(A.SB_ERR_INVALID_ARG, "an eval set needs labels")
        bm = None
        if d.base_margin is not None:
            bm = np.ascontiguousarray(np.broadcast_to(d.base_margin.reshape(d.n_rows, -1),
                                                      (d.n_rows, self.k)).reshape(-1), np.float32)
        eid = ctypes.c_int()
        A.check(A.lib().sb_booster_eval_add(self.h, A.ptr(d.data, ctypes.c_float), d.n_rows, d.n_cols, d.missing,
                                            A.ptr(d.labels, ctypes.c_float), A.ptr(d.weights, ctypes.c_float),
                                            A.ptr(bm, ctypes.c_float), ctypes.byref(eid)))
        self._eval_rows.append(d.n_rows)
        return eid.value

    def eval(self, metrics):
        """Metric values [n_eval_sets][len(metrics)] after the rounds grown so
        far; `metrics` are names (rmse, mae, logloss, error, mlogloss, merror)."""
        ids = [_metric_id(m) for m in metrics]
        n_e = len(self._eval_rows)
        out = np.zeros((max(n_e, 1), max(len(ids), 1)), np.float64)
        arr = (ctypes.c_int * max(len(ids), 1))(*ids)
        A.check(A.lib().sb_booster_eval(self.h, len(ids), arr, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out[:n_e, :len(ids)]

    def eval_margins(self, eval_id):
        """The margin cache of an eval set, [n_rows][n_outputs]."""
        out = np.zeros((self._eval_rows[eval_id], self.k), np.float32)
        A.check(A.lib().sb_booster_eval_margins(self.h, eval_id, A.ptr(out, ctypes.c_float)))
        return out

    def set_timing(self, on=True):
        A.check(A.lib().sb_booster_set_timing(self.h, 1 if on else 0))

    def set_graphs(self, on=True):
        """Replay steady-state rounds as one CUDA graph each (default on)."""
        A.check(A.lib().sb_booster_set_graphs(self.h, 1 if on else 0))

    def stats(self):
        s = A.SbBoosterStats()
        A.check(A.lib().sb_booster_stats_get(self.h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in A.SbBoosterStats._fields_}

    def reset_stats(self):
        A.check(A.lib().sb_booster_stats_reset(self.h))

    def _free(self, _A=A):
        _A.lib().sb_booster_destroy(self.h)


class Server(_Native):
    """The serving loop (sb_server): the model stays resident in HBM and margin
    / TreeSHAP requests from any thread are batched continuously on the
    device. `submit` returns a ticket; `wait` returns the request's output
    (the same array as `predict_margin` / `predict_contribs` would give) and
    its submit-to-done latency in ms."""

    KINDS = {"margin": A.SB_REQ_MARGIN, "contribs": A.SB_REQ_CONTRIBS}

    def __init__(self, model: BoostedModel, mem_bytes=0, n_slots=4, ctx: Context = None):
        self.model = model  # must outlive the loop
        self.ctx = ctx or model.ctx
        h = ctypes.c_void_p()
        A.check(A.lib().sb_server_create(self.ctx.h, model.h, mem_bytes, n_slots, ctypes.byref(h)))
        self.h = h
        self._adopt(self.ctx, model)
        self.k = model.n_outputs()
        self.f = model.info()[2]
        self._pending = {}

    def submit(self, x, kind="margin", missing=float("nan"), out=None):
        """Queues rows `x` [n][n_features] (kept referenced until `wait`)."""
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, self.f)
        n = x.shape[0]
        shape = (n, self.k) if kind == "margin" else (n, self.k, self.f + 1)
        if out is None:
            out = np.empty(shape, np.float32)
        t = ctypes.c_uint64()
        A.check(A.lib().sb_server_submit(self.h, self.KINDS[kind], A.ptr(x, ctypes.c_float), n, self.f,
                                         missing, A.ptr(out, ctypes.c_float), ctypes.byref(t)))
        self._pending[t.value] = (x, out)
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        lat = ctypes.c_double()
        st = A.lib().sb_server_wait(self.h, ticket, timeout_ms, ctypes.byref(lat))
        x, out = self._pending.pop(ticket)
        A.check(st)
        return out.reshape(-1), lat.value

    def stats(self):
        s = A.SbServerStats()
        A.check(A.lib().sb_server_stats_get(self.h, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_}

    def close(self):
        """Finishes every queued request, then stops the loop."""
        self._released = True
        self._drop()
        self._pending.clear()

    def _free(self, _A=A):
        _A.check(_A.lib().sb_server_destroy(self.h))
