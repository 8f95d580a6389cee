"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs load this module, as the checker or the timed CPU baseline. The struct
layouts below are declared independently of the product package; a test
checks that both match include/sb_gpu.h.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


class GradPair(ctypes.Structure):
    _fields_ = [("grad", ctypes.c_float), ("hess", ctypes.c_float)]


class GradStats(ctypes.Structure):
    _fields_ = [("grad", ctypes.c_double), ("hess", ctypes.c_double)]


class Node(ctypes.Structure):
    _fields_ = [("left", ctypes.c_int32), ("right", ctypes.c_int32), ("split_feature", ctypes.c_uint32),
                ("split_cond", ctypes.c_float), ("leaf_value", ctypes.c_float),
                ("sum_hess", ctypes.c_float), ("split_gain", ctypes.c_float),
                ("default_left", ctypes.c_uint8), ("is_categorical", ctypes.c_uint8),
                ("reserved", ctypes.c_uint16), ("cat_begin", ctypes.c_uint32),
                ("cat_end", ctypes.c_uint32)]


class Params(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("base_score", ctypes.c_double), ("eta", ctypes.c_double),
                ("gamma", ctypes.c_double), ("min_child_weight", ctypes.c_double),
                ("max_delta_step", ctypes.c_double), ("subsample", ctypes.c_double),
                ("colsample_bytree", ctypes.c_double), ("colsample_bylevel", ctypes.c_double),
                ("colsample_bynode", ctypes.c_double), ("lambda_", ctypes.c_double),
                ("alpha", ctypes.c_double), ("scale_pos_weight", ctypes.c_double),
                ("monotone", ctypes.POINTER(ctypes.c_int8)),
                ("interaction_offsets", ctypes.POINTER(ctypes.c_uint32)),
                ("interaction_features", ctypes.POINTER(ctypes.c_uint32)),
                ("objective", ctypes.c_int32), ("num_class", ctypes.c_int32),
                ("has_base_score", ctypes.c_int32), ("max_depth", ctypes.c_int32),
                ("max_leaves", ctypes.c_int32), ("grow_policy", ctypes.c_int32),
                ("max_bin", ctypes.c_int32), ("hist_precision", ctypes.c_int32),
                ("quantize_bits", ctypes.c_int32), ("n_monotone", ctypes.c_int32),
                ("n_interaction_groups", ctypes.c_int32), ("tree_method", ctypes.c_int32)]


class ModelView(ctypes.Structure):
    _fields_ = [("tree_node_offset", ctypes.POINTER(ctypes.c_int64)), ("nodes", ctypes.POINTER(Node)),
                ("tree_cat_offset", ctypes.POINTER(ctypes.c_int64)),
                ("categories", ctypes.POINTER(ctypes.c_uint32)),
                ("tree_weights", ctypes.POINTER(ctypes.c_float)), ("n_trees", ctypes.c_int32),
                ("num_class", ctypes.c_int32), ("n_features", ctypes.c_int32),
                ("objective", ctypes.c_int32), ("base_score", ctypes.c_float),
                ("reserved", ctypes.c_int32)]


NODE_DTYPE = np.dtype([
    ("left", "<i4"), ("right", "<i4"), ("split_feature", "<u4"), ("split_cond", "<f4"),
    ("leaf_value", "<f4"), ("sum_hess", "<f4"), ("split_gain", "<f4"), ("default_left", "u1"),
    ("is_categorical", "u1"), ("reserved", "<u2"), ("cat_begin", "<u4"), ("cat_end", "<u4")])

OBJ = {"reg:squarederror": 0, "reg:linear": 0, "reg:pseudohubererror": 1, "binary:logistic": 2,
       "reg:logistic": 2, "multi:softmax": 3, "multi:softprob": 4}

P = ctypes.c_void_p
SZ = ctypes.c_size_t
FP = ctypes.POINTER(ctypes.c_float)
U32P = ctypes.POINTER(ctypes.c_uint32)
U8P = ctypes.POINTER(ctypes.c_uint8)
I64P = ctypes.POINTER(ctypes.c_int64)
SIGS = {
    "orc_data_create": (P, [FP, SZ, SZ, U8P, ctypes.c_float, ctypes.c_int]),
    "orc_data_create_weighted": (P, [FP, SZ, SZ, U8P, ctypes.c_float, ctypes.c_int, FP]),
    "orc_data_destroy": (None, [P]),
    "orc_data_total_bins": (SZ, [P]),
    "orc_data_is_dense": (ctypes.c_int, [P]),
    "orc_data_cuts": (None, [P, U32P, FP, U8P]),
    "orc_data_dense_bins": (None, [P, U32P]),
    "orc_bin_of": (ctypes.c_uint32, [P, SZ, ctypes.c_float]),
    "orc_hist_build": (None, [P, U32P, SZ, ctypes.POINTER(GradPair), ctypes.POINTER(GradStats),
                              ctypes.c_int]),
    "orc_tree_build": (P, [P, ctypes.POINTER(Params), ctypes.POINTER(GradPair), U32P, SZ,
                           ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int]),
    "orc_train": (P, [P, FP, ctypes.POINTER(Params), FP, FP, FP, ctypes.c_int, ctypes.c_int, FP,
                      ctypes.POINTER(ctypes.c_double)]),
    "orc_train_dart": (P, [P, FP, ctypes.POINTER(Params), ctypes.c_double, ctypes.c_double, FP, FP, FP,
                           ctypes.c_int, ctypes.c_int, FP]),
    "orc_model_destroy": (None, [P]),
    "orc_model_sizes": (None, [P, ctypes.POINTER(ctypes.c_int32), I64P, I64P]),
    "orc_model_export": (None, [P, I64P, ctypes.POINTER(Node), I64P, U32P, FP, FP]),
    "orc_model_node_gaps": (None, [P, ctypes.POINTER(ctypes.c_double)]),
    "orc_predict_margin": (ctypes.c_int, [ctypes.POINTER(ModelView), FP, SZ, SZ, ctypes.c_float, FP,
                                          SZ, FP]),
    "orc_predict_contribs": (ctypes.c_int, [ctypes.POINTER(ModelView), FP, SZ, SZ, ctypes.c_float,
                                            FP]),
    "orc_predict_leaf": (ctypes.c_int, [ctypes.POINTER(ModelView), FP, SZ, SZ, ctypes.c_float, U32P]),
    "orc_predict_interactions": (ctypes.c_int, [ctypes.POINTER(ModelView), FP, SZ, SZ, ctypes.c_float,
                                                FP]),
    "orc_gradient": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_double, FP, FP, FP, SZ,
                            ctypes.POINTER(GradPair)]),
    "orc_pred_transform": (None, [ctypes.c_int, ctypes.c_int, FP, SZ]),
    "orc_metric": (ctypes.c_double, [ctypes.c_int, FP, FP, FP, SZ, ctypes.c_int]),
    "orc_base_margin": (ctypes.c_float, [ctypes.POINTER(Params), FP, FP, SZ]),
    "orc_quantize": (None, [ctypes.POINTER(GradPair), SZ, ctypes.c_int, ctypes.POINTER(GradPair),
                            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "orc_validate": (ctypes.c_int, [ctypes.POINTER(Params)]),
    "orc_sample_features": (ctypes.c_int, [SZ, ctypes.POINTER(Params), ctypes.c_uint64, ctypes.c_uint32,
                                           ctypes.c_uint64, U32P]),
    "orc_sample_rows": (SZ, [SZ, ctypes.POINTER(Params), ctypes.c_uint64, U32P]),
}


def _p(a, t):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(t))


def make_params(tp):
    """Oracle Params from a TrainingParams-like object (attribute names of
    the reference)."""
    p = Params()
    p.seed = tp.seed
    p.base_score = 0.0 if tp.base_score is None else float(tp.base_score)
    p.has_base_score = 0 if tp.base_score is None else 1
    p.eta, p.gamma, p.min_child_weight = tp.eta, tp.gamma, tp.min_child_weight
    p.max_delta_step, p.subsample = tp.max_delta_step, tp.subsample
    p.colsample_bytree, p.colsample_bylevel = tp.colsample_bytree, tp.colsample_bylevel
    p.colsample_bynode, p.lambda_, p.alpha = tp.colsample_bynode, tp.lambda_, tp.alpha
    p.scale_pos_weight = tp.scale_pos_weight
    p.objective = OBJ[tp.objective]
    p.num_class = tp.num_class
    p.max_depth, p.max_leaves = tp.max_depth, tp.max_leaves
    p.grow_policy = 1 if tp.grow_policy == "lossguide" else 0
    p.max_bin = tp.max_bin
    p.hist_precision = 1 if tp.hist_precision == "fixed" else 0
    p.tree_method = 1 if getattr(tp, "tree_method", "hist") == "approx" else 0
    p.quantize_bits = tp.quantize_bits
    keep = []
    if tp.monotone_constraints:
        m = np.asarray(tp.monotone_constraints, np.int8)
        keep.append(m)
        p.monotone = _p(m, ctypes.c_int8)
        p.n_monotone = len(m)
    if tp.interaction_constraints:
        offs, flat = [0], []
        for g in tp.interaction_constraints:
            flat += list(g)
            offs.append(len(flat))
        o = np.asarray(offs, np.uint32)
        fl = np.asarray(flat if flat else [0], np.uint32)
        keep += [o, fl]
        p.interaction_offsets = _p(o, ctypes.c_uint32)
        p.interaction_features = _p(fl, ctypes.c_uint32)
        p.n_interaction_groups = len(tp.interaction_constraints)
    return p, keep


class Oracle:
    def __init__(self):
        self.lib = ctypes.CDLL(LIB)
        for name, (res, args) in SIGS.items():
            fn = getattr(self.lib, name)
            fn.restype = res
            fn.argtypes = args

    # ---- data
    def data(self, x, ftypes=None, missing=float("nan"), max_bin=256):
        x = np.ascontiguousarray(x, np.float32)
        ft = None if ftypes is None else np.ascontiguousarray(ftypes, np.uint8)
        h = self.lib.orc_data_create(_p(x, ctypes.c_float), x.shape[0], x.shape[1],
                                     _p(ft, ctypes.c_uint8), missing, max_bin)
        if not h:
            raise ValueError("oracle rejected the dataset")
        return OData(self, h, x.shape[0], x.shape[1])

    def cuts(self, x, ftypes=None, missing=float("nan"), max_bin=256):
        return self.data(x, ftypes, missing, max_bin).cuts()

    def data_weighted(self, x, hessians, ftypes=None, missing=float("nan"), max_bin=256):
        """HistCuts::from_dmatrix_weighted (tree_method=approx) + GHistIndex."""
        x = np.ascontiguousarray(x, np.float32)
        w = np.ascontiguousarray(hessians, np.float32)
        assert w.size == x.shape[0]
        ft = None if ftypes is None else np.ascontiguousarray(ftypes, np.uint8)
        h = self.lib.orc_data_create_weighted(_p(x, ctypes.c_float), x.shape[0], x.shape[1],
                                              _p(ft, ctypes.c_uint8), missing, max_bin, _p(w, ctypes.c_float))
        if not h:
            raise ValueError("oracle rejected the dataset")
        return OData(self, h, x.shape[0], x.shape[1])

    # ---- trees / training
    def tree_build(self, d, params, gpair, rows, round_=0, k=0, threads=1):
        p, keep = make_params(params)
        g = np.ascontiguousarray(gpair, np.float32).reshape(-1, 2)
        r = np.ascontiguousarray(rows, np.uint32)
        h = self.lib.orc_tree_build(d.h, ctypes.byref(p), _p(g, GradPair), _p(r, ctypes.c_uint32),
                                    r.size, round_, k, threads)
        return OModel(self, h)

    def train(self, x, y, params, rounds, weights=None, base_margin=None, ftypes=None,
              missing=float("nan"), threads=1, want_metric=False, data=None):
        d = data if data is not None else self.data(x, ftypes, missing, params.max_bin)
        p, keep = make_params(params)
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        bm = None if base_margin is None else np.ascontiguousarray(base_margin, np.float32)
        k = params.num_class if params.objective.startswith("multi:") else 1
        margins = np.zeros((x.shape[0], k), np.float32)
        metric = np.zeros(max(rounds, 1), np.float64) if want_metric else None
        h = self.lib.orc_train(d.h, _p(x, ctypes.c_float), ctypes.byref(p), _p(y, ctypes.c_float),
                               _p(w, ctypes.c_float), _p(bm, ctypes.c_float), rounds, threads,
                               _p(margins, ctypes.c_float), _p(metric, ctypes.c_double))
        if not h:
            raise ValueError("oracle rejected the parameters")
        return {"model": OModel(self, h), "margins": margins,
                "metric": None if metric is None else metric[:rounds]}

    def train_dart(self, x, y, params, rounds, weights=None, base_margin=None, ftypes=None,
                   missing=float("nan"), threads=1):
        """dart_round (learner/train.rs:384-456); the model's export holds the
        tree weights."""
        d = self.data(x, ftypes, missing, params.max_bin)
        p, keep = make_params(params)
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        bm = None if base_margin is None else np.ascontiguousarray(base_margin, np.float32)
        k = params.num_class if params.objective.startswith("multi:") else 1
        margins = np.zeros((x.shape[0], k), np.float32)
        h = self.lib.orc_train_dart(d.h, _p(x, ctypes.c_float), ctypes.byref(p), float(params.rate_drop),
                                    float(params.skip_drop), _p(y, ctypes.c_float), _p(w, ctypes.c_float),
                                    _p(bm, ctypes.c_float), rounds, threads, _p(margins, ctypes.c_float))
        if not h:
            raise ValueError("oracle rejected the parameters")
        return {"model": OModel(self, h), "margins": margins}

    def sample_features(self, F, params, round_=0, k=0, nid=0):
        p, keep = make_params(params)
        out = np.zeros(F, np.uint32)
        m = self.lib.orc_sample_features(F, ctypes.byref(p), round_, k, nid, _p(out, ctypes.c_uint32))
        return out[:m]

    def sample_rows(self, n, params, round_=0):
        p, keep = make_params(params)
        out = np.zeros(n, np.uint32)
        m = self.lib.orc_sample_rows(n, ctypes.byref(p), round_, _p(out, ctypes.c_uint32))
        return out[:m]

    def validate(self, params):
        p, keep = make_params(params)
        return self.lib.orc_validate(ctypes.byref(p)) == 0

    # ---- objectives / metrics
    def gradient(self, objective, preds, labels, weights=None, num_class=0, spw=1.0):
        preds = np.ascontiguousarray(preds, np.float32)
        labels = np.ascontiguousarray(labels, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        out = np.zeros((preds.size, 2), np.float32)
        self.lib.orc_gradient(OBJ.get(objective, objective), num_class, spw, _p(preds, ctypes.c_float),
                              _p(labels, ctypes.c_float), _p(w, ctypes.c_float), labels.size,
                              _p(out, GradPair))
        return out

    def quantize(self, gpair, bits=16):
        g = np.ascontiguousarray(gpair, np.float32).reshape(-1, 2)
        out = np.zeros_like(g)
        sg, sh = ctypes.c_int(), ctypes.c_int()
        self.lib.orc_quantize(_p(g, GradPair), g.shape[0], bits, _p(out, GradPair), ctypes.byref(sg),
                              ctypes.byref(sh))
        return out, sg.value, sh.value

    def metric(self, kind, preds, labels, weights=None, num_class=0):
        preds = np.ascontiguousarray(preds, np.float32)
        labels = np.ascontiguousarray(labels, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        return self.lib.orc_metric(kind, _p(preds, ctypes.c_float), _p(labels, ctypes.c_float),
                                   _p(w, ctypes.c_float), labels.size, num_class)

    def transform(self, objective, preds, num_class=0):
        v = np.ascontiguousarray(preds, np.float32).copy()
        k = num_class if num_class >= 2 else 1
        self.lib.orc_pred_transform(OBJ.get(objective, objective), num_class, _p(v, ctypes.c_float),
                                    v.size // k)
        return v

    # ---- prediction on arbitrary ensembles
    def _view(self, arrays, base_score, num_class, n_features, objective=0):
        node_off, nodes, cat_off, cats = [np.ascontiguousarray(a) for a in arrays[:4]]
        weights = arrays[4] if len(arrays) > 4 else None
        cats = cats if len(cats) else np.zeros(1, np.uint32)
        v = ModelView()
        v.tree_node_offset = _p(node_off.astype(np.int64), ctypes.c_int64)
        keep = [node_off.astype(np.int64)]
        v.tree_node_offset = _p(keep[0], ctypes.c_int64)
        nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
        keep.append(nodes)
        v.nodes = nodes.ctypes.data_as(ctypes.POINTER(Node))
        co = np.ascontiguousarray(cat_off, np.int64)
        ca = np.ascontiguousarray(cats, np.uint32)
        keep += [co, ca]
        v.tree_cat_offset = _p(co, ctypes.c_int64)
        v.categories = _p(ca, ctypes.c_uint32)
        if weights is not None:
            w = np.ascontiguousarray(weights, np.float32)
            keep.append(w)
            v.tree_weights = _p(w, ctypes.c_float)
        v.n_trees = len(node_off) - 1
        v.num_class = num_class
        v.n_features = n_features
        v.objective = objective
        v.base_score = base_score
        return v, keep

    def predict_margin(self, arrays, x, base_score, num_class=0, missing=float("nan"),
                       base_margin=None, ntree_limit=0):
        x = np.ascontiguousarray(x, np.float32)
        v, keep = self._view(arrays, base_score, num_class, x.shape[1])
        k = num_class if num_class >= 2 else 1
        out = np.zeros(x.shape[0] * k, np.float32)
        bm = None if base_margin is None else np.ascontiguousarray(base_margin, np.float32)
        self.lib.orc_predict_margin(ctypes.byref(v), _p(x, ctypes.c_float), x.shape[0], x.shape[1],
                                    missing, _p(bm, ctypes.c_float), ntree_limit, _p(out, ctypes.c_float))
        return out

    def predict_contribs(self, arrays, x, base_score, num_class=0, missing=float("nan")):
        x = np.ascontiguousarray(x, np.float32)
        v, keep = self._view(arrays, base_score, num_class, x.shape[1])
        k = num_class if num_class >= 2 else 1
        out = np.zeros(x.shape[0] * k * (x.shape[1] + 1), np.float32)
        self.lib.orc_predict_contribs(ctypes.byref(v), _p(x, ctypes.c_float), x.shape[0], x.shape[1],
                                      missing, _p(out, ctypes.c_float))
        return out

    def predict_leaf(self, arrays, x, missing=float("nan")):
        """[n][n_trees] leaf node ids (predict_leaf, model.rs:330-341)."""
        x = np.ascontiguousarray(x, np.float32)
        v, keep = self._view(arrays, 0.0, 0, x.shape[1])
        out = np.zeros((x.shape[0], v.n_trees), np.uint32)
        self.lib.orc_predict_leaf(ctypes.byref(v), _p(x, ctypes.c_float), x.shape[0], x.shape[1], missing,
                                  _p(out, ctypes.c_uint32))
        return out

    def predict_interactions(self, arrays, x, base_score, num_class=0, missing=float("nan")):
        """[n][K][F+1][F+1] flattened (predict_interactions, shap.rs:395-509)."""
        x = np.ascontiguousarray(x, np.float32)
        v, keep = self._view(arrays, base_score, num_class, x.shape[1])
        k = num_class if num_class >= 2 else 1
        out = np.zeros(x.shape[0] * k * (x.shape[1] + 1) ** 2, np.float32)
        self.lib.orc_predict_interactions(ctypes.byref(v), _p(x, ctypes.c_float), x.shape[0], x.shape[1],
                                          missing, _p(out, ctypes.c_float))
        return out


class OData:
    def __init__(self, orc, h, n, f):
        self.orc, self.h, self.n, self.f = orc, h, n, f

    def total_bins(self):
        return self.orc.lib.orc_data_total_bins(self.h)

    def cuts(self):
        t = self.total_bins()
        off = np.zeros(self.f + 1, np.uint32)
        vals = np.zeros(t, np.float32)
        cat = np.zeros(self.f, np.uint8)
        self.orc.lib.orc_data_cuts(self.h, _p(off, ctypes.c_uint32), _p(vals, ctypes.c_float),
                                   _p(cat, ctypes.c_uint8))
        return off, vals, cat

    def global_bins(self):
        out = np.zeros((self.n, self.f), np.uint32)
        self.orc.lib.orc_data_dense_bins(self.h, _p(out, ctypes.c_uint32))
        return out

    def is_dense(self):
        return bool(self.orc.lib.orc_data_is_dense(self.h))

    def bin_of(self, f, v):
        return self.orc.lib.orc_bin_of(self.h, f, v)

    def hist(self, rows, gpair, threads=1):
        rows = np.ascontiguousarray(rows, np.uint32)
        g = np.ascontiguousarray(gpair, np.float32).reshape(-1, 2)
        out = np.zeros((self.total_bins(), 2), np.float64)
        self.orc.lib.orc_hist_build(self.h, _p(rows, ctypes.c_uint32), rows.size, _p(g, GradPair),
                                    _p(out, GradStats), threads)
        return out

    def __del__(self):
        if getattr(self, "h", None):
            self.orc.lib.orc_data_destroy(self.h)
            self.h = None


class OModel:
    def __init__(self, orc, h):
        self.orc, self.h = orc, h

    def export(self):
        nt, nn, nc = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        self.orc.lib.orc_model_sizes(self.h, ctypes.byref(nt), ctypes.byref(nn), ctypes.byref(nc))
        node_off = np.zeros(nt.value + 1, np.int64)
        nodes = np.zeros(nn.value, NODE_DTYPE)
        cat_off = np.zeros(nt.value + 1, np.int64)
        cats = np.zeros(max(nc.value, 1), np.uint32)
        w = np.zeros(max(nt.value, 1), np.float32)
        bs = ctypes.c_float()
        self.orc.lib.orc_model_export(self.h, _p(node_off, ctypes.c_int64),
                                      nodes.ctypes.data_as(ctypes.POINTER(Node)),
                                      _p(cat_off, ctypes.c_int64), _p(cats, ctypes.c_uint32),
                                      _p(w, ctypes.c_float), ctypes.byref(bs))
        self.base_score = bs.value
        return node_off, nodes, cat_off, cats[:nc.value], w[:nt.value]

    def gaps(self):
        _, nodes, _, _, _ = self.export()
        out = np.zeros(len(nodes), np.float64)
        self.orc.lib.orc_model_node_gaps(self.h, _p(out, ctypes.c_double))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            self.orc.lib.orc_model_destroy(self.h)
            self.h = None
