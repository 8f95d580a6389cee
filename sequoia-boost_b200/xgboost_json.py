"""XGBoost-format (JSON) model import and export, restating
crates/sequoia-boost/src/model/xgboost_json.rs.

The document layout is XGBoost's `Booster.save_model("m.json")` schema for a
`gbtree` booster: per tree, node-indexed parallel arrays (`left_children`,
`right_children`, `split_indices`, `split_conditions`, `default_left`,
`base_weights`, `loss_changes`, `sum_hessian`, ...). A node is a leaf when
`left_children[i] == -1`, and its weight is carried in `split_conditions[i]`
(and in `base_weights[i]`).

As in the reference (xgboost_json.rs:24-44):
  - only numeric splits round-trip: categorical splits, vector leaves and
    other booster kinds are not interpreted (`gblinear` / `dart` are rejected);
  - `base_score` is stored by XGBoost in the objective's output space, so
    export maps the margin through the objective's transform (scalar
    objectives only) and import maps it back with prob_to_margin.

The conversion works on the model's arrays (the form `BoostedModel.export`
returns and `BoostedModel.from_arrays` takes), so it runs on any host;
`BoostedModel.to_xgboost_json` / `from_xgboost_json` wrap it.
"""
import json
import math

import numpy as np

from . import _abi as A

INVALID_NODE = 2 ** 31 - 1  # XGBoost's parent of the root (kInvalidNodeId), xgboost_json.rs:53

OBJECTIVE_NAMES = {
    A.SB_OBJ_SQUARED_ERROR: "reg:squarederror",
    A.SB_OBJ_PSEUDOHUBER: "reg:pseudohubererror",
    A.SB_OBJ_LOGISTIC: "binary:logistic",
    A.SB_OBJ_SOFTMAX: "multi:softmax",
    A.SB_OBJ_SOFTPROB: "multi:softprob",
}
_LOGISTIC = ("binary:logistic", "reg:logistic")
_MULTICLASS = ("multi:softmax", "multi:softprob")
_SUPPORTED = ("reg:squarederror", "reg:linear", "reg:pseudohubererror") + _LOGISTIC + _MULTICLASS


class ModelFormatError(A.SbError):
    """SequoiaError::ModelFormat (error.rs): a document that is not a model
    this mirror can read."""

    def __init__(self, msg):
        super().__init__(A.SB_ERR_INVALID_ARG, f"model format: {msg}")
        self.detail = msg


def _f32(x):
    return float(np.float32(x))


def _link_export(margin, objective, num_class):
    """link_export, xgboost_json.rs:294-306: the forward transform for scalar
    objectives (sigmoid for logistic), the margin otherwise."""
    if objective in _LOGISTIC:
        x = np.float32(margin)
        with np.errstate(over="ignore"):
            if x >= 0:
                p = np.float32(1.0) / (np.float32(1.0) + np.exp(-x, dtype=np.float32))
            else:
                e = np.exp(x, dtype=np.float32)
                p = e / (np.float32(1.0) + e)
        return float(np.float32(p))
    return _f32(margin)


def _link_import(stored, objective, num_class):
    """link_import, xgboost_json.rs:308-314 with Objective::prob_to_margin
    (classification.rs:87-90 for logistic; the identity for the others)."""
    if objective in _LOGISTIC:
        p = min(max(np.float32(stored), np.float32(1e-6)), np.float32(1.0 - 1e-6))
        p = np.float32(p)
        return float(np.float32(np.log(np.float32(p / (np.float32(1.0) - p)), dtype=np.float32)))
    return _f32(stored)


def _objective_json(objective, num_class):
    """objective_to_json, xgboost_json.rs:322-338."""
    if objective in _MULTICLASS:
        return {"name": objective, "softmax_multiclass_param": {"num_class": str(num_class)}}
    if objective == "count:poisson":
        return {"name": objective, "poisson_regression_param": {"max_delta_step": "0.7"}}
    return {"name": objective, "reg_loss_param": {"scale_pos_weight": "1", "scale_pos_weight_default": "1"}}


def _tree_json(tid, nodes, num_feature):
    """tree_to_json, xgboost_json.rs:176-238."""
    n = len(nodes)
    leaf = nodes["left"] == -1
    parents = np.full(n, INVALID_NODE, np.int64)
    for i in np.nonzero(~leaf)[0]:
        parents[nodes["left"][i]] = i
        parents[nodes["right"][i]] = i
    left = [int(v) for v in nodes["left"]]
    right = [int(v) for v in nodes["right"]]
    split_indices = [0 if lf else int(f) for lf, f in zip(leaf, nodes["split_feature"])]
    split_conditions = [_f32(lv) if lf else _f32(c)
                        for lf, lv, c in zip(leaf, nodes["leaf_value"], nodes["split_cond"])]
    base_weights = [_f32(lv) if lf else 0.0 for lf, lv in zip(leaf, nodes["leaf_value"])]
    default_left = [1 if lf else int(d != 0) for lf, d in zip(leaf, nodes["default_left"])]
    loss_changes = [0.0 if lf else _f32(g) for lf, g in zip(leaf, nodes["split_gain"])]
    return {
        "id": tid,
        "tree_param": {"num_deleted": "0", "num_feature": str(num_feature), "num_nodes": str(n),
                       "size_leaf_vector": "0"},
        "left_children": left,
        "right_children": right,
        "parents": [int(p) for p in parents],
        "split_indices": split_indices,
        "split_conditions": split_conditions,
        "default_left": default_left,
        "base_weights": base_weights,
        "loss_changes": loss_changes,
        "sum_hessian": [_f32(h) for h in nodes["sum_hess"]],
        "split_type": [0] * n,  # numeric splits only
        "categories": [],
        "categories_nodes": [],
        "categories_segments": [],
        "categories_sizes": [],
    }


def arrays_to_xgboost_json(node_off, nodes, base_score, num_class, num_feature, objective):
    """export_xgboost_json, xgboost_json.rs:61-110, over a model's arrays;
    `objective` is the reference's objective name."""
    k = num_class if num_class >= 2 else 1
    n_trees = len(node_off) - 1
    trees = [_tree_json(t, nodes[node_off[t]:node_off[t + 1]], num_feature) for t in range(n_trees)]
    doc = {
        "version": [2, 0, 0],
        "learner": {
            "attributes": {},
            "feature_names": [],
            "feature_types": [],
            "gradient_booster": {
                "name": "gbtree",
                "model": {
                    "gbtree_model_param": {"num_parallel_tree": "1", "num_trees": str(n_trees)},
                    "tree_info": [t % k for t in range(n_trees)],
                    "trees": trees,
                },
            },
            "learner_model_param": {
                "base_score": str(np.float32(_link_export(base_score, objective, num_class))),
                "num_class": str(num_class),
                "num_feature": str(num_feature),
                "num_target": "1",
            },
            "objective": _objective_json(objective, num_class),
        },
    }
    return json.dumps(doc, indent=2)


def _scalar(v):
    """scalar_f64, xgboost_json.rs:347-356: a number, numeric string or bool."""
    if isinstance(v, bool):
        return 1.0 if v else 0.0
    if isinstance(v, (int, float)):
        return float(v)
    if isinstance(v, str):
        try:
            return float(v)
        except ValueError:
            return None
    return None


def _field(v, key):
    if not isinstance(v, dict) or key not in v:
        raise ModelFormatError(f"missing `{key}`")
    return v[key]


def _arr(tj, key):
    a = tj.get(key)
    if not isinstance(a, list):
        return None
    return [(_scalar(e) if _scalar(e) is not None else 0.0) for e in a]


def _tree_from_json(tj, node_dtype):
    """tree_from_json, xgboost_json.rs:241-291."""
    if not isinstance(tj, dict):
        raise ModelFormatError("a tree is not an object")
    left = _arr(tj, "left_children")
    if left is None:
        raise ModelFormatError("missing `left_children`")
    right = _arr(tj, "right_children")
    if right is None:
        raise ModelFormatError("missing `right_children`")
    cond = _arr(tj, "split_conditions")
    if cond is None:
        raise ModelFormatError("missing `split_conditions`")
    idx = _arr(tj, "split_indices") or []
    dleft = _arr(tj, "default_left") or []
    bw = _arr(tj, "base_weights") or []
    hess = _arr(tj, "sum_hessian") or []
    loss = _arr(tj, "loss_changes") or []

    def at(v, i):
        return v[i] if i < len(v) else 0.0

    n = len(left)
    nodes = np.zeros(n, node_dtype)
    for i in range(n):
        li = int(left[i])
        nodes["sum_hess"][i] = at(hess, i)
        nodes["is_categorical"][i] = 0
        if li == -1:
            lv = cond[i] if i < len(cond) else at(bw, i)
            nodes["left"][i] = -1
            nodes["right"][i] = -1
            nodes["leaf_value"][i] = lv
            nodes["default_left"][i] = 1
        else:
            ri = int(at(right, i))
            if not (0 <= li < n and 0 <= ri < n):
                raise ModelFormatError(f"node {i}: child out of range")
            nodes["left"][i] = li
            nodes["right"][i] = ri
            nodes["split_feature"][i] = int(at(idx, i))
            nodes["split_cond"][i] = at(cond, i)
            nodes["default_left"][i] = 1 if at(dleft, i) != 0.0 else 0
            nodes["split_gain"][i] = at(loss, i)
    return nodes


def xgboost_json_to_arrays(text, node_dtype):
    """import_xgboost_json, xgboost_json.rs:117-171: (node_off, nodes,
    cat_off, cats, base_score, num_class, num_feature, objective), base_score
    in margin space."""
    try:
        root = json.loads(text)
    except ValueError as e:
        raise ModelFormatError(f"not JSON: {e}") from None
    learner = _field(root, "learner")
    booster = _field(learner, "gradient_booster")
    name = booster.get("name", "gbtree") if isinstance(booster, dict) else "gbtree"
    if name != "gbtree":
        raise ModelFormatError(f"unsupported gradient_booster `{name}`: only `gbtree` is supported")
    model = _field(booster, "model")
    lmp = _field(learner, "learner_model_param")
    nf = _scalar(lmp.get("num_feature"))
    if nf is None:
        raise ModelFormatError("missing/invalid `num_feature`")
    nc = _scalar(lmp.get("num_class"))
    num_class = int(nc) if nc is not None else 0
    obj = learner.get("objective")
    objective = obj.get("name", "reg:squarederror") if isinstance(obj, dict) else "reg:squarederror"
    if objective not in _SUPPORTED:
        raise ModelFormatError(f"objective `{objective}` has no device transform here")
    trees_json = model.get("trees") if isinstance(model, dict) else None
    if not isinstance(trees_json, list):
        raise ModelFormatError("missing `model.trees` array")
    trees = []
    for i, tj in enumerate(trees_json):
        try:
            trees.append(_tree_from_json(tj, node_dtype))
        except ModelFormatError as e:
            raise ModelFormatError(f"tree {i}: {e.detail}") from None
    stored = _scalar(lmp.get("base_score"))
    if stored is None or not math.isfinite(stored):
        raise ModelFormatError("missing/invalid `base_score`")
    base = _link_import(np.float32(stored), objective, num_class)
    node_off = np.zeros(len(trees) + 1, np.int64)
    for t, nd in enumerate(trees):
        node_off[t + 1] = node_off[t] + len(nd)
    nodes = np.concatenate(trees) if trees else np.zeros(0, node_dtype)
    cat_off = np.zeros(len(trees) + 1, np.int64)
    return node_off, nodes, cat_off, np.zeros(0, np.uint32), base, num_class, int(nf), objective
