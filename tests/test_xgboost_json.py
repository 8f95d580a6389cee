"""XGBoost-format JSON import/export (model/xgboost_json.rs) on the host,
with the oracle as the predictor: the reference's own tests
(xgboost_json.rs:441-527) restated."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def xj(sb):
    from sequoia_boost_b200 import xgboost_json
    return xgboost_json


def _node_dtype(orc):
    from sb_pyoracle import NODE_DTYPE
    return NODE_DTYPE


def _roundtrip(xj, orc, x, y, p, rounds, objective):
    r = orc.train(x, y, p, rounds)
    arrays = r["model"].export()
    base = r["model"].base_score
    k = p.num_class if p.objective.startswith("multi:") else 0
    text = xj.arrays_to_xgboost_json(arrays[0], arrays[1], base, k, x.shape[1], objective)
    back = xj.xgboost_json_to_arrays(text, _node_dtype(orc))
    return arrays, base, back


def test_roundtrip_reg_preserves_predictions(sb, orc, xj):
    """xgboost_json.rs:441-457."""
    n = 120
    a = np.arange(n, dtype=np.float32) / np.float32(n)
    b = ((np.arange(n) * 7) % n).astype(np.float32) / np.float32(n)
    x = np.stack([a, b], axis=1)
    y = (2 * a - 3 * b + np.where(a > 0.5, 1.0, -1.0)).astype(np.float32)
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=3, eta=0.3)
    arrays, base, back = _roundtrip(xj, orc, x, y, p, 15, "reg:squarederror")
    off, nodes, coff, cats, base2, k2, f2, obj = back
    assert len(off) - 1 == len(arrays[0]) - 1 and f2 == 2 and obj == "reg:squarederror"
    before = orc.predict_margin(arrays, x, base, 0)
    after = orc.predict_margin((off, nodes, coff, cats), x, base2, k2)
    assert np.max(np.abs(before - after)) < 1e-5


def test_roundtrip_binary_preserves_predictions(sb, orc, xj):
    """xgboost_json.rs:459-486: base_score goes through the logit / sigmoid link."""
    n = 80
    x = (np.arange(n, dtype=np.float32) / np.float32(n)).reshape(-1, 1)
    y = (x[:, 0] > 0.4).astype(np.float32)
    p = sb.TrainingParams(objective="binary:logistic", max_depth=3, eta=0.3)
    arrays, base, back = _roundtrip(xj, orc, x, y, p, 20, "binary:logistic")
    off, nodes, coff, cats, base2, k2, f2, obj = back
    assert obj == "binary:logistic"
    assert abs(base2 - base) < 1e-4
    before = orc.transform(p.objective, orc.predict_margin(arrays, x, base, 0))
    after = orc.transform(p.objective, orc.predict_margin((off, nodes, coff, cats), x, base2, 0))
    assert np.max(np.abs(before - after)) < 1e-5


HAND_STUMP = """{
  "version": [2, 0, 0],
  "learner": {
    "gradient_booster": {
      "name": "gbtree",
      "model": {
        "gbtree_model_param": {"num_parallel_tree": "1", "num_trees": "1"},
        "tree_info": [0],
        "trees": [{
          "id": 0,
          "tree_param": {"num_nodes": "3", "num_feature": "1", "size_leaf_vector": "0"},
          "left_children":  [1, -1, -1],
          "right_children": [2, -1, -1],
          "parents":        [2147483647, 0, 0],
          "split_indices":  [0, 0, 0],
          "split_conditions": [1.5, 10.0, -10.0],
          "default_left":   [1, 0, 0],
          "base_weights":   [0.0, 10.0, -10.0],
          "loss_changes":   [42.0, 0.0, 0.0],
          "sum_hessian":    [8.0, 5.0, 3.0],
          "split_type":     [0, 0, 0]
        }]
      }
    },
    "learner_model_param": {"base_score": "0", "num_class": "0", "num_feature": "1"},
    "objective": {"name": "reg:squarederror"}
  }
}"""


def test_import_hand_written_stump_routes_correctly(sb, orc, xj):
    """xgboost_json.rs:488-540: a stump written by hand in XGBoost's schema."""
    off, nodes, coff, cats, base, k, f, obj = xj.xgboost_json_to_arrays(HAND_STUMP, _node_dtype(orc))
    assert len(off) - 1 == 1 and f == 1 and base == 0.0
    m = orc.predict_margin((off, nodes, coff, cats), np.array([[1.0], [2.0], [np.nan]], np.float32), base, k)
    assert np.allclose(m, [10.0, -10.0, 10.0], atol=1e-6)  # missing follows default_left


def test_unsupported_documents_are_rejected(sb, xj, orc):
    """xgboost_json.rs:542-548 (gblinear), and documents that are not models."""
    gbl = ('{"learner": {"gradient_booster": {"name": "gblinear"},'
           ' "learner_model_param": {"num_feature": "3", "base_score": "0"}}}')
    for text in (gbl, "not json", '{"learner": {}}',
                 HAND_STUMP.replace('"right_children": [2, -1, -1]', '"right_children": [7, -1, -1]')):
        with pytest.raises(xj.ModelFormatError):
            xj.xgboost_json_to_arrays(text, _node_dtype(orc))


def test_export_layout_matches_xgboost_schema(sb, orc, xj):
    import json
    x = np.random.default_rng(1).random((300, 4)).astype(np.float32)
    y = np.random.default_rng(2).integers(0, 3, 300).astype(np.float32)
    p = sb.TrainingParams(objective="multi:softprob", num_class=3, max_depth=2, eta=0.3)
    arrays, base, back = _roundtrip(xj, orc, x, y, p, 4, "multi:softprob")
    r = orc.train(x, y, p, 4)
    a = r["model"].export()
    doc = json.loads(xj.arrays_to_xgboost_json(a[0], a[1], r["model"].base_score, 3, 4, "multi:softprob"))
    gb = doc["learner"]["gradient_booster"]["model"]
    assert gb["tree_info"] == [t % 3 for t in range(12)]
    assert doc["learner"]["objective"]["softmax_multiclass_param"]["num_class"] == "3"
    t0 = gb["trees"][0]
    assert t0["parents"][0] == 2 ** 31 - 1
    leaf = [i for i, v in enumerate(t0["left_children"]) if v == -1]
    assert all(t0["split_conditions"][i] == t0["base_weights"][i] for i in leaf)
    off, nodes, coff, cats, base2, k2, f2, obj = back
    mb = orc.predict_margin(a, x, r["model"].base_score, 3)
    ma = orc.predict_margin((off, nodes, coff, cats), x, base2, k2)
    assert np.array_equal(mb, ma)
