"""predict_leaf and predict_interactions on the GPU against the oracle, and
the interaction-value properties the reference's own tests assert
(learner/shap.rs:662-778: row consistency, efficiency, symmetry)."""
import json
import os

import numpy as np
import pytest

from engines import GpuEngine
from gpu_helpers import mixed_data
from kat_checks import check_case

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [c for c in json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))["cases"]
         if c["kind"] == "interactions"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_interaction_reference_kats(case, sb, ctx):
    check_case(case, GpuEngine(sb, ctx), sb.TrainingParams)


def _model(sb, ctx, orc, kind, n=4000, f=10, rounds=12, depth=5):
    ft = None
    if kind == "categorical":
        x, ft = mixed_data(n, f, seed=31, n_cat=3, card=12)
    else:
        x, _ = mixed_data(n, f, seed=32)
    rng = np.random.default_rng(33)
    if kind == "multiclass":
        y = rng.integers(0, 3, len(x)).astype(np.float32)
        kw = dict(objective="multi:softprob", num_class=3, max_depth=depth, eta=0.3)
    else:
        y = (np.nan_to_num(x[:, 0]) * 2 - np.nan_to_num(x[:, 1]) * np.nan_to_num(x[:, 2])
             + 0.1 * rng.standard_normal(len(x))).astype(np.float32)
        kw = dict(objective="reg:squarederror", max_depth=depth, eta=0.3)
    p = sb.TrainingParams(**kw)
    r = orc.train(x, y, p, rounds, ftypes=ft)
    arrays, base = r["model"].export(), r["model"].base_score
    k = p.num_class if kind == "multiclass" else 0
    m = sb.BoostedModel.from_arrays(*arrays[:4], base, k, f, objective=p.objective, ctx=ctx)
    return m, arrays, base, k, x, ft


@pytest.mark.parametrize("kind", ["regression", "categorical", "multiclass"])
def test_predict_leaf_bit_exact(sb, ctx, orc, kind):
    m, arrays, base, k, x, ft = _model(sb, ctx, orc, kind)
    xt, _ = mixed_data(3000, 10, seed=34, n_cat=3 if kind == "categorical" else 0, card=14)
    got = m.predict_leaf(sb.DMatrix(xt))
    want = orc.predict_leaf(arrays, xt)
    assert got.dtype == np.uint32 and got.shape == (len(xt) * m.num_trees(),)
    assert np.array_equal(got, want.reshape(-1))
    # every id is a leaf of its tree
    ids = got.reshape(len(xt), -1)
    off, nodes = arrays[0], arrays[1]
    for t in range(ids.shape[1]):
        assert np.all(nodes["left"][off[t] + ids[:, t]] == -1)


@pytest.mark.parametrize("kind", ["regression", "categorical", "multiclass"])
def test_interactions_match_oracle(sb, ctx, orc, kind):
    m, arrays, base, k, x, ft = _model(sb, ctx, orc, kind, n=3000, f=8, rounds=8)
    xt, _ = mixed_data(150, 8, seed=35, n_cat=3 if kind == "categorical" else 0, card=14)
    kk = max(k, 1)
    w = 9
    got = m.predict_interactions(sb.DMatrix(xt)).reshape(len(xt), kk, w, w).astype(np.float64)
    want = orc.predict_interactions(arrays, xt, base, k).reshape(len(xt), kk, w, w).astype(np.float64)
    scale = max(1.0, float(np.max(np.abs(want))))
    assert np.max(np.abs(got - want)) <= 1e-4 * scale, float(np.max(np.abs(got - want)))
    # the reference's properties, against this build's own contributions and margins
    contribs = m.predict_contribs(sb.DMatrix(xt)).reshape(len(xt), kk, w).astype(np.float64)
    margin = m.predict_margin(sb.DMatrix(xt)).reshape(len(xt), kk).astype(np.float64)
    assert np.max(np.abs(got[:, :, :w - 1, :].sum(axis=3) - contribs[:, :, :w - 1])) < 1e-4
    if kind != "categorical":
        # the reference's TreeSHAP routes categorical nodes by `v < split_cond`
        # (shap.rs:207-211), not by category, so with categorical splits the
        # values need not add up to the margin; the oracle check above holds
        assert np.max(np.abs(got.sum(axis=(2, 3)) - (margin - base))) < 1e-4
    assert np.max(np.abs(got - got.transpose(0, 1, 3, 2))) < 1e-5


def test_interactions_of_a_deep_ensemble_add_up(sb, ctx, orc):
    """Depth-8 trees (paths of up to 9 elements) over 40 features."""
    x, _ = mixed_data(20000, 40, seed=36)
    rng = np.random.default_rng(37)
    y = (np.nan_to_num(x[:, :5]).sum(axis=1) + rng.standard_normal(len(x))).astype(np.float32)
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=8, eta=0.1)
    m = sb.train(p, sb.DMatrix(x, labels=y), 30, ctx=ctx)
    xt = x[:64]
    w = 41
    got = m.predict_interactions(sb.DMatrix(xt)).reshape(len(xt), w, w).astype(np.float64)
    contribs = m.predict_contribs(sb.DMatrix(xt)).reshape(len(xt), w).astype(np.float64)
    margin = m.predict_margin(sb.DMatrix(xt)).astype(np.float64)
    assert np.max(np.abs(got[:, :w - 1, :].sum(axis=2) - contribs[:, :w - 1])) < 1e-4
    assert np.max(np.abs(got.sum(axis=(1, 2)) - (margin - m.base_score()))) < 1e-4
    assert np.max(np.abs(got - got.transpose(0, 2, 1))) < 1e-5
    arrays = m.export()
    want = orc.predict_interactions(arrays, xt, m.base_score(), 0).reshape(len(xt), w, w)
    assert np.max(np.abs(got - want)) <= 1e-4 * max(1.0, float(np.max(np.abs(want))))


def test_interactions_and_leaf_edge_cases(sb, ctx, orc):
    m, arrays, base, k, x, ft = _model(sb, ctx, orc, "regression", n=2000, f=10, rounds=3)
    lib = sb._abi.lib()
    # zero rows through the C ABI (a DMatrix has at least one row)
    assert lib.sb_predict_leaf(m.h, None, 0, 10, float("nan"), None) == 0
    assert lib.sb_predict_interactions(m.h, None, 0, 10, float("nan"), None) == 0
    with pytest.raises(sb.SbError):
        m.predict_interactions(sb.DMatrix(np.zeros((3, 9), np.float32)))
    with pytest.raises(sb.SbError):
        m.predict_leaf(sb.DMatrix(np.zeros((3, 11), np.float32)))
