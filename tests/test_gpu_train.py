"""The boosting loop on the GPU (sb_train / sb_booster) against the oracle's
train_impl restatement."""
import json
import os

import numpy as np
import pytest

from engines import GpuEngine
from gpu_helpers import assert_trees_equal, mixed_data
from kat_checks import check_case

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [c for c in json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))["cases"]
         if c["kind"] in ("train", "train_cat_vs_num", "shap")
         and c["params"].get("grow_policy", 0) == 0]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_train_reference_kats(case, sb, ctx):
    check_case(case, GpuEngine(sb, ctx), sb.TrainingParams)


def _sine(n, f, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, f)).astype(np.float32)
    w = rng.uniform(-1, 1, f)
    y = (np.sin(x) @ w + 0.5 * x[:, 0] * x[:, 1] + rng.normal(0, 0.1, n)).astype(np.float32)
    return x, y


@pytest.mark.parametrize("sub", [1.0, 0.8])
def test_fixed_point_regression_model_bit_exact(sb, ctx, orc, sub):
    x, y = _sine(20000, 20, 1)
    x[np.random.default_rng(2).random(x.shape) < 0.05] = np.nan
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=6, eta=0.1, subsample=sub,
                          colsample_bytree=0.8, hist_precision="fixed", seed=4)
    m = sb.train(p, sb.DMatrix(x, labels=y), 8, ctx=ctx)
    ref = orc.train(x, y, p, 8)
    assert_trees_equal(m.export(), ref["model"].export())
    assert np.array_equal(m.predict_margin(sb.DMatrix(x)), ref["margins"].reshape(-1))


def test_booster_margins_follow_trees(sb, ctx, orc):
    """Device margins after each round equal the previous margins plus the new
    tree's leaf on the raw values (train.rs:326-328)."""
    x, y = _sine(10000, 10, 3)
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=5, eta=0.3, subsample=0.7,
                          hist_precision="fixed", seed=9)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    b = sb.Booster(gh, p, y)
    prev = b.margins().reshape(-1)
    for r in range(3):
        b.update(1)
        cur = b.margins().reshape(-1)
        arrays = b.model().export()
        last = tuple(a[-2:] if i in (0, 2) else a for i, a in enumerate(arrays[:4]))
        off, nodes, coff, cats = arrays[0][-2:], arrays[1], arrays[2][-2:], arrays[3]
        tree_only = (off - off[0], nodes[off[0]:off[1]], coff - coff[0], cats[coff[0]:coff[1]])
        add = orc.predict_margin(tree_only, x, 0.0, 0)
        assert np.array_equal(cur, (prev + add).astype(np.float32))
        prev = cur
        del last


def test_logistic_rounds_with_device_gradients(sb, ctx, orc):
    """Each round's tree equals the oracle's tree grown from the same round's
    device gradients (device expf may differ from glibc by an ulp, so the
    gradients are taken from the device)."""
    x, _ = mixed_data(20000, 12, seed=12)
    rng = np.random.default_rng(13)
    y = (rng.random(20000) < 1 / (1 + np.exp(-np.nan_to_num(x[:, 0]) * 2))).astype(np.float32)
    p = sb.TrainingParams(objective="binary:logistic", max_depth=6, eta=0.3, subsample=0.8,
                          colsample_bytree=0.8, hist_precision="fixed", seed=21)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    b = sb.Booster(gh, p, y)
    d = orc.data(x)
    for r in range(4):
        b.update(1)
        g = b.gradients()[0]
        rows = np.nonzero(b.row_mask(r))[0].astype(np.uint32)
        assert np.array_equal(rows, orc.sample_rows(len(x), p, r))
        gq, _, _ = orc.quantize(g, 16)
        om = orc.tree_build(d, p, gq, rows, round_=r)
        oa = om.export()
        # the booster stores eta-scaled leaves; the builder does not
        ga = b.model().export()
        t0, t1 = ga[0][r], ga[0][r + 1]
        gn = ga[1][t0:t1].copy()
        on = oa[1].copy()
        leaf = on["left"] == -1
        on["leaf_value"][leaf] = (on["leaf_value"][leaf] * np.float32(p.eta)).astype(np.float32)
        assert_trees_equal((np.array([0, t1 - t0]), gn, None, None), (oa[0], on, None, None),
                           check_cats=False)


@pytest.mark.parametrize("objective,metric", [("reg:squarederror", 0), ("binary:logistic", 1)])
@pytest.mark.parametrize("precision", ["fp32", "fixed"])
def test_metric_within_0p1_percent(sb, ctx, orc, objective, metric, precision):
    x, y = _sine(30000, 20, 5)
    if objective == "binary:logistic":
        y = (y > np.median(y)).astype(np.float32)
    p = sb.TrainingParams(objective=objective, max_depth=6, eta=0.1, subsample=0.8,
                          colsample_bytree=0.8, hist_precision=precision, seed=3)
    m = sb.train(p, sb.DMatrix(x, labels=y), 30, ctx=ctx)
    po = sb.TrainingParams(**{**p.__dict__, "hist_precision": "fp32"})
    ref = orc.train(x, y, po, 30)
    got = orc.metric(metric, m.predict(sb.DMatrix(x)), y)
    want = orc.metric(metric, orc.transform(objective, ref["margins"].reshape(-1)), y)
    assert abs(got - want) <= 1e-3 * want, (got, want)


def test_multiclass_softprob_trains(sb, ctx, orc):
    rng = np.random.default_rng(8)
    x = rng.random((6000, 8)).astype(np.float32)
    y = np.argmax(x[:, :3] + 0.1 * rng.standard_normal((6000, 3)), axis=1).astype(np.float32)
    p = sb.TrainingParams(objective="multi:softprob", num_class=3, max_depth=4, eta=0.3)
    m = sb.train(p, sb.DMatrix(x, labels=y), 20, ctx=ctx)
    assert m.num_trees() == 60
    pr = m.predict(sb.DMatrix(x)).reshape(-1, 3)
    assert np.allclose(pr.sum(axis=1), 1.0, atol=1e-5)
    ref = orc.train(x, y, p, 20)
    got = orc.metric(2, pr.reshape(-1), y, num_class=3)
    want = orc.metric(2, orc.transform(p.objective, ref["margins"].reshape(-1), 3), y, num_class=3)
    assert abs(got - want) <= 1e-3 * want, (got, want)


def test_zero_rounds_and_base_score(sb, ctx):
    x, y = _sine(500, 4, 1)
    p = sb.TrainingParams(objective="reg:squarederror", base_score=0.5)
    m = sb.train(p, sb.DMatrix(x, labels=y), 0, ctx=ctx)
    assert m.num_trees() == 0
    assert np.all(m.predict(sb.DMatrix(x)) == np.float32(0.5))


def test_graph_replayed_rounds_match_eager_rounds(sb, ctx):
    """Rounds replayed from a recorded CUDA graph give the same trees and
    margins as rounds launched kernel by kernel, across a tree-buffer growth
    (the graph is re-recorded) and a host read of the margins mid-way."""
    x, _ = mixed_data(30000, 16, seed=8)
    y = (np.nan_to_num(x[:, 0]) + 0.5 * np.nan_to_num(x[:, 1]) > 0).astype(np.float32)
    p = sb.TrainingParams(objective="binary:logistic", max_depth=6, eta=0.3, subsample=0.8,
                          colsample_bytree=0.8, hist_precision="fixed", seed=5)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    out = []
    for graphs in (True, False):
        b = sb.Booster(gh, p, y)
        b.set_graphs(graphs)
        for r in range(20):
            b.update(1)
            if r == 9:
                mid = b.margins().copy()
        out.append((b.model().export(), mid, b.margins()))
    (ma, mida, fa), (mb, midb, fb) = out
    assert_trees_equal(ma, mb)
    assert np.array_equal(mida, midb)
    assert np.array_equal(fa, fb)


@pytest.mark.parametrize("grow_policy", ["depthwise", "lossguide"])
def test_empty_row_draw_takes_one_row(sb, ctx, orc, grow_policy):
    """subsample so small that a round's Bernoulli draw keeps no row: the
    round takes the one fallback row (train.rs:472-474), every other row is
    routed through the tree for its leaf value, and the model and margins
    equal the oracle's."""
    x, y = _sine(500, 5, 7)
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=3, eta=0.5, subsample=1e-9,
                          min_child_weight=0.0, grow_policy=grow_policy, max_leaves=4 if grow_policy == "lossguide" else 0,
                          seed=11)
    m = sb.train(p, sb.DMatrix(x, labels=y), 3, ctx=ctx)
    ref = orc.train(x, y, p, 3)
    assert_trees_equal(m.export(), ref["model"].export())
    assert np.array_equal(m.predict_margin(sb.DMatrix(x)), ref["margins"].reshape(-1))


def test_row_grouping_does_not_change_the_model(sb, ctx):
    """Training on a narrow matrix with 1, 2, 4 or 8 rows per warp instruction
    of the histogram kernel (fixed point) gives bit-identical models."""
    from gpu_helpers import assert_trees_equal, hist_rows, mixed_data
    x, _ = mixed_data(30_000, 13, seed=61)
    y = (np.nan_to_num(x[:, 0]) - 0.5 * np.nan_to_num(x[:, 3]) > 0).astype(np.float32)
    p = sb.TrainingParams(objective="binary:logistic", max_depth=6, eta=0.3, subsample=0.8,
                          colsample_bytree=0.7, seed=5)
    d = sb.DMatrix(x, labels=y)
    models = []
    for rows in (1, 2, 4, 8):
        with hist_rows(rows):
            models.append(sb.train(p, d, 6, ctx=ctx))
    ref = models[0]
    for m in models[1:]:
        assert_trees_equal(m.export(), ref.export())
        assert np.array_equal(m.predict_margin(d), ref.predict_margin(d))
