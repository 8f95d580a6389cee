"""grow_lossguide (hist.rs:238-268) on the GPU against the oracle: the
per-tree priority queue pops nodes in the reference's order (Rust
BinaryHeap steps), so fixed-point trees match the oracle bit for bit, with
all K class trees of a round expanded step by step in the same launches."""
import json
import os

import numpy as np
import pytest

from engines import GpuEngine
from gpu_helpers import assert_trees_equal, leaf_ids, mixed_data, random_gpair
from kat_checks import check_case

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [c for c in json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))["cases"]
         if c.get("params", {}).get("grow_policy", 0) == 1]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_lossguide_reference_kats(case, sb, ctx):
    check_case(case, GpuEngine(sb, ctx), sb.TrainingParams)


VARIANTS = {
    "leaves8": dict(max_leaves=8, max_depth=0),
    "leaves31": dict(max_leaves=31, max_depth=0),
    "leaves64_depth5": dict(max_leaves=64, max_depth=5),
    "depth_only": dict(max_leaves=0, max_depth=4),
    "colsample": dict(max_leaves=40, max_depth=0, colsample_bytree=0.8, colsample_bylevel=0.7,
                      colsample_bynode=0.8, seed=3),
    "regularised": dict(max_leaves=48, max_depth=0, alpha=0.2, gamma=0.05, min_child_weight=3.0),
    "monotone": dict(max_leaves=48, max_depth=0, monotone_constraints=[1, -1, 0, 1]),
    "interaction": dict(max_leaves=48, max_depth=0, interaction_constraints=[[0, 1, 2], [3, 4], [5, 6, 7]]),
}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("logistic", [False, True])
def test_fixed_point_lossguide_tree_bit_exact(sb, ctx, orc, variant, logistic):
    n, f = 40000, 12
    x, _ = mixed_data(n, f, seed=17 + len(variant))
    g = random_gpair(n, seed=9, logistic=logistic)
    rng = np.random.default_rng(4)
    rows = np.sort(rng.choice(n, int(n * 0.8), replace=False)).astype(np.uint32)
    p = sb.TrainingParams(hist_precision="fixed", grow_policy="lossguide", **VARIANTS[variant])
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    m, row_leaf = sb.HistTreeBuilder(p, ctx=ctx).build(gh, g, rows, round=2, return_row_leaf=True)
    gq, _, _ = orc.quantize(g, 16)
    om = orc.tree_build(orc.data(x), p, gq, rows, round_=2)
    ga, oa = m.export(), om.export()
    assert len(ga[1]) > 7, "tree too small to be a useful check"
    assert_trees_equal(ga, oa)
    want = leaf_ids(oa[1], oa[3], x)
    in_subset = np.zeros(n, bool)
    in_subset[rows] = True
    assert np.array_equal(row_leaf[in_subset], want[in_subset])
    assert np.all(row_leaf[~in_subset] == -1)


def test_fixed_point_lossguide_categorical_tree_bit_exact(sb, ctx, orc):
    n, f = 30000, 10
    x, ft = mixed_data(n, f, seed=23, n_cat=3, card=20)
    g = random_gpair(n, seed=12)
    rows = np.arange(n, dtype=np.uint32)
    p = sb.TrainingParams(hist_precision="fixed", grow_policy="lossguide", max_leaves=32, max_depth=0)
    gh = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), ctx=ctx)
    m = sb.HistTreeBuilder(p, ctx=ctx).build(gh, g, rows)
    gq, _, _ = orc.quantize(g, 16)
    om = orc.tree_build(orc.data(x, ft), p, gq, rows)
    ga, oa = m.export(), om.export()
    assert ga[1]["is_categorical"].any(), "expected categorical splits"
    assert_trees_equal(ga, oa)


def test_lossguide_multiclass_rounds_bit_exact(sb, ctx, orc):
    """softprob with lossguide: all class trees of a round grow in the same
    launches. Round 0 (equal margins) matches the oracle's whole model; each
    later class tree matches the oracle's tree grown from that round's device
    gradients (device expf may differ from glibc's by an ulp)."""
    n, f = 20000, 10
    rng = np.random.default_rng(31)
    x = rng.standard_normal((n, f)).astype(np.float32)
    x[rng.random(x.shape) < 0.05] = np.nan
    w = rng.standard_normal((f, 3))
    y = np.argmax(np.nan_to_num(x) @ w + rng.gumbel(size=(n, 3)), axis=1).astype(np.float32)
    p = sb.TrainingParams(objective="multi:softprob", num_class=3, grow_policy="lossguide", max_leaves=24,
                          max_depth=0, eta=0.3, subsample=0.8, colsample_bytree=0.8, hist_precision="fixed",
                          monotone_constraints=[1, -1], seed=6)
    m = sb.train(p, sb.DMatrix(x, labels=y), 1, ctx=ctx)
    ref = orc.train(x, y, p, 1)
    assert_trees_equal(m.export(), ref["model"].export())
    assert np.array_equal(m.predict_margin(sb.DMatrix(x)), ref["margins"].reshape(-1))

    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    b = sb.Booster(gh, p, y)
    d = orc.data(x)
    for r in range(3):
        b.update(1)
        grads = b.gradients()
        rows = np.nonzero(b.row_mask(r))[0].astype(np.uint32)
        ga = b.model().export()
        for k in range(3):
            gq, _, _ = orc.quantize(grads[k], 16)
            oa = orc.tree_build(d, p, gq, rows, round_=r, k=k).export()
            t0, t1 = ga[0][3 * r + k], ga[0][3 * r + k + 1]
            gn = ga[1][t0:t1].copy()
            on = oa[1].copy()
            leaf = on["left"] == -1  # the booster stores eta-scaled leaves
            on["leaf_value"][leaf] = (on["leaf_value"][leaf] * np.float32(p.eta)).astype(np.float32)
            assert_trees_equal((np.array([0, t1 - t0]), gn, None, None), (oa[0], on, None, None),
                               check_cats=False)


def test_lossguide_graph_rounds_match_eager_rounds(sb, ctx):
    x, _ = mixed_data(20000, 10, seed=41)
    y = (np.nan_to_num(x[:, 0]) > 0).astype(np.float32)
    p = sb.TrainingParams(objective="binary:logistic", grow_policy="lossguide", max_leaves=20, max_depth=0,
                          eta=0.3, hist_precision="fixed", seed=2)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    out = []
    for graphs in (True, False):
        b = sb.Booster(gh, p, y)
        b.set_graphs(graphs)
        b.update(6)
        out.append((b.model().export(), b.margins()))
    assert_trees_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
