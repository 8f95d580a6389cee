"""HistTreeBuilder::build on the GPU against the oracle.

Fixed-point form: gradients are rounded to the per-call power-of-two grid;
the oracle grows its tree from the same rounded values, and every f64 sum is
then exact on both sides, so the trees must match bit for bit: structure,
thresholds, default directions, leaf values, sum_hess, gains, categories and
the row-to-leaf assignment. FP32 form: structure must match wherever the
oracle's best-vs-runner-up gain gap exceeds the tolerance."""
import json
import os
import zlib

import numpy as np
import pytest

from engines import GpuEngine
from gpu_helpers import LAYOUTS, assert_trees_equal, hist_layout, leaf_ids, mixed_data, random_gpair
from kat_checks import check_case

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [c for c in json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))["cases"]
         if c["kind"] in ("leaf_weight", "split_gain", "tree", "tree_same")
         and c["params"].get("grow_policy", 0) == 0]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_tree_reference_kats(case, sb, ctx):
    check_case(case, GpuEngine(sb, ctx), sb.TrainingParams)


VARIANTS = {
    "plain": dict(max_depth=6),
    "deep_subset": dict(max_depth=8, lambda_=0.5),
    "colsample": dict(max_depth=6, colsample_bytree=0.8, colsample_bylevel=0.7, colsample_bynode=0.8,
                      seed=11),
    "regularised": dict(max_depth=5, alpha=0.3, max_delta_step=4.0, gamma=0.05, min_child_weight=3.0),
    "monotone": dict(max_depth=6, monotone_constraints=[1, -1, 0, 1]),
    "interaction": dict(max_depth=6, interaction_constraints=[[0, 1, 2], [3, 4], [5, 6, 7, 8]]),
}


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("logistic", [False, True])
def test_fixed_point_tree_bit_exact(sb, ctx, orc, variant, logistic, layout):
    n, f = 40000, 12
    x, _ = mixed_data(n, f, seed=zlib.crc32(variant.encode()) % 1000)
    g = random_gpair(n, seed=5, logistic=logistic)
    rng = np.random.default_rng(6)
    rows = np.sort(rng.choice(n, int(n * 0.8), replace=False)).astype(np.uint32)
    p = sb.TrainingParams(hist_precision="fixed", **VARIANTS[variant])
    with hist_layout(layout):
        gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    m, row_leaf = sb.HistTreeBuilder(p, ctx=ctx).build(gh, g, rows, round=3, return_row_leaf=True)
    gq, _, _ = orc.quantize(g, 16)
    om = orc.tree_build(orc.data(x), p, gq, rows, round_=3)
    ga, oa = m.export(), om.export()
    assert len(ga[1]) > 7, "tree too small to be a useful check"
    assert_trees_equal(ga, oa)
    # row-to-node assignment: every subset row ends in the same leaf
    want = leaf_ids(oa[1], oa[3], x)
    in_subset = np.zeros(n, bool)
    in_subset[rows] = True
    assert np.array_equal(row_leaf[in_subset], want[in_subset])
    assert np.all(row_leaf[~in_subset] == -1)


@pytest.mark.parametrize("layout", LAYOUTS)
def test_fixed_point_categorical_tree_bit_exact(sb, ctx, orc, layout):
    n, f = 30000, 10
    x, ft = mixed_data(n, f, seed=21, n_cat=3, card=24)
    g = random_gpair(n, seed=8)
    rows = np.arange(n, dtype=np.uint32)
    p = sb.TrainingParams(hist_precision="fixed", max_depth=6)
    with hist_layout(layout):
        gh = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), ctx=ctx)
    m = sb.HistTreeBuilder(p, ctx=ctx).build(gh, g, rows)
    gq, _, _ = orc.quantize(g, 16)
    om = orc.tree_build(orc.data(x, ft), p, gq, rows)
    ga, oa = m.export(), om.export()
    assert ga[1]["is_categorical"].any(), "expected categorical splits"
    assert_trees_equal(ga, oa)


def _compare_structure(gn, on, gaps, tol):
    """BFS over the oracle tree; below a node whose gain gap is within tol
    the two trees may legitimately differ."""
    stack = [(0, 0)]
    checked = 0
    while stack:
        gi, oi = stack.pop()
        a, b = gn[gi], on[oi]
        if b["left"] == -1:
            assert a["left"] == -1, ("oracle leaf, gpu split", oi)
            assert abs(a["leaf_value"] - b["leaf_value"]) <= 1e-4 * max(1.0, abs(b["leaf_value"]))
            checked += 1
            continue
        if abs(gaps[oi]) <= tol * max(1.0, abs(b["split_gain"])):
            continue
        assert a["left"] != -1, ("gpu leaf, oracle split", oi)
        assert (a["split_feature"], a["split_cond"], a["default_left"]) == \
            (b["split_feature"], b["split_cond"], b["default_left"]), (oi, a, b)
        stack.append((a["left"], b["left"]))
        stack.append((a["right"], b["right"]))
        checked += 1
    return checked


@pytest.mark.parametrize("variant", ["plain", "colsample", "monotone"])
def test_fp32_tree_structure(sb, ctx, orc, variant):
    n, f = 40000, 12
    x, _ = mixed_data(n, f, seed=31)
    g = random_gpair(n, seed=9, logistic=True)
    rows = np.arange(n, dtype=np.uint32)
    p = sb.TrainingParams(hist_precision="fp32", **VARIANTS[variant])
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    m = sb.HistTreeBuilder(p, ctx=ctx).build(gh, g, rows, round=1)
    om = orc.tree_build(orc.data(x), p, g, rows, round_=1)
    gaps = om.gaps()
    checked = _compare_structure(m.export()[1], om.export()[1], gaps, 1e-5)
    assert checked > 10


@pytest.mark.parametrize("scale", [3e-3, 1e-3])
def test_near_tie_gains_follow_sequential_rule(sb, ctx, orc, scale):
    """Small gradients put many candidate gains within 1e-6 of each other, and
    duplicated columns give exactly equal gains: the device must reproduce
    consider's sequential `g > best + 1e-6` rule exactly (fixed-point form)."""
    n = 4000
    rng = np.random.default_rng(17)
    base = rng.standard_normal((n, 4)).astype(np.float32)
    x = np.concatenate([base, base[:, ::-1], np.round(base, 1), base[:, :2]], axis=1)
    g = np.stack([rng.standard_normal(n) * scale, np.ones(n)], axis=1).astype(np.float32)
    rows = np.arange(n, dtype=np.uint32)
    p = sb.TrainingParams(hist_precision="fixed", max_depth=5, min_child_weight=0.0, lambda_=1.0)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    m = sb.HistTreeBuilder(p, ctx=ctx).build(gh, g, rows)
    gq, _, _ = orc.quantize(g, 16)
    om = orc.tree_build(orc.data(x), p, gq, rows)
    assert_trees_equal(m.export(), om.export())
