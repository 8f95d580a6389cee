"""predict_margin / predict / predict_contribs on the GPU against the oracle."""
import numpy as np
import pytest

from gpu_helpers import mixed_data

pytestmark = pytest.mark.gpu


def _model(orc, x, y, ft=None, **kw):
    from sequoia_boost_b200 import TrainingParams
    p = TrainingParams(**kw)
    r = orc.train(x, y, p, 20, ftypes=ft)
    return p, r["model"].export(), r["model"].base_score


@pytest.mark.parametrize("kind", ["regression", "categorical", "multiclass"])
def test_margins_bit_exact(sb, ctx, orc, kind):
    ft = None
    if kind == "categorical":
        x, ft = mixed_data(8000, 10, seed=3, n_cat=3, card=12)
    else:
        x, _ = mixed_data(8000, 10, seed=4)
    rng = np.random.default_rng(5)
    if kind == "multiclass":
        y = rng.integers(0, 4, len(x)).astype(np.float32)
        kw = dict(objective="multi:softprob", num_class=4, max_depth=4, eta=0.3)
    else:
        y = (np.nan_to_num(x[:, 0]) * 2 + rng.standard_normal(len(x))).astype(np.float32)
        kw = dict(objective="reg:squarederror", max_depth=6, eta=0.2)
    p, arrays, base = _model(orc, x, y, ft, **kw)
    k = p.num_class if kind == "multiclass" else 0
    m = sb.BoostedModel.from_arrays(*arrays[:4], base, k, x.shape[1], objective=p.objective, ctx=ctx)
    xt, _ = mixed_data(3000, 10, seed=99, n_cat=3 if kind == "categorical" else 0, card=14)
    got = m.predict_margin(sb.DMatrix(xt))
    full = orc.predict_margin(arrays, xt, base, k)
    assert np.array_equal(got, full)
    for lim in (1, 7):
        got = m.predict_margin_limited(sb.DMatrix(xt), lim)
        want = orc.predict_margin(arrays, xt, base, k, ntree_limit=lim)
        assert np.array_equal(got, want)
    pr = m.predict(sb.DMatrix(xt))
    assert np.allclose(pr, orc.transform(p.objective, full, max(k, 0)), rtol=1e-6, atol=1e-7)


def test_base_margin_overrides_base_score(sb, ctx, orc):
    x, _ = mixed_data(2000, 6, seed=6)
    y = np.random.default_rng(1).standard_normal(2000).astype(np.float32)
    p, arrays, base = _model(orc, x, y, max_depth=4)
    m = sb.BoostedModel.from_arrays(*arrays[:4], base, 0, 6, ctx=ctx)
    bm = np.linspace(-1, 1, 2000).astype(np.float32)
    got = m.predict_margin(sb.DMatrix(x, base_margin=bm))
    want = orc.predict_margin(arrays, x, base, 0, base_margin=bm)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("multiclass", [False, True])
def test_contribs_match_oracle_and_add_up(sb, ctx, orc, multiclass):
    x, _ = mixed_data(1500, 8, seed=7)
    rng = np.random.default_rng(2)
    if multiclass:
        y = rng.integers(0, 3, len(x)).astype(np.float32)
        kw = dict(objective="multi:softprob", num_class=3, max_depth=4, eta=0.3)
        k = 3
    else:
        y = (np.nan_to_num(x[:, 1]) - np.nan_to_num(x[:, 2]) + 0.1 * rng.standard_normal(len(x)))
        y = y.astype(np.float32)
        kw = dict(objective="reg:squarederror", max_depth=6, eta=0.3)
        k = 0
    p, arrays, base = _model(orc, x, y, **kw)
    m = sb.BoostedModel.from_arrays(*arrays[:4], base, k, 8, objective=p.objective, ctx=ctx)
    got = m.predict_contribs(sb.DMatrix(x))
    want = orc.predict_contribs(arrays, x, base, k)
    assert np.max(np.abs(got - want)) < 1e-4
    kk = max(k, 1)
    margin = orc.predict_margin(arrays, x, base, k).reshape(len(x), kk)
    sums = got.reshape(len(x), kk, 9).astype(np.float64).sum(axis=2)
    assert np.max(np.abs(sums - margin)) < 1e-4


def test_dimension_mismatch(sb, ctx, orc):
    x, _ = mixed_data(500, 6, seed=6)
    y = np.zeros(500, np.float32)
    p, arrays, base = _model(orc, x, y, max_depth=2)
    m = sb.BoostedModel.from_arrays(*arrays[:4], base, 0, 6, ctx=ctx)
    with pytest.raises(sb.SbError):
        m.predict_margin(sb.DMatrix(x[:, :5]))


def test_margins_bit_exact_many_classes_and_trees(sb, ctx, orc):
    """More than 16 classes (the running sums leave shared memory) and more
    trees than one chunk of the prediction kernel: random stumps and depth-2
    trees, against the oracle's sequential sum."""
    from sequoia_boost_b200.api import NODE_DTYPE
    rng = np.random.default_rng(17)
    K, rounds, f = 20, 15, 6  # 300 trees
    trees = []
    for t in range(K * rounds):
        nd = np.zeros(3, NODE_DTYPE)
        nd["left"] = [1, -1, -1]
        nd["right"] = [2, -1, -1]
        nd["split_feature"][0] = rng.integers(0, f)
        nd["split_cond"][0] = rng.standard_normal()
        nd["default_left"][0] = rng.integers(0, 2)
        nd["leaf_value"][1:] = rng.standard_normal(2).astype(np.float32) * 0.1
        nd["sum_hess"] = [10.0, 4.0, 6.0]
        trees.append(nd)
    nodes = np.concatenate(trees)
    off = np.arange(0, 3 * len(trees) + 1, 3, dtype=np.int64)
    coff = np.zeros(len(trees) + 1, np.int64)
    cats = np.zeros(1, np.uint32)
    arrays = (off, nodes, coff, cats)
    m = sb.BoostedModel.from_arrays(off, nodes, coff, cats, 0.25, K, f, objective="multi:softprob", ctx=ctx)
    x, _ = mixed_data(777, f, seed=18)
    got = m.predict_margin(sb.DMatrix(x))
    want = orc.predict_margin(arrays, x, 0.25, K)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("objective", ["reg:squarederror", "binary:logistic", "multi:softprob"])
def test_xgboost_json_roundtrip_on_device(sb, ctx, tmp_path, objective):
    """BoostedModel.save_xgboost_json / load_xgboost_json (model.rs:446-455):
    a numeric model comes back with the same trees; margins agree within
    the base_score link's rounding (xgboost_json.rs:459-486)."""
    x, _ = mixed_data(4000, 8, seed=11)
    rng = np.random.default_rng(12)
    kw = dict(objective=objective, max_depth=4, eta=0.3)
    if objective == "multi:softprob":
        kw["num_class"] = 3
        y = rng.integers(0, 3, len(x)).astype(np.float32)
    elif objective == "binary:logistic":
        y = (np.nan_to_num(x[:, 0]) > 0).astype(np.float32)
    else:
        y = (np.nan_to_num(x[:, 0]) + rng.standard_normal(len(x))).astype(np.float32)
    m = sb.train(sb.TrainingParams(**kw), sb.DMatrix(x, labels=y), 10, ctx=ctx)
    path = tmp_path / "m.json"
    m.save_xgboost_json(str(path))
    r = sb.BoostedModel.load_xgboost_json(str(path), ctx=ctx)
    assert r.num_trees() == m.num_trees() and r.objective_name() == objective
    a, b = m.export(), r.export()
    for key in ("left", "right", "split_feature", "split_cond", "leaf_value", "default_left"):
        assert np.array_equal(a[1][key], b[1][key]), key
    d = sb.DMatrix(x)
    assert np.max(np.abs(m.predict(d) - r.predict(d))) < 1e-5


def _chain_data(n, f, seed):
    """y = the number of leading features (0, 1, 2, ...) above 0.1: every node
    of the chain x_0 > 0.1, x_1 > 0.1, ... has its best split on the next
    feature, so a lossguide tree grows one path through all f features."""
    rng = np.random.default_rng(seed)
    x = rng.random((n, f), dtype=np.float32)
    y = np.cumprod(x > 0.1, axis=1).sum(axis=1).astype(np.float32)
    return x, y


def _max_distinct_features(nodes, lo, hi):
    """Most distinct split features on a root-to-leaf path of one tree."""
    best = 0
    stack = [(0, frozenset())]
    while stack:
        i, feats = stack.pop()
        nd = nodes[lo + i]
        if nd["left"] == -1:
            best = max(best, len(feats))
            continue
        fs = feats | {int(nd["split_feature"])}
        stack.append((int(nd["left"]), fs))
        stack.append((int(nd["right"]), fs))
    return best


@pytest.mark.parametrize("f", [12, 30])
def test_contribs_of_deep_lossguide_paths(sb, ctx, orc, f):
    """shap.rs:321-367 on paths longer than the table form (10 features) and
    the register form (12) hold: lossguide trees with max_depth 0 whose paths
    split on 12 and on 30 distinct features. Contributions match the oracle's
    recursion within 1e-4 and add up to the margins."""
    x, y = _chain_data(40_000, f, seed=f)
    p = sb.TrainingParams(objective="reg:squarederror", grow_policy="lossguide", max_leaves=64, max_depth=0,
                          eta=0.5)
    r = orc.train(x, y, p, 3)
    arrays, base = r["model"].export(), r["model"].base_score
    off, nodes = arrays[0], arrays[1]
    deepest = max(_max_distinct_features(nodes, off[t], off[t + 1]) for t in range(len(off) - 1))
    assert deepest >= min(f, 20), deepest
    m = sb.BoostedModel.from_arrays(*arrays[:4], base, 0, f, objective=p.objective, ctx=ctx)
    xt = x[:3000]
    got = m.predict_contribs(sb.DMatrix(xt))
    want = orc.predict_contribs(arrays, xt, base, 0)
    assert np.max(np.abs(got - want)) < 1e-4
    margin = orc.predict_margin(arrays, xt, base, 0)
    sums = got.reshape(len(xt), f + 1).astype(np.float64).sum(axis=1)
    assert np.max(np.abs(sums - margin)) < 1e-4
