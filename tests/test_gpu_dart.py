"""booster=dart (learner/train.rs:384-456) over the device booster: the
reference's DART test restated, DART without dropout equal to gbtree, and
the tree weights honoured by prediction (model.rs:130-145)."""
import numpy as np
import pytest

from gpu_helpers import mixed_data

pytestmark = pytest.mark.gpu


def _step(sb, n):
    x = (np.arange(n, dtype=np.float32) / np.float32(n)).reshape(-1, 1)
    return x, (x[:, 0] >= 0.5).astype(np.float32)


def test_dart_trains_reduces_error_and_roundtrips(sb, ctx, orc):
    """train.rs:895-930: rate_drop 0.1, 60 rounds on the step data."""
    x, y = _step(sb, 120)
    d = sb.DMatrix(x, labels=y)
    p = sb.TrainingParams(objective="reg:squarederror", booster="dart", rate_drop=0.1, max_depth=3, eta=0.3)
    m = sb.train(p, d, 60, ctx=ctx)
    assert m.num_trees() == 60
    pred = m.predict(d)
    rmse = float(np.sqrt(np.mean((pred.astype(np.float64) - y) ** 2)))
    assert rmse < 0.1, rmse
    off, nodes, coff, cats, w = m.export()
    assert np.any(w < 1.0) and np.all(w > 0.0)  # some trees were dropped and rescaled
    # the weighted sum is what prediction computes (oracle as the checker)
    want = orc.predict_margin((off, nodes, coff, cats, w), x, m.base_score(), 0)
    assert np.array_equal(m.predict_margin(d), want)
    # the model's arrays, weights included, round-trip through the ABI
    r = sb.BoostedModel.from_arrays(off, nodes, coff, cats, m.base_score(), 0, 1, weights=w, ctx=ctx)
    assert np.max(np.abs(r.predict(d) - pred)) < 1e-6


@pytest.mark.parametrize("objective", ["reg:squarederror", "multi:softprob"])
def test_dart_without_dropout_is_gbtree(sb, ctx, objective):
    """skip_drop 1: no round drops a tree, every weight stays 1, and the
    trees are gbtree's (fixed point, so the histograms are order-free)."""
    x, _ = mixed_data(5000, 8, seed=61)
    rng = np.random.default_rng(62)
    kw = dict(objective=objective, max_depth=4, eta=0.3, subsample=0.8, hist_precision="fixed", seed=3)
    if objective == "multi:softprob":
        kw["num_class"] = 3
        y = rng.integers(0, 3, len(x)).astype(np.float32)
    else:
        y = (np.nan_to_num(x[:, 0]) + 0.1 * rng.standard_normal(len(x))).astype(np.float32)
    d = sb.DMatrix(x, labels=y)
    g = sb.train(sb.TrainingParams(**kw), d, 6, ctx=ctx)
    m = sb.train(sb.TrainingParams(booster="dart", rate_drop=0.5, skip_drop=1.0, **kw), d, 6, ctx=ctx)
    a, b = g.export(), m.export()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert np.all(b[4] == 1.0)
    assert np.array_equal(g.predict_margin(d), m.predict_margin(d))


def test_dart_multiclass_learns(sb, ctx):
    x, _ = mixed_data(4000, 6, seed=63)
    y = (np.nan_to_num(x[:, 0]) > 0).astype(np.float32) + (np.nan_to_num(x[:, 1]) > 0.5).astype(np.float32)
    p = sb.TrainingParams(objective="multi:softprob", num_class=3, booster="dart", rate_drop=0.2, max_depth=4,
                          eta=0.3)
    m = sb.train(p, sb.DMatrix(x, labels=y), 20, ctx=ctx)
    pr = m.predict(sb.DMatrix(x)).reshape(-1, 3)
    assert np.mean(np.argmax(pr, axis=1) == y) > 0.9
    with pytest.raises(sb.SbError):
        sb.train_with_eval(p, sb.DMatrix(x, labels=y), 2, [(sb.DMatrix(x, labels=y), "t")], ctx=ctx)


@pytest.mark.parametrize("objective", ["reg:squarederror", "reg:pseudohubererror"])
def test_dart_matches_the_oracle_restatement(sb, ctx, orc, objective):
    """dart_round (train.rs:384-456) against the oracle's restatement with the
    same dropout stream: the trees, their weights (1/(k+1) for new trees,
    k/(k+1) for dropped ones) and the margins equal the oracle's bit for bit
    on the default fixed-point form."""
    x, _ = mixed_data(6000, 8, seed=71)
    rng = np.random.default_rng(72)
    y = (np.sin(np.nan_to_num(x[:, 0])) + np.nan_to_num(x[:, 1]) + 0.1 * rng.standard_normal(len(x))).astype(np.float32)
    p = sb.TrainingParams(objective=objective, booster="dart", rate_drop=0.3, skip_drop=0.1, max_depth=4, eta=0.3,
                          subsample=0.8, seed=13)
    m = sb.train(p, sb.DMatrix(x, labels=y), 10, ctx=ctx)
    ref = orc.train_dart(x, y, p, 10)
    got, want = m.export(), ref["model"].export()
    from gpu_helpers import assert_trees_equal
    assert_trees_equal(got, want)
    assert np.array_equal(got[4], want[4])
    assert np.any(got[4] < 1.0)
    assert np.array_equal(m.predict_margin(sb.DMatrix(x)), ref["margins"].reshape(-1))
