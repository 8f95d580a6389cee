"""tree_method=approx on the GPU against the oracle's restatement of
HistCuts::from_dmatrix_weighted (data/quantile.rs:81-122, :253-316) and of
the Prepared::Approx round (learner/train.rs:46-53).

The weighted cuts must equal the oracle's bit for bit for the same hessians:
the device adds the weights in value order in f64 exactly as the reference's
sequential `cum += w as f64`, and places cuts with the same comparisons."""
import math

import numpy as np
import pytest

from gpu_helpers import assert_trees_equal, mixed_data

pytestmark = pytest.mark.gpu


def _same_index(gh, od):
    got_off, got_vals, got_cat = gh.cuts()
    want_off, want_vals, want_cat = od.cuts()
    assert np.array_equal(got_off, want_off)
    assert np.array_equal(got_vals.view(np.uint32), want_vals.view(np.uint32))
    assert np.array_equal(got_cat, want_cat)
    assert np.array_equal(gh.global_bins(), od.global_bins())


def _logistic_hessians(n, seed):
    rng = np.random.default_rng(seed)
    p = 1.0 / (1.0 + np.exp(-rng.standard_normal(n) * 3))
    return np.maximum(p * (1 - p), 1e-16).astype(np.float32)


@pytest.mark.parametrize("max_bin", [16, 256])
def test_weighted_cuts_regression_shape(sb, ctx, orc, max_bin):
    """100k x 30 N(0,1) features (the regression workload's shape) with
    logistic-like hessians spanning many magnitudes."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal((100_000, 30)).astype(np.float32)
    h = _logistic_hessians(x.shape[0], 4)
    gh = sb.GHistIndex.weighted(sb.DMatrix(x), h, max_bin=max_bin, ctx=ctx)
    _same_index(gh, orc.data_weighted(x, h, max_bin=max_bin))


def test_weighted_cuts_binary_mixed_shape(sb, ctx, orc, datagen):
    """The binary workload's columns (normal, lognormal, Bernoulli, 10% NaN)
    at 200k rows, with the hessians of a logistic round."""
    x, y = datagen.binary_mixed(n=200_000, seed=5, chunk=100_000)
    p = np.clip(np.nanmean(np.nan_to_num(x[:, :5]), axis=1) * 0.5 + 0.5, 0.01, 0.99)
    h = (p * (1 - p)).astype(np.float32)
    gh = sb.GHistIndex.weighted(sb.DMatrix(x), h, max_bin=256, ctx=ctx)
    _same_index(gh, orc.data_weighted(x, h, max_bin=256))


def test_weighted_cuts_edge_cases(sb, ctx, orc):
    """Ties across weight boundaries, +0.0 and -0.0, few distinct values,
    categorical columns, an all-missing column, zero weights and a column
    whose weights are all zero (unweighted positions)."""
    n = 20_000
    rng = np.random.default_rng(8)
    x = np.zeros((n, 8), np.float32)
    x[:, 0] = np.round(rng.standard_normal(n) * 4) / 4          # heavy ties
    x[:, 1] = np.where(rng.random(n) < 0.5, -0.0, 0.0)          # signed zeros among others
    x[:200, 1] = rng.standard_normal(200)
    x[:, 2] = rng.integers(0, 5, n)                               # few distinct values
    x[:, 3] = rng.integers(0, 40, n)                              # categorical
    x[:, 4] = np.nan                                              # all missing
    x[:, 5] = rng.standard_normal(n)
    x[rng.random(n) < 0.3, 5] = np.nan
    x[:, 6] = rng.exponential(1.0, n)
    x[:, 7] = rng.standard_normal(n)
    ft = np.zeros(8, np.uint8)
    ft[3] = 1
    h = rng.uniform(0.0, 1.0, n).astype(np.float32)
    h[rng.random(n) < 0.2] = 0.0
    for weights in (h, np.zeros(n, np.float32), np.ones(n, np.float32)):
        d = sb.DMatrix(x, feature_types=ft)
        for mb in (8, 64):
            gh = sb.GHistIndex.weighted(d, weights, max_bin=mb, ctx=ctx)
            _same_index(gh, orc.data_weighted(x, weights, ftypes=ft, max_bin=mb))


def test_unit_weights_reproduce_hist_cuts(sb, ctx):
    """With all weights equal the weighted cuts are the hist cuts
    (build_feature_cuts_weighted's doc, quantile.rs:248-252)."""
    x, _ = mixed_data(30_000, 12, seed=2)
    a = sb.GHistIndex(sb.DMatrix(x), max_bin=64, ctx=ctx).cuts()
    b = sb.GHistIndex.weighted(sb.DMatrix(x), np.ones(len(x), np.float32), max_bin=64, ctx=ctx).cuts()
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_weighted_cuts_reject_bad_hessians(sb, ctx):
    x, _ = mixed_data(100, 3, seed=1)
    for bad in (-1.0, np.nan, np.inf):
        h = np.ones(100, np.float32)
        h[7] = bad
        with pytest.raises(sb.SbError):
            sb.GHistIndex.weighted(sb.DMatrix(x), h, ctx=ctx)


@pytest.mark.parametrize("objective", ["reg:squarederror", "reg:pseudohubererror"])
@pytest.mark.parametrize("sampling", [False, True])
def test_approx_training_bit_exact(sb, ctx, orc, objective, sampling):
    """Whole approx trainings on the default fixed-point form: every round's
    weighted cuts, trees and margins equal the oracle's (these objectives'
    gradients round identically on both sides)."""
    rng = np.random.default_rng(11)
    n, f = 20_000, 16
    x = rng.standard_normal((n, f)).astype(np.float32)
    x[rng.random(x.shape) < 0.05] = np.nan
    y = (np.sin(np.nan_to_num(x[:, 0])) * 2 + np.nan_to_num(x[:, 1]) * np.nan_to_num(x[:, 2])
         + rng.normal(0, 0.2, n)).astype(np.float32)
    kw = dict(subsample=0.8, colsample_bytree=0.8, seed=3) if sampling else {}
    p = sb.TrainingParams(objective=objective, tree_method="approx", max_depth=5, eta=0.3, max_bin=64, **kw)
    m = sb.train(p, sb.DMatrix(x, labels=y), 6, ctx=ctx)
    ref = orc.train(x, y, p, 6)
    assert_trees_equal(m.export(), ref["model"].export())
    assert np.array_equal(m.predict_margin(sb.DMatrix(x)), ref["margins"].reshape(-1))


def test_approx_multiclass_first_round_bit_exact(sb, ctx, orc):
    """softprob: round 0 starts from equal margins, so both sides weight the
    cuts of each class with the same hessians; the K trees match."""
    rng = np.random.default_rng(21)
    n, f = 15_000, 10
    x = rng.standard_normal((n, f)).astype(np.float32)
    y = np.argmax(x[:, :3] + rng.gumbel(size=(n, 3)), axis=1).astype(np.float32)
    p = sb.TrainingParams(objective="multi:softprob", num_class=3, tree_method="approx", max_depth=4,
                          max_bin=32, eta=0.3)
    m = sb.train(p, sb.DMatrix(x, labels=y), 1, ctx=ctx)
    ref = orc.train(x, y, p, 1)
    assert_trees_equal(m.export(), ref["model"].export())


def _step_dataset(n):  # train.rs:543-555
    x = (np.arange(n) / n).astype(np.float32).reshape(n, 1)
    y = (x[:, 0] >= 0.5).astype(np.float32)
    return x, y


def test_approx_reduces_training_error(sb, ctx):
    """train.rs:631-645."""
    x, y = _step_dataset(120)
    p = sb.TrainingParams(objective="reg:squarederror", tree_method="approx", max_depth=3, eta=0.3)
    m = sb.train(p, sb.DMatrix(x, labels=y), 50, ctx=ctx)
    assert m.num_trees() == 50
    rmse = math.sqrt(float(np.mean((m.predict(sb.DMatrix(x)).astype(np.float64) - y) ** 2)))
    assert rmse < 0.05, rmse


def test_approx_and_hist_reach_similar_accuracy(sb, ctx):
    """train.rs:647-668."""
    x, y = _step_dataset(120)

    def rmse(method):
        p = sb.TrainingParams(objective="reg:squarederror", tree_method=method, max_depth=3, eta=0.3)
        m = sb.train(p, sb.DMatrix(x, labels=y), 60, ctx=ctx)
        return math.sqrt(float(np.mean((m.predict(sb.DMatrix(x)).astype(np.float64) - y) ** 2)))

    ra, rh = rmse("approx"), rmse("hist")
    assert ra < 0.05 and rh < 0.05
    assert abs(ra - rh) < 0.02


def test_approx_is_deterministic_and_rejects_boosters(sb, ctx):
    x, _ = mixed_data(8000, 6, seed=4)
    y = (np.nan_to_num(x[:, 0]) > 0).astype(np.float32)
    p = sb.TrainingParams(objective="binary:logistic", tree_method="approx", max_depth=4, subsample=0.7, seed=9)
    d = sb.DMatrix(x, labels=y)
    a = sb.train(p, d, 5, ctx=ctx).predict(d)
    b = sb.train(p, d, 5, ctx=ctx).predict(d)
    assert np.array_equal(a, b)
    with pytest.raises(sb.SbError):
        sb.Booster(sb.GHistIndex(d, ctx=ctx), p, y)
    with pytest.raises(sb.SbError):
        sb.TrainingParams(tree_method="exact").to_c()
