"""The oracle's restatement of tree_method=approx (HistCuts::
from_dmatrix_weighted, data/quantile.rs:81-122 and :253-316, and the
Prepared::Approx round, learner/train.rs:46-53) against the reference's
stated properties and its approx tests (train.rs:631-668)."""
import math

import numpy as np
import pytest


def _params(sb, **kw):
    return sb.TrainingParams(objective="reg:squarederror", **kw)


def test_equal_weights_give_the_unweighted_cuts(orc):
    """quantile.rs:248-252: with all weights equal the weighted cuts are the
    unweighted ones."""
    rng = np.random.default_rng(0)
    x = rng.standard_normal((6000, 4)).astype(np.float32)
    x[:, 3] = np.round(x[:, 3] * 3)
    for w in (1.0, 0.25):
        for mb in (8, 64, 256):
            a = orc.data(x, max_bin=mb).cuts()
            b = orc.data_weighted(x, np.full(len(x), w, np.float32), max_bin=mb).cuts()
            for u, v in zip(a, b):
                assert np.array_equal(u, v), (w, mb)


def test_zero_weights_fall_back_to_unweighted_positions(orc):
    rng = np.random.default_rng(1)
    x = rng.standard_normal((3000, 3)).astype(np.float32)
    a = orc.data(x, max_bin=32).cuts()
    b = orc.data_weighted(x, np.zeros(len(x), np.float32), max_bin=32).cuts()
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_weighted_cuts_follow_the_weights(orc):
    """Cut invariants (quantile.rs:329-389) hold, and heavier weights on the
    high values pull the cuts toward them."""
    rng = np.random.default_rng(2)
    x = rng.standard_normal((20000, 1)).astype(np.float32)
    w = np.where(x[:, 0] > 1.0, 50.0, 1.0).astype(np.float32)
    off, vals, _ = orc.data_weighted(x, w, max_bin=32).cuts()
    assert off[-1] - off[0] <= 33
    assert np.all(np.diff(vals) > 0)
    assert vals[-1] > x.max()  # the sentinel
    _, uvals, _ = orc.data(x, max_bin=32).cuts()
    assert np.sum(vals > 1.0) > np.sum(uvals > 1.0)


def _step(n):  # train.rs:543-555
    x = (np.arange(n) / n).astype(np.float32).reshape(n, 1)
    return x, (x[:, 0] >= 0.5).astype(np.float32)


def test_oracle_approx_reduces_training_error(orc, sb):
    """train.rs:631-645."""
    x, y = _step(120)
    p = _params(sb, tree_method="approx", max_depth=3, eta=0.3)
    r = orc.train(x, y, p, 50)
    assert len(r["model"].export()[0]) - 1 == 50
    rmse = math.sqrt(float(np.mean((r["margins"].reshape(-1).astype(np.float64) - y) ** 2)))
    assert rmse < 0.05


@pytest.mark.parametrize("objective", ["reg:squarederror", "binary:logistic"])
def test_oracle_approx_and_hist_reach_similar_accuracy(orc, sb, objective):
    """train.rs:647-668 (and the same closeness for a logistic objective)."""
    x, y = _step(120)
    out = {}
    for method in ("approx", "hist"):
        p = sb.TrainingParams(objective=objective, tree_method=method, max_depth=3, eta=0.3)
        m = orc.train(x, y, p, 60)["margins"].reshape(-1).astype(np.float64)
        pred = 1 / (1 + np.exp(-m)) if objective == "binary:logistic" else m
        out[method] = math.sqrt(float(np.mean((pred - y) ** 2)))
    assert out["approx"] < 0.05 and out["hist"] < 0.05
    assert abs(out["approx"] - out["hist"]) < 0.02


def test_oracle_dart_dropout_matches_the_host_loop(orc, sb):
    """The oracle's DART draws the dropout sets of api.dart_dropout (the same
    sb_dart_key stream), so without any dropped tree it is gbtree, and with
    dropout its tree weights follow 1/(k+1), k/(k+1)."""
    x, y = _step(200)
    kw = dict(objective="reg:squarederror", max_depth=3, eta=0.3, hist_precision="fixed")
    g = orc.train(x, y, sb.TrainingParams(**kw), 8)
    dd = orc.train_dart(x, y, sb.TrainingParams(booster="dart", rate_drop=0.5, skip_drop=1.0, **kw), 8)
    for a, b in zip(g["model"].export()[:2], dd["model"].export()[:2]):
        assert np.array_equal(a, b)
    assert np.all(dd["model"].export()[4] == 1.0)
    p = sb.TrainingParams(booster="dart", rate_drop=0.3, skip_drop=0.1, seed=5, **kw)
    r = orc.train_dart(x, y, p, 12)
    w = np.ones(0, np.float32)
    from sequoia_boost_b200.api import dart_dropout
    for rnd in range(12):  # restate the weight bookkeeping from the host loop's dropout sets
        drop = dart_dropout(p.seed, rnd, len(w), p.rate_drop, p.skip_drop)
        kd = np.float32(len(drop))
        w = np.concatenate([w, [np.float32(1.0) / (kd + np.float32(1.0))]]).astype(np.float32)
        if drop:
            w[drop] = w[drop] * (kd / (kd + np.float32(1.0)))
    assert np.array_equal(r["model"].export()[4], w)
