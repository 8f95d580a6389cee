"""Eval sets and early stopping on the device (train_with_eval,
learner/train.rs:121-140, 243-379): the margin caches against
predict_margin, the metrics against metric/mod.rs restated in numpy, and the
reference's early-stopping test."""
import math

import numpy as np
import pytest

from gpu_helpers import mixed_data

pytestmark = pytest.mark.gpu


def _step_dataset(sb, n):
    """train.rs:543-555."""
    x = (np.arange(n, dtype=np.float32) / np.float32(n)).reshape(-1, 1)
    y = (x[:, 0] >= 0.5).astype(np.float32)
    return sb.DMatrix(x, labels=y)


def test_early_stopping_sets_best_iteration(sb, ctx):
    """train.rs:1327-1342: the training set as its own eval set."""
    d = _step_dataset(sb, 80)
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=3, eta=0.3)
    res = sb.train_with_eval(p, d, 200, [(d, "train")], early_stopping_rounds=5, ctx=ctx)
    assert res.model.num_trees() < 200
    assert res.model.best_iteration() is not None
    assert len(res.history) > 0 and res.history[0].scores[0][:2] == ("train", "rmse")
    # the best round's score is the smallest, and it is 5 rounds before the stop
    vals = [h.scores[-1][2] for h in res.history]
    best = res.model.best_iteration()
    assert len(vals) == best + 6 and min(vals) == vals[best]
    # predict and predict_margin use the best round's trees (model.rs:213-226)
    lim = (best + 1)
    assert np.array_equal(res.model.predict_margin(d), res.model.predict_margin_limited(d, lim))
    assert np.array_equal(res.model.predict(d), res.model.predict_margin_limited(d, lim))


def _restated(name, preds, y, w, k):
    """metric/mod.rs:37-262 in numpy (f64)."""
    w = np.ones(len(y)) if w is None else w.astype(np.float64)
    p = preds.astype(np.float64).reshape(len(y), k)
    y64 = y.astype(np.float64)
    if name == "rmse":
        return math.sqrt(np.sum(w * (p[:, 0] - y64) ** 2) / np.sum(w))
    if name == "mae":
        return np.sum(w * np.abs(p[:, 0] - y64)) / np.sum(w)
    if name == "logloss":
        q = np.clip(p[:, 0], 1e-15, 1 - 1e-15)
        return np.sum(w * -(y64 * np.log(q) + (1 - y64) * np.log(1 - q))) / np.sum(w)
    if name == "error":
        return np.sum(w * ((preds.reshape(-1) > 0.5) != (y > 0.5))) / np.sum(w)
    if name == "mlogloss":
        q = np.clip(p[np.arange(len(y)), y.astype(int)], 1e-15, 1.0)
        return np.sum(-w * np.log(q)) / np.sum(w)
    if name == "merror":
        pr = preds.reshape(len(y), k)
        best = np.zeros(len(y), int)
        for c in range(1, k):
            best = np.where(pr[:, c] > pr[np.arange(len(y)), best], c, best)
        return np.sum(w * (best != y.astype(int))) / np.sum(w)
    raise ValueError(name)


@pytest.mark.parametrize("kind", ["regression", "binary", "multiclass", "categorical"])
def test_eval_caches_and_metrics(sb, ctx, kind):
    ft = None
    if kind == "categorical":
        x, ft = mixed_data(6000, 10, seed=51, n_cat=3, card=12)
    else:
        x, _ = mixed_data(6000, 10, seed=52)
    rng = np.random.default_rng(53)
    xe = x[:2000].copy()
    xe[rng.random(xe.shape) < 0.05] = np.nan
    signal = np.nan_to_num(x[:, 0]) - np.nan_to_num(x[:, 1])
    if kind == "multiclass":
        y = rng.integers(0, 3, len(x)).astype(np.float32)
        kw = dict(objective="multi:softprob", num_class=3, eval_metric=["mlogloss", "merror"])
        k = 3
    elif kind == "binary":
        y = (signal + rng.standard_normal(len(x)) > 0).astype(np.float32)
        kw = dict(objective="binary:logistic", eval_metric=["logloss", "error"])
        k = 1
    else:
        y = (signal + 0.1 * rng.standard_normal(len(x))).astype(np.float32)
        kw = dict(objective="reg:squarederror", eval_metric=["rmse", "mae"])
        k = 1
    p = sb.TrainingParams(max_depth=5, eta=0.3, subsample=0.8, **kw)
    ye = y[:2000]
    we = rng.uniform(0.5, 2.0, 2000).astype(np.float32)
    dtrain = sb.DMatrix(x, labels=y, feature_types=ft)
    gh = sb.GHistIndex(dtrain, ctx=ctx)
    b = sb.Booster(gh, p, y, ctx=ctx)
    de = sb.DMatrix(xe, labels=ye, weights=we, feature_types=ft)
    e0 = b.add_eval(de)
    bm = rng.standard_normal((2000, k)).astype(np.float32) * 0.1
    e1 = b.add_eval(sb.DMatrix(xe, labels=ye, base_margin=bm, feature_types=ft))
    done = 0
    for target in (1, 4, 9):
        b.update(target - done)
        done = target
        vals = b.eval(p.eval_metric)
        m = b.model()
        got0 = b.eval_margins(e0)
        want0 = m.predict_margin_limited(sb.DMatrix(xe), 0).reshape(2000, k)
        assert np.array_equal(got0, want0), target  # the cache is predict_margin's sum
        got1 = b.eval_margins(e1)
        want1 = m.predict_margin_limited(sb.DMatrix(xe, base_margin=bm), 0).reshape(2000, k)
        assert np.array_equal(got1, want1), target
        preds0 = m.predict(sb.DMatrix(xe))
        preds1 = m.predict(sb.DMatrix(xe, base_margin=bm))
        for j, name in enumerate(p.eval_metric):
            r0 = _restated(name, preds0, ye, we, k)
            r1 = _restated(name, preds1, ye, None, k)
            assert abs(vals[e0, j] - r0) <= 1e-9 * max(1.0, abs(r0)), (name, vals[e0, j], r0)
            assert abs(vals[e1, j] - r1) <= 1e-9 * max(1.0, abs(r1)), (name, vals[e1, j], r1)


def test_eval_history_and_metric_errors(sb, ctx):
    x, _ = mixed_data(3000, 6, seed=54)
    y = np.nan_to_num(x[:, 0]).astype(np.float32)
    d = sb.DMatrix(x, labels=y)
    dv = sb.DMatrix(x[:500], labels=y[:500])
    # default precision (fixed point): the histograms, and so the trees, do not
    # depend on the order of atomic additions, so two trainings are equal
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=4)
    res = sb.train_with_eval(p, d, 12, [(d, "train"), (dv, "valid")], ctx=ctx)
    assert len(res.history) == 12 and res.model.num_trees() == 12
    assert [s[:2] for s in res.history[0].scores] == [("train", "rmse"), ("valid", "rmse")]
    tr = [h.scores[0][2] for h in res.history]
    assert tr[-1] < tr[0]  # training error goes down
    assert res.model.best_iteration() is None
    assert np.array_equal(res.model.predict_margin(d), sb.train(p, d, 12, ctx=ctx).predict_margin(d))
    with pytest.raises(sb.SbError):
        sb.train_with_eval(sb.TrainingParams(eval_metric=["mlogloss"]), d, 2, [(dv, "v")], ctx=ctx)
    with pytest.raises(sb.SbError):
        sb.train_with_eval(sb.TrainingParams(eval_metric=["auc"]), d, 2, [(dv, "v")], ctx=ctx)
