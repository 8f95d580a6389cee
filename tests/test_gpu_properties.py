"""The reference's property tests (crates/sequoia-boost/tests/properties.rs)
restated over seeded random cases on the GPU path, with default histogram
precision:

  training_is_deterministic   (:40-46)  same data, params and seed -> equal
                                        predictions, bit for bit
  monotone_increasing_holds   (:81-104) predictions never decrease along an
                                        increasing-constrained feature

The reference draws 48 proptest cases of 40 rows x 3 features; here the same
shapes run over seeded cases, plus larger matrices on which many CTAs add
into the same histogram bins, where the order of atomic additions would show
up if the histograms depended on it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROWS, COLS = 40, 3


def _dataset(seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-10.0, 10.0, ROWS * COLS).astype(np.float32).reshape(ROWS, COLS)
    y = rng.uniform(-5.0, 5.0, ROWS).astype(np.float32)
    return x, y


def _base_params(sb, seed):  # properties.rs:23-33
    return sb.TrainingParams(objective="reg:squarederror", max_depth=3, eta=0.3, subsample=0.8,
                             colsample_bytree=0.8, seed=seed)


@pytest.mark.parametrize("case", range(12))
def test_training_is_deterministic(sb, ctx, case):
    x, y = _dataset(1000 + case)
    seed = int(np.random.default_rng(case).integers(0, 10_000))
    d = sb.DMatrix(x, labels=y)
    p = _base_params(sb, seed)
    a = sb.train(p, d, 15, ctx=ctx).predict(d)
    b = sb.train(p, d, 15, ctx=ctx).predict(d)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("objective,num_class", [("reg:squarederror", 0), ("binary:logistic", 0),
                                                 ("multi:softprob", 4)])
def test_training_is_deterministic_at_scale(sb, ctx, objective, num_class):
    """400k rows x 24 features: every histogram bin collects additions from
    many CTAs and warps. Two trainings with default parameters give the same
    trees and predictions bit for bit."""
    rng = np.random.default_rng(5)
    n, f = 400_000, 24
    x = rng.standard_normal((n, f)).astype(np.float32)
    x[rng.random(x.shape) < 0.05] = np.nan
    s = np.nan_to_num(x[:, 0]) + 0.5 * np.nan_to_num(x[:, 1]) * np.nan_to_num(x[:, 2])
    if objective == "binary:logistic":
        y = (s + rng.standard_normal(n) > 0).astype(np.float32)
    elif num_class:
        y = np.clip(np.floor(s + 2), 0, num_class - 1).astype(np.float32)
    else:
        y = (s + rng.normal(0, 0.1, n)).astype(np.float32)
    p = sb.TrainingParams(objective=objective, num_class=num_class, max_depth=7, eta=0.1, subsample=0.8,
                          colsample_bytree=0.8, seed=11)
    assert p.hist_precision == "fixed"  # the default form
    d = sb.DMatrix(x, labels=y)
    m1 = sb.train(p, d, 12, ctx=ctx)
    m2 = sb.train(p, d, 12, ctx=ctx)
    e1, e2 = m1.export(), m2.export()
    for a, b in zip(e1[:4], e2[:4]):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    assert np.array_equal(m1.predict(d), m2.predict(d))


def _assert_monotone(x_col, preds, direction):
    idx = np.argsort(x_col, kind="stable")
    prev = -np.inf if direction > 0 else np.inf
    for i in idx:  # properties.rs:96-102
        if direction > 0:
            assert preds[i] >= prev - 1e-4, (preds[i], prev)
            prev = max(prev, preds[i])
        else:
            assert preds[i] <= prev + 1e-4, (preds[i], prev)
            prev = min(prev, preds[i])


@pytest.mark.parametrize("case", range(12))
def test_monotone_increasing_holds(sb, ctx, case):
    rng = np.random.default_rng(2000 + case)
    x = rng.uniform(-10.0, 10.0, ROWS).astype(np.float32).reshape(ROWS, 1)
    y = rng.uniform(-5.0, 5.0, ROWS).astype(np.float32)
    d = sb.DMatrix(x, labels=y)
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=4, eta=0.3,
                          monotone_constraints=[sb.Monotone.INCREASING])
    preds = sb.train(p, d, 20, ctx=ctx).predict(d)
    _assert_monotone(x[:, 0], preds, +1)


@pytest.mark.parametrize("grow_policy", ["depthwise", "lossguide"])
def test_monotone_constraints_hold_on_a_grid(sb, ctx, grow_policy):
    """Larger case: 6 features, +1 on feature 0 and -1 on feature 1. Sweeping
    one constrained feature over a grid with the others held fixed, the
    prediction moves only in the constrained direction."""
    rng = np.random.default_rng(17)
    n, f = 50_000, 6
    x = rng.standard_normal((n, f)).astype(np.float32)
    y = (np.sin(3 * x[:, 0]) + x[:, 0] - np.cos(2 * x[:, 1]) - x[:, 1] + x[:, 2] * x[:, 3]
         + rng.normal(0, 0.3, n)).astype(np.float32)
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=6, eta=0.3, grow_policy=grow_policy,
                          max_leaves=48 if grow_policy == "lossguide" else 0,
                          monotone_constraints=[1, -1, 0, 0, 0, 0], seed=2)
    m = sb.train(p, sb.DMatrix(x, labels=y), 30, ctx=ctx)
    grid = np.linspace(-3, 3, 121).astype(np.float32)
    base = x[:64]
    for feat, direction in ((0, +1), (1, -1)):
        q = np.repeat(base, grid.size, axis=0)
        q[:, feat] = np.tile(grid, base.shape[0])
        pr = m.predict(sb.DMatrix(q)).reshape(base.shape[0], grid.size)
        steps = np.diff(pr.astype(np.float64), axis=1) * direction
        assert np.all(steps >= -1e-6), (feat, float(steps.min()))
