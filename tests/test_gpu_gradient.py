"""Objective::gradient on the device (sb_objective_gradient, the same device
code as the boosting rounds' gradients) against the reference's gradient
known answers and the oracle's restatement.

Squared error and pseudo-Huber use only correctly rounded IEEE operations
(sub, mul, add, div, sqrt), so the device pairs equal the oracle's bit for
bit. Logistic and softmax call `expf`, which may differ from glibc's by an
ulp: a probability then moves by about 1.2e-7, and g = p - y and
h = p (1 - p) move by that times the row's weight. The tolerance per pair is
4e-7 relative plus 3e-7 times the largest row weight (scale_pos_weight
included)."""
import json
import os
import zlib

import numpy as np
import pytest

from engines import GpuEngine
from kat_checks import check_case

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [c for c in json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))["cases"]
         if c["kind"] == "gradient"]
EXP_REL, EXP_ABS = 4e-7, 3e-7


def _close(got, want, wmax=1.0):
    err = np.abs(got.astype(np.float64) - want)
    return np.all(err <= EXP_REL * np.abs(want) + EXP_ABS * wmax), float(np.max(err))


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_gradient_reference_kats(case, sb, ctx):
    """regression.rs:91-119, classification.rs:97-138, multiclass.rs:110-141."""
    check_case(case, GpuEngine(sb, ctx), sb.TrainingParams)


def _inputs(objective, n, k, seed):
    rng = np.random.default_rng(seed)
    preds = (rng.standard_normal(n * k) * 3).astype(np.float32)
    if objective.startswith("multi:"):
        labels = rng.integers(0, k, n).astype(np.float32)
    elif objective == "binary:logistic":
        labels = (rng.random(n) < 0.3).astype(np.float32)
    else:
        labels = (rng.standard_normal(n) * 2).astype(np.float32)
    weights = rng.uniform(0.1, 3.0, n).astype(np.float32)
    return preds, labels, weights


OBJ = [("reg:squarederror", 0, True), ("reg:pseudohubererror", 0, True), ("binary:logistic", 0, False),
       ("multi:softprob", 7, False)]


@pytest.mark.parametrize("objective,num_class,exact", OBJ, ids=[o[0] for o in OBJ])
@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("spw", [1.0, 3.5])
def test_device_gradient_matches_oracle(sb, ctx, orc, objective, num_class, exact, weighted, spw):
    if spw != 1.0 and objective != "binary:logistic":
        pytest.skip("scale_pos_weight only applies to the logistic objective")
    k = max(num_class, 1)
    n = 50_000
    preds, labels, weights = _inputs(objective, n, k, seed=zlib.crc32(f"{objective}{weighted}".encode()) % 997)
    w = weights if weighted else None
    got = sb.objective_gradient(objective, preds, labels, w, num_class=num_class, scale_pos_weight=spw,
                                ctx=ctx)
    want = orc.gradient(objective, preds, labels, w, num_class, spw)
    assert got.shape == want.shape == (n * k, 2)
    if exact:
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    else:
        ok, worst = _close(got, want, (float(weights.max()) if weighted else 1.0) * spw)
        assert ok, worst


def test_softmax_labels_cast_like_rust(sb, ctx, orc):
    """`labels[i] as usize` saturates: negative and NaN labels select class 0,
    fractions truncate, labels >= K select no class."""
    labels = np.array([-1.0, np.nan, 2.7, 5.0, 0.0, 1.0], np.float32)
    preds = np.linspace(-1, 1, labels.size * 3).astype(np.float32)
    got = sb.objective_gradient("multi:softmax", preds, labels, num_class=3, ctx=ctx)
    want = orc.gradient("multi:softmax", preds, labels, None, 3)
    assert _close(got, want)[0]
    g = got[:, 0].reshape(-1, 3)
    assert g[0, 0] < 0 and g[1, 0] < 0 and g[2, 2] < 0  # class 0, class 0, class 2 are the targets
    assert np.all(g[3] > 0)  # label 5 >= K: no class is the target


def test_gradient_rejects_bad_arguments(sb, ctx):
    with pytest.raises(sb.SbError):
        sb.objective_gradient("multi:softprob", np.zeros(4, np.float32), np.zeros(4, np.float32), num_class=1,
                              ctx=ctx)
    with pytest.raises(sb.SbError):
        sb.objective_gradient("binary:logistic", np.zeros(4, np.float32), np.zeros(4, np.float32),
                              scale_pos_weight=0.0, ctx=ctx)


ROUND_OBJ = [("reg:squarederror", 0, True, 1.0), ("reg:pseudohubererror", 0, True, 1.0),
             ("binary:logistic", 0, False, 2.5), ("multi:softprob", 4, False, 1.0)]


@pytest.mark.parametrize("objective,num_class,exact,spw", ROUND_OBJ, ids=[o[0] for o in ROUND_OBJ])
def test_round_gradients_with_weights_match_oracle(sb, ctx, orc, objective, num_class, exact, spw):
    """The gradients a boosting round computes from the booster's margins, with
    sample weights (and scale_pos_weight for the logistic objective), equal the
    oracle's Objective::gradient on the same margins (train.rs:297-302)."""
    n, f = 30_000, 8
    rng = np.random.default_rng(13)
    x = rng.standard_normal((n, f)).astype(np.float32)
    k = max(num_class, 1)
    if objective.startswith("multi:"):
        y = rng.integers(0, k, n).astype(np.float32)
    elif objective == "binary:logistic":
        y = (x[:, 0] + rng.standard_normal(n) > 0.5).astype(np.float32)
    else:
        y = (np.sin(x[:, 0]) + 0.3 * x[:, 1] + rng.normal(0, 0.1, n)).astype(np.float32)
    w = rng.uniform(0.2, 2.0, n).astype(np.float32)
    p = sb.TrainingParams(objective=objective, num_class=num_class, max_depth=4, eta=0.3,
                          scale_pos_weight=spw, seed=3)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    b = sb.Booster(gh, p, y, weights=w)
    for _ in range(2):
        b.update(1)
        m_prev = b.margins().reshape(n, k).copy()
        b.update(1)
        got = b.gradients().reshape(k, n, 2).transpose(1, 0, 2).reshape(-1, 2)
        want = orc.gradient(objective, m_prev.reshape(-1), y, w, num_class, spw)
        if exact:
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        else:
            ok, worst = _close(got, want, float(w.max()) * spw)
            assert ok, worst


@pytest.mark.parametrize("objective", ["reg:pseudohubererror", "reg:squarederror"])
def test_weighted_training_bit_exact(sb, ctx, orc, objective):
    """Training with sample weights (and pseudo-Huber) on the default
    fixed-point form: trees and margins equal the oracle's bit for bit."""
    n, f = 20_000, 12
    rng = np.random.default_rng(29)
    x = rng.standard_normal((n, f)).astype(np.float32)
    x[rng.random(x.shape) < 0.05] = np.nan
    y = (np.sin(np.nan_to_num(x[:, 0])) * 3 + np.nan_to_num(x[:, 1]) + rng.normal(0, 0.3, n)).astype(np.float32)
    w = rng.uniform(0.1, 4.0, n).astype(np.float32)
    p = sb.TrainingParams(objective=objective, max_depth=5, eta=0.2, subsample=0.9, seed=8)
    m = sb.train(p, sb.DMatrix(x, labels=y, weights=w), 6, ctx=ctx)
    ref = orc.train(x, y, p, 6, weights=w)
    from gpu_helpers import assert_trees_equal
    assert_trees_equal(m.export(), ref["model"].export())
    assert np.array_equal(m.predict_margin(sb.DMatrix(x)), ref["margins"].reshape(-1))
