"""Sampling contract (include/sb_sampling.h) against the reference's sampler
tests (tree/sampler.rs:73-108, learner/train.rs:465-489). The Rust stream
(rand 0.8 StdRng) is unpinned; sizes, order, determinism and the
at-least-one rule are pinned."""
import numpy as np


def test_pass_through_when_ratios_one(orc, sb):  # sampler.rs:79-84
    p = sb.TrainingParams()
    assert list(orc.sample_features(10, p)) == list(range(10))


def test_composes_bylevel_and_bynode(orc, sb):  # sampler.rs:86-94
    p = sb.TrainingParams(colsample_bylevel=0.5, colsample_bynode=0.5, seed=42)
    f = orc.sample_features(100, p, nid=3)
    assert len(f) == 25  # round(0.5*100)=50, round(0.5*50)=25
    assert np.all(np.diff(f.astype(np.int64)) > 0)
    assert f.max() < 100


def test_deterministic_for_seed(orc, sb):  # sampler.rs:96-101
    p = sb.TrainingParams(colsample_bylevel=0.6, seed=7)
    assert list(orc.sample_features(50, p, nid=1)) == list(orc.sample_features(50, p, nid=1))
    q = sb.TrainingParams(colsample_bylevel=0.6, seed=8)
    assert list(orc.sample_features(50, p, nid=1)) != list(orc.sample_features(50, q, nid=1))


def test_always_at_least_one(orc, sb):  # sampler.rs:103-107
    p = sb.TrainingParams(colsample_bylevel=0.01, colsample_bynode=0.01, seed=1)
    assert len(orc.sample_features(3, p, nid=0)) >= 1


def test_bytree_pool_size(orc, sb):  # train.rs:479-489
    p = sb.TrainingParams(colsample_bytree=0.8, seed=3)
    for r in range(5):
        f = orc.sample_features(100, p, round_=r)
        assert len(f) == 80 and np.all(np.diff(f.astype(np.int64)) > 0)


def test_row_subsample_bernoulli(orc, sb):  # train.rs:465-476
    p = sb.TrainingParams(subsample=0.8, seed=5)
    rows = orc.sample_rows(100_000, p, round_=2)
    assert abs(len(rows) / 100_000 - 0.8) < 0.01
    assert np.all(np.diff(rows.astype(np.int64)) > 0)
    assert len(orc.sample_rows(100, sb.TrainingParams(subsample=1.0))) == 100
    tiny = orc.sample_rows(3, sb.TrainingParams(subsample=1e-9, seed=1))
    assert len(tiny) == 1  # at least one row
