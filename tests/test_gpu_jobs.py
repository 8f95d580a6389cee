"""sb_train_many: independent jobs of uneven sizes trained together give, job
by job, the same model as training each job alone (fixed point: bit-exact)."""
import numpy as np
import pytest

from gpu_helpers import assert_trees_equal

pytestmark = pytest.mark.gpu


def test_jobs_together_equal_jobs_alone(sb, ctx):
    from sequoia_boost_b200 import datagen
    specs = datagen.small_jobs(n_jobs=12, seed=5)
    jobs = []
    for i, s in enumerate(specs):
        n = min(len(s["x"]), 20000)
        objective = "reg:squarederror" if i % 3 else "binary:logistic"
        y = s["y"][:n] if objective.startswith("reg") else (s["y"][:n] > 0).astype(np.float32)
        p = sb.TrainingParams(objective=objective, max_depth=s["max_depth"], eta=s["eta"], max_bin=64,
                              subsample=0.9 if i % 2 else 1.0, hist_precision="fixed", seed=i)
        jobs.append((p, sb.DMatrix(s["x"][:n], labels=y), 3 + (i % 5)))
    together = sb.train_many(jobs, n_streams=4, ctx=ctx)
    for (p, d, rounds), m in zip(jobs, together):
        alone = sb.train(p, d, rounds, ctx=ctx)
        assert m.num_trees() == rounds
        assert_trees_equal(m.export(), alone.export())
        assert np.array_equal(m.predict_margin(d), alone.predict_margin(d))


def test_a_failing_job_reports_its_status(sb, ctx):
    x = np.random.default_rng(0).standard_normal((500, 4)).astype(np.float32)
    y = np.zeros(500, np.float32)
    good = sb.TrainingParams(max_depth=3)
    bad = sb.TrainingParams(objective="multi:softprob", num_class=0)  # invalid
    with pytest.raises(sb.SbError):
        sb.train_many([(good, sb.DMatrix(x, labels=y), 2), (bad, sb.DMatrix(x, labels=y), 2)], ctx=ctx)


def test_mixed_jobs_batched_and_pooled_equal_alone(sb, ctx):
    """Depthwise fixed-point jobs train as one batch (one launch per kernel
    step for all of them), a multiclass job among them with 3 class trees per
    round beside single-tree jobs; a lossguide job and an FP32 job go through
    the stream pool in the same call. Every fixed-point model equals the one
    trained alone bit for bit; the FP32 job's margins agree within 1e-5."""
    rng = np.random.default_rng(11)

    def data(n, f):
        x = rng.standard_normal((n, f)).astype(np.float32)
        x[rng.random(x.shape) < 0.05] = np.nan
        return x, (np.nan_to_num(x[:, 0]) * 2 + np.nan_to_num(x[:, 1]) + rng.normal(0, 0.3, n)).astype(np.float32)

    jobs = []
    for i in range(6):
        x, y = data(3000 + 2500 * i, 10 + 3 * i)
        p = sb.TrainingParams(max_depth=(3, 5, 7)[i % 3], eta=0.3, max_bin=64, colsample_bytree=0.8, seed=i)
        jobs.append((p, sb.DMatrix(x, labels=y), 4 + i % 3))
    x, y = data(6000, 12)
    yk = np.digitize(y, [-1.0, 1.0]).astype(np.float32)
    jobs.append((sb.TrainingParams(objective="multi:softprob", num_class=3, max_depth=4, eta=0.3, seed=7),
                 sb.DMatrix(x, labels=yk), 5))
    x, y = data(5000, 9)
    jobs.append((sb.TrainingParams(grow_policy="lossguide", max_leaves=20, max_depth=0, seed=8),
                 sb.DMatrix(x, labels=y), 4))
    x, y = data(4000, 8)
    jobs.append((sb.TrainingParams(hist_precision="fp32", max_depth=5, seed=9), sb.DMatrix(x, labels=y), 4))
    together = sb.train_many(jobs, n_streams=3, ctx=ctx)
    for (p, d, rounds), m in zip(jobs, together):
        alone = sb.train(p, d, rounds, ctx=ctx)
        k = max(p.num_class, 1)
        assert m.num_trees() == rounds * k
        if p.hist_precision == "fixed":
            assert_trees_equal(m.export(), alone.export())
            assert np.array_equal(m.predict_margin(d), alone.predict_margin(d))
        else:
            assert np.allclose(m.predict_margin(d), alone.predict_margin(d), rtol=1e-5, atol=1e-5)
