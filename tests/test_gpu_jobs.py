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
