"""Seeded synthetic datasets with the shapes and distributions of the
benchmark workloads (no public dataset is involved; every call with the same
arguments returns the same bytes).

  regression_sine   100k x 30, x ~ N(0,1), y = sum w_j sin(x_j) + 0.5 x0 x1 + N(0, 0.1^2)
  binary_mixed      10M x 100: 70 N(0,1), 20 lognormal(0,1), 10 Bernoulli(0.05),
                    10% MCAR NaN, y ~ Bernoulli(sigmoid(v.x + 10 random pair products))
  multiclass_uniform 2M x 200 U(0,1), 10 classes = argmax of 10 random projections
                    + Gumbel(0,1), features 195..199 categorical (32 integer codes)
  small_jobs        256 regression jobs, rows log-uniform in [1k, 200k], 20..50 features
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np


def regression_sine(n=100_000, f=30, seed=0):
    rng = np.random.default_rng(seed)
    w = rng.uniform(-1.0, 1.0, f)
    x = rng.standard_normal((n, f), dtype=np.float32)
    y = np.sin(x.astype(np.float64)) @ w + 0.5 * x[:, 0].astype(np.float64) * x[:, 1]
    y += rng.normal(0.0, 0.1, n)
    return x, y.astype(np.float32)


def _binary_chunk(args):
    seed_seq, n, v, pairs = args
    rng = np.random.default_rng(seed_seq)
    x = np.empty((n, 100), np.float32)
    x[:, :70] = rng.standard_normal((n, 70), dtype=np.float32)
    x[:, 70:90] = np.exp(rng.standard_normal((n, 20), dtype=np.float32))
    x[:, 90:] = (rng.random((n, 10), dtype=np.float32) < 0.05).astype(np.float32)
    logit = x.astype(np.float64) @ v
    for a, b in pairs:
        logit += x[:, a].astype(np.float64) * x[:, b]
    y = (rng.random(n) < 1.0 / (1.0 + np.exp(-logit))).astype(np.float32)
    x[rng.random((n, 100), dtype=np.float32) < 0.10] = np.nan  # MCAR, after the label
    return x, y


def binary_mixed(n=10_000_000, seed=1, chunk=500_000, threads=8):
    """The label uses the complete values (missing treated as observed before
    masking); 10% of entries are then replaced by NaN."""
    root = np.random.SeedSequence(seed)
    rng = np.random.default_rng(root.spawn(1)[0])
    v = rng.normal(0.0, 0.3, 100)
    pairs = [tuple(rng.choice(100, 2, replace=False)) for _ in range(10)]
    sizes = [min(chunk, n - i) for i in range(0, n, chunk)]
    seqs = root.spawn(len(sizes) + 1)[1:]
    x = np.empty((n, 100), np.float32)
    y = np.empty(n, np.float32)
    jobs = [(s, m, v, pairs) for s, m in zip(seqs, sizes)]
    offs = np.cumsum([0] + sizes)
    with ThreadPoolExecutor(threads) as ex:
        for i, (xc, yc) in enumerate(ex.map(_binary_chunk, jobs)):
            x[offs[i]:offs[i + 1]] = xc
            y[offs[i]:offs[i + 1]] = yc
    return x, y


def multiclass_uniform(n=2_000_000, f=200, k=10, seed=2, n_cat=5, card=32):
    rng = np.random.default_rng(seed)
    x = rng.random((n, f), dtype=np.float32)
    cat_cols = list(range(f - n_cat, f))
    for c in cat_cols:
        x[:, c] = rng.integers(0, card, n).astype(np.float32)
    w = rng.standard_normal((f, k))
    scores = x.astype(np.float64) @ w + rng.gumbel(0.0, 1.0, (n, k))
    y = scores.argmax(axis=1).astype(np.float32)
    ftypes = np.zeros(f, np.uint8)
    ftypes[cat_cols] = 1
    return x, y, ftypes


def small_jobs(n_jobs=256, seed=3):
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_jobs):
        n = int(np.exp(rng.uniform(np.log(1_000), np.log(200_000))))
        f = int(rng.integers(20, 51))
        x, y = regression_sine(n, f, seed=seed * 100_000 + j)
        jobs.append({"x": x, "y": y, "max_depth": int(rng.choice([4, 6, 8])),
                     "eta": float(rng.choice([0.05, 0.1, 0.3]))})
    return jobs
