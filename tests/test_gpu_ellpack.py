"""The device ELLPACK's code width. The reference stores its bins as u16 or
u32 by the total bin count (GHistIndex::from_dmatrix, data/ghist.rs:48-82,
the tagged storage behind `bins()` at :117); the device index stores one byte
per entry when every feature has at most 255 bins (max_bin 64 in the
many-jobs workload: 65 local bins), and two bytes otherwise: a numeric
feature has up to max_bin + 1 bins once the sentinel is pushed
(quantile.rs:232-243, :319-323), so max_bin 255 or 256 can need 256 or 257.
Codes, histograms and models are checked bit-exact against the oracle, and
against the same index with two-byte codes forced (SB_HIST_CODES=2)."""
import contextlib
import os

import numpy as np
import pytest

from gpu_helpers import assert_trees_equal, hist_layout, hist_rows, mixed_data, random_gpair

pytestmark = pytest.mark.gpu
MISSING_GLOBAL = np.iinfo(np.uint32).max


@contextlib.contextmanager
def code_width(nbytes):
    """Indexes built inside the block keep `nbytes`-byte codes where the
    shape allows one byte (2: always two bytes; None: by the bin counts)."""
    old = os.environ.get("SB_HIST_CODES")
    if nbytes is None:
        os.environ.pop("SB_HIST_CODES", None)
    else:
        os.environ["SB_HIST_CODES"] = str(nbytes)
    try:
        yield
    finally:
        if old is None:
            os.environ.pop("SB_HIST_CODES", None)
        else:
            os.environ["SB_HIST_CODES"] = old


def _u8_global_bins(gh):
    """Global bins decoded from the stored one-byte codes: feature f at
    position f holds its local bin, or its bin count when missing."""
    off, _, _ = gh.cuts()
    n, f, _ = gh.info()
    codes = gh.codes()
    lay = gh.layout()
    assert codes.dtype == np.uint8 and codes.shape == (n, lay["row_stride"])
    assert np.all(codes[:, f:] == 0xFF)  # row padding
    local = codes[:, :f].astype(np.int64)
    nb = np.diff(off.astype(np.int64))
    assert np.all(local <= nb[None, :])
    out = (off[:-1].astype(np.int64)[None, :] + local).astype(np.uint32)
    out[local == nb[None, :]] = MISSING_GLOBAL
    return out


@pytest.mark.parametrize("max_bin", [16, 64, 254])
def test_u8_codes_are_the_oracle_bins(sb, ctx, orc, max_bin):
    x, ft = mixed_data(40_000, 37, seed=max_bin, n_cat=3, card=20)
    gh = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), max_bin=max_bin, ctx=ctx)
    lay = gh.layout()
    assert lay["layout"] == "tiled" and lay["code_bytes"] == 1, lay
    want = orc.data(x, ft, max_bin=max_bin).global_bins()
    got = _u8_global_bins(gh)
    bad = np.argwhere(got != want)
    assert bad.size == 0, (bad[:5], got[tuple(bad[0])], want[tuple(bad[0])])
    assert np.array_equal(gh.global_bins(), want)  # the feature-major copy


def test_two_byte_escape_at_256_bins(sb, ctx, orc):
    """254 distinct values give 255 bins (the values and the sentinel): one
    byte. 255 distinct values give 256 bins: the index keeps two bytes, and
    its bins still equal the oracle's."""
    rng = np.random.default_rng(3)
    n = 6000
    base = rng.integers(0, 50, (n, 5)).astype(np.float32)  # 51 bins each
    for distinct, width in ((254, 1), (255, 2)):
        x = base.copy()
        x[:, 2] = rng.integers(0, distinct, n).astype(np.float32)
        x[:distinct, 2] = np.arange(distinct, dtype=np.float32)  # every value present
        gh = sb.GHistIndex(sb.DMatrix(x), max_bin=256, ctx=ctx)
        off, _, _ = gh.cuts()
        assert off[3] - off[2] == distinct + 1
        assert gh.layout()["code_bytes"] == width
        want = orc.data(x, max_bin=256).global_bins()
        assert np.array_equal(gh.global_bins(), want)
        if width == 1:
            assert np.array_equal(_u8_global_bins(gh), want)


def test_lanes_layout_keeps_two_bytes(sb, ctx):
    x, _ = mixed_data(5000, 20, seed=4)
    with hist_layout("lanes"):
        gh = sb.GHistIndex(sb.DMatrix(x), max_bin=64, ctx=ctx)
    lay = gh.layout()
    assert lay["layout"] == "lanes" and lay["code_bytes"] == 2
    assert gh.codes().dtype == np.uint16


@pytest.mark.parametrize("f,rows", [(30, None), (30, 8), (100, None), (200, None)])
def test_u8_fixed_point_histograms_exact(sb, ctx, orc, f, rows):
    """200 features of 65 bins need two feature tiles (at most 128 features
    each), so the second tile's entry table is read at a non-zero offset."""
    n = 60_000
    x, ft = mixed_data(n, f, seed=f, n_cat=2, card=16)
    g = random_gpair(n, seed=5)
    sel = np.arange(0, n, 3, dtype=np.uint32)
    with hist_rows(rows):
        gh = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), max_bin=64, ctx=ctx)
        with code_width(2):
            gh2 = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), max_bin=64, ctx=ctx)
    assert gh.layout()["code_bytes"] == 1 and gh2.layout()["code_bytes"] == 2
    got = sb.GpuBackend("fixed", quantize_bits=16, ctx=ctx).build(gh, sel, g)
    gq, _, _ = orc.quantize(g, 16)
    want = orc.data(x, ft, max_bin=64).hist(sel, gq, threads=1)
    assert np.array_equal(got, want)
    assert np.array_equal(sb.GpuBackend("fixed", quantize_bits=16, ctx=ctx).build(gh2, sel, g), got)
    # FP32 accumulation within 1e-5 of each bin's mass
    got32 = sb.GpuBackend("fp32", ctx=ctx).build(gh, sel, g)
    d = orc.data(x, ft, max_bin=64)
    want64 = d.hist(sel, g, threads=8)
    mag = d.hist(sel, np.abs(g), threads=8)
    assert np.all(np.abs(got32 - want64) <= 1e-5 * mag + 1e-12)


@pytest.mark.parametrize("grow_policy", ["depthwise", "lossguide"])
def test_u8_training_bit_exact_against_the_oracle(sb, ctx, orc, grow_policy):
    x, ft = mixed_data(20_000, 24, seed=9, n_cat=2, card=12)
    y = (np.nan_to_num(x[:, 0]) - 0.7 * np.nan_to_num(x[:, 3]) + 0.3 * (x[:, -1] == 2)).astype(np.float32)
    kw = dict(max_depth=6) if grow_policy == "depthwise" else dict(max_depth=0, max_leaves=24)
    p = sb.TrainingParams(objective="reg:squarederror", grow_policy=grow_policy, eta=0.3, max_bin=64,
                          subsample=0.8, colsample_bytree=0.8, hist_precision="fixed", seed=3, **kw)
    d = sb.DMatrix(x, labels=y, feature_types=ft)
    m = sb.train(p, d, 6, ctx=ctx)
    ref = orc.train(x, y, p, 6, ftypes=ft)
    assert_trees_equal(m.export(), ref["model"].export())
    assert np.array_equal(m.predict_margin(d), ref["margins"].reshape(-1))


@pytest.mark.parametrize("grow_policy", ["depthwise", "lossguide"])
def test_u8_and_u16_models_identical(sb, ctx, grow_policy):
    """Multiclass with categorical features (the lossguide round routes every
    row through its trees with the row-major codes): the same models with
    one- and two-byte codes."""
    x, ft = mixed_data(15_000, 18, seed=21, n_cat=2, card=10)
    y = np.digitize(np.nan_to_num(x[:, 0]) + 0.5 * np.nan_to_num(x[:, 1]), [-0.5, 0.5]).astype(np.float32)
    kw = dict(max_depth=5) if grow_policy == "depthwise" else dict(max_depth=0, max_leaves=20)
    p = sb.TrainingParams(objective="multi:softprob", num_class=3, grow_policy=grow_policy, eta=0.3,
                          max_bin=64, subsample=0.9, colsample_bytree=0.8, seed=8, **kw)
    d = sb.DMatrix(x, labels=y, feature_types=ft)
    m1 = sb.train(p, d, 5, ctx=ctx)
    with code_width(2):
        m2 = sb.train(p, d, 5, ctx=ctx)
    assert_trees_equal(m1.export(), m2.export())
    assert np.array_equal(m1.predict_margin(d), m2.predict_margin(d))


def test_batched_jobs_with_u8_codes_equal_u16_alone(sb, ctx):
    """Jobs at the many-jobs shape (max_bin 64) train batched with one-byte
    codes; each model equals the job trained alone with two-byte codes."""
    rng = np.random.default_rng(31)
    jobs = []
    for i in range(5):
        n, f = 4000 + 3000 * i, 20 + 6 * i
        x = rng.standard_normal((n, f)).astype(np.float32)
        x[rng.random(x.shape) < 0.05] = np.nan
        y = (np.sin(np.nan_to_num(x[:, 0])) + np.nan_to_num(x[:, 1]) + rng.normal(0, 0.1, n)).astype(np.float32)
        p = sb.TrainingParams(max_depth=(4, 6, 8)[i % 3], eta=(0.05, 0.1, 0.3)[i % 3], max_bin=64, seed=i)
        jobs.append((p, sb.DMatrix(x, labels=y), 4))
    together = sb.train_many(jobs, ctx=ctx)
    with code_width(2):
        for (p, d, rounds), m in zip(jobs, together):
            alone = sb.train(p, d, rounds, ctx=ctx)
            assert_trees_equal(m.export(), alone.export())
            assert np.array_equal(m.predict_margin(d), alone.predict_margin(d))
