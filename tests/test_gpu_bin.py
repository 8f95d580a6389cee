"""K1/K2 on the GPU: quantile cuts and bins bit-exact against the oracle
(HistCuts::from_dmatrix + GHistIndex::from_dmatrix)."""
import numpy as np
import pytest

from gpu_helpers import mixed_data

pytestmark = pytest.mark.gpu


def _compare(sb, ctx, orc, x, ft=None, max_bin=256, missing=float("nan")):
    gh = sb.GHistIndex(sb.DMatrix(x, feature_types=ft, missing=missing), max_bin=max_bin, ctx=ctx)
    off, vals, cat = gh.cuts()
    d = orc.data(x, ft, missing=missing, max_bin=max_bin)
    o_off, o_vals, o_cat = d.cuts()
    assert np.array_equal(off, o_off), np.nonzero(off != o_off)
    bad = np.nonzero(vals != o_vals)[0]
    assert bad.size == 0, (bad[:5], vals[bad[:5]], o_vals[bad[:5]])
    assert np.array_equal(cat, o_cat)
    gb = gh.global_bins()
    ob = d.global_bins()
    bad = np.argwhere(gb != ob)
    assert bad.size == 0, (bad[:5], gb[tuple(bad[0])], ob[tuple(bad[0])])
    return gh


@pytest.mark.parametrize("max_bin", [16, 64, 256])
def test_cuts_bins_normal(sb, ctx, orc, max_bin):
    x = np.random.default_rng(1).standard_normal((20000, 30)).astype(np.float32)
    _compare(sb, ctx, orc, x, max_bin=max_bin)


def test_cuts_bins_mixed_missing(sb, ctx, orc):
    x, _ = mixed_data(30000, 40, seed=2, nan_frac=0.1)
    _compare(sb, ctx, orc, x)


def test_cuts_bins_binary_mixed_shape(sb, ctx, orc, datagen):
    x, _ = datagen.binary_mixed(n=40_000, seed=11, chunk=10_000)
    _compare(sb, ctx, orc, x)


def test_cuts_bins_categorical(sb, ctx, orc):
    x, ft = mixed_data(20000, 16, seed=3, n_cat=4, card=32)
    _compare(sb, ctx, orc, x, ft)


def test_edge_values(sb, ctx, orc):
    rng = np.random.default_rng(4)
    n = 5000
    x = np.zeros((n, 8), np.float32)
    x[:, 0] = 5.0                                     # constant feature
    x[:, 1] = np.nan                                  # all missing
    x[:, 2] = rng.integers(0, 3, n)                   # few distinct
    x[:, 3] = np.where(rng.random(n) < 0.5, -0.0, 0.0)  # signed zeros
    x[:, 4] = rng.standard_normal(n)
    x[:5, 4] = [np.inf, -np.inf, np.inf, 1e38, -1e-45]
    x[:, 5] = np.round(rng.standard_normal(n), 1)     # heavy ties, > max_bin distinct
    x[:, 6] = rng.standard_normal(n) * 1e-30          # tiny magnitudes
    x[:, 7] = rng.integers(0, 300, n)                 # 300 distinct integers
    _compare(sb, ctx, orc, x, max_bin=256)
    _compare(sb, ctx, orc, x, max_bin=16)


def test_single_row_and_sentinel_missing(sb, ctx, orc):
    x = np.array([[1.5, -2.0, 7.0]], np.float32)
    _compare(sb, ctx, orc, x)
    y = np.random.default_rng(5).integers(-3, 4, (1000, 3)).astype(np.float32)
    _compare(sb, ctx, orc, y, missing=-3.0)  # -3 entries are missing


def test_nan_with_numeric_sentinel_is_rejected(sb, ctx):
    x = np.array([[1.0], [np.nan], [2.0]], np.float32)
    with pytest.raises(sb.SbError):
        sb.GHistIndex(sb.DMatrix(x, missing=-1.0), ctx=ctx)


def test_empty_dataset_is_rejected(sb, ctx):
    with pytest.raises(sb.SbError):
        sb.DMatrix(np.zeros((0, 3), np.float32))
