"""Shapes the smaller parity tests do not reach, bit-exact against the oracle
on the fixed-point form:
  - more features than one shared-memory histogram tile holds (>= 200
    features of 257 bins: the histogram kernel runs several feature tiles);
  - the multiclass lossguide configuration (10 classes, 200 features, 5
    categorical features of cardinality 32 at 195-199, monotone +1 / -1 on
    features 0 and 1, max_leaves 255 with max_depth 0) at reduced rows;
  - 20-bit quantisation with more rows per CTA than one shared partial may
    hold, so the kernel splits a CTA's rows into several flushed pieces."""
import numpy as np
import pytest

from gpu_helpers import LAYOUTS, assert_trees_equal, hist_layout, leaf_ids, mixed_data, random_gpair

pytestmark = pytest.mark.gpu
# One histogram tile holds (bins + features) * 8 bytes in the shared memory a
# CTA may opt into (227 KB on a B200, less 4 KB kept free).
TILE_BYTES = 227 * 1024 - 4096


def _tiles_needed(gh):
    return ((gh.total_bins + gh.info()[1]) * 8 + TILE_BYTES - 1) // TILE_BYTES


@pytest.mark.parametrize("layout", LAYOUTS)
def test_multi_tile_tree_bit_exact(sb, ctx, orc, layout):
    n, f = 30_000, 210
    x, _ = mixed_data(n, f, seed=71)
    g = random_gpair(n, seed=72, logistic=True)
    rng = np.random.default_rng(73)
    rows = np.sort(rng.choice(n, int(n * 0.8), replace=False)).astype(np.uint32)
    p = sb.TrainingParams(max_depth=7, colsample_bytree=0.9, seed=5)
    with hist_layout(layout):
        gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    assert _tiles_needed(gh) >= 2, "the index must need more than one histogram tile"
    m, row_leaf = sb.HistTreeBuilder(p, ctx=ctx).build(gh, g, rows, round=1, return_row_leaf=True)
    gq, _, _ = orc.quantize(g, 16)
    om = orc.tree_build(orc.data(x), p, gq, rows, round_=1)
    ga, oa = m.export(), om.export()
    assert len(ga[1]) > 31
    assert ga[1]["split_feature"][ga[1]["left"] != -1].max() >= 128, "splits should use later tiles"
    assert_trees_equal(ga, oa)
    want = leaf_ids(oa[1], oa[3], x)
    assert np.array_equal(row_leaf[rows], want[rows])


@pytest.mark.parametrize("layout", LAYOUTS)
def test_multi_tile_histogram_exact(sb, ctx, orc, layout):
    n, f = 20_000, 240
    x, _ = mixed_data(n, f, seed=75)
    g = random_gpair(n, seed=76)
    rows = np.arange(0, n, 3, dtype=np.uint32)
    with hist_layout(layout):
        gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    assert _tiles_needed(gh) >= 2
    got = sb.GpuBackend("fixed", quantize_bits=16, ctx=ctx).build(gh, rows, g)
    gq, _, _ = orc.quantize(g, 16)
    want = orc.data(x).hist(rows, gq)
    assert np.array_equal(got, want)


def _c2_data(n, seed):
    """The multiclass lossguide workload's distribution: U(0,1) features, 5
    categorical features (cardinality 32) at 195-199, 10 classes = argmax of
    10 random projections plus Gumbel(0,1) noise."""
    rng = np.random.default_rng(seed)
    f, k = 200, 10
    x = rng.random((n, f), dtype=np.float32)
    x[:, 195:] = rng.integers(0, 32, (n, 5)).astype(np.float32)
    w = rng.standard_normal((f, k)).astype(np.float32)
    y = np.argmax(x @ w + rng.gumbel(size=(n, k)), axis=1).astype(np.float32)
    ft = np.zeros(f, np.uint8)
    ft[195:] = 1
    return x, y, ft


def _c2_params(sb):
    return sb.TrainingParams(objective="multi:softprob", num_class=10, grow_policy="lossguide", max_leaves=255,
                             max_depth=0, eta=0.3, monotone_constraints=[1, -1], seed=4)


@pytest.mark.parametrize("layout", LAYOUTS)
def test_multiclass_lossguide_workload_round0_bit_exact(sb, ctx, orc, layout):
    """Round 0 starts from equal margins, so device and oracle gradients are
    equal: the whole model (10 trees of up to 255 leaves) matches bit for bit."""
    x, y, ft = _c2_data(12_000, seed=81)
    p = _c2_params(sb)
    with hist_layout(layout):
        m = sb.train(p, sb.DMatrix(x, labels=y, feature_types=ft), 1, ctx=ctx)
    ref = orc.train(x, y, p, 1, ftypes=ft)
    ga = m.export()
    assert ga[0].size == 11
    assert ga[1]["is_categorical"].any(), "expected categorical splits"
    assert (ga[1]["left"] == -1).sum() > 10 * 10, "trees should grow past 10 leaves"
    assert_trees_equal(ga, ref["model"].export())
    assert np.array_equal(m.predict_margin(sb.DMatrix(x)), ref["margins"].reshape(-1))


def test_multiclass_lossguide_workload_later_rounds_bit_exact(sb, ctx, orc):
    """Later rounds: each class tree equals the oracle's tree grown from the
    round's device gradients (device expf may differ from glibc's by an ulp)."""
    x, y, ft = _c2_data(8_000, seed=82)
    p = _c2_params(sb)
    gh = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), ctx=ctx)
    b = sb.Booster(gh, p, y)
    d = orc.data(x, ft)
    b.update(1)
    b.update(1)
    grads = b.gradients()
    ga = b.model().export()
    rows = np.nonzero(b.row_mask(1))[0].astype(np.uint32)
    for k in range(10):
        gq, _, _ = orc.quantize(grads[k], 16)
        oa = orc.tree_build(d, p, gq, rows, round_=1, k=k).export()
        t0, t1 = ga[0][10 + k], ga[0][10 + k + 1]
        gn = ga[1][t0:t1].copy()
        on = oa[1].copy()
        leaf = on["left"] == -1  # the booster stores eta-scaled leaves
        on["leaf_value"][leaf] = (on["leaf_value"][leaf] * np.float32(p.eta)).astype(np.float32)
        c0, c1 = ga[2][10 + k], ga[2][10 + k + 1]
        assert_trees_equal((np.array([0, t1 - t0]), gn, np.array([0, c1 - c0]), ga[3][c0:c1]),
                           (oa[0], on, oa[2], oa[3]))


@pytest.mark.parametrize("layout", LAYOUTS)
def test_fixed_point_flush_split_bit_exact(sb, ctx, orc, layout):
    """quantize_bits = 20 lets a CTA fold at most 2046 rows into one shared
    partial; 420k rows spread over the grid give every CTA more than that at
    the root, so its rows are split into several flushed pieces."""
    n, f = 420_000, 8
    x, _ = mixed_data(n, f, seed=91)
    g = random_gpair(n, seed=92, logistic=True)
    rows = np.arange(n, dtype=np.uint32)
    import torch
    with hist_layout(layout):
        gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    # the histogram grid holds one 1024-thread CTA per SM
    assert n / torch.cuda.get_device_properties(0).multi_processor_count > 2046
    got = sb.GpuBackend("fixed", quantize_bits=20, ctx=ctx).build(gh, rows, g)
    gq, _, _ = orc.quantize(g, 20)
    d = orc.data(x)
    assert np.array_equal(got, d.hist(rows, gq, threads=8))
    p = sb.TrainingParams(max_depth=6, quantize_bits=20)
    m = sb.HistTreeBuilder(p, ctx=ctx).build(gh, g, rows)
    om = orc.tree_build(d, p, gq, rows, threads=8)
    assert_trees_equal(m.export(), om.export())
