"""K4/K5 through the HistogramBackend seam (sb_hist_build / sb_hist_subtract)
against CpuBackend::build of the oracle."""
import json
import os

import numpy as np
import pytest

from engines import GpuEngine
from gpu_helpers import LAYOUTS, hist_layout, hist_rows, mixed_data, random_gpair
from kat_checks import check_case

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [c for c in json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))["cases"]
         if c["kind"] in ("hist", "subtract")]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_hist_reference_kats(case, sb, ctx):
    check_case(case, GpuEngine(sb, ctx), sb.TrainingParams)


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("n,f,frac", [(2000, 10, 1.0), (60000, 40, 0.7), (200000, 100, 0.5)])
def test_fp32_within_1e5_of_f64(sb, ctx, orc, n, f, frac, layout):
    x, _ = mixed_data(n, f, seed=n)
    g = random_gpair(n, seed=1, logistic=True)
    rng = np.random.default_rng(2)
    rows = np.sort(rng.choice(n, int(n * frac), replace=False)).astype(np.uint32)
    with hist_layout(layout):
        gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    got = sb.GpuBackend("fp32", ctx=ctx).build(gh, rows, g)
    d = orc.data(x)
    want = d.hist(rows, g, threads=8)
    mag = d.hist(rows, np.abs(g), threads=8)  # sum of |g| and |h| per bin
    err = np.abs(got - want)
    # relative to the bin's absolute mass (1e-5), with an absolute floor for
    # near-empty bins
    assert np.all(err <= 1e-5 * mag + 1e-12), float(np.max(err / (mag + 1e-30)))


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("bits,f", [(12, 30), (16, 30), (20, 30), (16, 50), (16, 100)])
def test_fixed_point_is_exact(sb, ctx, orc, bits, f, layout):
    n = 100000
    x, _ = mixed_data(n, f, seed=7, n_cat=2, card=16)
    ft = np.zeros(f, np.uint8)
    ft[-2:] = 1
    g = random_gpair(n, seed=3)
    rows = np.arange(0, n, 3, dtype=np.uint32)
    with hist_layout(layout):
        gh = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), ctx=ctx)
    got = sb.GpuBackend("fixed", quantize_bits=bits, ctx=ctx).build(gh, rows, g)
    gq, _, _ = orc.quantize(g, bits)
    want = orc.data(x, ft).hist(rows, gq, threads=1)
    assert np.array_equal(got, want)
    # and deterministic across calls
    again = sb.GpuBackend("fixed", quantize_bits=bits, ctx=ctx).build(gh, rows, g)
    assert np.array_equal(got, again)


@pytest.mark.parametrize("rows_per_step", [1, 2, 4, 8])
@pytest.mark.parametrize("f", [6, 14])
def test_rows_per_warp_instruction(sb, ctx, orc, rows_per_step, f):
    """The TILED kernel with 1, 2, 4 or 8 rows sharing a warp instruction (a
    narrow matrix leaves most lanes idle with one row): fixed point exact
    against the oracle, FP32 within 1e-5 of each bin's mass, on sampled rows
    that end mid-batch."""
    n = 50_000
    x, _ = mixed_data(n, f, seed=40 + f, n_cat=1, card=9)
    ft = np.zeros(f, np.uint8)
    ft[-1] = 1
    g = random_gpair(n, seed=41, logistic=True)
    rng = np.random.default_rng(42)
    rows = np.sort(rng.choice(n, 37_777, replace=False)).astype(np.uint32)
    with hist_rows(rows_per_step):
        gh = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), ctx=ctx)
    d = orc.data(x, ft)
    got = sb.GpuBackend("fixed", quantize_bits=16, ctx=ctx).build(gh, rows, g)
    gq, _, _ = orc.quantize(g, 16)
    assert np.array_equal(got, d.hist(rows, gq, threads=8))
    got32 = sb.GpuBackend("fp32", ctx=ctx).build(gh, rows, g)
    want = d.hist(rows, g, threads=8)
    mag = d.hist(rows, np.abs(g), threads=8)
    assert np.all(np.abs(got32 - want) <= 1e-5 * mag + 1e-12)


def test_empty_rows_give_zero_histogram(sb, ctx):
    x, _ = mixed_data(1000, 5, seed=9)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    out = sb.GpuBackend(ctx=ctx).build(gh, np.zeros(0, np.uint32), random_gpair(1000))
    assert not out.any()


def test_dimension_mismatch_is_reported(sb, ctx):
    x, _ = mixed_data(100, 5, seed=9)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    with pytest.raises(sb.SbError):
        sb.GpuBackend(ctx=ctx).build(gh, np.arange(10, dtype=np.uint32), random_gpair(99))


@pytest.mark.parametrize("layout", LAYOUTS)
def test_local_bins_do_not_depend_on_layout(sb, ctx, layout):
    """The exported local bins (GHistIndex::bins) are the same whichever
    layout the histogram kernel reads."""
    x, ft = mixed_data(5000, 37, seed=4, n_cat=3, card=9)
    with hist_layout(None):
        ref = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), ctx=ctx).local_bins()
    with hist_layout(layout):
        got = sb.GHistIndex(sb.DMatrix(x, feature_types=ft), ctx=ctx).local_bins()
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("f", [24, 60, 100])
def test_autotuned_index_is_exact(sb, ctx, orc, f):
    """Indexes of 200k rows and more with at most 64 features time every
    choice that fits their shape (TILED with 1, 2, 4 or 8 rows per warp
    instruction, LANES with 1 or 2 positions per lane) and keep the fastest;
    whichever wins, the histograms are exact."""
    n = 250_000
    x, _ = mixed_data(n, f, seed=f)
    g = random_gpair(n, seed=f + 1)
    rows = np.arange(1, n, 2, dtype=np.uint32)
    with hist_layout(None):
        gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    got = sb.GpuBackend("fixed", quantize_bits=16, ctx=ctx).build(gh, rows, g)
    gq, _, _ = orc.quantize(g, 16)
    assert np.array_equal(got, orc.data(x).hist(rows, gq, threads=8))
