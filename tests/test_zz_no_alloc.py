"""sb_hist_build_static (the histogram build that allocates no device memory)
against sb_hist_build on the same inputs. Collected after every other test
file, so it also runs after the rest of the suite has used the device."""
import ctypes

import numpy as np
import pytest

from gpu_helpers import mixed_data, random_gpair

pytestmark = pytest.mark.gpu


def _static_build(sb, ctx, gh, d_rows, m, d_gpair, n, d_out, total):
    lib = sb._abi.lib()
    return lib.sb_hist_build_static(ctx.h, gh.h, ctypes.c_void_p(d_rows), m, ctypes.c_void_p(d_gpair), n,
                                    ctypes.c_void_p(d_out), total)


def test_static_scratch_build_matches_sb_hist_build_twice(sb, ctx, orc):
    import torch
    n, f = 60000, 24
    x, _ = mixed_data(n, f, seed=11)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    total = gh.total_bins
    rng = np.random.default_rng(5)
    dev = torch.device("cuda", 0)
    # two calls in a row with different rows and gradients: the second must not
    # see anything the first left in the shared scratch
    for call, frac in enumerate((0.6, 0.35)):
        g = random_gpair(n, seed=20 + call, logistic=True)
        rows = np.sort(rng.choice(n, int(n * frac), replace=False)).astype(np.uint32)
        want = sb.GpuBackend("fp32", ctx=ctx).build(gh, rows, g)
        d_rows = torch.from_numpy(rows.astype(np.int32)).to(dev)
        d_g = torch.from_numpy(np.ascontiguousarray(g, np.float32)).to(dev)
        d_out = torch.full((total, 2), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = _static_build(sb, ctx, gh, d_rows.data_ptr(), rows.size, d_g.data_ptr(), n, d_out.data_ptr(),
                           total)
        assert rc == 0, sb._abi.lib().sb_last_error()
        got = d_out.cpu().numpy()
        # both are FP32 shared-memory partials summed into f64 with atomics in
        # a different order: equal within 1e-5 of each bin's absolute mass
        mag = sb.GpuBackend("fp32", ctx=ctx).build(gh, rows, np.abs(g))
        err = np.abs(got - want)
        assert np.all(err <= 1e-5 * mag + 1e-12), (call, float(np.max(err / (mag + 1e-30))))
        # and against the oracle's f64 CpuBackend::build on the same rows
        ref = orc.data(x).hist(rows, g)
        err = np.abs(got - ref)
        assert np.all(err <= 1e-5 * mag + 1e-12), (call, float(np.max(err / (mag + 1e-30))))


def test_static_scratch_rejects_bad_rows_and_large_indexes(sb, ctx):
    import torch
    dev = torch.device("cuda", 0)
    n, f = 2000, 6
    x, _ = mixed_data(n, f, seed=3)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    total = gh.total_bins
    d_g = torch.zeros((n, 2), dtype=torch.float32, device=dev)
    d_out = torch.zeros((total, 2), dtype=torch.float64, device=dev)
    d_rows = torch.tensor([0, 5, n], dtype=torch.int32, device=dev)  # one id out of range
    torch.cuda.synchronize()
    rc = _static_build(sb, ctx, gh, d_rows.data_ptr(), 3, d_g.data_ptr(), n, d_out.data_ptr(), total)
    assert rc == sb._abi.SB_ERR_INVALID_ARG
    assert b"not below n_rows" in sb._abi.lib().sb_last_error()

    # 2100 features of 257 bins: about 541,800 histogram bins, above the scratch limit
    rng = np.random.default_rng(1)
    big = rng.normal(size=(300, 2100)).astype(np.float32)
    gb = sb.GHistIndex(sb.DMatrix(big), ctx=ctx)
    tb = gb.total_bins
    assert tb + 2100 > (8 << 20) // 16
    d_gb = torch.zeros((300, 2), dtype=torch.float32, device=dev)
    d_ob = torch.zeros((tb, 2), dtype=torch.float64, device=dev)
    d_rb = torch.arange(300, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    rc = _static_build(sb, ctx, gb, d_rb.data_ptr(), 300, d_gb.data_ptr(), 300, d_ob.data_ptr(), tb)
    assert rc == sb._abi.SB_ERR_UNSUPPORTED
    assert b"SB_STATIC_SCRATCH_BYTES" in sb._abi.lib().sb_last_error()


def test_static_scratch_through_a_second_context(sb, ctx, orc):
    """A second context on the same device reuses the scratch address the
    first context's calls looked up; its results match sb_hist_build and the
    oracle."""
    import torch
    n, f = 30000, 16
    x, _ = mixed_data(n, f, seed=14)
    ctx2 = sb.Context(0)
    gh2 = sb.GHistIndex(sb.DMatrix(x), ctx=ctx2)
    total = gh2.total_bins
    g = random_gpair(n, seed=33)
    rows = np.arange(1, n, 2, dtype=np.uint32)
    dev = torch.device("cuda", 0)
    d_rows = torch.from_numpy(rows.astype(np.int32)).to(dev)
    d_g = torch.from_numpy(np.ascontiguousarray(g, np.float32)).to(dev)
    want = sb.GpuBackend("fp32", ctx=ctx2).build(gh2, rows, g)
    mag = sb.GpuBackend("fp32", ctx=ctx2).build(gh2, rows, np.abs(g))
    ref = orc.data(x).hist(rows, g)
    for _ in range(2):
        d_out = torch.full((total, 2), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = _static_build(sb, ctx2, gh2, d_rows.data_ptr(), rows.size, d_g.data_ptr(), n, d_out.data_ptr(),
                           total)
        assert rc == 0, sb._abi.lib().sb_last_error()
        got = d_out.cpu().numpy()
        assert np.all(np.abs(got - want) <= 1e-5 * mag + 1e-12)
        assert np.all(np.abs(got - ref) <= 1e-5 * mag + 1e-12)


def test_static_scratch_from_a_second_context(sb, ctx, orc):
    """A second context on the same device uses the array address that the
    first context's call looked up (one lookup per device)."""
    import torch
    dev = torch.device("cuda", 0)
    n, f = 20000, 12
    x, _ = mixed_data(n, f, seed=23)
    g = random_gpair(n, seed=7, logistic=True)
    rows = np.arange(0, n, 2, dtype=np.uint32)
    d_rows = torch.from_numpy(rows.astype(np.int32)).to(dev)
    d_g = torch.from_numpy(np.ascontiguousarray(g, np.float32)).to(dev)
    ref = orc.data(x).hist(rows, g)
    mag = orc.data(x).hist(rows, np.abs(g))
    ctx2 = sb.Context(0)
    for c in (ctx, ctx2):
        gh = sb.GHistIndex(sb.DMatrix(x), ctx=c)
        total = gh.total_bins
        d_out = torch.full((total, 2), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = _static_build(sb, c, gh, d_rows.data_ptr(), rows.size, d_g.data_ptr(), n, d_out.data_ptr(), total)
        assert rc == 0, sb._abi.lib().sb_last_error()
        err = np.abs(d_out.cpu().numpy() - ref)
        assert np.all(err <= 1e-5 * mag + 1e-12), float(np.max(err / (mag + 1e-30)))


@pytest.mark.filterwarnings("ignore:The CUDA Graph is empty")
def test_static_scratch_refuses_a_capturing_stream(sb, ctx):
    """While the context's stream records a CUDA graph the call returns
    SB_ERR_UNSUPPORTED before it enqueues anything; the capture then ends with
    an empty graph and the context stays usable."""
    import torch
    dev = torch.device("cuda", 0)
    n, f = 2000, 6
    x, _ = mixed_data(n, f, seed=3)
    gh = sb.GHistIndex(sb.DMatrix(x), ctx=ctx)
    total = gh.total_bins
    d_g = torch.zeros((n, 2), dtype=torch.float32, device=dev)
    d_out = torch.zeros((total, 2), dtype=torch.float64, device=dev)
    d_rows = torch.arange(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        rc = _static_build(sb, ctx, gh, d_rows.data_ptr(), n, d_g.data_ptr(), n, d_out.data_ptr(), total)
    assert rc == sb._abi.SB_ERR_UNSUPPORTED
    assert b"captured" in sb._abi.lib().sb_last_error()
    del graph
    rc = _static_build(sb, ctx, gh, d_rows.data_ptr(), n, d_g.data_ptr(), n, d_out.data_ptr(), total)
    assert rc == 0, sb._abi.lib().sb_last_error()
