"""The serving loop (sb_server): each request's result is the same alone and in
a mix of concurrent requests, admission follows the memory budget, and
shutdown drains the queue."""
import threading

import numpy as np
import pytest

from gpu_helpers import mixed_data

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served(sb, ctx):
    x, _ = mixed_data(20000, 12, seed=21)
    y = (np.nan_to_num(x[:, 0]) - np.nan_to_num(x[:, 3]) > 0).astype(np.float32)
    p = sb.TrainingParams(objective="binary:logistic", max_depth=6, eta=0.3, hist_precision="fixed", seed=2)
    m = sb.train(p, sb.DMatrix(x, labels=y), 40, ctx=ctx)
    return m, x


def _requests(x, seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(0, np.log(3000))))
        lo = int(rng.integers(0, x.shape[0] - n))
        kind = "contribs" if rng.random() < 0.2 else "margin"
        out.append((kind, np.ascontiguousarray(x[lo:lo + n])))
    return out


def test_results_alone_equal_results_in_the_mix(sb, served):
    m, x = served
    reqs = _requests(x, 1, 60)
    alone = []
    for kind, xr in reqs:
        d = sb.DMatrix(xr)
        alone.append(m.predict_margin(d) if kind == "margin" else m.predict_contribs(d))
    srv = sb.Server(m, mem_bytes=256 << 20, n_slots=4)
    try:
        # everything submitted at once from two threads: batches of mixed sizes
        tickets = [None] * len(reqs)

        def submit(idx):
            for i in idx:
                tickets[i] = srv.submit(reqs[i][1], kind=reqs[i][0])
        th = [threading.Thread(target=submit, args=(range(j, len(reqs), 2),)) for j in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for i, (kind, xr) in enumerate(reqs):
            got, lat = srv.wait(tickets[i], timeout_ms=60000)
            assert lat >= 0.0
            if kind == "margin":
                assert np.array_equal(got, alone[i]), i  # bit-identical margins
            else:
                # TreeSHAP accumulates in f64 with atomics: order-dependent last bits
                assert np.max(np.abs(got - alone[i])) <= 1e-5 * max(1.0, np.max(np.abs(alone[i]))), i
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["batches"] < len(reqs)  # requests were joined into batches
        assert st["max_batch_requests"] > 1
    finally:
        srv.close()


def test_small_and_large_margin_lanes(sb, served):
    """Margin requests on both sides of the small-lane bound (4096 rows) and
    TreeSHAP requests, submitted together, each get their own rows' results."""
    m, x = served
    rng = np.random.default_rng(5)
    sizes = [1, 4096, 4097, 19000, 37, 4095, 12000, 2, 8000, 4096]
    reqs = []
    for i, n in enumerate(sizes):
        idx = rng.integers(0, x.shape[0], n)
        reqs.append(("contribs" if i % 5 == 4 else "margin", np.ascontiguousarray(x[idx])))
    srv = sb.Server(m, mem_bytes=512 << 20, n_slots=2)
    try:
        tickets = [srv.submit(xr, kind=k) for k, xr in reqs]
        for (kind, xr), t in zip(reqs, tickets):
            got, _ = srv.wait(t, timeout_ms=60000)
            d = sb.DMatrix(xr)
            if kind == "margin":
                assert np.array_equal(got, m.predict_margin(d)), len(xr)
            else:
                want = m.predict_contribs(d)
                assert np.max(np.abs(got - want)) <= 1e-5 * max(1.0, np.max(np.abs(want)))
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
    finally:
        srv.close()


def test_admission_waits_for_memory_and_rejects_what_never_fits(sb, served):
    m, x = served
    # a budget that holds a few 2000-row margin batches, not all of them
    srv = sb.Server(m, mem_bytes=2 << 20, n_slots=4)
    try:
        xs = [np.ascontiguousarray(x[i * 2000:(i + 1) * 2000]) for i in range(6)]
        ts = [srv.submit(xi) for xi in xs]
        for xi, t in zip(xs, ts):
            got, _ = srv.wait(t, timeout_ms=60000)
            assert np.array_equal(got, m.predict_margin(sb.DMatrix(xi)))
        assert srv.stats()["mem_peak"] <= 2 << 20
        big = srv.submit(x[:20000], kind="contribs")  # far above the budget
        with pytest.raises(sb.SbError):
            srv.wait(big, timeout_ms=60000)
    finally:
        srv.close()


def test_close_finishes_queued_requests(sb, served):
    m, x = served
    srv = sb.Server(m, mem_bytes=64 << 20, n_slots=2)
    outs = []
    for i in range(10):
        xi = np.ascontiguousarray(x[i * 500:(i + 1) * 500])
        outs.append((srv.submit(xi), xi))
    pend = dict(srv._pending)
    srv.close()  # drains: every queued request has been computed
    for t, xi in outs:
        assert np.array_equal(pend[t][1].reshape(-1), m.predict_margin(sb.DMatrix(xi)))
