#!/usr/bin/env python
"""Benchmark of the hist training path on the 10M x 100 binary workload.

A step is one boosting round (gradients, row sampling, one depth-8 tree,
margin update) over all 10M rows of the synthetic `binary_mixed` dataset
(70 N(0,1), 20 lognormal, 10 Bernoulli(0.05) features, 10% NaN;
binary:logistic, max_depth 8, max_bin 256, eta 0.05, subsample 0.8,
colsample_bytree 0.8), with the fixed-point histogram form by default.

  value : Mrow-rounds/s with the binned matrix resident in HBM (CUDA events
          on the library's stream, max over ranks).
  e2e   : the same metric through the public C ABI call sb_train() from
          pinned host buffers: upload, cuts + binning, K rounds, model
          download.
  roofline : the histogram kernel (dominant), algorithmic bytes / device time.
  cpu_baseline : the C++ restatement of the reference CPU hist path, all
          host threads, on a bounded row sample, rounds only.

`--impl reference` times the reference's CPU path (the oracle port: the Rust
reference cannot be built here) with all host threads on a bounded sample of
the same workload.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

# The serving loop keeps several streams in flight; with the default 8
# hardware work queues, streams alias onto shared queues and a margin kernel
# can wait behind a TreeSHAP kernel of another stream. Must be set before the
# process's first CUDA call.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
METRIC = "train Mrow-rounds/s at matched RMSE; serving predict p50/p99 ms vs plain GPU"
UNIT = "Mrow-rounds/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=10_000_000)
    ap.add_argument("--precision", default="fixed", choices=["fixed", "fp32"])
    ap.add_argument("--cpu-rows", type=int, default=250_000)
    ap.add_argument("--cpu-rounds", type=int, default=20)
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-c0", action="store_true")
    ap.add_argument("--no-c2", action="store_true")
    ap.add_argument("--no-c3", action="store_true")
    ap.add_argument("--c2-rows", type=int, default=2_000_000)
    ap.add_argument("--c2-rounds", type=int, default=5)
    ap.add_argument("--c3-jobs", type=int, default=256)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--only", choices=["c0", "c2", "c3", "serve", "prediction", "index"], default=None,
                    help="run one extra leg alone on GPU 0 and print its JSON (profiling aid)")
    ap.add_argument("--index-reps", type=int, default=3)
    ap.add_argument("--serve-requests", type=int, default=1000)
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-train-rows", type=int, default=1_000_000)
    return ap.parse_args()


def params_for(sb, precision):
    return sb.TrainingParams(objective="binary:logistic", max_depth=8, max_bin=256, eta=0.05,
                             subsample=0.8, colsample_bytree=0.8, hist_precision=precision, seed=7)


def config_of(args, n):
    return {"workload": f"binary_mixed {n} x 100 (binary:logistic, depth 8, max_bin 256, eta 0.05, "
                        "subsample 0.8, colsample_bytree 0.8)",
            "n_rows": n, "n_features": 100, "rounds_per_step": 1, "precision": args.precision,
            "l2": "inputs larger than L2 (ELLPACK 2 B/entry = 2.1 GB at 10M rows)",
            "parallelism": f"replicas x{args.gpus}"}


class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.tmp,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.06)
        self.proc.terminate()
        self.proc.wait()
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_launch():
    """dram read+write bytes of one histogram launch, from the committed ncu
    summary of the same kernel (scaled to this workload), or None."""
    path = os.path.join(ROOT, "profiles", "k_hist_traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return d
    except (OSError, ValueError):
        return None


def logloss(margin, y):
    p = 1.0 / (1.0 + np.exp(-margin.astype(np.float64)))
    p = np.clip(p, 1e-15, 1 - 1e-15)
    return float(np.mean(-(y * np.log(p) + (1 - y) * np.log(1 - p))))


def cpu_leg(x, y, args, sb, threads, rounds, rows):
    """The oracle (C++ restatement of the reference CPU hist path) on the first
    `rows` rows: binning timed apart, then one `rounds`-round training with
    `threads` host threads. Returns (rows, seconds of the rounds, seconds of
    binning, train logloss after the rounds)."""
    import __graft_entry__ as ge
    orc = ge._load_module("sb_pyoracle", os.path.join(ROOT, "oracle", "pyoracle.py")).Oracle()
    xs = np.ascontiguousarray(x[:rows])
    ys = np.ascontiguousarray(y[:rows])
    p = params_for(sb, "fp32")
    t0 = time.perf_counter()
    d = orc.data(xs, max_bin=256)
    t_bin = time.perf_counter() - t0
    t0 = time.perf_counter()
    r = orc.train(xs, ys, p, rounds, threads=threads, data=d)
    t_rounds = time.perf_counter() - t0
    return xs.shape[0], t_rounds, t_bin, logloss(r["margins"].reshape(-1), ys)


def matched_quality(sb, ctx, x, y, rows, rounds, oracle_logloss):
    """Train logloss after the same rounds on the same row sample: the GPU's
    fixed-point and FP32 forms against the oracle (f64 histograms of f32
    gradients, as the reference CPU hist path)."""
    xs = np.ascontiguousarray(x[:rows])
    ys = np.ascontiguousarray(y[:rows])
    d = sb.DMatrix(xs, labels=ys)
    out = {"rows": rows, "rounds": rounds, "oracle_logloss": oracle_logloss}
    for prec in ("fixed", "fp32"):
        m = sb.train(params_for(sb, prec), d, rounds, ctx=ctx)
        ll = logloss(m.predict_margin(sb.DMatrix(xs)), ys)
        out[f"{prec}_logloss"] = ll
        out[f"{prec}_rel_diff"] = abs(ll - oracle_logloss) / oracle_logloss
    out["within_0.1pct"] = max(out["fixed_rel_diff"], out["fp32_rel_diff"]) < 1e-3
    return out


def c0_leg(sb, ctx, args):
    """The 100k x 30 regression workload (regression_sine; reg:squarederror,
    100 rounds, depth 6, max_bin 256, eta 0.1, lambda 1, base_score 0.5, no
    sampling), end to end from host buffers including binning: one sb_train()
    call on the GPU (best of 3) and the oracle on ONE host thread (as the
    reference's README times its 1.77 s)."""
    import __graft_entry__ as ge
    from sequoia_boost_b200 import datagen
    x, y = datagen.regression_sine(100_000, 30, seed=args.seed)
    p = sb.TrainingParams(objective="reg:squarederror", max_depth=6, max_bin=256, eta=0.1, lambda_=1.0,
                          base_score=0.5)
    rmse = lambda pr: float(np.sqrt(np.mean((pr.astype(np.float64) - y) ** 2)))  # noqa: E731
    sb.train(p, sb.DMatrix(x, labels=y), 100, ctx=ctx)  # warm-up
    best = math.inf
    for _ in range(3):
        t0 = time.perf_counter()
        m = sb.train(p, sb.DMatrix(x, labels=y), 100, ctx=ctx)
        best = min(best, time.perf_counter() - t0)
    gpu_rmse = rmse(m.predict(sb.DMatrix(x)))
    orc = ge._load_module("sb_pyoracle", os.path.join(ROOT, "oracle", "pyoracle.py")).Oracle()
    p32 = sb.TrainingParams(**{**p.__dict__, "hist_precision": "fp32"})
    t0 = time.perf_counter()
    d = orc.data(x, max_bin=256)
    r = orc.train(x, y, p32, 100, threads=1, data=d)
    t_cpu = time.perf_counter() - t0
    return {"workload": "regression_sine 100000 x 30, reg:squarederror, 100 rounds, depth 6, max_bin 256, "
                        "eta 0.1, lambda 1, base_score 0.5",
            "gpu_e2e_s": best, "gpu_mrow_rounds_per_s": 100_000 * 100 / best / 1e6, "gpu_train_rmse": gpu_rmse,
            "oracle_1thread_s": t_cpu, "oracle_mrow_rounds_per_s": 100_000 * 100 / t_cpu / 1e6,
            "oracle_train_rmse": rmse(r["margins"].reshape(-1)),
            "speedup_e2e": t_cpu / best,
            "reference_readme": "1.77 s on 1 thread (README.md:117-125), U(0,1) polynomial data of the same "
                                "shape; this oracle time calibrates the port against it"}


def _pct(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q)) if len(v) else None


def _latency_summary(lat, rows, kinds, wall):
    lat = np.asarray(lat)
    m = kinds == 0
    small = m & (rows <= 4096)
    return {"p50_ms_margin": _pct(lat[m], 50), "p99_ms_margin": _pct(lat[m], 99),
            "p99_ms_margin_le4096_rows": _pct(lat[small], 99),
            "p50_ms_contribs": _pct(lat[~m], 50), "p99_ms_contribs": _pct(lat[~m], 99),
            "rows_per_s": float(rows.sum() / wall)}


def serving_model(sb, ctx, args, torch):
    """The serving workload's model: 1000 trees of depth 8 (binary:logistic)
    trained on binary_mixed rows, and a pool of 65,536 request rows (N(0,1),
    10% NaN, pinned host memory)."""
    from sequoia_boost_b200 import datagen
    n = args.serve_train_rows
    x, y = datagen.binary_mixed(n=n, seed=args.seed + 100)
    xd = torch.from_numpy(x).to(f"cuda:{ctx.device}")
    gh = sb.GHistIndex.from_device(xd.data_ptr(), n, x.shape[1], max_bin=256, ctx=ctx)
    del xd
    b = sb.Booster(gh, params_for(sb, "fixed"), y, ctx=ctx)
    b.update(1000)
    model = b.model()
    del b, gh, x, y
    rng = np.random.default_rng(args.seed + 200)
    pool = rng.standard_normal((65536, 100)).astype(np.float32)
    pool[rng.random(pool.shape) < 0.1] = np.nan
    pool = torch.from_numpy(pool).pin_memory().numpy()
    return model, pool, rng


def prediction_figures(sb, model, pool):
    """Whole-call throughput of predict_contribs, predict_interactions and
    predict_leaf on the serving model (host buffers, copies included), best
    of 3 after one untimed call."""
    out = {}
    for name, rows, fn in (("contribs_rows_per_s", 4096, model.predict_contribs),
                           ("interactions_rows_per_s", 128, model.predict_interactions),
                           ("leaf_rows_per_s", 65536, model.predict_leaf)):
        d = sb.DMatrix(pool[:rows])
        fn(d)
        best = math.inf
        for _ in range(3):
            t0 = time.perf_counter()
            fn(d)
            best = min(best, time.perf_counter() - t0)
        out[name] = rows / best
    return out


def index_leg(sb, ctx, args, torch):
    """The index build of the bench workload (quantile cuts and binning,
    HistCuts::from_dmatrix + GHistIndex::from_dmatrix) from X already on the
    device, and the pinned-host upload of X that precedes it in sb_train."""
    from sequoia_boost_b200 import datagen
    x, _ = datagen.binary_mixed(n=args.rows, seed=args.seed)
    xp = torch.from_numpy(x).pin_memory()
    xd = torch.empty(x.shape, dtype=torch.float32, device="cuda")
    h2d = []
    for _ in range(args.index_reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xd.copy_(xp, non_blocking=True)
        torch.cuda.synchronize()
        h2d.append(time.perf_counter() - t0)
    build = []
    for _ in range(args.index_reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gh = sb.GHistIndex.from_device(xd.data_ptr(), x.shape[0], x.shape[1], max_bin=256, ctx=ctx)
        ctx.synchronize()
        build.append(time.perf_counter() - t0)
        lay = gh.layout()
        del gh
    return {"workload": f"binary_mixed {x.shape[0]} x {x.shape[1]}, max_bin 256",
            "build_ms": [round(t * 1e3, 2) for t in build], "h2d_ms": [round(t * 1e3, 2) for t in h2d],
            "h2d_gbs": x.nbytes / min(h2d) / 1e9, "code_bytes": lay["code_bytes"], "layout": lay["layout"]}


def prediction_leg(sb, ctx, args, torch):
    model, pool, _ = serving_model(sb, ctx, args, torch)
    return {"workload": f"1000-tree depth-8 binary:logistic ensemble (trained on {args.serve_train_rows} "
                        "binary_mixed rows), 100 features", "prediction": prediction_figures(sb, model, pool)}


def serving_leg(sb, ctx, args, torch):
    """The serving workload: a 1000-tree depth-8 ensemble trained on the
    binary_mixed data (100 features), a Poisson request stream, rows per
    request log-uniform in [1, 65536] (N(0,1) with 10% NaN), 90% margin and
    10% TreeSHAP. Continuous batching (sb_server) against the same stream
    served one request at a time by sb_predict_margin / sb_predict_contribs
    ("plain GPU"). Latency = scheduled arrival to result on the host."""
    import threading
    n = args.serve_train_rows
    model, pool, rng = serving_model(sb, ctx, args, torch)
    F = 100
    N = args.serve_requests
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, N))
    rows = np.clip(np.exp(rng.uniform(0.0, np.log(65536.0), N)).astype(np.int64), 1, 65536)
    kinds = (rng.random(N) < 0.1).astype(np.int64)  # 1 = TreeSHAP
    offs = np.array([rng.integers(0, 65536 - r + 1) for r in rows])
    outs = [torch.empty(int(r) * (1 if k == 0 else F + 1), dtype=torch.float32).pin_memory().numpy()
            for r, k in zip(rows, kinds)]

    def run_batched():
        srv = sb.Server(model, mem_bytes=0, n_slots=8, ctx=ctx)
        for i in range(8):  # warm-up
            srv.wait(srv.submit(pool[:512], kind="contribs" if i % 4 == 3 else "margin"))
        tickets = [None] * N
        sub = np.zeros(N)
        t0 = time.perf_counter() + 0.01

        def submitter():
            for i in range(N):
                d = t0 + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                sub[i] = time.perf_counter()
                lo = int(offs[i])
                tickets[i] = srv.submit(pool[lo:lo + rows[i]], kind="contribs" if kinds[i] else "margin",
                                        out=outs[i])
        th = threading.Thread(target=submitter)
        th.start()
        lat = np.zeros(N)
        for i in range(N):
            while tickets[i] is None:
                time.sleep(0.0001)
            _, l_ms = srv.wait(tickets[i])
            lat[i] = l_ms + (sub[i] - (t0 + arrivals[i])) * 1e3
        th.join()
        wall = max(time.perf_counter() - t0, 1e-9)
        st = srv.stats()
        srv.close()
        out = _latency_summary(lat, rows, kinds, wall)
        out.update({"batches": st["batches"], "max_batch_requests": st["max_batch_requests"],
                    "memory_waits": st["memory_waits"], "mem_budget_bytes": st["mem_bytes"],
                    "mem_peak_bytes": st["mem_peak"]})
        return out

    def run_plain():
        for _ in range(4):
            model.predict_margin(sb.DMatrix(pool[:512]))
        model.predict_contribs(sb.DMatrix(pool[:512]))
        lat = np.zeros(N)
        t0 = time.perf_counter() + 0.01
        for i in range(N):
            d = t0 + arrivals[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            lo = int(offs[i])
            dm = sb.DMatrix(pool[lo:lo + rows[i]])
            if kinds[i]:
                model.predict_contribs(dm)
            else:
                model.predict_margin(dm)
            lat[i] = (time.perf_counter() - (t0 + arrivals[i])) * 1e3
        wall = max(time.perf_counter() - t0, 1e-9)
        return _latency_summary(lat, rows, kinds, wall)

    batched = run_batched()
    plain = run_plain()
    pred = prediction_figures(sb, model, pool)
    return {"workload": f"1000-tree depth-8 binary:logistic ensemble (trained on {n} binary_mixed rows), "
                        f"{N} requests, Poisson {args.serve_rate:g} req/s, rows log-uniform [1, 65536], "
                        "10% NaN, 90% margin / 10% TreeSHAP",
            "batched": batched, "plain_gpu": plain,
            "requests_margin": int((kinds == 0).sum()), "requests_contribs": int(kinds.sum()),
            "prediction": pred}


def c2_leg(sb, ctx, args, torch):
    """The multiclass lossguide workload: multiclass_uniform 2M x 200 (U(0,1),
    features 195-199 categorical with 32 codes), 10 classes, multi:softprob,
    lossguide with max_leaves 255 and max_depth 0, max_bin 256, monotone +1 on
    feature 0 and -1 on feature 1; all 10 class trees of a round grow in the
    same launches. A step is one round (10 trees); CUDA events on the
    library's stream."""
    from sequoia_boost_b200 import datagen
    n = args.c2_rows
    x, y, ft = datagen.multiclass_uniform(n=n, seed=args.seed + 2)
    xd = torch.from_numpy(x).to(f"cuda:{ctx.device}")
    gh = sb.GHistIndex.from_device(xd.data_ptr(), n, x.shape[1], max_bin=256, feature_types=ft, ctx=ctx)
    del xd
    p = sb.TrainingParams(objective="multi:softprob", num_class=10, grow_policy="lossguide", max_leaves=255,
                          max_depth=0, max_bin=256, eta=0.3, monotone_constraints=[1, -1], seed=7)
    b = sb.Booster(gh, p, y, ctx=ctx)
    b.update(2)
    stream = torch.cuda.ExternalStream(ctx.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    e0.record(stream)
    b.update(args.c2_rounds)
    e1.record(stream)
    ctx.synchronize()
    ms = e0.elapsed_time(e1)
    b.set_timing(True)
    b.reset_stats()
    b.update(1)
    st = b.stats()
    m = b.margins().reshape(n, 10).astype(np.float64)
    m -= m.max(axis=1, keepdims=True)
    lp = m - np.log(np.exp(m).sum(axis=1, keepdims=True))
    mll = float(-np.mean(lp[np.arange(n), y.astype(np.int64)]))
    out = {"workload": f"multiclass_uniform {n} x 200, 10 classes, lossguide max_leaves 255, 5 categorical, "
                       "monotone on features 0 and 1", "value": n * args.c2_rounds / (ms / 1e3) / 1e6,
           "unit": UNIT, "ms_per_round": ms / args.c2_rounds, "rounds_timed": args.c2_rounds,
           "hist_ms_per_launch": st["hist_ms"] / max(st["hist_launches"], 1),
           "hist_launches_per_round": st["hist_launches"], "train_mlogloss": mll}
    del b, gh
    return out


def c3_leg(sb, ctx, args):
    """256 independent regression jobs (small_jobs: rows log-uniform in [1k,
    200k], 20-50 N(0,1) features, max_depth in {4,6,8}, eta in {0.05, 0.1,
    0.3}, 100 rounds, max_bin 64) trained together by one sb_train_many call
    from host buffers (upload, binning, rounds, model download)."""
    from sequoia_boost_b200 import datagen
    jobs = datagen.small_jobs(n_jobs=args.c3_jobs, seed=args.seed + 3)
    spec = [(sb.TrainingParams(objective="reg:squarederror", max_depth=j["max_depth"], eta=j["eta"], max_bin=64),
             sb.DMatrix(j["x"], labels=j["y"]), 100) for j in jobs]
    sb.train_many(spec[:4], ctx=ctx)  # warm-up
    # the same call with one round each: upload, binning and set-up alone
    t0 = time.perf_counter()
    sb.train_many([(p, d, 1) for p, d, _ in spec], n_streams=32, ctx=ctx)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    models = sb.train_many(spec, n_streams=32, ctx=ctx)
    t = time.perf_counter() - t0
    rows = sum(j["x"].shape[0] for j in jobs)
    assert all(m is not None for m in models)
    return {"workload": f"{len(jobs)} regression jobs, {rows} rows in total, 20-50 features, 100 rounds each, "
                        "max_bin 64, one sb_train_many call (32 streams)",
            "value": rows * 100 / t / 1e6, "unit": UNIT, "seconds": t, "seconds_one_round": t_setup}


def run_reference(args):
    """The reference arm: the reference's CPU hist path (oracle port), all host
    threads, a bounded sample of the same workload per step."""
    import __graft_entry__ as ge
    sb = ge.load_package()
    from sequoia_boost_b200 import datagen
    threads = os.cpu_count() or 1
    rows = args.cpu_rows
    x, y = datagen.binary_mixed(n=rows, seed=args.seed, chunk=min(rows, 500_000))
    orc = ge._load_module("sb_pyoracle", os.path.join(ROOT, "oracle", "pyoracle.py")).Oracle()
    d = orc.data(x, max_bin=256)
    p = params_for(sb, "fp32")
    for _ in range(args.warmup):
        orc.train(x, y, p, 1, threads=threads, data=d)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.train(x, y, p, 1, threads=threads, data=d)
    t = time.perf_counter() - t0
    value = rows * args.steps / t / 1e6
    cfg = config_of(args, args.rows)
    cfg["sample_rows"] = rows
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"first {rows} rows of binary_mixed, one round per step "
                                       "(binning excluded); the Rust reference cannot be built here"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def max_over_ranks(ms, dist, device=None):
    """The job's time for a step range: the slowest rank's device time."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, n, steps, ms):
    """Whole-job Mrow-rounds/s: every rank's replica trains n rows per round."""
    return world * n * steps / (ms / 1e3) / 1e6


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    import torch
    import __graft_entry__ as ge
    torch.cuda.set_device(local)
    if args.only:
        sb = ge.load_package()
        ctx = sb.Context(local)
        leg = {"c0": lambda: c0_leg(sb, ctx, args), "c2": lambda: c2_leg(sb, ctx, args, torch),
               "c3": lambda: c3_leg(sb, ctx, args), "serve": lambda: serving_leg(sb, ctx, args, torch),
               "prediction": lambda: prediction_leg(sb, ctx, args, torch),
               "index": lambda: index_leg(sb, ctx, args, torch)}[args.only]
        print(json.dumps({"leg": args.only, **leg()}), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    sb = ge.load_package()
    from sequoia_boost_b200 import datagen
    ctx = sb.Context(local)
    n = args.rows
    x, y = datagen.binary_mixed(n=n, seed=args.seed + rank)
    p = params_for(sb, args.precision)
    xd = torch.from_numpy(x).to(f"cuda:{local}")
    gh = sb.GHistIndex.from_device(xd.data_ptr(), n, x.shape[1], max_bin=256, ctx=ctx)
    del xd
    torch.cuda.synchronize()
    b = sb.Booster(gh, p, y, ctx=ctx)
    for _ in range(args.warmup):
        b.update(1)
    stream = torch.cuda.ExternalStream(ctx.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    l0 = ctx.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        b.update(1)
    e1.record(stream)
    launches = ctx.launch_count() - l0
    ctx.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if dist:
        ms = max_over_ranks(ms, dist, f"cuda:{local}")
        dist.barrier()
    value = job_value(world, n, args.steps, ms)

    # roofline of the histogram kernel: algorithmic bytes / device time
    b.set_timing(True)
    b.reset_stats()
    b.update(min(args.steps, 5))
    st = b.stats()
    b.set_timing(False)
    peak, peak_kind = peaks()
    achieved = st["hist_bytes"] / (st["hist_ms"] / 1e3) / 1e9 if st["hist_ms"] > 0 else None
    tr = traffic_per_launch()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": None if achieved is None else achieved / peak, "peak_kind": peak_kind,
                "traffic": None if tr is None else tr.get("bytes_per_launch"),
                "kernel": f"k_hist<{'fixed' if args.precision == 'fixed' else 'fp32'}>",
                "launches_timed": st["hist_launches"],
                "bytes_per_launch": st["hist_bytes"] / max(st["hist_launches"], 1),
                "ms_per_launch": st["hist_ms"] / max(st["hist_launches"], 1),
                "hist_share_of_round": st["hist_ms"] / st["round_ms"] if st["round_ms"] else None}
    rounds_total = args.warmup + args.steps + min(args.steps, 5)
    quality = {"train_logloss_fixed": logloss(b.margins().reshape(-1), y), "rounds": rounds_total,
               "quant_err_grad": st["quant_err_grad"], "quant_err_hess": st["quant_err_hess"]}
    del b

    fp32 = None
    if args.precision == "fixed" and not args.no_fp32:
        # the plain FP32 histogram form on the same resident index, same rounds
        b32 = sb.Booster(gh, params_for(sb, "fp32"), y, ctx=ctx)
        for _ in range(args.warmup):
            b32.update(1)
        ctx.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            b32.update(1)
        e1.record(stream)
        ctx.synchronize()
        ms32 = max_over_ranks(e0.elapsed_time(e1), dist, f"cuda:{local}")
        b32.set_timing(True)
        b32.reset_stats()
        b32.update(min(args.steps, 5))
        st32 = b32.stats()
        quality["train_logloss_fp32"] = logloss(b32.margins().reshape(-1), y)
        quality["fixed_vs_fp32_rel_diff"] = (abs(quality["train_logloss_fixed"] - quality["train_logloss_fp32"])
                                             / quality["train_logloss_fp32"])
        fp32 = {"value": job_value(world, n, args.steps, ms32), "unit": UNIT, "ms_per_step": ms32 / args.steps,
                "hist_ms_per_launch": st32["hist_ms"] / max(st32["hist_launches"], 1),
                "fixed_over_fp32": value / job_value(world, n, args.steps, ms32)}
        del b32
    del gh

    e2e = None
    if not args.no_e2e and rank == 0:
        xp = torch.from_numpy(x).pin_memory()
        yp = torch.from_numpy(y).pin_memory()
        xh = xp.numpy()
        yh = yp.numpy()
        # two whole calls, the faster one reported: a single call's time
        # varied by up to 60 ms between calls of one process (host side)
        calls = []
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            m = sb.train(p, sb.DMatrix(xh, labels=yh), args.steps, ctx=ctx)
            t1 = time.perf_counter()
            calls.append(t1 - t0)
        off, nodes, coff, cats, w = m.export()
        d2h = nodes.nbytes + off.nbytes + coff.nbytes + cats.nbytes
        e2e = {"value": n * args.steps / min(calls) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": (xh.nbytes + yh.nbytes) / args.steps,
               "d2h_bytes_per_step": d2h / args.steps,
               "calls_s": [round(c, 4) for c in calls],
               "note": "sb_train() from pinned host X/y: upload, cuts+binning, "
                       f"{args.steps} rounds, model download, the faster of two calls; bytes amortised per round"}
        del m, xp, yp

    cpu = None
    matched = None
    c0 = None
    if not args.no_cpu and rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        rows, t_rounds, t_bin, orc_ll = cpu_leg(x, y, args, sb, threads, args.cpu_rounds, args.cpu_rows)
        cpu = {"value": rows * args.cpu_rounds / t_rounds / 1e6, "unit": UNIT, "cores": threads,
               "kind": "port",
               "sample": f"first {rows} rows, one {args.cpu_rounds}-round training, binning excluded "
                         f"(binning {t_bin:.1f} s single-threaded)"}
        matched = matched_quality(sb, ctx, x, y, rows, args.cpu_rounds, orc_ll)
        if not args.no_c0:
            c0 = c0_leg(sb, ctx, args)
    serving = None
    if not args.no_serve and rank == 0:
        serving = serving_leg(sb, ctx, args, torch)
    c2 = c2_leg(sb, ctx, args, torch) if not args.no_c2 and rank == 0 else None
    c3 = c3_leg(sb, ctx, args) if not args.no_c3 and rank == 0 else None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "i64" if args.precision == "fixed" else "f32", "data": "synthetic",
                "config": config_of(args, n), "clocks": clk, "gpu_launches": launches,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "quality": quality,
                "fp32_arm": fp32, "matched_quality": matched, "c0": c0, "c2": c2, "c3": c3,
                "serving": serving}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
