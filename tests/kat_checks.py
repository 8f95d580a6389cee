"""Checks of the reference's known-answer tests (tests/golden/reference_kats.json)
against an engine: the CPU oracle or the CUDA path. Each check restates the
assertion of the reference test named in the case's `ref`."""
import math

import numpy as np


def params_of(sb_params_cls, d):
    p = sb_params_cls()
    for k, v in d.items():
        if k == "lambda":
            p.lambda_ = v
        elif k == "grow_policy":
            p.grow_policy = "lossguide" if v == 1 else "depthwise"
        elif k == "objective":
            p.objective = {0: "reg:squarederror", 2: "binary:logistic", 4: "multi:softprob"}[v]
        elif k == "monotone":
            p.monotone_constraints = v
        elif k == "interaction":
            p.interaction_constraints = v
        else:
            setattr(p, k, v)
    return p


def xarr(rows):
    return np.asarray([[np.nan if v is None else v for v in r] for r in rows], np.float32)


def gparr(g):
    return np.asarray(g, np.float32).reshape(-1, 2)


def leaf_of(nodes, cats, row):
    nid = 0
    while nodes["left"][nid] != -1:
        nd = nodes[nid]
        v = row[nd["split_feature"]]
        if np.isnan(v):
            left = bool(nd["default_left"])
        elif nd["is_categorical"]:
            c = 0 if not v > 0 else int(v)
            left = c in set(cats[nd["cat_begin"]:nd["cat_end"]].tolist())
        else:
            left = v < nd["split_cond"]
        nid = nd["left"] if left else nd["right"]
    return nid


def paths(nodes):
    out = []

    def walk(i, acc):
        if nodes["left"][i] == -1:
            out.append(list(acc))
            return
        acc.append(int(nodes["split_feature"][i]))
        walk(nodes["left"][i], acc)
        walk(nodes["right"][i], acc)
        acc.pop()
    walk(0, [])
    return out


def check_case(case, engine, Params):
    kind = case["kind"]
    if kind in ("leaf_weight", "split_gain", "tree", "tree_same"):
        x = xarr(case["x"])
        g = gparr(case["gpair"])
        p = params_of(Params, case["params"])
        nodes, cats = engine.tree(x, g, p)
        if kind == "leaf_weight":
            assert len(nodes) == 1, case["name"]
            assert np.float32(nodes["leaf_value"][0]) == np.float32(case["expected_leaf"]), case["name"]
        elif kind == "split_gain":
            assert len(nodes) == 3
            assert np.float32(nodes["split_gain"][0]) == np.float32(case["expected_gain"])
            assert [np.float32(nodes["leaf_value"][1]), np.float32(nodes["leaf_value"][2])] == \
                [np.float32(v) for v in case["expected_leaves"]]
        elif kind == "tree_same":
            nodes_b, _ = engine.tree(x, g, params_of(Params, case["params_b"]))
            assert len(nodes) == len(nodes_b)
            for r in range(len(x)):
                assert nodes["leaf_value"][leaf_of(nodes, cats, x[r])] == \
                    nodes_b["leaf_value"][leaf_of(nodes_b, cats, x[r])]
        else:
            if "expected_num_nodes" in case:
                assert len(nodes) == case["expected_num_nodes"], (case["name"], len(nodes))
            if "expected_pred" in case:
                for r, v in case["expected_pred"].items():
                    got = nodes["leaf_value"][leaf_of(nodes, cats, x[int(r)])]
                    assert abs(got - v) < case["tol"], (case["name"], r, got, v)
            if "expected_pred_all" in case:
                for r, v in enumerate(case["expected_pred_all"]):
                    got = nodes["leaf_value"][leaf_of(nodes, cats, x[r])]
                    assert abs(got - v) < case["tol"], (case["name"], r, got, v)
            if "expected_max_leaves" in case:
                assert int((nodes["left"] == -1).sum()) <= case["expected_max_leaves"]
            if "expected_monotone" in case:
                order = np.argsort(x[:, 0], kind="stable")
                prev = -np.inf
                for r in order:
                    pv = nodes["leaf_value"][leaf_of(nodes, cats, x[r])]
                    assert pv >= prev - 1e-5, (case["name"], pv, prev)
                    prev = pv
            if "expected_path_groups" in case:
                groups = case["expected_path_groups"]
                for path in paths(nodes):
                    hits = [any(f in grp for f in path) for grp in groups]
                    assert sum(hits) <= 1, (case["name"], path)
        return
    if kind == "cuts":
        x = xarr(case["x"])
        off, vals, _ = engine.cuts(x, case["max_bin"])
        for f, want in enumerate(case["expected_cuts"]):
            got = vals[off[f]:off[f + 1]]
            assert np.array_equal(got, np.asarray(want, np.float32)), (case["name"], f, got, want)
        gb = engine.global_bins(x, case["max_bin"])
        if "expected_strict_bins" in case:
            b = [engine.bin_of(x, case["max_bin"], 0, v) for v in case["expected_strict_bins"]]
            assert all(b[i] < b[i + 1] for i in range(len(b) - 1)), b
        if "expected_max_bins" in case:
            assert off[1] - off[0] <= case["expected_max_bins"]
            col = gb[:, 0]
            assert np.all(np.diff(col[np.argsort(x[:, 0], kind="stable")].astype(np.int64)) >= 0)
        if case.get("check_threshold_consistency"):
            s, e = int(off[0]), int(off[1])
            for target in range(s, e - 1):
                thr = vals[target]
                for r in range(len(x)):
                    assert (x[r, 0] < thr) == (gb[r, 0] <= target)
        if "expected_row_len" in case:
            assert list((gb != 0xFFFFFFFF).sum(axis=1)) == case["expected_row_len"]
        return
    if kind == "hist":
        if "x" in case:
            x = xarr(case["x"])
            g = gparr(case["gpair"])
        else:
            n = case["n"]
            i = np.arange(n)
            x = (i % 251).astype(np.float32).reshape(-1, 1)
            g = np.stack([((i * 7) % 13 - 6).astype(np.float32), np.ones(n, np.float32)], axis=1)
        rows = np.arange(len(x), dtype=np.uint32)
        h = engine.hist(x, case["max_bin"], rows, g)
        want = np.asarray(case["expected_hist"], np.float64)
        assert h.shape == want.shape, (h.shape, want.shape)
        assert np.max(np.abs(h - want)) < case["tol"], case["name"]
        return
    if kind == "subtract":
        left = np.asarray(case["left"], np.float64)
        right = np.asarray(case["right"], np.float64)
        parent = left + right
        got = engine.subtract(parent, left)
        assert np.max(np.abs(got - right)) < case["tol"]
        return
    if kind == "route":
        nodes = np.zeros(len(case["nodes"]), engine.NODE_DTYPE)
        for i, nd in enumerate(case["nodes"]):
            nodes[i]["split_feature"], nodes[i]["split_cond"], nodes[i]["default_left"] = nd[0], nd[1], nd[2]
            nodes[i]["left"], nodes[i]["right"], nodes[i]["leaf_value"], nodes[i]["sum_hess"] = nd[3:7]
            nodes[i]["is_categorical"] = 1 if nd[7] else 0
            if nd[7]:
                nodes[i]["cat_begin"], nodes[i]["cat_end"] = nd[8], nd[9]
        cats = np.asarray(case["cats"] or [0], np.uint32)
        arrays = (np.array([0, len(nodes)], np.int64), nodes, np.array([0, len(case["cats"])], np.int64),
                  cats)
        x = xarr(case["rows"])
        got = engine.predict(arrays, x, 0.0, 0)
        assert np.array_equal(got, np.asarray(case["expected"], np.float32)), (case["name"], got)
        return
    if kind == "gradient":
        got = engine.gradient(case["objective"], np.asarray(case["preds"], np.float32),
                              np.asarray(case["labels"], np.float32), case.get("weights"),
                              case.get("num_class", 0), case.get("scale_pos_weight", 1.0))
        want = np.asarray(case["expected"], np.float64)
        assert np.max(np.abs(got.astype(np.float64) - want)) <= case["tol"] + 1e-7, (case["name"], got)
        return
    if kind == "train":
        x = xarr(case["x"])
        y = np.asarray(case["y"], np.float32)
        p = params_of(Params, case["params"])
        bm = None if "base_margin" not in case else np.asarray(case["base_margin"], np.float32)
        res = engine.train(x, y, p, case["rounds"], base_margin=bm)
        e = case["expect"]
        k = p.num_class if p.objective.startswith("multi:") else 1
        if "num_trees" in e:
            assert res["num_trees"] == e["num_trees"]
        preds = res["predict"]
        if "rmse_below" in e:
            rmse = math.sqrt(float(np.mean((preds.astype(np.float64) - y) ** 2)))
            assert rmse < e["rmse_below"], (case["name"], rmse)
        if "prob_first_below" in e:
            assert preds[0] < e["prob_first_below"] and preds[-1] > e["prob_last_above"], preds[[0, -1]]
        if "pred_equals" in e:
            assert np.all(np.abs(preds - e["pred_equals"]) < e["tol"])
        if "probs_sum_to_one" in e:
            pr = preds.reshape(-1, k)
            assert np.all(np.abs(pr.sum(axis=1) - 1.0) < e["probs_sum_to_one"])
            acc = float(np.mean(pr.argmax(axis=1) == y))
            assert acc > e["accuracy_above"], acc
        if "margin_equals_base_margin" in e:
            assert np.all(np.abs(res["margin"] - bm) < e["margin_equals_base_margin"])
        return
    if kind == "train_cat_vs_num":
        x = xarr(case["x"])
        y = np.asarray(case["y"], np.float32)
        p = params_of(Params, case["params"])
        rn = engine.train(x, y, p, case["rounds"])
        rc = engine.train(x, y, p, case["rounds"], ftypes=np.ones(1, np.uint8))
        rmse = lambda pr: math.sqrt(float(np.mean((pr.astype(np.float64) - y) ** 2)))  # noqa: E731
        assert rmse(rc["predict"]) < case["expect"]["rmse_cat_below"]
        assert rmse(rn["predict"]) > case["expect"]["rmse_num_above"]
        return
    if kind == "shap":
        x = xarr(case["x"])
        y = np.asarray(case["y"], np.float32)
        p = params_of(Params, case["params"])
        res = engine.train(x, y, p, case["rounds"], want_contribs=True)
        k = p.num_class if p.objective.startswith("multi:") else 1
        contribs = res["contribs"].reshape(len(x), k, x.shape[1] + 1).astype(np.float64)
        margin = res["margin"].reshape(len(x), k).astype(np.float64)
        err = np.max(np.abs(contribs.sum(axis=2) - margin))
        assert err < case["tol"], (case["name"], err)
        if "zero_feature" in case:
            f = case["zero_feature"]
            assert res["feature_unused"](f)
            assert np.max(np.abs(contribs[:, :, f])) < case["zero_tol"]
        return
    if kind == "interactions":
        x = xarr(case["x"])
        y = np.asarray(case["y"], np.float32)
        p = params_of(Params, case["params"])
        res = engine.train(x, y, p, case["rounds"], want_contribs=True, want_interactions=True)
        k = p.num_class if p.objective.startswith("multi:") else 1
        w = x.shape[1] + 1
        inter = res["interactions"].reshape(len(x), k, w, w).astype(np.float64)
        contribs = res["contribs"].reshape(len(x), k, w).astype(np.float64)
        margin = res["margin"].reshape(len(x), k).astype(np.float64)
        row_err = np.max(np.abs(inter[:, :, :w - 1, :].sum(axis=3) - contribs[:, :, :w - 1]))
        eff_err = np.max(np.abs(inter.sum(axis=(2, 3)) - (margin - res["base_score"])))
        sym_err = np.max(np.abs(inter - inter.transpose(0, 1, 3, 2)))
        assert row_err < case["tol_row"], (case["name"], row_err)
        assert eff_err < case["tol_eff"], (case["name"], eff_err)
        assert sym_err < case["tol_sym"], (case["name"], sym_err)
        return
    raise AssertionError(f"unknown kind {kind}")
