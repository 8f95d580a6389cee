"""Writes tests/golden/reference_kats.json: the known-answer tests and
invariants that the reference's own unit tests hold for the hist path.

The reference (pgarrett-scripps/sequoia-boost) is Rust and cannot be built
here, so its tests cannot be run to produce outputs. Each case below restates
one reference test: the same inputs (built by the same formula), and the
expected answer that test asserts. Where a test compares against a brute-force
computation (histogram == brute force, hist == exact greedy tree, cut values),
the expected numbers are computed here in plain Python, independently of the
C++ oracle and the CUDA path, so that both are pinned to them.

Run:  python tests/golden/make_reference_kats.py
"""
import json
import math
import os
import struct

HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x):
    return struct.unpack("<f", struct.pack("<f", x))[0]


def next_up_f32(x):
    b = struct.unpack("<I", struct.pack("<f", x))[0]
    if x == 0.0:
        return struct.unpack("<f", struct.pack("<I", 1))[0]
    b = b + 1 if x > 0 else b - 1
    return struct.unpack("<f", struct.pack("<I", b))[0]


def feature_cuts(vals, max_bin):
    """build_feature_cuts + push_max_sentinel, quantile.rs:203-245, :319-323."""
    sv = sorted(vals)
    if not sv:
        return [0.0]
    out = []
    distinct = 1 + sum(1 for a, b in zip(sv, sv[1:]) if a != b)
    if distinct <= max_bin:
        out.append(sv[0])
        out += [b for a, b in zip(sv, sv[1:]) if a != b]
    else:
        n = len(sv)
        last = -math.inf
        for b in range(1, max_bin + 1):
            q = b / max_bin
            idx = min(max(math.ceil(q * n), 1) - 1, n - 1)
            if sv[idx] > last:
                out.append(sv[idx])
                last = sv[idx]
    if out[-1] <= sv[-1]:
        out.append(next_up_f32(sv[-1]))
    return out


def bin_of(cuts, v):
    """numeric HistCuts::bin_of (local index), quantile.rs:166-181."""
    k = sum(1 for c in cuts if c <= v)
    return min(k, len(cuts) - 1)


def exact_tree_predict(x, g, h, max_depth, lam, mcw):
    """Exact greedy regression tree on one feature (ColMaker-style), used by
    hist.rs:1003-1046 as the oracle for the hist builder. Depthwise, ties keep
    the first split (strictly greater than best + 1e-6)."""
    n = len(x)

    def gain(G, H):
        return 0.0 if (H < mcw or H <= 0) else G * G / (H + lam)

    def weight(G, H):
        return 0.0 if (H < mcw or H <= 0) else -G / (H + lam)

    pred = [0.0] * n

    def grow(rows, depth):
        G = sum(g[r] for r in rows)
        H = sum(h[r] for r in rows)
        best = (0.0, None)
        if depth < max_depth:
            order = sorted(rows, key=lambda r: x[r])
            gl = hl = 0.0
            for i in range(len(order) - 1):
                gl += g[order[i]]
                hl += h[order[i]]
                if x[order[i]] == x[order[i + 1]]:
                    continue
                gr, hr = G - gl, H - hl
                if hl < mcw or hr < mcw:
                    continue
                lc = gain(gl, hl) + gain(gr, hr) - gain(G, H)
                if lc > best[0] + 1e-6:
                    best = (lc, (x[order[i]] + x[order[i + 1]]) / 2)
        if best[1] is None or best[0] <= 1e-6:
            w = weight(G, H)
            for r in rows:
                pred[r] = w
            return
        thr = best[1]
        grow([r for r in rows if x[r] < thr], depth + 1)
        grow([r for r in rows if x[r] >= thr], depth + 1)

    grow(list(range(n)), 0)
    return pred


def hist_brute(x, gp, cuts):
    hist = [[0.0, 0.0] for _ in cuts]
    for xi, (gg, hh) in zip(x, gp):
        b = bin_of(cuts, xi)
        hist[b][0] += gg
        hist[b][1] += hh
    return hist


def main():
    cases = []

    # ---- gain / weight closed forms, tree/gain.rs:128-200, constraints.rs:136-178
    # Each is a one-distinct-value dataset: the root cannot split, so its leaf
    # weight is calc_weight_bounded(G, H).
    for name, ref, G, H, params, w in [
        ("weight_closed_form", "tree/gain.rs:149-156", -4.0, 2.0, {"lambda": 1.0}, 4.0 / 3.0),
        ("l1_reduces_weight", "tree/gain.rs:158-164", -4.0, 2.0, {"lambda": 1.0, "alpha": 1.0}, 1.0),
        ("max_delta_step_clamps", "tree/gain.rs:166-177", -100.0, 1.0,
         {"lambda": 0.0, "max_delta_step": 1.0, "min_child_weight": 0.0}, 1.0),
        ("min_child_weight_zeros", "tree/gain.rs:179-190", -4.0, 0.5,
         {"lambda": 1.0, "min_child_weight": 1.0}, 0.0),
    ]:
        cases.append({"name": name, "ref": ref, "kind": "leaf_weight",
                      "x": [[0.0], [0.0]], "gpair": [[G / 2, H / 2], [G / 2, H / 2]],
                      "params": dict(params, max_depth=1), "expected_leaf": f32(w)})

    # split gain: left (-4,2), right (4,2), parent (0,4) -> 16/3 + 16/3 - 0
    cases.append({"name": "split_gain_positive", "ref": "tree/gain.rs:192-200 + constraints.rs:150-158",
                  "kind": "split_gain", "x": [[0.0], [1.0]], "gpair": [[-4.0, 2.0], [4.0, 2.0]],
                  "params": {"lambda": 1.0, "min_child_weight": 0.0, "max_depth": 1},
                  "expected_gain": f32(32.0 / 3.0),
                  "expected_leaves": [f32(4.0 / 3.0), f32(-4.0 / 3.0)]})

    # ---- tree builder, tree/builder/hist.rs:779-1046
    cases.append({"name": "splits_on_separating_feature", "ref": "tree/builder/hist.rs:779-801",
                  "kind": "tree", "x": [[0.0], [0.0], [1.0], [1.0]],
                  "gpair": [[1, 1], [1, 1], [-1, 1], [-1, 1]],
                  "params": {"max_depth": 1, "lambda": 0.0, "min_child_weight": 0.0, "gamma": 0.0},
                  "expected_num_nodes": 3, "expected_pred": {"0": -1.0, "2": 1.0}, "tol": 1e-6})
    cases.append({"name": "no_split_below_gamma", "ref": "tree/builder/hist.rs:803-820",
                  "kind": "tree", "x": [[0.0], [1.0]], "gpair": [[1, 1], [-1, 1]],
                  "params": {"max_depth": 3, "gamma": 1e9}, "expected_num_nodes": 1})
    n = 64
    cases.append({"name": "lossguide_respects_max_leaves", "ref": "tree/builder/hist.rs:822-845",
                  "kind": "tree", "x": [[float(i)] for i in range(n)],
                  "gpair": [[1.0 if i % 2 == 0 else -1.0, 1.0] for i in range(n)],
                  "params": {"grow_policy": 1, "max_leaves": 4, "max_depth": 0,
                             "min_child_weight": 0.0, "gamma": 0.0, "lambda": 0.0},
                  "expected_max_leaves": 4})
    n = 60
    xs = [f32(i / n) for i in range(n)]
    cases.append({"name": "monotone_increasing_is_enforced", "ref": "tree/builder/hist.rs:847-883",
                  "kind": "tree", "x": [[v] for v in xs],
                  "gpair": [[f32(-(abs(v - 0.5) - 0.25)), 1.0] for v in xs],
                  "params": {"max_depth": 4, "min_child_weight": 0.0, "gamma": 0.0, "lambda": 1.0,
                             "monotone": [1]},
                  "expected_monotone": [0, 1]})
    four = []
    gp4 = []
    for i in range(32):
        four.append([float(i % 2), float(i % 4), float(i % 8), float(i % 16)])
        gp4.append([1.0 if i % 2 == 0 else -1.0, 1.0])
    cases.append({"name": "interaction_constraints_confine_paths", "ref": "tree/builder/hist.rs:904-962",
                  "kind": "tree", "x": four, "gpair": gp4,
                  "params": {"max_depth": 4, "min_child_weight": 0.0, "gamma": 0.0, "lambda": 0.0,
                             "interaction": [[0, 1], [2, 3]]},
                  "expected_path_groups": [[0, 1], [2, 3]]})
    cases.append({"name": "empty_interaction_constraints_noop", "ref": "tree/builder/hist.rs:964-1001",
                  "kind": "tree_same", "x": four, "gpair": gp4,
                  "params": {"max_depth": 4, "min_child_weight": 0.0, "gamma": 0.0, "lambda": 0.0},
                  "params_b": {"max_depth": 4, "min_child_weight": 0.0, "gamma": 0.0, "lambda": 0.0,
                               "interaction": []}})
    n = 60
    xs = [f32(i * f32(0.1)) for i in range(n)]
    gs = [f32(math.sin(f32(v - 3.0))) for v in xs]
    exact = exact_tree_predict(xs, gs, [1.0] * n, 3, 1.0, 1.0)
    cases.append({"name": "hist_matches_exact_on_small_problem", "ref": "tree/builder/hist.rs:1003-1046",
                  "kind": "tree", "x": [[v] for v in xs], "gpair": [[g, 1.0] for g in gs],
                  "params": {"max_depth": 3, "lambda": 1.0, "min_child_weight": 1.0, "gamma": 0.0},
                  "expected_pred_all": [f32(v) for v in exact], "tol": 1e-5})

    # ---- cuts and binning, data/quantile.rs:325-390, data/ghist.rs:173-214
    x = [0.0, 1.0, 2.0, 1.0]
    cases.append({"name": "few_distinct_values_one_bin_each", "ref": "data/quantile.rs:329-340",
                  "kind": "cuts", "x": [[v] for v in x], "max_bin": 256,
                  "expected_cuts": [feature_cuts(x, 256)], "expected_strict_bins": [0.0, 1.0, 2.0]})
    x = [float(i) for i in range(1000)]
    cases.append({"name": "monotone_binning", "ref": "data/quantile.rs:342-359",
                  "kind": "cuts", "x": [[v] for v in x], "max_bin": 16,
                  "expected_cuts": [feature_cuts(x, 16)], "expected_max_bins": 17})
    x = [5.0, 5.0, 5.0]
    cases.append({"name": "constant_feature_never_collides", "ref": "data/quantile.rs:361-367",
                  "kind": "cuts", "x": [[v] for v in x], "max_bin": 256,
                  "expected_cuts": [feature_cuts(x, 256)]})
    x = [float(i) for i in range(10)]
    cases.append({"name": "split_threshold_consistency", "ref": "data/quantile.rs:369-389",
                  "kind": "cuts", "x": [[v] for v in x], "max_bin": 256,
                  "expected_cuts": [feature_cuts(x, 256)], "check_threshold_consistency": True})
    cases.append({"name": "bins_roundtrip_dense", "ref": "data/ghist.rs:177-191",
                  "kind": "cuts", "x": [[0.0, 10.0], [1.0, 20.0]], "max_bin": 256,
                  "expected_cuts": [feature_cuts([0.0, 1.0], 256), feature_cuts([10.0, 20.0], 256)],
                  "expected_row_len": [2, 2]})
    cases.append({"name": "missing_entries_absent", "ref": "data/ghist.rs:193-201",
                  "kind": "cuts", "x": [[0.0, None], [1.0, 2.0]], "max_bin": 256,
                  "expected_cuts": [feature_cuts([0.0, 1.0], 256), feature_cuts([2.0], 256)],
                  "expected_row_len": [1, 2]})

    # ---- histogram backend, tree/hist/mod.rs:121-204
    n = 200
    x = [float(i % 17) for i in range(n)]
    gp = [[f32(f32(i) * f32(0.1) - 5.0), 1.0] for i in range(n)]
    cuts = feature_cuts(x, 32)
    cases.append({"name": "build_matches_brute_force", "ref": "tree/hist/mod.rs:352-371",
                  "kind": "hist", "x": [[v] for v in x], "gpair": gp, "max_bin": 32,
                  "expected_hist": hist_brute(x, gp, cuts), "tol": 1e-4})
    n = 20000
    x = [float(i % 251) for i in range(n)]
    gp = [[float((i * 7) % 13) - 6.0, 1.0] for i in range(n)]
    cuts = feature_cuts(x, 64)
    cases.append({"name": "parallel_matches_sequential_large", "ref": "tree/hist/mod.rs:393-417",
                  "kind": "hist", "x_formula": "i % 251", "n": n,
                  "gpair_formula": "((i*7) % 13) - 6, 1", "max_bin": 64,
                  "expected_hist": hist_brute(x, gp, cuts), "tol": 1e-2})
    cases.append({"name": "subtraction_identity", "ref": "tree/hist/mod.rs:373-391",
                  "kind": "subtract",
                  "left": [[float(i), 1.0] for i in range(8)],
                  "right": [[-(float(i)) * 0.5, 2.0] for i in range(8)], "tol": 1e-12})

    # ---- routing, tree/regtree.rs:251-308
    cases.append({"name": "routing_stump", "ref": "tree/regtree.rs:255-279, :299-307",
                  "kind": "route",
                  "nodes": [[0, 0.5, 1, 1, 2, 0.0, 10.0, False], [0, 0.0, 1, -1, -1, -1.0, 5.0, False],
                            [0, 0.0, 1, -1, -1, 2.0, 5.0, False]],
                  "cats": [], "rows": [[0.2], [0.9], [None], [0.1]],
                  "expected": [-1.0, 2.0, -1.0, -1.0]})
    cases.append({"name": "routing_categorical_set_membership", "ref": "tree/regtree.rs:281-297",
                  "kind": "route",
                  "nodes": [[0, 0.0, 0, 1, 2, 0.0, 10.0, True, 0, 2],
                            [0, 0.0, 1, -1, -1, -1.0, 5.0, False], [0, 0.0, 1, -1, -1, 2.0, 5.0, False]],
                  "cats": [0, 2], "rows": [[0.0], [2.0], [1.0], [3.0], [9.0], [None]],
                  "expected": [-1.0, -1.0, 2.0, 2.0, 2.0, 2.0]})

    # ---- objectives, objective/*.rs tests
    cases.append({"name": "squared_error_gradient", "ref": "objective/regression.rs:91-113",
                  "kind": "gradient", "objective": 0, "preds": [2.0, 0.0, -1.0],
                  "labels": [1.0, 0.5, -3.0], "expected": [[1.0, 1.0], [-0.5, 1.0], [2.0, 1.0]],
                  "tol": 0.0})
    cases.append({"name": "squared_error_weighted", "ref": "objective/regression.rs:98-107",
                  "kind": "gradient", "objective": 0, "preds": [2.0], "labels": [1.0],
                  "weights": [4.0], "expected": [[4.0, 4.0]], "tol": 0.0})
    cases.append({"name": "logistic_gradient", "ref": "objective/classification.rs:104-114",
                  "kind": "gradient", "objective": 2, "preds": [0.0], "labels": [1.0],
                  "expected": [[-0.5, 0.25]], "tol": 1e-6})
    cases.append({"name": "logistic_scale_pos_weight", "ref": "objective/classification.rs:116-129",
                  "kind": "gradient", "objective": 2, "preds": [0.0, 0.0], "labels": [1.0, 0.0],
                  "scale_pos_weight": 3.0, "expected": [[-1.5, 0.75], [0.5, 0.25]], "tol": 1e-6})
    third = 1.0 / 3.0
    cases.append({"name": "softmax_gradient_layout", "ref": "objective/multiclass.rs:116-140",
                  "kind": "gradient", "objective": 4, "num_class": 3, "preds": [0.0] * 6,
                  "labels": [0.0, 2.0],
                  "expected": [[third - 1, 2 * third * (1 - third)], [third, 2 * third * (1 - third)],
                               [third, 2 * third * (1 - third)], [third, 2 * third * (1 - third)],
                               [third, 2 * third * (1 - third)], [third - 1, 2 * third * (1 - third)]],
                  "tol": 1e-6})

    # ---- end to end, learner/train.rs:536-1343 (thresholds the reference asserts)
    step = lambda n: ([[f32(i / n)] for i in range(n)],  # noqa: E731
                      [1.0 if f32(i / n) >= 0.5 else 0.0 for i in range(n)])
    x, y = step(100)
    cases.append({"name": "regression_reduces_training_error", "ref": "learner/train.rs:557-573",
                  "kind": "train", "x": x, "y": y, "rounds": 50,
                  "params": {"objective": 0, "max_depth": 3, "eta": 0.3},
                  "expect": {"num_trees": 50, "rmse_below": 0.05}})
    cases.append({"name": "binary_logistic_separates_classes", "ref": "learner/train.rs:575-589",
                  "kind": "train", "x": x, "y": y, "rounds": 50,
                  "params": {"objective": 2, "max_depth": 3, "eta": 0.3},
                  "expect": {"prob_first_below": 0.1, "prob_last_above": 0.9}})
    x10, y10 = step(10)
    cases.append({"name": "base_score_only_model_predicts_mean", "ref": "learner/train.rs:591-605",
                  "kind": "train", "x": x10, "y": y10, "rounds": 0,
                  "params": {"objective": 0},
                  "expect": {"pred_equals": f32(sum(y10) / 10.0), "tol": 1e-6}})
    x120, y120 = step(120)
    cases.append({"name": "hist_reaches_accuracy", "ref": "learner/train.rs:607-628",
                  "kind": "train", "x": x120, "y": y120, "rounds": 60,
                  "params": {"objective": 0, "max_depth": 3, "eta": 0.3},
                  "expect": {"rmse_below": 0.05}})
    cases.append({"name": "lossguide_trains_end_to_end", "ref": "learner/train.rs:670-685",
                  "kind": "train", "x": x120, "y": y120, "rounds": 60,
                  "params": {"objective": 0, "grow_policy": 1, "max_leaves": 16, "eta": 0.3},
                  "expect": {"rmse_below": 0.06}})
    n = 150
    xm = [[f32(i / n)] for i in range(n)]
    ym = [0.0 if v[0] < f32(0.33) else (1.0 if v[0] < f32(0.66) else 2.0) for v in xm]
    cases.append({"name": "multiclass_softprob_learns_three_classes", "ref": "learner/train.rs:699-748",
                  "kind": "train", "x": xm, "y": ym, "rounds": 60,
                  "params": {"objective": 4, "num_class": 3, "max_depth": 3, "eta": 0.3},
                  "expect": {"num_trees": 180, "probs_sum_to_one": 1e-4, "accuracy_above": 0.95}})
    xc, yc = [], []
    for _ in range(40):
        for c in [0.0, 1.0, 2.0, 3.0]:
            xc.append([c])
            yc.append(1.0 if int(c) % 2 == 1 else 0.0)
    cases.append({"name": "categorical_split_beats_numeric", "ref": "learner/train.rs:958-1005",
                  "kind": "train_cat_vs_num", "x": xc, "y": yc, "rounds": 40,
                  "params": {"objective": 0, "max_depth": 1, "eta": 0.3},
                  "expect": {"rmse_cat_below": 0.02, "rmse_num_above": 0.05}})
    x50, y50 = step(50)
    cases.append({"name": "base_margin_is_the_initial_margin", "ref": "learner/train.rs:1092-1108",
                  "kind": "train", "x": x50, "y": y50, "rounds": 0,
                  "base_margin": [f32(f32(i) * f32(0.01) - 0.25) for i in range(50)],
                  "params": {"objective": 0}, "expect": {"margin_equals_base_margin": 1e-6}})

    # ---- TreeSHAP, learner/shap.rs:512-779
    def make_data(n, nf):
        x = [[((i * 31 + j * 17 + 7) % 97) / 97.0 for j in range(nf)] for i in range(n)]
        x = [[f32(v) for v in row] for row in x]
        y = [f32(f32(2.0 * row[0]) - f32(1.5 * row[1]) + 0.3) for row in x]
        return x, y
    xs_, ys_ = make_data(80, 5)
    cases.append({"name": "additivity_single_output", "ref": "learner/shap.rs:539-571",
                  "kind": "shap", "x": xs_, "y": ys_, "rounds": 30,
                  "params": {"objective": 0, "max_depth": 4, "eta": 0.3}, "tol": 1e-4})
    n, nf, k = 90, 4, 3
    xmc = [[f32(((i * 13 + j * 29 + 3) % 101) / 101.0) for j in range(nf)] for i in range(n)]
    ymc = [float(i % k) for i in range(n)]
    cases.append({"name": "additivity_multiclass", "ref": "learner/shap.rs:573-614",
                  "kind": "shap", "x": xmc, "y": ymc, "rounds": 15,
                  "params": {"objective": 4, "num_class": 3, "max_depth": 3, "eta": 0.3},
                  "tol": 1e-4})
    n = 70
    xu = []
    yu = []
    for i in range(n):
        r = [f32(((i * 7 + 1) % 53) / 53.0), f32(((i * 11 + 2) % 53) / 53.0),
             f32(((i * 5 + 3) % 53) / 53.0), 0.5]
        xu.append(r)
        yu.append(f32(f32(3.0 * r[0]) - f32(2.0 * r[1])))
    cases.append({"name": "unused_feature_has_zero_contribution", "ref": "learner/shap.rs:616-660",
                  "kind": "shap", "x": xu, "y": yu, "rounds": 25,
                  "params": {"objective": 0, "max_depth": 4, "eta": 0.3}, "tol": 1e-4,
                  "zero_feature": 3, "zero_tol": 1e-6})

    # ---- TreeSHAP interaction values, learner/shap.rs:662-778: each feature
    # row of a matrix sums to the feature's contribution (row consistency),
    # the matrix sums to margin - base_score (efficiency), and the matrix is
    # symmetric
    cases.append({"name": "interactions_single_output", "ref": "learner/shap.rs:666-715",
                  "kind": "interactions", "x": xs_, "y": ys_, "rounds": 30,
                  "params": {"objective": 0, "max_depth": 4, "eta": 0.3},
                  "tol_row": 1e-4, "tol_eff": 1e-4, "tol_sym": 1e-5})
    cases.append({"name": "interactions_multiclass", "ref": "learner/shap.rs:716-778",
                  "kind": "interactions", "x": xmc, "y": ymc, "rounds": 15,
                  "params": {"objective": 4, "num_class": 3, "max_depth": 3, "eta": 0.3},
                  "tol_row": 1e-4, "tol_eff": 1e-4, "tol_sym": 1e-5})

    with open(os.path.join(HERE, "reference_kats.json"), "w") as fh:
        json.dump({"generated_by": "tests/golden/make_reference_kats.py",
                   "source": "unit tests of pgarrett-scripps/sequoia-boost, crates/sequoia-boost/src",
                   "cases": cases}, fh, indent=None, separators=(",", ":"))
    print(f"wrote {len(cases)} cases")


if __name__ == "__main__":
    main()
