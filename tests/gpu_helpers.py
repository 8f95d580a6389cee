"""Helpers shared by the GPU parity tests."""
import contextlib
import os

import numpy as np

# The histogram's bin-code layouts: "tiled" (a feature's bins contiguous in
# shared memory) and "lanes" (each lane of a warp owns its features' bins in
# its own bank). An index picks one by shape; SB_HIST_LAYOUT forces one for
# the indexes built while it is set.
LAYOUTS = ["tiled", "lanes"]


@contextlib.contextmanager
def hist_layout(name):
    """Indexes built inside the block use the given layout (None: by shape)."""
    old = os.environ.get("SB_HIST_LAYOUT")
    if name is None:
        os.environ.pop("SB_HIST_LAYOUT", None)
    else:
        os.environ["SB_HIST_LAYOUT"] = name
    try:
        yield
    finally:
        if old is None:
            os.environ.pop("SB_HIST_LAYOUT", None)
        else:
            os.environ["SB_HIST_LAYOUT"] = old


@contextlib.contextmanager
def hist_rows(rows):
    """Indexes built inside the block give the TILED histogram kernel `rows`
    rows (1, 2, 4 or 8) per warp instruction (None: by the feature count)."""
    old = os.environ.get("SB_HIST_ROWS")
    if rows is None:
        os.environ.pop("SB_HIST_ROWS", None)
    else:
        os.environ["SB_HIST_ROWS"] = str(rows)
    try:
        yield
    finally:
        if old is None:
            os.environ.pop("SB_HIST_ROWS", None)
        else:
            os.environ["SB_HIST_ROWS"] = old


def mixed_data(n, f=12, seed=0, nan_frac=0.1, n_cat=0, card=8):
    """N(0,1), lognormal and Bernoulli columns, NaN holes, optional
    categorical columns at the end."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, f)).astype(np.float32)
    if f >= 6:
        x[:, f // 3:f // 2] = np.exp(x[:, f // 3:f // 2])
        x[:, f // 2:f // 2 + 2] = (rng.random((n, 2)) < 0.05).astype(np.float32)
    for c in range(n_cat):
        x[:, f - 1 - c] = rng.integers(0, card, n).astype(np.float32)
    x[rng.random((n, f)) < nan_frac] = np.nan
    ft = np.zeros(f, np.uint8)
    ft[f - n_cat:] = 1 if n_cat else 0
    return x, ft


def random_gpair(n, seed=0, logistic=False):
    rng = np.random.default_rng(seed)
    if logistic:
        p = rng.random(n).astype(np.float32)
        y = (rng.random(n) < 0.3).astype(np.float32)
        return np.stack([p - y, np.maximum(p * (1 - p), 1e-16)], axis=1).astype(np.float32)
    return np.stack([rng.standard_normal(n), np.ones(n)], axis=1).astype(np.float32)


def assert_trees_equal(gpu_arrays, orc_arrays, check_cats=True):
    go, gn, gco, gc = gpu_arrays[:4]
    oo, on, oco, oc = orc_arrays[:4]
    assert np.array_equal(go, oo), ("tree offsets", go, oo)
    for name in gn.dtype.names:
        if name == "reserved":
            continue
        a, b = gn[name], on[name]
        if not np.array_equal(a, b):
            i = int(np.nonzero(a != b)[0][0])
            raise AssertionError(f"field {name} differs first at node {i}: gpu {a[i]} oracle {b[i]}\n"
                                 f"gpu node {gn[i]}\noracle node {on[i]}")
    if check_cats:
        assert np.array_equal(gco, oco)
        assert np.array_equal(gc, oc)


def leaf_ids(nodes, cats, x):
    out = np.zeros(len(x), np.int32)
    for r in range(len(x)):
        nid = 0
        while nodes["left"][nid] != -1:
            nd = nodes[nid]
            v = x[r, nd["split_feature"]]
            if np.isnan(v):
                left = bool(nd["default_left"])
            elif nd["is_categorical"]:
                c = 0 if not v > 0 else int(v)
                left = c in set(cats[nd["cat_begin"]:nd["cat_end"]].tolist())
            else:
                left = v < nd["split_cond"]
            nid = nd["left"] if left else nd["right"]
        out[r] = nid
    return out
