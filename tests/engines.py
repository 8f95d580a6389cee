"""Two engines behind one interface for the KAT checks: the CPU oracle and
the CUDA path (through the C ABI)."""
import numpy as np


class OracleEngine:
    def __init__(self, orc):
        self.o = orc
        from sb_pyoracle import NODE_DTYPE
        self.NODE_DTYPE = NODE_DTYPE

    def tree(self, x, g, p):
        d = self.o.data(x, max_bin=p.max_bin)
        m = self.o.tree_build(d, p, g, np.arange(len(x), dtype=np.uint32))
        off, nodes, coff, cats, _ = m.export()
        return nodes, cats

    def cuts(self, x, max_bin, ftypes=None):
        return self.o.data(x, ftypes, max_bin=max_bin).cuts()

    def global_bins(self, x, max_bin):
        return self.o.data(x, max_bin=max_bin).global_bins()

    def bin_of(self, x, max_bin, f, v):
        return self.o.data(x, max_bin=max_bin).bin_of(f, v)

    def hist(self, x, max_bin, rows, g):
        d = self.o.data(x, max_bin=max_bin)
        h1 = d.hist(rows, g, threads=1)
        h8 = d.hist(rows, g, threads=8)
        assert np.max(np.abs(h1 - h8)) < 1e-6  # parallel == sequential (hist/mod.rs:393-417)
        return h1

    def subtract(self, parent, child):
        return parent - child

    def predict(self, arrays, x, base, k):
        return self.o.predict_margin(arrays, x, base, k)

    def gradient(self, obj, preds, labels, weights, k, spw):
        w = None if weights is None else np.asarray(weights, np.float32)
        return self.o.gradient(obj, preds, labels, w, k, spw)

    def train(self, x, y, p, rounds, base_margin=None, ftypes=None, want_contribs=False,
              want_interactions=False):
        r = self.o.train(x, y, p, rounds, base_margin=base_margin, ftypes=ftypes)
        arrays = r["model"].export()
        base = r["model"].base_score
        k = p.num_class if p.objective.startswith("multi:") else 1
        margin = self.o.predict_margin(arrays, x, base, p.num_class,
                                       base_margin=None if base_margin is None else base_margin)
        out = {"num_trees": len(arrays[0]) - 1, "margin": margin,
               "predict": self.o.transform(p.objective, margin, p.num_class)}
        assert np.array_equal(margin, r["margins"].reshape(-1))
        if want_contribs:
            out["contribs"] = self.o.predict_contribs(arrays, x, base, p.num_class)
            nodes = arrays[1]
            out["feature_unused"] = lambda f: not np.any((nodes["left"] != -1) & (nodes["split_feature"] == f))
        if want_interactions:
            out["interactions"] = self.o.predict_interactions(arrays, x, base, p.num_class)
            out["base_score"] = base
        del k
        return out


class GpuEngine:
    def __init__(self, sb, ctx):
        self.sb = sb
        self.ctx = ctx
        from sequoia_boost_b200.api import NODE_DTYPE
        self.NODE_DTYPE = NODE_DTYPE

    def _g(self, x, max_bin, ftypes=None):
        return self.sb.GHistIndex(self.sb.DMatrix(x, feature_types=ftypes), max_bin=max_bin, ctx=self.ctx)

    def tree(self, x, g, p):
        gh = self._g(x, p.max_bin)
        m = self.sb.HistTreeBuilder(p, ctx=self.ctx).build(gh, g, np.arange(len(x), dtype=np.uint32))
        off, nodes, coff, cats, _ = m.export()
        return nodes, cats

    def cuts(self, x, max_bin, ftypes=None):
        return self._g(x, max_bin, ftypes).cuts()

    def global_bins(self, x, max_bin):
        return self._g(x, max_bin).global_bins()

    def bin_of(self, x, max_bin, f, v):
        gh = self._g(x, max_bin)
        off, vals, _ = gh.cuts()
        sl = vals[off[f]:off[f + 1]]
        return int(off[f] + min(np.searchsorted(sl, v, side="right"), len(sl) - 1))

    def hist(self, x, max_bin, rows, g):
        gh = self._g(x, max_bin)
        return self.sb.GpuBackend("fp32", ctx=self.ctx).build(gh, rows, g)

    def subtract(self, parent, child):
        return self.sb.GpuBackend(ctx=self.ctx).subtract(parent, child)

    def predict(self, arrays, x, base, k):
        m = self.sb.BoostedModel.from_arrays(arrays[0], arrays[1], arrays[2], arrays[3], base, k,
                                             x.shape[1], ctx=self.ctx)
        return m.predict_margin(self.sb.DMatrix(x))

    def gradient(self, obj, preds, labels, weights, k, spw):
        w = None if weights is None else np.asarray(weights, np.float32)
        return self.sb.objective_gradient(obj, preds, labels, w, num_class=k, scale_pos_weight=spw,
                                          ctx=self.ctx)

    def train(self, x, y, p, rounds, base_margin=None, ftypes=None, want_contribs=False,
              want_interactions=False):
        d = self.sb.DMatrix(x, labels=y, base_margin=base_margin, feature_types=ftypes)
        m = self.sb.train(p, d, rounds, ctx=self.ctx)
        dx = self.sb.DMatrix(x, base_margin=base_margin)
        out = {"num_trees": m.num_trees(), "margin": m.predict_margin(dx), "predict": m.predict(dx)}
        if want_contribs:
            out["contribs"] = m.predict_contribs(self.sb.DMatrix(x))
            nodes = m.export()[1]
            out["feature_unused"] = lambda f: not np.any((nodes["left"] != -1) & (nodes["split_feature"] == f))
        if want_interactions:
            out["interactions"] = m.predict_interactions(self.sb.DMatrix(x))
            out["base_score"] = m.base_score()
        return out
