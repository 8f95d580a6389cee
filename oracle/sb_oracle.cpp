// sb_oracle.cpp — TEST INFRASTRUCTURE ONLY (see sb_oracle.h).
//
// A CPU restatement of the reference's `tree_method=hist` path, function by
// function. Every function names the reference file:line it follows (paths
// relative to crates/sequoia-boost/src/ of pgarrett-scripps/sequoia-boost).
// f64 is kept wherever the reference keeps it; the file must be compiled
// without -ffast-math and with -ffp-contract=off so that every f64/f32
// operation rounds exactly as the Rust code's does.
//
// Deliberate, documented differences from the reference:
//  * Random streams: include/sb_sampling.h replaces rand 0.8 StdRng (the
//    crate is not vendored and has no lock file, so its stream is unpinned).
//    Per-node column subsets are keyed by node id rather than drawn from one
//    sequential stream; with colsample_bylevel = colsample_bynode = 1 (the
//    defaults and every benchmark configuration) no draw happens at all.
//  * CpuBackend's rayon `reduce` sums per-thread partials in an unspecified
//    tree order; here they are summed in chunk order.
//  * The lossguide max-heap restates Rust std's BinaryHeap (sift_up on push,
//    sift_down_to_bottom + sift_up on pop) so equal-gain pop order matches.

#include "sb_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../include/sb_sampling.h"

namespace {

constexpr double K_RT_EPS = 1e-6;  // tree/builder/hist.rs:22
constexpr size_t PARALLEL_THRESHOLD = 32768;  // tree/hist/mod.rs:55
constexpr double INF = std::numeric_limits<double>::infinity();

// ------------------------------------------------------------ thread pool
// Stands in for rayon's global pool: a fixed set of workers that run the
// chunks of one parallel call.
class Pool {
 public:
  explicit Pool(int n) : n_(n) {
    for (int i = 0; i < n_ - 1; ++i) workers_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
      gen_++;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  int size() const { return n_; }
  void run(int nchunks, const std::function<void(int)>& f) {
    if (nchunks <= 0) return;
    if (n_ <= 1 || nchunks == 1) {
      for (int c = 0; c < nchunks; ++c) f(c);
      return;
    }
    auto job = std::make_shared<Job>();
    job->f = &f;
    job->total = nchunks;
    {
      std::lock_guard<std::mutex> g(mu_);
      job_ = job;
      gen_++;
    }
    cv_.notify_all();
    work(*job);
    std::unique_lock<std::mutex> g(job->mu);
    job->cv.wait(g, [&] { return job->done == job->total; });
  }

 private:
  struct Job {
    const std::function<void(int)>* f = nullptr;
    int total = 0;
    std::atomic<int> next{0};
    int done = 0;
    std::mutex mu;
    std::condition_variable cv;
  };
  static void work(Job& j) {
    for (;;) {
      int c = j.next.fetch_add(1);
      if (c >= j.total) break;
      (*j.f)(c);
      std::lock_guard<std::mutex> g(j.mu);
      if (++j.done == j.total) j.cv.notify_all();
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
        job = job_;
      }
      if (job) work(*job);
    }
  }
  int n_;
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::shared_ptr<Job> job_;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

Pool* get_pool(int threads) {
  static std::mutex mu;
  static std::vector<std::unique_ptr<Pool>> pools;
  std::lock_guard<std::mutex> g(mu);
  for (auto& p : pools)
    if (p->size() == threads) return p.get();
  pools.emplace_back(new Pool(threads));
  return pools.back().get();
}

// ---------------------------------------------------------------- helpers
inline bool is_missing(float v, float missing) {  // data/dmatrix.rs:10-16
  return std::isnan(missing) ? std::isnan(v) : v == missing;
}

inline uint32_t f32_as_u32(float v) {  // Rust `f32 as u32`: saturating, NaN -> 0
  if (std::isnan(v) || v <= 0.0f) return 0;
  if (v >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)v;
}

struct GS {  // GradStats, tree/gain.rs:18-48
  double g = 0, h = 0;
  void add(GS o) { g += o.g; h += o.h; }
  GS sub(GS o) const { return GS{g - o.g, h - o.h}; }
};

struct Reg {  // RegParams, gain.rs:52-74
  double lambda, alpha, mds, mcw;
};

double threshold_l1(double g, double a) {  // gain.rs:78-86
  if (g > a) return g - a;
  if (g < -a) return g + a;
  return 0.0;
}
double clamp_f64(double x, double lo, double hi) {  // f64::clamp
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
double calc_weight(GS s, const Reg& r) {  // gain.rs:91-100
  if (s.h < r.mcw || s.h <= 0.0) return 0.0;
  double w = -threshold_l1(s.g, r.alpha) / (s.h + r.lambda);
  if (r.mds > 0.0) w = clamp_f64(w, -r.mds, r.mds);
  return w;
}
double calc_gain(GS s, const Reg& r) {  // gain.rs:105-119
  if (s.h < r.mcw || s.h <= 0.0) return 0.0;
  if (r.mds == 0.0) {
    double t = threshold_l1(s.g, r.alpha);
    return (t * t) / (s.h + r.lambda);
  }
  double w = calc_weight(s, r);
  double t = threshold_l1(s.g, r.alpha);
  return -(2.0 * t * w + (s.h + r.lambda) * w * w);
}

struct Bounds {  // constraints.rs:45-67
  double lo = -INF, hi = INF;
  double clamp(double w) const { return clamp_f64(w, lo, hi); }
};
double calc_weight_bounded(GS s, const Reg& r, Bounds b) {  // constraints.rs:70-79
  if (s.h < r.mcw || s.h <= 0.0) return b.clamp(0.0);
  double w = -threshold_l1(s.g, r.alpha) / (s.h + r.lambda);
  if (r.mds > 0.0) w = clamp_f64(w, -r.mds, r.mds);
  return b.clamp(w);
}
double gain_at_weight(GS s, const Reg& r, double w) {  // constraints.rs:84-90
  if (s.h < r.mcw || s.h <= 0.0) return 0.0;
  double t = threshold_l1(s.g, r.alpha);
  return -(2.0 * t * w + (s.h + r.lambda) * w * w);
}
void child_bounds(Bounds p, int dir, double wl, double wr, Bounds* l, Bounds* rr) {
  // constraints.rs:94-124
  if (dir == 0) { *l = p; *rr = p; return; }
  double mid = 0.5 * (wl + wr);
  if (dir > 0) { *l = Bounds{p.lo, mid}; *rr = Bounds{mid, p.hi}; }
  else { *l = Bounds{mid, p.hi}; *rr = Bounds{p.lo, mid}; }
}
bool satisfies(int dir, double wl, double wr) {  // constraints.rs:128-134
  if (dir > 0) return wl <= wr;
  if (dir < 0) return wl >= wr;
  return true;
}
int64_t total_cmp_key(double x) {  // f64::total_cmp
  int64_t b;
  std::memcpy(&b, &x, 8);
  b ^= (int64_t)(((uint64_t)(b >> 63)) >> 1);
  return b;
}

// ------------------------------------------------------------------ cuts
struct Cuts {  // HistCuts, data/quantile.rs:20-31
  size_t F = 0;
  std::vector<uint32_t> off;  // F+1
  std::vector<float> vals;
  std::vector<uint8_t> is_cat;
  size_t total() const { return vals.size(); }
  // bin_of, quantile.rs:166-181
  uint32_t bin_of(size_t f, float v) const {
    uint32_t s = off[f], e = off[f + 1];
    const float* sl = vals.data() + s;
    size_t len = e - s;
    if (is_cat[f]) {
      // binary_search_by(partial_cmp): exact match or 0.
      size_t lo = 0, hi = len;
      while (lo < hi) {
        size_t mid = lo + (hi - lo) / 2;
        if (sl[mid] < v) lo = mid + 1;
        else if (sl[mid] > v) hi = mid;
        else return s + (uint32_t)mid;
      }
      return s;
    }
    size_t lo = 0, hi = len;  // partition_point(c <= v)
    while (lo < hi) {
      size_t mid = lo + (hi - lo) / 2;
      if (sl[mid] <= v) lo = mid + 1; else hi = mid;
    }
    size_t local = std::min(lo, len == 0 ? 0 : len - 1);
    return s + (uint32_t)local;
  }
};

void build_categorical_cuts(const std::vector<float>& sv, std::vector<float>& out) {
  // quantile.rs:187-200
  if (sv.empty()) { out.push_back(0.0f); return; }
  out.push_back(sv[0]);
  for (size_t i = 1; i < sv.size(); ++i)
    if (sv[i - 1] != sv[i]) out.push_back(sv[i]);
}

void push_max_sentinel(std::vector<float>& out, float max_val) {  // quantile.rs:319-323
  if (out.back() <= max_val) out.push_back(std::nextafterf(max_val, INFINITY));
}

void build_feature_cuts(const std::vector<float>& sv, size_t max_bin, std::vector<float>& out) {
  // quantile.rs:203-245
  if (sv.empty()) { out.push_back(0.0f); return; }
  float max_val = sv.back();
  size_t distinct = 1;
  for (size_t i = 1; i < sv.size(); ++i)
    if (sv[i - 1] != sv[i]) distinct++;
  if (distinct <= max_bin) {
    out.push_back(sv[0]);
    for (size_t i = 1; i < sv.size(); ++i)
      if (sv[i - 1] != sv[i]) out.push_back(sv[i]);
  } else {
    size_t n = sv.size();
    float last = -INFINITY;
    for (size_t b = 1; b <= max_bin; ++b) {
      double q = (double)b / (double)max_bin;
      size_t c = (size_t)std::ceil(q * (double)n);
      size_t idx = std::min(std::max(c, (size_t)1) - 1, n - 1);
      float v = sv[idx];
      if (v > last) { out.push_back(v); last = v; }
    }
  }
  push_max_sentinel(out, max_val);
}

// Hessian-weighted cuts of tree_method=approx, quantile.rs:253-316: `sv`
// holds ascending (value, weight) pairs (a stable sort by value keeps row
// order among equal values).
void build_feature_cuts_weighted(const std::vector<std::pair<float, float>>& sv, size_t max_bin,
                                 std::vector<float>& out) {
  if (sv.empty()) { out.push_back(0.0f); return; }
  const float max_val = sv.back().first;
  size_t distinct = 1;
  for (size_t i = 1; i < sv.size(); ++i)
    if (sv[i - 1].first != sv[i].first) distinct++;
  if (distinct <= max_bin) {  // every distinct value is a cut; weights do not matter
    out.push_back(sv[0].first);
    for (size_t i = 1; i < sv.size(); ++i)
      if (sv[i - 1].first != sv[i].first) out.push_back(sv[i].first);
  } else {
    double total = 0.0;  // the sequential f64 sum of the weights in value order
    for (const auto& p : sv) total += (double)p.second;
    float last = -INFINITY;
    if (total > 0.0) {
      const double step = total / (double)max_bin;
      double cum = 0.0;
      size_t b = 1;
      for (const auto& p : sv) {
        cum += (double)p.second;
        while (b <= max_bin && cum + 1e-12 >= (double)b * step) {
          if (p.first > last) { out.push_back(p.first); last = p.first; }
          b++;
        }
      }
    } else {  // all weights zero: the unweighted positions
      const size_t n = sv.size();
      for (size_t b = 1; b <= max_bin; ++b) {
        const double q = (double)b / (double)max_bin;
        const size_t c = (size_t)std::ceil(q * (double)n);
        const size_t idx = std::min(std::max(c, (size_t)1) - 1, n - 1);
        const float v = sv[idx].first;
        if (v > last) { out.push_back(v); last = v; }
      }
    }
  }
  push_max_sentinel(out, max_val);
}

// ---------------------------------------------------------------- ghist
}  // namespace

struct orc_data {
  size_t n = 0, F = 0;
  float missing = NAN;
  Cuts cuts;
  std::vector<size_t> row_ptr;  // GHistIndex CSR, data/ghist.rs:34-41
  std::vector<uint32_t> bins;   // global bins
  bool dense = true;
};

struct OTree {  // RegTree, tree/regtree.rs:74-83
  std::vector<sb_node> nodes;
  std::vector<uint32_t> cats;
  std::vector<double> gaps;
};

struct orc_model {  // BoostedModel, learner/model.rs:34-54
  std::vector<OTree> trees;
  std::vector<float> weights;
  float base_score = 0;
  int num_class = 0;
  int n_features = 0;
  int objective = 0;
};

namespace {

sb_node leaf_node(float value, float sum_hess) {  // Node::leaf, regtree.rs:51-65
  sb_node n;
  std::memset(&n, 0, sizeof(n));
  n.left = -1;
  n.right = -1;
  n.leaf_value = value;
  n.sum_hess = sum_hess;
  n.default_left = 1;
  return n;
}

// feature_bin_at / feature_bin, ghist.rs:134-170. Returns -1 for missing.
inline int64_t feature_bin_at(const orc_data& d, size_t r, size_t f, uint32_t fs, uint32_t fe) {
  if (d.dense) return d.bins[d.row_ptr[r] + f];
  for (size_t i = d.row_ptr[r]; i < d.row_ptr[r + 1]; ++i) {
    uint32_t b = d.bins[i];
    if (b >= fs && b < fe) return b;
  }
  return -1;
}

// accumulate, tree/hist/mod.rs:95-119
void accumulate(const orc_data& d, const uint32_t* rows, size_t m, const sb_gradpair* gp, GS* out) {
  const size_t* rp = d.row_ptr.data();
  const uint32_t* bins = d.bins.data();
  for (size_t i = 0; i < m; ++i) {
    size_t r = rows[i];
    double g = (double)gp[r].grad, h = (double)gp[r].hess;
    for (size_t k = rp[r]; k < rp[r + 1]; ++k) {
      GS& o = out[bins[k]];
      o.g += g;
      o.h += h;
    }
  }
}

// CpuBackend::build, tree/hist/mod.rs:58-89
void hist_build(const orc_data& d, const uint32_t* rows, size_t m, const sb_gradpair* gp,
                GS* out, int threads) {
  size_t total = d.cuts.total();
  std::fill(out, out + total, GS{});
  if (threads <= 1 || m < PARALLEL_THRESHOLD) {
    accumulate(d, rows, m, gp, out);
    return;
  }
  size_t grain = (m + threads - 1) / threads;
  int nchunks = (int)((m + grain - 1) / grain);
  std::vector<std::vector<GS>> partial(nchunks);
  get_pool(threads)->run(nchunks, [&](int c) {
    partial[c].assign(total, GS{});
    size_t b = (size_t)c * grain, e = std::min(m, b + grain);
    accumulate(d, rows + b, e - b, gp, partial[c].data());
  });
  for (int c = 0; c < nchunks; ++c)
    for (size_t i = 0; i < total; ++i) out[i].add(partial[c][i]);
}

// ---------------------------------------------------------- tree builder
struct Best {  // BestSplit, hist.rs:24-63
  double loss_chg = 0.0;
  uint32_t feature = 0;
  size_t split_bin = 0;
  bool default_left = true;
  GS left, right;
  double wl = 0.0, wr = 0.0;
  bool is_cat = false;
  std::vector<uint32_t> cat_left;
  double runner_up = -INF;  // best gain of every other candidate
  bool found() const { return loss_chg > K_RT_EPS; }
};

struct NodeEntry {  // hist.rs:66-77
  uint32_t nid = 0;
  size_t depth = 0;
  std::vector<uint32_t> rows;
  std::vector<GS> hist;
  Best best;
  Bounds bounds;
  bool has_allowed = false;
  std::vector<uint32_t> allowed;
};

struct Sampler {  // ColumnSampler (tree/sampler.rs) over sb_sampling.h keys
  std::vector<uint32_t> pool;
  double bylevel = 1, bynode = 1;
  uint64_t tree_key = 0;
  std::vector<uint32_t> sample(uint64_t nid) const {
    std::vector<uint32_t> v = pool;
    if (bylevel >= 1.0 && bynode >= 1.0) return v;
    sb_splitmix g{sb_node_key(tree_key, nid)};
    int len = sb_subsample(v.data(), (int)v.size(), bylevel, &g);
    len = sb_subsample(v.data(), len, bynode, &g);
    v.resize(len);
    return v;
  }
};

Sampler make_sampler(size_t F, const sb_train_params& p, uint64_t round, uint64_t k) {
  // make_column_sampler + sample_features, train.rs:479-489, :516-534
  Sampler s;
  s.pool.resize(F);
  for (size_t i = 0; i < F; ++i) s.pool[i] = (uint32_t)i;
  s.tree_key = sb_tree_key(p.seed, round, k);
  if (p.colsample_bytree < 1.0) {
    sb_splitmix g{s.tree_key};
    int len = sb_subsample(s.pool.data(), (int)F, p.colsample_bytree, &g);
    s.pool.resize(len);
  }
  s.bylevel = p.colsample_bylevel;
  s.bynode = p.colsample_bynode;
  return s;
}

class Builder {  // HistTreeBuilder, hist.rs:98-131
 public:
  Builder(const sb_train_params& p, size_t F) : p_(p) {
    reg_ = Reg{p.lambda, p.alpha, p.max_delta_step, p.min_child_weight};
    dirs_.assign(F, 0);
    for (int i = 0; i < p.n_monotone && (size_t)i < F; ++i) dirs_[i] = p.monotone ? p.monotone[i] : 0;
    // MonotoneConstraints::dir returns 0 beyond the list; is_active over the list
    active_ = false;
    for (int i = 0; i < p.n_monotone; ++i)
      if (p.monotone && p.monotone[i] != 0) active_ = true;
    // build_interaction_sets, hist.rs:715-731
    has_inter_ = p.n_interaction_groups > 0;
    if (has_inter_) {
      inter_.assign(F, {});
      in_group_.assign(F, 0);
      for (int gi = 0; gi < p.n_interaction_groups; ++gi) {
        uint32_t b = p.interaction_offsets[gi], e = p.interaction_offsets[gi + 1];
        for (uint32_t a = b; a < e; ++a) {
          uint32_t f = p.interaction_features[a];
          if (f >= F) continue;
          in_group_[f] = 1;
          for (uint32_t c = b; c < e; ++c) inter_[f].push_back(p.interaction_features[c]);
        }
      }
      for (auto& v : inter_) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
      }
    }
  }
  int dir(size_t f) const { return f < dirs_.size() ? dirs_[f] : 0; }

  OTree build(const orc_data& d, const sb_gradpair* gp, const uint32_t* subset, size_t m,
              const Sampler& sampler, int threads) {  // hist.rs:139-202
    size_t total_bins = d.cuts.total();
    GS root_stats;
    for (size_t i = 0; i < m; ++i)
      root_stats.add(GS{(double)gp[subset[i]].grad, (double)gp[subset[i]].hess});
    std::vector<GS> root_hist(total_bins);
    hist_build(d, subset, m, gp, root_hist.data(), threads);

    OTree tree;
    tree.nodes.push_back(leaf_node(0.0f, (float)root_stats.h));
    stats_ = {root_stats};
    bounds_ = {Bounds{}};
    gaps_.assign(1, INF);

    std::vector<uint32_t> root_feats = sampler.sample(0);
    NodeEntry root;
    root.nid = 0;
    root.depth = 0;
    root.rows.assign(subset, subset + m);
    root.best = evaluate(d.cuts, root_hist, root_stats, root_feats, Bounds{}, false, {});
    root.hist = std::move(root_hist);
    if (p_.grow_policy == SB_GROW_DEPTHWISE)
      grow_depthwise(tree, d, gp, sampler, std::move(root), threads);
    else
      grow_lossguide(tree, d, gp, sampler, std::move(root), threads);

    for (size_t id = 0; id < tree.nodes.size(); ++id) {  // hist.rs:193-200
      if (tree.nodes[id].left == -1) {
        double w = calc_weight_bounded(stats_[id], reg_, bounds_[id]);
        tree.nodes[id].leaf_value = (float)w;
      }
    }
    tree.gaps = gaps_;
    return tree;
  }

 private:
  size_t depth_limit() const {  // hist.rs:204-210
    return p_.max_depth == 0 ? std::numeric_limits<size_t>::max() : (size_t)p_.max_depth;
  }
  bool valid(const Best& b) const {  // hist.rs:271-276
    return b.found() && b.loss_chg > p_.gamma && b.left.h >= reg_.mcw && b.right.h >= reg_.mcw;
  }

  void grow_depthwise(OTree& tree, const orc_data& d, const sb_gradpair* gp, const Sampler& s,
                      NodeEntry root, int threads) {  // hist.rs:212-236
    size_t limit = depth_limit();
    std::vector<NodeEntry> frontier;
    frontier.push_back(std::move(root));
    size_t depth = 0;
    while (depth < limit && !frontier.empty()) {
      std::vector<NodeEntry> next;
      for (auto& e : frontier) {
        if (valid(e.best)) {
          NodeEntry l, r;
          split(tree, d, gp, s, std::move(e), threads, &l, &r);
          next.push_back(std::move(l));
          next.push_back(std::move(r));
        }
      }
      frontier = std::move(next);
      depth++;
    }
  }

  // Rust std BinaryHeap (max-heap) restated for equal-key pop order.
  static bool le(const NodeEntry& a, const NodeEntry& b) {  // a <= b under Ord
    return total_cmp_key(a.best.loss_chg) <= total_cmp_key(b.best.loss_chg);
  }
  static void sift_up(std::vector<NodeEntry>& h, size_t start, size_t pos) {
    NodeEntry hole = std::move(h[pos]);
    while (pos > start) {
      size_t parent = (pos - 1) / 2;
      if (le(hole, h[parent])) break;
      h[pos] = std::move(h[parent]);
      pos = parent;
    }
    h[pos] = std::move(hole);
  }
  static void sift_down_to_bottom(std::vector<NodeEntry>& h, size_t pos) {
    size_t end = h.size(), start = pos;
    NodeEntry hole = std::move(h[pos]);
    size_t child = 2 * pos + 1;
    while (end >= 2 && child <= end - 2) {
      child += le(h[child], h[child + 1]) ? 1 : 0;
      h[pos] = std::move(h[child]);
      pos = child;
      child = 2 * pos + 1;
    }
    if (child == end - 1) {
      h[pos] = std::move(h[child]);
      pos = child;
    }
    h[pos] = std::move(hole);
    sift_up(h, start, pos);
  }
  static void heap_push(std::vector<NodeEntry>& h, NodeEntry e) {
    h.push_back(std::move(e));
    sift_up(h, 0, h.size() - 1);
  }
  static NodeEntry heap_pop(std::vector<NodeEntry>& h) {
    NodeEntry item = std::move(h.back());
    h.pop_back();
    if (!h.empty()) {
      std::swap(item, h[0]);
      sift_down_to_bottom(h, 0);
    }
    return item;
  }

  void grow_lossguide(OTree& tree, const orc_data& d, const sb_gradpair* gp, const Sampler& s,
                      NodeEntry root, int threads) {  // hist.rs:238-268
    size_t limit = depth_limit();
    size_t max_leaves = p_.max_leaves == 0 ? std::numeric_limits<size_t>::max() : (size_t)p_.max_leaves;
    std::vector<NodeEntry> heap;
    heap_push(heap, std::move(root));
    size_t n_leaves = 1;
    while (!heap.empty()) {
      NodeEntry e = heap_pop(heap);
      if (n_leaves >= max_leaves) break;
      if (e.depth >= limit || !valid(e.best)) continue;
      NodeEntry l, r;
      split(tree, d, gp, s, std::move(e), threads, &l, &r);
      n_leaves++;
      heap_push(heap, std::move(l));
      heap_push(heap, std::move(r));
    }
  }

  void split(OTree& tree, const orc_data& d, const sb_gradpair* gp, const Sampler& s,
             NodeEntry e, int threads, NodeEntry* lo, NodeEntry* ro) {  // hist.rs:280-411
    const Cuts& cuts = d.cuts;
    const Best& b = e.best;
    int dr = dir(b.feature);
    Bounds lb, rb;
    child_bounds(e.bounds, dr, b.wl, b.wr, &lb, &rb);
    uint32_t fs = cuts.off[b.feature], fe = cuts.off[b.feature + 1];

    uint32_t left_id = (uint32_t)tree.nodes.size(), right_id = left_id + 1;
    tree.nodes.push_back(leaf_node((float)b.wl, (float)b.left.h));
    tree.nodes.push_back(leaf_node((float)b.wr, (float)b.right.h));
    sb_node& pn = tree.nodes[e.nid];
    pn.split_feature = b.feature;
    pn.default_left = b.default_left ? 1 : 0;
    pn.left = (int32_t)left_id;
    pn.right = (int32_t)right_id;
    if (b.is_cat) {  // expand_categorical, regtree.rs:159-186
      pn.is_categorical = 1;
      pn.cat_begin = (uint32_t)tree.cats.size();
      tree.cats.insert(tree.cats.end(), b.cat_left.begin(), b.cat_left.end());
      pn.cat_end = (uint32_t)tree.cats.size();
    } else {  // expand, regtree.rs:129-151
      pn.split_cond = cuts.vals[b.split_bin];
    }
    pn.split_gain = (float)b.loss_chg;
    stats_.push_back(b.left);
    bounds_.push_back(lb);
    stats_.push_back(b.right);
    bounds_.push_back(rb);
    gaps_.push_back(INF);
    gaps_.push_back(INF);
    gaps_[e.nid] = b.loss_chg - b.runner_up;

    std::vector<uint32_t> lrows, rrows;
    for (uint32_t r : e.rows) {
      int64_t bin = feature_bin_at(d, r, b.feature, fs, fe);
      bool go_left;
      if (bin >= 0) {
        if (b.is_cat) {
          uint32_t cv = f32_as_u32(cuts.vals[bin]);
          go_left = std::find(b.cat_left.begin(), b.cat_left.end(), cv) != b.cat_left.end();
        } else {
          go_left = (size_t)bin <= b.split_bin;
        }
      } else {
        go_left = b.default_left;
      }
      (go_left ? lrows : rrows).push_back(r);
    }

    size_t total_bins = e.hist.size();
    std::vector<GS> lh(total_bins), rh(total_bins);
    if (lrows.size() <= rrows.size()) {
      hist_build(d, lrows.data(), lrows.size(), gp, lh.data(), threads);
      for (size_t i = 0; i < total_bins; ++i) rh[i] = e.hist[i].sub(lh[i]);
    } else {
      hist_build(d, rrows.data(), rrows.size(), gp, rh.data(), threads);
      for (size_t i = 0; i < total_bins; ++i) lh[i] = e.hist[i].sub(rh[i]);
    }

    bool child_has_allowed = false;
    std::vector<uint32_t> child_allowed;
    if (has_inter_) {  // intersect_allowed, hist.rs:736-747
      bool feat_has = in_group_[b.feature] != 0;
      if (!e.has_allowed && !feat_has) {
        child_has_allowed = false;
      } else if (!e.has_allowed) {
        child_has_allowed = true;
        child_allowed = inter_[b.feature];
      } else if (!feat_has) {
        child_has_allowed = true;
        child_allowed = e.allowed;
      } else {
        child_has_allowed = true;
        for (uint32_t f : e.allowed)
          if (std::binary_search(inter_[b.feature].begin(), inter_[b.feature].end(), f))
            child_allowed.push_back(f);
      }
    }

    std::vector<uint32_t> lf = s.sample(left_id);
    Best left_best = evaluate(cuts, lh, b.left, lf, lb, child_has_allowed, child_allowed);
    std::vector<uint32_t> rf = s.sample(right_id);
    Best right_best = evaluate(cuts, rh, b.right, rf, rb, child_has_allowed, child_allowed);

    lo->nid = left_id; lo->depth = e.depth + 1; lo->rows = std::move(lrows); lo->hist = std::move(lh);
    lo->best = std::move(left_best); lo->bounds = lb; lo->has_allowed = child_has_allowed; lo->allowed = child_allowed;
    ro->nid = right_id; ro->depth = e.depth + 1; ro->rows = std::move(rrows); ro->hist = std::move(rh);
    ro->best = std::move(right_best); ro->bounds = rb; ro->has_allowed = child_has_allowed; ro->allowed = std::move(child_allowed);
  }

  // consider / consider_cat, hist.rs:549-596, :659-706
  void consider(Best& best, GS l, GS r, double parent_gain, Bounds bnd, int dr, uint32_t f,
                size_t bin, bool dleft, const std::vector<uint32_t>* cats) {
    double g, wl = 0.0, wr = 0.0;
    if (active_) {
      wl = calc_weight_bounded(l, reg_, bnd);
      wr = calc_weight_bounded(r, reg_, bnd);
      if (!satisfies(dr, wl, wr)) return;
      g = gain_at_weight(l, reg_, wl) + gain_at_weight(r, reg_, wr) - parent_gain;
    } else {
      g = calc_gain(l, reg_) + calc_gain(r, reg_) - parent_gain;
    }
    if (g > best.loss_chg + K_RT_EPS) {
      if (best.found() || best.loss_chg != 0.0) best.runner_up = std::max(best.runner_up, best.loss_chg);
      best.loss_chg = g;
      best.feature = f;
      best.split_bin = cats ? 0 : bin;
      best.default_left = cats ? false : dleft;
      best.left = l;
      best.right = r;
      best.wl = wl;
      best.wr = wr;
      best.is_cat = cats != nullptr;
      best.cat_left = cats ? *cats : std::vector<uint32_t>{};
    } else {
      best.runner_up = std::max(best.runner_up, g);
    }
  }

  Best evaluate(const Cuts& cuts, const std::vector<GS>& hist, GS total,
                const std::vector<uint32_t>& feats_in, Bounds bnd, bool has_allowed,
                const std::vector<uint32_t>& allowed) {  // hist.rs:418-542
    Best best;
    double mcw = reg_.mcw;
    std::vector<uint32_t> feats;
    if (has_allowed) {
      for (uint32_t f : feats_in)
        if (std::binary_search(allowed.begin(), allowed.end(), f)) feats.push_back(f);
    } else {
      feats = feats_in;
    }
    double parent_gain = active_
        ? gain_at_weight(total, reg_, calc_weight_bounded(total, reg_, bnd))
        : calc_gain(total, reg_);
    for (uint32_t f : feats) {
      size_t fs = cuts.off[f], fe = cuts.off[f + 1];
      if (fe <= fs + 1) continue;
      int dr = dir(f);
      if (cuts.is_cat[f]) {  // evaluate_categorical, hist.rs:607-653
        std::vector<size_t> order;
        for (size_t i = fs; i < fe; ++i)
          if (hist[i].h > 0.0) order.push_back(i);
        if (order.size() < 2) continue;
        double lam = reg_.lambda;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
          return total_cmp_key(hist[a].g / (hist[a].h + lam)) <
                 total_cmp_key(hist[b].g / (hist[b].h + lam));
        });
        GS left;
        std::vector<uint32_t> cats_left;
        for (size_t oi = 0; oi + 1 < order.size(); ++oi) {
          size_t bin = order[oi];
          left.add(hist[bin]);
          cats_left.push_back(f32_as_u32(cuts.vals[bin]));
          GS right = total.sub(left);
          if (left.h < mcw || right.h < mcw) continue;
          consider(best, left, right, parent_gain, bnd, dr, f, 0, false, &cats_left);
        }
        continue;
      }
      GS present;
      for (size_t i = fs; i < fe; ++i) present.add(hist[i]);
      GS missing = total.sub(present);
      bool has_missing = missing.h > 1e-6;
      GS acc;
      for (size_t i = fs; i < fe; ++i) {
        acc.add(hist[i]);
        if (i + 1 >= fe) break;
        GS la = acc, ra = total.sub(acc);
        if (la.h >= mcw && ra.h >= mcw) consider(best, la, ra, parent_gain, bnd, dr, f, i, false, nullptr);
        if (has_missing) {
          GS lb = acc;
          lb.add(missing);
          GS rb = present.sub(acc);
          if (lb.h >= mcw && rb.h >= mcw) consider(best, lb, rb, parent_gain, bnd, dr, f, i, true, nullptr);
        }
      }
    }
    return best;
  }

  const sb_train_params& p_;
  Reg reg_;
  std::vector<int> dirs_;
  bool active_ = false;
  bool has_inter_ = false;
  std::vector<std::vector<uint32_t>> inter_;
  std::vector<uint8_t> in_group_;
  std::vector<GS> stats_;
  std::vector<Bounds> bounds_;
  std::vector<double> gaps_;
};

// ------------------------------------------------------------ objectives
float sigmoid(float x) {  // objective/classification.rs:7-15
  if (x >= 0.0f) return 1.0f / (1.0f + std::exp(-x));
  float e = std::exp(x);
  return e / (1.0f + e);
}
void softmax_inplace(float* row, int k) {  // objective/multiclass.rs:14-30
  float mx = -INFINITY;
  for (int c = 0; c < k; ++c)
    if (row[c] > mx) mx = row[c];
  float sum = 0.0f;
  for (int c = 0; c < k; ++c) {
    row[c] = std::exp(row[c] - mx);
    sum += row[c];
  }
  float inv = 1.0f / sum;
  for (int c = 0; c < k; ++c) row[c] *= inv;
}
int n_outputs(int objective, int num_class) {
  return (objective == SB_OBJ_SOFTMAX || objective == SB_OBJ_SOFTPROB) ? num_class : 1;
}

double weighted_label_mean(const float* labels, const float* w, size_t n) {  // objective/mod.rs:~110
  if (w) {
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < n; ++i) {
      num += (double)labels[i] * (double)w[i];
      den += (double)w[i];
    }
    return den > 0.0 ? num / den : 0.0;
  }
  if (n == 0) return 0.0;
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += (double)labels[i];
  return s / (double)n;
}

std::vector<float> init_margin(const float* bm, size_t bm_len, size_t n, int k, float base) {
  // init_margin, train.rs:496-511
  std::vector<float> m(n * k, base);
  if (bm) {
    if (bm_len == n * k) std::memcpy(m.data(), bm, n * k * sizeof(float));
    else if (bm_len == n)
      for (size_t r = 0; r < n; ++r)
        for (int c = 0; c < k; ++c) m[r * k + c] = bm[r];
  }
  return m;
}

// RegTree::leaf_id_with over a dense row, regtree.rs:213-242
size_t leaf_id(const OTree& t, const float* row, float missing) {
  size_t nid = 0;
  for (;;) {
    const sb_node& nd = t.nodes[nid];
    if (nd.left == -1) return nid;
    float v = row[nd.split_feature];
    bool go_left;
    if (is_missing(v, missing)) go_left = nd.default_left != 0;
    else if (nd.is_categorical) {
      uint32_t c = f32_as_u32(v);
      go_left = false;
      for (uint32_t i = nd.cat_begin; i < nd.cat_end; ++i)
        if (t.cats[i] == c) { go_left = true; break; }
    } else go_left = v < nd.split_cond;
    nid = go_left ? (size_t)nd.left : (size_t)nd.right;
  }
}

void view_to_trees(const sb_model_view* v, std::vector<OTree>& trees) {
  trees.resize(v->n_trees);
  for (int t = 0; t < v->n_trees; ++t) {
    trees[t].nodes.assign(v->nodes + v->tree_node_offset[t], v->nodes + v->tree_node_offset[t + 1]);
    if (v->categories && v->tree_cat_offset)
      trees[t].cats.assign(v->categories + v->tree_cat_offset[t],
                           v->categories + v->tree_cat_offset[t + 1]);
  }
}

// ------------------------------------------------------------- TreeSHAP
struct PathEl {  // learner/shap.rs:33-42
  int64_t feature;
  double zero, one, pweight;
};
void extend_path(std::vector<PathEl>& path, double z, double o, int64_t f) {  // shap.rs:49-68
  size_t ud = path.size();
  path.push_back(PathEl{f, z, o, ud == 0 ? 1.0 : 0.0});
  double denom = (double)(ud + 1);
  for (size_t ii = ud; ii-- > 0;) {
    double pw = path[ii].pweight;
    path[ii + 1].pweight += o * pw * (double)(ii + 1) / denom;
    path[ii].pweight = z * pw * (double)(ud - ii) / denom;
  }
}
void unwind_path(std::vector<PathEl>& path, size_t pi) {  // shap.rs:72-94
  size_t ud = path.size() - 1;
  double o = path[pi].one, z = path[pi].zero;
  double next = path[ud].pweight;
  double denom = (double)(ud + 1);
  for (size_t ii = ud; ii-- > 0;) {
    if (o != 0.0) {
      double tmp = path[ii].pweight;
      path[ii].pweight = next * denom / ((double)(ii + 1) * o);
      next = tmp - path[ii].pweight * z * (double)(ud - ii) / denom;
    } else if (z != 0.0) {
      path[ii].pweight = path[ii].pweight * denom / (z * (double)(ud - ii));
    }
  }
  for (size_t ii = pi; ii < ud; ++ii) {
    path[ii].feature = path[ii + 1].feature;
    path[ii].zero = path[ii + 1].zero;
    path[ii].one = path[ii + 1].one;
  }
  path.pop_back();
}
double unwound_path_sum(const std::vector<PathEl>& path, size_t pi) {  // shap.rs:98-116
  size_t ud = path.size() - 1;
  double o = path[pi].one, z = path[pi].zero;
  double next = path[ud].pweight;
  double denom = (double)(ud + 1);
  double total = 0.0;
  for (size_t ii = ud; ii-- > 0;) {
    if (o != 0.0) {
      double tmp = next * denom / ((double)(ii + 1) * o);
      total += tmp;
      next = path[ii].pweight - tmp * z * (double)(ud - ii) / denom;
    } else if (z != 0.0) {
      total += (path[ii].pweight / z) / ((double)(ud - ii) / denom);
    }
  }
  return total;
}
void tree_shap_cond(const OTree& t, size_t nidx, std::vector<PathEl> path, double pz, double po,
                    int64_t pf, const float* row, float missing, double* phi, int cond, int64_t cf,
                    double cfrac) {
  // tree_shap_cond, shap.rs:165-283: cond 0 = ordinary TreeSHAP; +1 / -1 =
  // feature cf fixed present / absent (kept off the path, its weight carried
  // in cfrac)
  if (cfrac == 0.0) return;
  if (cond == 0 || cf != pf) extend_path(path, pz, po, pf);
  const sb_node& nd = t.nodes[nidx];
  size_t ud = path.size() - 1;
  if (nd.left == -1) {
    double leaf = (double)nd.leaf_value;
    for (size_t i = 1; i <= ud; ++i) {
      double w = unwound_path_sum(path, i);
      const PathEl& el = path[i];
      phi[el.feature] += w * (el.one - el.zero) * leaf * cfrac;
    }
    return;
  }
  float v = row[nd.split_feature];
  // The reference routes by `v < split_cond` here even at categorical nodes.
  bool go_left = is_missing(v, missing) ? nd.default_left != 0 : v < nd.split_cond;
  size_t hot = go_left ? nd.left : nd.right, cold = go_left ? nd.right : nd.left;
  double cover = (double)nd.sum_hess;
  double hz = 0.0, cz = 0.0;
  if (cover > 0.0) {
    hz = (double)t.nodes[hot].sum_hess / cover;
    cz = (double)t.nodes[cold].sum_hess / cover;
  }
  int64_t si = nd.split_feature;
  double iz = 1.0, io = 1.0;
  for (size_t i = 1; i <= ud; ++i) {
    if (path[i].feature == si) {
      iz = path[i].zero;
      io = path[i].one;
      unwind_path(path, i);
      break;
    }
  }
  double hot_cf = cfrac, cold_cf = cfrac;
  if (cond > 0 && si == cf) cold_cf = 0.0;
  else if (cond < 0 && si == cf) {
    hot_cf *= hz;
    cold_cf *= cz;
  }
  tree_shap_cond(t, hot, path, hz * iz, io, si, row, missing, phi, cond, cf, hot_cf);
  tree_shap_cond(t, cold, std::move(path), cz * iz, 0.0, si, row, missing, phi, cond, cf, cold_cf);
}
void tree_shap(const OTree& t, size_t nidx, std::vector<PathEl> path, double pz, double po,
               int64_t pf, const float* row, float missing, double* phi) {
  tree_shap_cond(t, nidx, std::move(path), pz, po, pf, row, missing, phi, 0, -1, 1.0);
}
double node_mean_value(const OTree& t, size_t id) {  // shap.rs:288-302
  const sb_node& nd = t.nodes[id];
  if (nd.left == -1) return (double)nd.leaf_value;
  double cover = (double)nd.sum_hess;
  if (cover <= 0.0) return 0.0;
  double lc = (double)t.nodes[nd.left].sum_hess, rc = (double)t.nodes[nd.right].sum_hess;
  return (lc * node_mean_value(t, nd.left) + rc * node_mean_value(t, nd.right)) / cover;
}

int scale_exp(float m, int bits) {
  if (!(m > 0.0f) || !std::isfinite(m)) return 0;
  int e = std::ilogb(m);
  int s = (bits - 1) - e;
  if (s > 100) s = 100;
  if (s < -100) s = -100;
  return s;
}

}  // namespace

// =================================================================== C ABI
extern "C" {

// HistCuts::from_dmatrix (quantile.rs:39-70) or, with `hessians` (one per
// row), HistCuts::from_dmatrix_weighted (quantile.rs:81-122), then
// GHistIndex::from_dmatrix.
orc_data* orc_data_create_weighted(const float* X, size_t n, size_t F, const uint8_t* ftypes, float missing,
                                   int max_bin, const float* hessians);

orc_data* orc_data_create(const float* X, size_t n, size_t F, const uint8_t* ftypes, float missing,
                          int max_bin) {
  return orc_data_create_weighted(X, n, F, ftypes, missing, max_bin, nullptr);
}

orc_data* orc_data_create_weighted(const float* X, size_t n, size_t F, const uint8_t* ftypes, float missing,
                                   int max_bin, const float* hessians) {
  if (!X || n == 0 || F == 0 || max_bin < 2) return nullptr;
  if (!std::isnan(missing))
    for (size_t i = 0; i < n * F; ++i)
      if (std::isnan(X[i])) return nullptr;
  orc_data* d = new orc_data;
  d->n = n;
  d->F = F;
  d->missing = missing;
  Cuts& c = d->cuts;
  c.F = F;
  c.off.push_back(0);
  c.is_cat.assign(F, 0);
  std::vector<float> col;
  std::vector<std::pair<float, float>> wcol;
  for (size_t f = 0; f < F; ++f) {  // from_dmatrix, quantile.rs:39-70 (to_csc order)
    col.clear();
    wcol.clear();
    for (size_t r = 0; r < n; ++r) {
      float v = X[r * F + f];
      if (is_missing(v, missing)) continue;
      col.push_back(v);
      if (hessians) wcol.emplace_back(v, hessians[r]);
    }
    std::stable_sort(col.begin(), col.end(), [](float a, float b) { return a < b; });
    if (ftypes && ftypes[f] == SB_FEAT_CATEGORICAL) {
      c.is_cat[f] = 1;
      build_categorical_cuts(col, c.vals);
    } else if (hessians) {  // from_dmatrix_weighted, quantile.rs:103-114
      std::stable_sort(wcol.begin(), wcol.end(),
                       [](const std::pair<float, float>& a, const std::pair<float, float>& b) {
                         return a.first < b.first;
                       });
      build_feature_cuts_weighted(wcol, (size_t)max_bin, c.vals);
    } else {
      build_feature_cuts(col, (size_t)max_bin, c.vals);
    }
    c.off.push_back((uint32_t)c.vals.size());
  }
  d->row_ptr.reserve(n + 1);
  d->row_ptr.push_back(0);
  d->bins.reserve(n * F);
  for (size_t r = 0; r < n; ++r) {  // GHistIndex::from_dmatrix, ghist.rs:48-82
    size_t cnt = 0;
    for (size_t f = 0; f < F; ++f) {
      float v = X[r * F + f];
      if (is_missing(v, missing)) continue;
      d->bins.push_back(c.bin_of(f, v));
      cnt++;
    }
    if (cnt != F) d->dense = false;
    d->row_ptr.push_back(d->bins.size());
  }
  return d;
}

void orc_data_destroy(orc_data* d) { delete d; }
size_t orc_data_total_bins(const orc_data* d) { return d->cuts.total(); }
int orc_data_is_dense(const orc_data* d) { return d->dense ? 1 : 0; }

void orc_data_cuts(const orc_data* d, uint32_t* off, float* vals, uint8_t* is_cat) {
  if (off) std::memcpy(off, d->cuts.off.data(), (d->F + 1) * sizeof(uint32_t));
  if (vals) std::memcpy(vals, d->cuts.vals.data(), d->cuts.total() * sizeof(float));
  if (is_cat) std::memcpy(is_cat, d->cuts.is_cat.data(), d->F);
}

void orc_data_dense_bins(const orc_data* d, uint32_t* out) {
  for (size_t r = 0; r < d->n; ++r) {
    for (size_t f = 0; f < d->F; ++f) out[r * d->F + f] = 0xFFFFFFFFu;
    for (size_t i = d->row_ptr[r]; i < d->row_ptr[r + 1]; ++i) {
      uint32_t b = d->bins[i];
      size_t f = std::upper_bound(d->cuts.off.begin(), d->cuts.off.end(), b) - d->cuts.off.begin() - 1;
      out[r * d->F + f] = b;
    }
  }
}

uint32_t orc_bin_of(const orc_data* d, size_t f, float v) { return d->cuts.bin_of(f, v); }

void orc_hist_build(const orc_data* d, const uint32_t* rows, size_t m, const sb_gradpair* gpair,
                    sb_gradstats* out, int threads) {
  std::vector<GS> h(d->cuts.total());
  hist_build(*d, rows, m, gpair, h.data(), threads);
  for (size_t i = 0; i < h.size(); ++i) out[i] = sb_gradstats{h[i].g, h[i].h};
}

orc_model* orc_tree_build(const orc_data* d, const sb_train_params* p, const sb_gradpair* gpair,
                          const uint32_t* rows, size_t m, uint64_t round, uint32_t k, int threads) {
  Sampler s = make_sampler(d->F, *p, round, k);
  Builder b(*p, d->F);
  orc_model* mdl = new orc_model;
  mdl->trees.push_back(b.build(*d, gpair, rows, m, s, threads));
  mdl->weights.push_back(1.0f);
  mdl->n_features = (int)d->F;
  mdl->objective = p->objective;
  mdl->num_class = p->num_class;
  return mdl;
}

int orc_sample_features(size_t F, const sb_train_params* p, uint64_t round, uint32_t k, uint64_t nid,
                        uint32_t* out) {
  Sampler s = make_sampler(F, *p, round, k);
  std::vector<uint32_t> v = s.sample(nid);
  std::memcpy(out, v.data(), v.size() * 4);
  return (int)v.size();
}

size_t orc_sample_rows(size_t n, const sb_train_params* p, uint64_t round, uint32_t* out) {
  size_t m = 0;  // sample_rows, train.rs:465-476
  if (p->subsample >= 1.0) {
    for (size_t r = 0; r < n; ++r) out[m++] = (uint32_t)r;
    return m;
  }
  uint64_t rk = sb_round_key(p->seed, round);
  for (size_t r = 0; r < n; ++r)
    if (sb_u01(sb_row_draw(rk, r)) < p->subsample) out[m++] = (uint32_t)r;
  if (m == 0) out[m++] = (uint32_t)sb_row_fallback(rk, n);
  return m;
}

int orc_validate(const sb_train_params* p) {  // params.rs:197-261
  auto unit = [](double v) { return v >= 0.0 && v <= 1.0; };
  auto pos = [](double v) { return !std::isnan(v) && v > 0.0; };
  auto nonneg = [](double v) { return !std::isnan(v) && v >= 0.0; };
  if (!pos(p->eta) || !nonneg(p->gamma) || !nonneg(p->min_child_weight) ||
      !nonneg(p->max_delta_step) || !nonneg(p->lambda) || !nonneg(p->alpha) ||
      !pos(p->scale_pos_weight))
    return 1;
  if (!unit(p->subsample) || p->subsample == 0.0) return 1;
  if (!unit(p->colsample_bytree) || !unit(p->colsample_bylevel) || !unit(p->colsample_bynode)) return 1;
  if (p->max_bin < 2) return 1;
  if (p->grow_policy == SB_GROW_LOSSGUIDE && p->max_leaves == 0 && p->max_depth == 0) return 1;
  if ((p->objective == SB_OBJ_SOFTMAX || p->objective == SB_OBJ_SOFTPROB) && p->num_class < 2) return 1;
  return 0;
}

void orc_gradient(int objective, int num_class, double spw, const float* preds, const float* labels,
                  const float* weights, size_t n, sb_gradpair* out) {
  switch (objective) {
    case SB_OBJ_SQUARED_ERROR:  // regression.rs:18-40
      for (size_t i = 0; i < n; ++i) {
        float g = preds[i] - labels[i];
        out[i] = weights ? sb_gradpair{g * weights[i], weights[i]} : sb_gradpair{g, 1.0f};
      }
      break;
    case SB_OBJ_PSEUDOHUBER:  // regression.rs:51-85
      for (size_t i = 0; i < n; ++i) {
        float w = weights ? weights[i] : 1.0f;
        float dd = preds[i] - labels[i];
        float s = 1.0f + dd * dd;
        float sq = std::sqrt(s);
        out[i] = sb_gradpair{(dd / sq) * w, (1.0f / (s * sq)) * w};
      }
      break;
    case SB_OBJ_LOGISTIC: {  // classification.rs:50-71
      float sp = (float)spw;
      for (size_t i = 0; i < n; ++i) {
        float y = labels[i];
        float p = sigmoid(preds[i]);
        float w = weights ? weights[i] : 1.0f;
        if (y == 1.0f) w *= sp;
        float grad = (p - y) * w;
        float hess = std::max(p * (1.0f - p), 1e-16f) * w;
        out[i] = sb_gradpair{grad, hess};
      }
      break;
    }
    default: {  // softmax, multiclass.rs:64-91
      int k = num_class;
      std::vector<float> probs(k);
      for (size_t i = 0; i < n; ++i) {
        std::memcpy(probs.data(), preds + i * k, k * sizeof(float));
        softmax_inplace(probs.data(), k);
        float w = weights ? weights[i] : 1.0f;
        // `labels[i] as usize` saturates: negative and NaN labels are class 0
        const uint32_t label = f32_as_u32(labels[i]);
        for (int c = 0; c < k; ++c) {
          float p = probs[c];
          float target = ((uint32_t)c == label) ? 1.0f : 0.0f;
          float grad = (p - target) * w;
          float hess = std::max(2.0f * p * (1.0f - p) * w, 1e-16f);
          out[i * k + c] = sb_gradpair{grad, hess};
        }
      }
    }
  }
}

void orc_pred_transform(int objective, int num_class, float* preds, size_t n) {
  if (objective == SB_OBJ_LOGISTIC)
    for (size_t i = 0; i < n; ++i) preds[i] = sigmoid(preds[i]);
  else if (objective == SB_OBJ_SOFTMAX || objective == SB_OBJ_SOFTPROB)
    for (size_t i = 0; i < n; ++i) softmax_inplace(preds + i * num_class, num_class);
}

double orc_metric(int kind, const float* preds, const float* labels, const float* weights, size_t n,
                  int num_class) {  // metric/mod.rs:40-64, :91-116, :201-228
  double acc = 0.0, wsum = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double w = weights ? (double)weights[i] : 1.0;
    if (kind == 0) {
      double dd = (double)preds[i] - (double)labels[i];
      acc += w * dd * dd;
    } else if (kind == 1) {
      double p = clamp_f64((double)preds[i], 1e-15, 1.0 - 1e-15);
      double y = (double)labels[i];
      acc += w * -(y * std::log(p) + (1.0 - y) * std::log(1.0 - p));
    } else {
      double p = clamp_f64((double)preds[i * num_class + (size_t)labels[i]], 1e-15, 1.0);
      acc += -w * std::log(p);
    }
    wsum += w;
  }
  if (wsum <= 0.0) return 0.0;
  return kind == 0 ? std::sqrt(acc / wsum) : acc / wsum;
}

float orc_base_margin(const sb_train_params* p, const float* labels, const float* weights, size_t n) {
  // train.rs:203-210 with base_margin / prob_to_margin of each objective
  if (p->objective == SB_OBJ_SOFTMAX || p->objective == SB_OBJ_SOFTPROB) return 0.0f;
  if (p->has_base_score) {
    float bs = (float)p->base_score;
    if (p->objective == SB_OBJ_LOGISTIC) {  // classification.rs:~99-102
      float pp = bs < 1e-6f ? 1e-6f : (bs > 1.0f - 1e-6f ? 1.0f - 1e-6f : bs);
      return std::log(pp / (1.0f - pp));
    }
    return bs;
  }
  double mean = weighted_label_mean(labels, weights, n);
  if (p->objective == SB_OBJ_LOGISTIC) {  // classification.rs:~93-98
    double pp = clamp_f64(mean, 1e-6, 1.0 - 1e-6);
    return (float)std::log(pp / (1.0 - pp));
  }
  return (float)mean;
}

void orc_quantize(const sb_gradpair* in, size_t n, int bits, sb_gradpair* out, int* shift_g,
                  int* shift_h) {
  float mg = 0.0f, mh = 0.0f;
  for (size_t i = 0; i < n; ++i) {
    mg = std::max(mg, std::fabs(in[i].grad));
    mh = std::max(mh, std::fabs(in[i].hess));
  }
  int sg = scale_exp(mg, bits), sh = scale_exp(mh, bits);
  for (size_t i = 0; i < n; ++i) {
    float qg = std::nearbyint(std::ldexp(in[i].grad, sg));
    float qh = std::nearbyint(std::ldexp(in[i].hess, sh));
    out[i].grad = std::ldexp(qg, -sg);
    out[i].hess = std::ldexp(qh, -sh);
  }
  if (shift_g) *shift_g = sg;
  if (shift_h) *shift_h = sh;
}

orc_model* orc_train(const orc_data* d, const float* X, const sb_train_params* p, const float* labels,
                     const float* weights, const float* base_margin, int rounds, int threads,
                     float* margins_out, double* metric_out) {
  // train_impl, learner/train.rs:183-383 (gbtree, hist, no eval sets)
  if (orc_validate(p) != 0 || !labels) return nullptr;
  size_t n = d->n, F = d->F;
  int K = n_outputs(p->objective, p->num_class);
  float base = orc_base_margin(p, labels, weights, n);
  orc_model* mdl = new orc_model;
  mdl->base_score = base;
  mdl->num_class = p->num_class;
  mdl->n_features = (int)F;
  mdl->objective = p->objective;
  std::vector<float> margin = init_margin(base_margin, base_margin ? n : 0, n, K, base);
  std::vector<sb_gradpair> gpair(n * K), gk(n);
  std::vector<uint32_t> rows;
  Builder builder(*p, F);
  int bits = p->quantize_bits > 0 ? p->quantize_bits : 16;
  std::vector<float> preds;
  for (int round = 0; round < rounds; ++round) {
    orc_gradient(p->objective, p->num_class, p->scale_pos_weight, margin.data(), labels, weights, n,
                 gpair.data());
    rows.clear();  // sample_rows, train.rs:465-476
    if (p->subsample >= 1.0) {
      for (size_t r = 0; r < n; ++r) rows.push_back((uint32_t)r);
    } else {
      uint64_t rk = sb_round_key(p->seed, (uint64_t)round);
      for (size_t r = 0; r < n; ++r)
        if (sb_u01(sb_row_draw(rk, r)) < p->subsample) rows.push_back((uint32_t)r);
      if (rows.empty()) rows.push_back((uint32_t)sb_row_fallback(rk, n));
    }
    for (int k = 0; k < K; ++k) {
      for (size_t r = 0; r < n; ++r) gk[r] = gpair[r * K + k];
      const orc_data* dk = d;
      std::unique_ptr<orc_data> dw;
      if (p->tree_method == SB_TREE_APPROX) {  // Prepared::Approx, train.rs:46-53
        std::vector<float> hess(n);
        for (size_t r = 0; r < n; ++r) hess[r] = gk[r].hess;
        dw.reset(orc_data_create_weighted(X, n, F, d->cuts.is_cat.data(), d->missing, p->max_bin, hess.data()));
        if (!dw) {
          delete mdl;
          return nullptr;
        }
        dk = dw.get();
      }
      if (p->hist_precision == SB_HIST_FIXED) orc_quantize(gk.data(), n, bits, gk.data(), nullptr, nullptr);
      Sampler s = make_sampler(F, *p, (uint64_t)round, (uint64_t)k);
      OTree t = builder.build(*dk, gk.data(), rows.data(), rows.size(), s, threads);
      float eta = (float)p->eta;
      for (auto& nd : t.nodes)  // scale_leaves, regtree.rs:201-207
        if (nd.left == -1) nd.leaf_value *= eta;
      for (size_t r = 0; r < n; ++r)  // train.rs:326-328
        margin[r * K + k] += t.nodes[leaf_id(t, X + r * F, d->missing)].leaf_value;
      mdl->trees.push_back(std::move(t));
      mdl->weights.push_back(1.0f);
    }
    if (metric_out) {
      preds = margin;
      orc_pred_transform(p->objective, p->num_class, preds.data(), n);
      int kind = p->objective == SB_OBJ_LOGISTIC ? 1 : (K > 1 ? 2 : 0);
      metric_out[round] = orc_metric(kind, preds.data(), labels, weights, n, p->num_class);
    }
  }
  if (margins_out) std::memcpy(margins_out, margin.data(), n * K * sizeof(float));
  return mdl;
}

// dart_round (learner/train.rs:384-456) with the dropout draws taken from the
// SplitMix64 stream keyed by sb_dart_key (the reference's rand 0.8 StdRng is
// not available); row and column sampling use the hist path's keys. Tree
// weights come back in weights_out (one per tree, n_trees = rounds * K).
orc_model* orc_train_dart(const orc_data* d, const float* X, const sb_train_params* p, double rate_drop,
                          double skip_drop, const float* labels, const float* weights, const float* base_margin,
                          int rounds, int threads, float* margins_out) {
  if (orc_validate(p) != 0 || !labels) return nullptr;
  const size_t n = d->n, F = d->F;
  const int K = n_outputs(p->objective, p->num_class);
  const float base = orc_base_margin(p, labels, weights, n);
  orc_model* mdl = new orc_model;
  mdl->base_score = base;
  mdl->num_class = p->num_class;
  mdl->n_features = (int)F;
  mdl->objective = p->objective;
  const std::vector<float> init = init_margin(base_margin, base_margin ? n : 0, n, K, base);
  std::vector<sb_gradpair> gpair(n * K), gk(n);
  std::vector<uint32_t> rows;
  std::vector<float> margin(n * K);
  Builder builder(*p, F);
  const int bits = p->quantize_bits > 0 ? p->quantize_bits : 16;
  for (int round = 0; round < rounds; ++round) {
    // 1. the dropout set (train.rs:397-425)
    const size_t existing = mdl->trees.size();
    std::vector<size_t> drop;
    sb_splitmix g{sb_dart_key(p->seed, (uint64_t)round)};
    const bool skip = sb_u01(sb_splitmix_next(&g)) < skip_drop;
    if (!skip && existing > 0) {
      for (size_t i = 0; i < existing; ++i)
        if (sb_u01(sb_splitmix_next(&g)) < rate_drop) drop.push_back(i);
      if (drop.empty()) drop.push_back((size_t)sb_splitmix_bounded(&g, existing));
    }
    // 2. the ensemble's margins without the dropout set (model.rs:130-145)
    std::vector<uint8_t> dropped(existing, 0);
    for (size_t i : drop) dropped[i] = 1;
    margin = init;
    for (size_t t = 0; t < existing; ++t) {
      if (dropped[t]) continue;
      const float w = mdl->weights[t];
      const size_t cls = t % K;
      for (size_t r = 0; r < n; ++r)
        margin[r * K + cls] += w * mdl->trees[t].nodes[leaf_id(mdl->trees[t], X + r * F, d->missing)].leaf_value;
    }
    orc_gradient(p->objective, p->num_class, p->scale_pos_weight, margin.data(), labels, weights, n,
                 gpair.data());
    // 3. one new tree per output, weight 1 / (k + 1)
    rows.clear();
    if (p->subsample >= 1.0) {
      for (size_t r = 0; r < n; ++r) rows.push_back((uint32_t)r);
    } else {
      const uint64_t rk = sb_round_key(p->seed, (uint64_t)round);
      for (size_t r = 0; r < n; ++r)
        if (sb_u01(sb_row_draw(rk, r)) < p->subsample) rows.push_back((uint32_t)r);
      if (rows.empty()) rows.push_back((uint32_t)sb_row_fallback(rk, n));
    }
    const float kd = (float)drop.size();
    const float new_weight = 1.0f / (kd + 1.0f);
    for (int k = 0; k < K; ++k) {
      for (size_t r = 0; r < n; ++r) gk[r] = gpair[r * K + k];
      if (p->hist_precision == SB_HIST_FIXED) orc_quantize(gk.data(), n, bits, gk.data(), nullptr, nullptr);
      Sampler smp = make_sampler(F, *p, (uint64_t)round, (uint64_t)k);
      OTree t = builder.build(*d, gk.data(), rows.data(), rows.size(), smp, threads);
      const float eta = (float)p->eta;
      for (auto& nd : t.nodes)  // scale_leaves, regtree.rs:201-207
        if (nd.left == -1) nd.leaf_value *= eta;
      mdl->trees.push_back(std::move(t));
      mdl->weights.push_back(new_weight);
    }
    // 4. the dropped trees scaled by k / (k + 1)
    const float factor = kd / (kd + 1.0f);
    for (size_t i : drop) mdl->weights[i] *= factor;
  }
  if (margins_out) {  // the final model's margins with its tree weights
    margin = init;
    for (size_t t = 0; t < mdl->trees.size(); ++t) {
      const float w = mdl->weights[t];
      const size_t cls = t % K;
      for (size_t r = 0; r < n; ++r)
        margin[r * K + cls] += w * mdl->trees[t].nodes[leaf_id(mdl->trees[t], X + r * F, d->missing)].leaf_value;
    }
    std::memcpy(margins_out, margin.data(), n * K * sizeof(float));
  }
  return mdl;
}

void orc_model_destroy(orc_model* m) { delete m; }

void orc_model_sizes(const orc_model* m, int32_t* n_trees, int64_t* n_nodes, int64_t* n_cats) {
  int64_t nn = 0, nc = 0;
  for (auto& t : m->trees) {
    nn += (int64_t)t.nodes.size();
    nc += (int64_t)t.cats.size();
  }
  if (n_trees) *n_trees = (int32_t)m->trees.size();
  if (n_nodes) *n_nodes = nn;
  if (n_cats) *n_cats = nc;
}

void orc_model_export(const orc_model* m, int64_t* node_off, sb_node* nodes, int64_t* cat_off,
                      uint32_t* cats, float* weights, float* base_score) {
  int64_t no = 0, co = 0;
  for (size_t t = 0; t < m->trees.size(); ++t) {
    const OTree& tr = m->trees[t];
    if (node_off) node_off[t] = no;
    if (cat_off) cat_off[t] = co;
    if (nodes) std::memcpy(nodes + no, tr.nodes.data(), tr.nodes.size() * sizeof(sb_node));
    if (cats && !tr.cats.empty()) std::memcpy(cats + co, tr.cats.data(), tr.cats.size() * 4);
    if (weights) weights[t] = m->weights[t];
    no += (int64_t)tr.nodes.size();
    co += (int64_t)tr.cats.size();
  }
  if (node_off) node_off[m->trees.size()] = no;
  if (cat_off) cat_off[m->trees.size()] = co;
  if (base_score) *base_score = m->base_score;
}

void orc_model_node_gaps(const orc_model* m, double* out) {
  size_t o = 0;
  for (auto& t : m->trees)
    for (double g : t.gaps) out[o++] = g;
}

int orc_predict_margin(const sb_model_view* v, const float* X, size_t n, size_t F, float missing,
                       const float* base_margin, size_t ntree_limit, float* out) {
  // predict_margin_limited, learner/model.rs:231-285
  std::vector<OTree> trees;
  view_to_trees(v, trees);
  int K = v->num_class >= 2 ? v->num_class : 1;
  size_t limit = ntree_limit == 0 ? trees.size() : std::min(ntree_limit, trees.size());
  for (size_t i = 0; i < n * K; ++i) out[i] = v->base_score;
  if (base_margin) std::memcpy(out, base_margin, n * K * sizeof(float));
  for (size_t t = 0; t < limit; ++t) {
    float w = v->tree_weights ? v->tree_weights[t] : 1.0f;
    size_t cls = t % K;
    for (size_t r = 0; r < n; ++r)
      out[r * K + cls] += w * trees[t].nodes[leaf_id(trees[t], X + r * F, missing)].leaf_value;
  }
  return 0;
}

int orc_predict_contribs(const sb_model_view* v, const float* X, size_t n, size_t F, float missing,
                         float* out) {
  // predict_contribs, learner/shap.rs:321-367
  std::vector<OTree> trees;
  view_to_trees(v, trees);
  int K = v->num_class >= 2 ? v->num_class : 1;
  size_t width = F + 1;
  std::vector<double> means(trees.size());
  for (size_t t = 0; t < trees.size(); ++t) means[t] = node_mean_value(trees[t], 0);
  double base = (double)v->base_score;
  std::vector<double> acc(K * width);
  for (size_t r = 0; r < n; ++r) {
    std::fill(acc.begin(), acc.end(), 0.0);
    for (int c = 0; c < K; ++c) acc[c * width + F] += base;
    for (size_t t = 0; t < trees.size(); ++t) {
      size_t off = (t % K) * width;
      tree_shap(trees[t], 0, {}, 1.0, 1.0, -1, X + r * F, missing, acc.data() + off);
      acc[off + F] += means[t];
    }
    for (size_t i = 0; i < K * width; ++i) out[r * K * width + i] = (float)acc[i];
  }
  return 0;
}

int orc_predict_leaf(const sb_model_view* v, const float* X, size_t n, size_t F, float missing,
                     uint32_t* out) {
  // predict_leaf, learner/model.rs:330-341: [n][T] leaf node ids
  std::vector<OTree> trees;
  view_to_trees(v, trees);
  const size_t T = trees.size();
  for (size_t r = 0; r < n; ++r)
    for (size_t t = 0; t < T; ++t) out[r * T + t] = (uint32_t)leaf_id(trees[t], X + r * F, missing);
  return 0;
}

int orc_predict_interactions(const sb_model_view* v, const float* X, size_t n, size_t F, float missing,
                             float* out) {
  // predict_interactions, learner/shap.rs:395-509: [n][K][F+1][F+1]
  std::vector<OTree> trees;
  view_to_trees(v, trees);
  const int K = v->num_class >= 2 ? v->num_class : 1;
  const size_t width = F + 1, mw = width * width;
  std::vector<double> means(trees.size());
  for (size_t t = 0; t < trees.size(); ++t) means[t] = node_mean_value(trees[t], 0);
  std::vector<double> diag(K * width), on(K * width), off(K * width), mat(K * mw);
  for (size_t r = 0; r < n; ++r) {
    const float* row = X + r * F;
    std::fill(diag.begin(), diag.end(), 0.0);
    std::fill(mat.begin(), mat.end(), 0.0);
    for (size_t t = 0; t < trees.size(); ++t) {
      const size_t base = (t % K) * width;
      tree_shap_cond(trees[t], 0, {}, 1.0, 1.0, -1, row, missing, diag.data() + base, 0, -1, 1.0);
      diag[base + F] += means[t];
    }
    for (int c = 0; c < K; ++c)
      for (size_t j = 0; j < width; ++j) mat[c * mw + j * width + j] = diag[c * width + j];
    for (size_t j = 0; j < F; ++j) {
      std::fill(on.begin(), on.end(), 0.0);
      std::fill(off.begin(), off.end(), 0.0);
      for (size_t t = 0; t < trees.size(); ++t) {
        const size_t base = (t % K) * width;
        tree_shap_cond(trees[t], 0, {}, 1.0, 1.0, -1, row, missing, on.data() + base, 1, (int64_t)j, 1.0);
        tree_shap_cond(trees[t], 0, {}, 1.0, 1.0, -1, row, missing, off.data() + base, -1, (int64_t)j, 1.0);
      }
      for (int c = 0; c < K; ++c)
        for (size_t kk = 0; kk < width; ++kk) {
          const double val = 0.5 * (on[c * width + kk] - off[c * width + kk]);
          mat[c * mw + j * width + kk] += val;
          mat[c * mw + j * width + j] -= val;
        }
    }
    for (size_t i = 0; i < K * mw; ++i) out[r * K * mw + i] = (float)mat[i];
  }
  return 0;
}

}  // extern "C"
