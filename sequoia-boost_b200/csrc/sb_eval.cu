// sb_eval.cu — eval sets on the device: the incremental margin caches and
// the per-round metrics of train_impl (learner/train.rs:243-246, 319-347),
// with the pointwise metrics of metric/mod.rs:37-262.
//
// An eval set's rows, labels, weights and margins are uploaded once. After
// each boosting round, sb_booster_eval adds the round's K trees into the
// cache (one thread per (row, class), the trees in order, f32 adds: the same
// sums as predict_margin, train.rs:330-335), transforms a copy of the
// margins with the objective's pred_transform, and reduces the metrics in
// f64, per block and then over blocks in a fixed order, so a value does not
// depend on scheduling. Only the metric values cross to the host, which is
// what early stopping (train.rs:350-379) needs.
#include <algorithm>

#include "sb_internal.cuh"

namespace sb {
namespace {

constexpr int EVAL_THREADS = 256;
constexpr int EVAL_MAX_BLOCKS = 1024;

__device__ __forceinline__ bool eval_missing(float v, float missing) {
  return isnan(missing) ? isnan(v) : (v == missing);
}

// RegTree::predict_row over one device tree (regtree.rs:213-242).
__device__ __forceinline__ float tree_leaf(const sb_node* nd, const uint32_t* cats, const float* row,
                                           float missing) {
  int nid = 0;
  for (;;) {
    const sb_node& x = nd[nid];
    if (x.left < 0) return x.leaf_value;
    const float v = row[x.split_feature];
    bool go_left;
    if (eval_missing(v, missing)) {
      go_left = x.default_left != 0;
    } else if (x.is_categorical) {
      const uint32_t c = f32_as_u32(v);
      go_left = false;
      for (uint32_t i = x.cat_begin; i < x.cat_end; ++i)
        if (cats[i] == c) {
          go_left = true;
          break;
        }
    } else {
      go_left = v < x.split_cond;
    }
    nid = go_left ? x.left : x.right;
  }
}

__global__ void k_eval_add(BoosterTrees T, const float* __restrict__ X, size_t n, float missing, int r0, int r1,
                           float* __restrict__ margin) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t K = (size_t)T.K;
  if (i >= n * K) return;
  const size_t r = i / K;
  const int k = (int)(i - r * K);
  const float* row = X + r * T.n_features;
  float m = margin[i];
  for (int rd = r0; rd < r1; ++rd) {
    const size_t t = (size_t)rd * K + k;
    m = __fadd_rn(m, tree_leaf(T.nodes + t * T.maxn, T.cats ? T.cats + t * T.cat_cap : nullptr, row, missing));
  }
  margin[i] = m;
}

// Per block: for each requested metric, (sum, weight sum) over its rows.
__global__ void __launch_bounds__(EVAL_THREADS)
    k_eval_metrics(const float* __restrict__ margin, const float* __restrict__ labels,
                   const float* __restrict__ weights, size_t n, int K, int objective, const int* __restrict__ metrics,
                   int nm, double* __restrict__ partial) {
  __shared__ double s_sum[SB_EVAL_MAX_METRICS][EVAL_THREADS / 32], s_w[EVAL_THREADS / 32];
  double acc[SB_EVAL_MAX_METRICS];
  for (int j = 0; j < SB_EVAL_MAX_METRICS; ++j) acc[j] = 0.0;
  double wsum = 0.0;
  float row[SB_EVAL_MAX_CLASSES];
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    for (int c = 0; c < K; ++c) row[c] = margin[r * K + c];
    pred_transform_row(row, K, objective);
    const double w = weights ? (double)weights[r] : 1.0;
    const float y = labels[r];
    wsum += w;
    for (int j = 0; j < nm; ++j) {
      double v = 0.0;
      switch (metrics[j]) {
        case SB_METRIC_RMSE: {
          const double d = (double)row[0] - (double)y;
          v = w * d * d;
          break;
        }
        case SB_METRIC_MAE:
          v = w * fabs((double)row[0] - (double)y);
          break;
        case SB_METRIC_LOGLOSS: {
          const double p = fmin(fmax((double)row[0], 1e-15), 1.0 - 1e-15);
          const double yy = (double)y;
          v = w * -(yy * log(p) + (1.0 - yy) * log(1.0 - p));
          break;
        }
        case SB_METRIC_ERROR:
          v = ((row[0] > 0.5f) != (y > 0.5f)) ? w : 0.0;
          break;
        case SB_METRIC_MLOGLOSS: {
          const int lab = (int)y;
          const double p = fmin(fmax((double)row[lab], 1e-15), 1.0);
          v = -w * log(p);
          break;
        }
        case SB_METRIC_MERROR: {
          int best = 0;
          for (int c = 1; c < K; ++c)
            if (row[c] > row[best]) best = c;
          v = best != (int)y ? w : 0.0;
          break;
        }
        default:
          break;
      }
      acc[j] += v;
    }
  }
  // block reduction in a fixed order: warp shuffles, then warps in order
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    wsum += __shfl_down_sync(0xFFFFFFFFu, wsum, o);
    for (int j = 0; j < SB_EVAL_MAX_METRICS; ++j) acc[j] += __shfl_down_sync(0xFFFFFFFFu, acc[j], o);
  }
  if (lane == 0) {
    s_w[warp] = wsum;
    for (int j = 0; j < SB_EVAL_MAX_METRICS; ++j) s_sum[j][warp] = acc[j];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tw = 0.0;
    for (int i = 0; i < EVAL_THREADS / 32; ++i) tw += s_w[i];
    partial[(size_t)blockIdx.x * (SB_EVAL_MAX_METRICS + 1)] = tw;
    for (int j = 0; j < nm; ++j) {
      double t = 0.0;
      for (int i = 0; i < EVAL_THREADS / 32; ++i) t += s_sum[j][i];
      partial[(size_t)blockIdx.x * (SB_EVAL_MAX_METRICS + 1) + 1 + j] = t;
    }
  }
}

// Sums the blocks in order and finishes each metric (rmse: the root of the
// weighted mean; the others: the weighted mean; 0 when the weights sum to 0).
__global__ void k_eval_finish(const double* __restrict__ partial, int blocks, const int* __restrict__ metrics,
                              int nm, double* __restrict__ out) {
  const int j = threadIdx.x;
  if (j >= nm) return;
  double w = 0.0, s = 0.0;
  for (int b = 0; b < blocks; ++b) {
    w += partial[(size_t)b * (SB_EVAL_MAX_METRICS + 1)];
    s += partial[(size_t)b * (SB_EVAL_MAX_METRICS + 1) + 1 + j];
  }
  double v = w > 0.0 ? s / w : 0.0;
  if (metrics[j] == SB_METRIC_RMSE) v = w > 0.0 ? sqrt(v) : 0.0;
  out[j] = v;
}

}  // namespace
}  // namespace sb

extern "C" {

int sb_booster_eval_add(sb_booster* b, const float* X, size_t n_rows, size_t n_cols, float missing,
                        const float* labels, const float* weights, const float* base_margin, int* eval_id) {
  using namespace sb;
  SB_REQUIRE(b && X && labels && eval_id, SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_rows > 0, SB_ERR_INVALID_ARG, "empty eval set");
  BoosterTrees T;
  SB_TRY(booster_trees(b, &T));
  SB_REQUIRE(n_cols == T.n_features, SB_ERR_DIMENSION, "dimension mismatch: expected %zu features, got %zu",
             T.n_features, n_cols);
  SB_REQUIRE(T.K <= SB_EVAL_MAX_CLASSES, SB_ERR_UNSUPPORTED, "eval sets support up to %d classes",
             SB_EVAL_MAX_CLASSES);
  if (T.K > 1)
    for (size_t i = 0; i < n_rows; ++i)
      SB_REQUIRE(labels[i] >= 0.0f && labels[i] < (float)T.K && labels[i] == (float)(int)labels[i],
                 SB_ERR_INVALID_ARG, "eval label %zu (%g) is not a class index below %d", i, labels[i], T.K);
  sb_ctx* ctx = T.ctx;
  SB_CUDA(cudaSetDevice(ctx->device));
  std::unique_ptr<EvalSet> e(new EvalSet);
  e->n = n_rows;
  e->missing = missing;
  const size_t K = (size_t)T.K;
  SB_TRY(e->X.alloc(ctx, n_rows * n_cols));
  SB_TRY(e->labels.alloc(ctx, n_rows));
  SB_TRY(e->margin.alloc(ctx, n_rows * K));
  SB_CUDA(cudaMemcpyAsync(e->X.p, X, e->X.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  SB_CUDA(cudaMemcpyAsync(e->labels.p, labels, e->labels.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  if (weights) {
    SB_TRY(e->weights.alloc(ctx, n_rows));
    SB_CUDA(cudaMemcpyAsync(e->weights.p, weights, e->weights.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  }
  // init_margin (train.rs:240-241): the dataset's base_margin ([n][K]), else
  // the booster's base score in every slot
  std::vector<float> m0(n_rows * K, T.base_score);
  if (base_margin) std::copy(base_margin, base_margin + n_rows * K, m0.begin());
  SB_CUDA(cudaMemcpyAsync(e->margin.p, m0.data(), m0.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  auto& ev = booster_evals(b);
  *eval_id = (int)ev.size();
  ev.push_back(std::move(e));
  return SB_OK;
}

int sb_booster_eval(sb_booster* b, int n_metrics, const int* metrics, double* out) {
  using namespace sb;
  SB_REQUIRE(b && (metrics || n_metrics == 0) && (out || n_metrics == 0), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_metrics >= 0 && n_metrics <= SB_EVAL_MAX_METRICS, SB_ERR_INVALID_ARG,
             "n_metrics must be in [0, %d]", SB_EVAL_MAX_METRICS);
  BoosterTrees T;
  SB_TRY(booster_trees(b, &T));
  for (int j = 0; j < n_metrics; ++j) {
    const int mtr = metrics[j];
    SB_REQUIRE(mtr >= SB_METRIC_RMSE && mtr <= SB_METRIC_MERROR, SB_ERR_UNSUPPORTED, "unknown metric %d", mtr);
    const bool multi = mtr == SB_METRIC_MLOGLOSS || mtr == SB_METRIC_MERROR;
    SB_REQUIRE(multi == (T.K > 1), SB_ERR_INVALID_ARG, "metric %d does not apply to a model with %d outputs", mtr,
               T.K);
  }
  sb_ctx* ctx = T.ctx;
  SB_CUDA(cudaSetDevice(ctx->device));
  auto& ev = booster_evals(b);
  DBuf<int> d_metrics;
  DBuf<double> d_partial, d_out;
  if (n_metrics) {
    SB_TRY(d_metrics.alloc(ctx, n_metrics));
    SB_TRY(d_out.alloc(ctx, std::max<size_t>(ev.size(), 1) * n_metrics));
    SB_TRY(d_partial.alloc(ctx, (size_t)EVAL_MAX_BLOCKS * (SB_EVAL_MAX_METRICS + 1)));
    SB_CUDA(cudaMemcpyAsync(d_metrics.p, metrics, n_metrics * 4, cudaMemcpyHostToDevice, ctx->stream));
  }
  for (size_t i = 0; i < ev.size(); ++i) {
    EvalSet& e = *ev[i];
    const size_t nk = e.n * (size_t)T.K;
    if (e.rounds_in_margin < T.rounds_done) {
      SB_LAUNCH(ctx, k_eval_add, (unsigned)((nk + 255) / 256), 256, 0, T, e.X.p, e.n, e.missing,
                e.rounds_in_margin, T.rounds_done, e.margin.p);
      e.rounds_in_margin = T.rounds_done;
    }
    if (!n_metrics) continue;
    const unsigned blocks =
        (unsigned)std::min<size_t>((e.n + EVAL_THREADS - 1) / EVAL_THREADS, (size_t)EVAL_MAX_BLOCKS);
    SB_LAUNCH(ctx, k_eval_metrics, blocks, EVAL_THREADS, 0, e.margin.p, e.labels.p, e.weights.p, e.n, T.K,
              T.objective, d_metrics.p, n_metrics, d_partial.p);
    SB_LAUNCH(ctx, k_eval_finish, 1, 32, 0, d_partial.p, (int)blocks, d_metrics.p, n_metrics,
              d_out.p + i * n_metrics);
  }
  if (n_metrics && !ev.empty()) {
    SB_CUDA(cudaMemcpyAsync(out, d_out.p, ev.size() * n_metrics * 8, cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  return SB_OK;
}

int sb_booster_eval_margins(sb_booster* b, int eval_id, float* out) {
  using namespace sb;
  SB_REQUIRE(b && out, SB_ERR_INVALID_ARG, "NULL argument");
  auto& ev = booster_evals(b);
  SB_REQUIRE(eval_id >= 0 && (size_t)eval_id < ev.size(), SB_ERR_INVALID_ARG, "unknown eval set %d", eval_id);
  SB_TRY(sb_booster_eval(b, 0, nullptr, nullptr));  // bring every cache up to date
  BoosterTrees T;
  SB_TRY(booster_trees(b, &T));
  EvalSet& e = *ev[eval_id];
  SB_CUDA(cudaMemcpyAsync(out, e.margin.p, e.margin.bytes(), cudaMemcpyDeviceToHost, T.ctx->stream));
  SB_CUDA(cudaStreamSynchronize(T.ctx->stream));
  return SB_OK;
}

int sb_model_set_best_iteration(sb_model* m, int64_t best_iteration) {
  SB_REQUIRE(m, SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(best_iteration >= -1, SB_ERR_INVALID_ARG, "best_iteration must be >= -1");
  m->best_iteration = best_iteration;
  return SB_OK;
}

int sb_model_best_iteration(const sb_model* m, int64_t* best_iteration) {
  SB_REQUIRE(m && best_iteration, SB_ERR_INVALID_ARG, "NULL argument");
  *best_iteration = m->best_iteration;
  return SB_OK;
}

}  // extern "C"
