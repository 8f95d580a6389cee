// sb_predict.cu — ensemble prediction (K9): the device copy of a model, margins,
// predict and predict_leaf. TreeSHAP (K10) is in sb_shap.cu.
//
// Replaces BoostedModel::predict_margin_limited (learner/model.rs:231-285),
// predict (:291-300, with pred_transform of objective/classification.rs:
// :73-77 and multiclass.rs:93-99), predict_leaf (:330-341) and
// node_mean_value (learner/shap.rs:288-302).
//
// Margins: phase 1 routes every (row, tree) pair in parallel and stores the
// leaf value tree-major; phase 2 sums each (row, class) over its trees in
// tree order with separate f32 multiply and add, which is exactly the
// reference's accumulation, so margins are bit-identical.
#include <cmath>
#include <cstring>
#include <functional>

#include "sb_internal.cuh"

namespace sb {
namespace {

constexpr uint32_t NF_DEFAULT_LEFT = 1u << 30;
constexpr uint32_t NF_CATEGORICAL = 1u << 31;
constexpr uint32_t NF_FEATURE = (1u << 30) - 1;

struct PredDev {
  const int4* nodes;        // {feat|flags, cond (leaf value for leaves / cat_begin), left, right}
  const int* cat_end;       // per node (categorical nodes only)
  const int64_t* tree_off;  // [n_trees + 1]
  const uint32_t* cats;     // global category pool
  const float* weights;
  int n_trees;
};

__device__ __forceinline__ bool is_missing_d(float v, float missing, bool miss_nan) {
  return miss_nan ? isnan(v) : (v == missing);
}

// RegTree::leaf_id_with over a dense row (regtree.rs:213-242): the leaf's
// node index, and its packed node in *leaf.
__device__ __forceinline__ int route_to_leaf(const PredDev& P, int t, const float* row, float missing,
                                             bool miss_nan, int4* leaf) {
  const int4* nd = P.nodes + P.tree_off[t];
  int nid = 0;
  for (;;) {
    int4 x = __ldg(nd + nid);
    if (x.z < 0) {
      *leaf = x;
      return nid;
    }
    uint32_t ff = (uint32_t)x.x;
    float v = row[ff & NF_FEATURE];
    bool go_left;
    if (is_missing_d(v, missing, miss_nan)) {
      go_left = (ff & NF_DEFAULT_LEFT) != 0;
    } else if (ff & NF_CATEGORICAL) {
      uint32_t c = f32_as_u32(v);
      go_left = false;
      for (int i = x.y; i < P.cat_end[P.tree_off[t] + nid]; ++i)
        if (P.cats[i] == c) {
          go_left = true;
          break;
        }
    } else {
      go_left = v < __int_as_float(x.y);
    }
    nid = go_left ? x.z : x.w;
  }
}

// The leaf value of one tree for a dense row.
__device__ __forceinline__ float route(const PredDev& P, int t, const float* row, float missing,
                                       bool miss_nan) {
  int4 x;
  route_to_leaf(P, t, row, missing, miss_nan, &x);
  return __int_as_float(x.y);
}

// predict_leaf (model.rs:330-341): out [n][T] leaf node ids, one thread per
// (row, tree) with the tree index fastest, so the stores are coalesced and a
// warp reads one row.
__global__ void k_leaf_ids(PredDev P, const float* __restrict__ X, size_t n, int F, float missing,
                           uint32_t* __restrict__ out) {
  const size_t T = (size_t)P.n_trees;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * T) return;
  const size_t r = i / T;
  const int t = (int)(i - r * T);
  int4 x;
  out[i] = (uint32_t)route_to_leaf(P, t, X + r * F, missing, isnan(missing), &x);
}

// Margins in two phases. Phase 1 routes every (row, tree) pair in parallel
// (a thread takes one row through a few consecutive trees) and stores the
// leaf values tree-major. Phase 2 adds them per (row, class) in tree order
// with separate f32 multiply and add, which is the reference's accumulation
// (predict_margin_limited), so margins are bit-identical: a block takes
// PRED_ROWS rows, stages chunks of PRED_CHUNK trees' leaf values through
// shared memory with coalesced loads from all its warps, and warp 0 (lane =
// row) runs the ordered sums.
constexpr int PRED_ROWS = 32;
constexpr int PRED_WARPS = 4;
constexpr int PRED_CHUNK = 128;

__global__ void k_leaf_values(PredDev P, const float* __restrict__ X, size_t n, int F, float missing,
                              int tree_limit, int trees_per_block, float* __restrict__ buf) {
  const bool miss_nan = isnan(missing);
  size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const float* row = X + r * F;
  int t0 = blockIdx.y * trees_per_block;
  int t1 = min(tree_limit, t0 + trees_per_block);
  for (int t = t0; t < t1; ++t) buf[(size_t)t * n + r] = route(P, t, row, missing, miss_nan);
}

__global__ void __launch_bounds__(PRED_ROWS * PRED_WARPS)
    k_margin_sum(PredDev P, const float* __restrict__ buf, size_t n, int K, int tree_limit, float base,
                 const float* __restrict__ base_margin, int bm_kind, float* __restrict__ out) {
  __shared__ float leaf_s[PRED_CHUNK][PRED_ROWS];
  __shared__ float acc_s[16][PRED_ROWS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t r = (size_t)blockIdx.x * PRED_ROWS + lane;
  const bool in = r < n;
  // the running sums: shared memory for up to 16 classes, else `out` itself
  const bool in_smem = K <= 16;
  auto acc = [&](int c) -> float& { return in_smem ? acc_s[c][lane] : out[(in ? r : 0) * K + c]; };
  if (warp == 0 && (in || in_smem))
    for (int c = 0; c < K; ++c) {
      float a = base;
      if (in && bm_kind == 1) a = base_margin[r * K + c];  // n*K
      else if (in && bm_kind == 2) a = base_margin[r];     // n
      acc(c) = a;
    }
  for (int t0 = 0; t0 < tree_limit; t0 += PRED_CHUNK) {
    const int t1 = min(tree_limit, t0 + PRED_CHUNK);
    for (int t = t0 + warp; t < t1; t += PRED_WARPS) leaf_s[t - t0][lane] = in ? buf[(size_t)t * n + r] : 0.0f;
    __syncthreads();
    if (warp == 0 && (in || in_smem)) {
      if (K == 1) {
        float a = acc(0);
        for (int t = t0; t < t1; ++t) {
          const float w = P.weights ? P.weights[t] : 1.0f;
          a = __fadd_rn(a, __fmul_rn(w, leaf_s[t - t0][lane]));
        }
        acc(0) = a;
      } else {
        for (int t = t0; t < t1; ++t) {
          const float w = P.weights ? P.weights[t] : 1.0f;
          float& a = acc(t % K);
          a = __fadd_rn(a, __fmul_rn(w, leaf_s[t - t0][lane]));
        }
      }
    }
    __syncthreads();
  }
  if (warp == 0 && in && in_smem)
    for (int c = 0; c < K; ++c) out[r * K + c] = acc_s[c][lane];
}

// Both phases over n rows, in chunks of `chunk` rows (buf holds chunk * T floats).
int margins(sb_ctx* ctx, cudaStream_t st, const PredDev& P, const float* d_X, size_t n, size_t F, float missing,
            int K, int limit, float base, const float* d_bm, int bm_kind, float* d_buf, size_t chunk, float* d_out) {
  for (size_t r0 = 0; r0 < n; r0 += chunk) {
    const size_t nb = std::min(chunk, n - r0);
    if (limit > 0) {
      const int tpb = nb < 16384 ? 2 : 8;  // small batches: more (row, tree) pairs in flight
      dim3 grid((unsigned)((nb + 127) / 128), (unsigned)((limit + tpb - 1) / tpb));
      SB_LAUNCH_ON(ctx, st, k_leaf_values, grid, 128, 0, P, d_X + r0 * F, nb, (int)F, missing, limit, tpb, d_buf);
    }
    const float* bm = d_bm ? d_bm + (bm_kind == 1 ? r0 * K : r0) : nullptr;
    SB_LAUNCH_ON(ctx, st, k_margin_sum, (unsigned)((nb + PRED_ROWS - 1) / PRED_ROWS), PRED_ROWS * PRED_WARPS, 0, P,
                 d_buf, nb, K, limit, base, bm, bm ? bm_kind : 0, d_out + r0 * K);
  }
  return SB_OK;
}

__global__ void k_transform(float* __restrict__ v, size_t n, int K, int objective) {
  size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  pred_transform_row(v + r * K, K, objective);
}

}  // namespace

int tree_depth(const HostTree& t) {
  std::vector<int> depth(t.nodes.size(), 0);
  int mx = 0;
  for (size_t i = 0; i < t.nodes.size(); ++i) {
    const sb_node& nd = t.nodes[i];
    if (nd.left >= 0) {
      depth[nd.left] = depth[i] + 1;
      depth[nd.right] = depth[i] + 1;
      mx = std::max(mx, depth[i] + 1);
    }
  }
  return mx;
}

double node_mean_value(const HostTree& t, int id) {  // shap.rs:288-302
  const sb_node& nd = t.nodes[id];
  if (nd.left < 0) return (double)nd.leaf_value;
  double cover = (double)nd.sum_hess;
  if (cover <= 0.0) return 0.0;
  double lc = (double)t.nodes[nd.left].sum_hess, rc = (double)t.nodes[nd.right].sum_hess;
  return (lc * node_mean_value(t, nd.left) + rc * node_mean_value(t, nd.right)) / cover;
}

int model_upload(sb_model* m) {
  if (m->dev_valid) return SB_OK;
  sb_ctx* ctx = m->ctx;
  DevEnsemble& D = m->dev;
  const int T = (int)m->trees.size();
  std::vector<int64_t> off(T + 1, 0);
  for (int t = 0; t < T; ++t) off[t + 1] = off[t] + (int64_t)m->trees[t].nodes.size();
  std::vector<int4> packed(off[T]);
  std::vector<int> catend(off[T], 0);
  std::vector<uint32_t> cats;
  int maxd = 0;
  for (int t = 0; t < T; ++t) {
    const HostTree& tr = m->trees[t];
    int cat_base = (int)cats.size();
    cats.insert(cats.end(), tr.cats.begin(), tr.cats.end());
    for (size_t i = 0; i < tr.nodes.size(); ++i) {
      const sb_node& nd = tr.nodes[i];
      int4 x;
      uint32_t ff = nd.split_feature & NF_FEATURE;
      if (nd.default_left) ff |= NF_DEFAULT_LEFT;
      if (nd.is_categorical && nd.left >= 0) ff |= NF_CATEGORICAL;
      x.x = (int)ff;
      if (nd.left < 0) {
        float lv = nd.leaf_value;
        std::memcpy(&x.y, &lv, 4);
      } else if (nd.is_categorical) {
        x.y = cat_base + (int)nd.cat_begin;
        catend[off[t] + i] = cat_base + (int)nd.cat_end;
      } else {
        float c = nd.split_cond;
        std::memcpy(&x.y, &c, 4);
      }
      x.z = nd.left;
      x.w = nd.right;
      packed[off[t] + i] = x;
    }
    maxd = std::max(maxd, tree_depth(tr));
  }
  SB_TRY(D.nodes.alloc(ctx, std::max<size_t>(packed.size(), 1)));
  SB_TRY(D.tree_off.alloc(ctx, T + 1));
  SB_TRY(D.cats.alloc(ctx, std::max<size_t>(cats.size(), 1)));
  SB_TRY(D.weights.alloc(ctx, std::max(T, 1)));
  cudaStream_t st = ctx->stream;
  if (!packed.empty()) {
    SB_CUDA(cudaMemcpyAsync(D.nodes.p, packed.data(), packed.size() * 16, cudaMemcpyHostToDevice, st));
  }
  SB_CUDA(cudaMemcpyAsync(D.tree_off.p, off.data(), (T + 1) * 8, cudaMemcpyHostToDevice, st));
  if (!cats.empty()) SB_CUDA(cudaMemcpyAsync(D.cats.p, cats.data(), cats.size() * 4, cudaMemcpyHostToDevice, st));
  if (T) SB_CUDA(cudaMemcpyAsync(D.weights.p, m->weights.data(), T * 4, cudaMemcpyHostToDevice, st));
  SB_TRY(D.cat_end.alloc(ctx, std::max<size_t>(catend.size(), 1)));
  if (!catend.empty())
    SB_CUDA(cudaMemcpyAsync(D.cat_end.p, catend.data(), catend.size() * 4, cudaMemcpyHostToDevice, st));
  std::vector<double> means(T);
  for (int t = 0; t < T; ++t) means[t] = node_mean_value(m->trees[t], 0);
  SB_TRY(D.tree_mean.alloc(ctx, std::max(T, 1)));
  if (T) SB_CUDA(cudaMemcpyAsync(D.tree_mean.p, means.data(), T * 8, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaStreamSynchronize(st));
  D.n_trees = T;
  D.max_depth = maxd;
  m->dev_valid = true;
  return SB_OK;
}

// Rows per phase-1 chunk, so that the tree-major leaf buffer stays <= 64 MB.
size_t margin_chunk_rows(const sb_model* m) {
  const size_t T = (size_t)std::max(m->dev.n_trees, 1);
  return std::max<size_t>(1024, (size_t)(64ull << 20) / (T * 4));
}

int predict_margin_device(sb_model* m, const float* d_X, size_t n, size_t F, float missing,
                          const float* d_base_margin, int bm_kind, size_t ntree_limit, float* d_out) {
  sb_ctx* ctx = m->ctx;
  SB_TRY(model_upload(m));
  const int Kc = m->num_class >= 2 ? m->num_class : 1;
  const int T = m->dev.n_trees;
  const int limit = ntree_limit == 0 ? T : (int)std::min<size_t>(ntree_limit, (size_t)T);
  PredDev P;
  P.nodes = m->dev.nodes.p;
  P.cat_end = m->dev.cat_end.p;
  P.tree_off = m->dev.tree_off.p;
  P.cats = m->dev.cats.p;
  P.weights = m->dev.weights.p;
  P.n_trees = T;
  if (n == 0) return SB_OK;
  const size_t chunk = std::min(n, margin_chunk_rows(m));  // leaf buffer <= 64 MB
  DBuf<float> buf;
  if (limit > 0) SB_TRY(buf.alloc(ctx, (size_t)limit * chunk));
  return margins(ctx, ctx->stream, P, d_X, n, F, missing, Kc, limit, m->base_score, d_base_margin, bm_kind, buf.p,
                 chunk, d_out);
}

// ---- batch launchers on an explicit stream with caller-owned buffers (used
// by the serving loop; the model must be resident, see model_upload)

int margin_batch(sb_model* m, cudaStream_t st, const float* d_X, size_t n, size_t F, float missing,
                 float* d_buf, size_t buf_rows, float* d_out) {
  sb_ctx* ctx = m->ctx;
  const int Kc = m->num_class >= 2 ? m->num_class : 1;
  PredDev P;
  P.nodes = m->dev.nodes.p;
  P.cat_end = m->dev.cat_end.p;
  P.tree_off = m->dev.tree_off.p;
  P.cats = m->dev.cats.p;
  P.weights = m->dev.weights.p;
  P.n_trees = m->dev.n_trees;
  if (n == 0) return SB_OK;
  return margins(ctx, st, P, d_X, n, F, missing, Kc, m->dev.n_trees, m->base_score, nullptr, 0, d_buf, buf_rows,
                 d_out);
}

}  // namespace sb

extern "C" {

int sb_predict_margin(sb_model* m, const float* X, size_t n_rows, size_t n_cols, float missing,
                      const float* base_margin, size_t ntree_limit, float* out) {
  using namespace sb;
  SB_REQUIRE(m && out && (X || n_rows == 0), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_cols == (size_t)m->n_features, SB_ERR_DIMENSION,
             "dimension mismatch: expected %d features, got %zu", m->n_features, n_cols);
  if (n_rows == 0) return SB_OK;
  sb_ctx* ctx = m->ctx;
  SB_CUDA(cudaSetDevice(ctx->device));
  const int K = m->num_class >= 2 ? m->num_class : 1;
  DBuf<float> dX, dbm, dout;
  SB_TRY(dX.alloc(ctx, n_rows * n_cols));
  SB_TRY(dout.alloc(ctx, n_rows * K));
  SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  if (base_margin) {
    SB_TRY(dbm.alloc(ctx, n_rows * K));
    SB_CUDA(cudaMemcpyAsync(dbm.p, base_margin, dbm.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  }
  SB_TRY(predict_margin_device(m, dX.p, n_rows, n_cols, missing, dbm.p, 1, ntree_limit, dout.p));
  SB_CUDA(cudaMemcpyAsync(out, dout.p, dout.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_predict(sb_model* m, const float* X, size_t n_rows, size_t n_cols, float missing,
               const float* base_margin, float* out) {
  using namespace sb;
  SB_REQUIRE(m && out && (X || n_rows == 0), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_cols == (size_t)m->n_features, SB_ERR_DIMENSION,
             "dimension mismatch: expected %d features, got %zu", m->n_features, n_cols);
  if (n_rows == 0) return SB_OK;
  sb_ctx* ctx = m->ctx;
  SB_CUDA(cudaSetDevice(ctx->device));
  const int K = m->num_class >= 2 ? m->num_class : 1;
  DBuf<float> dX, dbm, dout;
  SB_TRY(dX.alloc(ctx, n_rows * n_cols));
  SB_TRY(dout.alloc(ctx, n_rows * K));
  SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  if (base_margin) {
    SB_TRY(dbm.alloc(ctx, n_rows * K));
    SB_CUDA(cudaMemcpyAsync(dbm.p, base_margin, dbm.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  }
  // predict uses the effective tree count: (best_iteration + 1) * K after
  // early stopping, else all trees (model.rs:213-219)
  const size_t limit = m->best_iteration >= 0 ? (size_t)(m->best_iteration + 1) * K : 0;
  SB_TRY(predict_margin_device(m, dX.p, n_rows, n_cols, missing, dbm.p, 1, limit, dout.p));
  SB_LAUNCH(ctx, k_transform, (unsigned)((n_rows + 255) / 256), 256, 0, dout.p, n_rows, K, m->objective);
  SB_CUDA(cudaMemcpyAsync(out, dout.p, dout.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_predict_contribs(sb_model* m, const float* X, size_t n_rows, size_t n_cols, float missing,
                        float* out) {
  using namespace sb;
  SB_REQUIRE(m && out && (X || n_rows == 0), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_cols == (size_t)m->n_features, SB_ERR_DIMENSION,
             "dimension mismatch: expected %d features, got %zu", m->n_features, n_cols);
  if (n_rows == 0) return SB_OK;
  sb_ctx* ctx = m->ctx;
  SB_CUDA(cudaSetDevice(ctx->device));
  const int K = m->num_class >= 2 ? m->num_class : 1;
  DBuf<float> dX, dout;
  SB_TRY(dX.alloc(ctx, n_rows * n_cols));
  SB_TRY(dout.alloc(ctx, n_rows * K * (n_cols + 1)));
  SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  SB_TRY(predict_contribs_device(m, dX.p, n_rows, n_cols, missing, dout.p));
  SB_CUDA(cudaMemcpyAsync(out, dout.p, dout.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_predict_leaf(sb_model* m, const float* X, size_t n_rows, size_t n_cols, float missing, uint32_t* out) {
  using namespace sb;
  SB_REQUIRE(m && (out || n_rows == 0) && (X || n_rows == 0), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_cols == (size_t)m->n_features, SB_ERR_DIMENSION,
             "dimension mismatch: expected %d features, got %zu", m->n_features, n_cols);
  sb_ctx* ctx = m->ctx;
  SB_CUDA(cudaSetDevice(ctx->device));
  SB_TRY(model_upload(m));
  const size_t T = (size_t)m->dev.n_trees;
  if (n_rows == 0 || T == 0) return SB_OK;
  PredDev P;
  P.nodes = m->dev.nodes.p;
  P.cat_end = m->dev.cat_end.p;
  P.tree_off = m->dev.tree_off.p;
  P.cats = m->dev.cats.p;
  P.weights = m->dev.weights.p;
  P.n_trees = (int)T;
  DBuf<float> dX;
  DBuf<uint32_t> dout;
  SB_TRY(dX.alloc(ctx, n_rows * n_cols));
  SB_TRY(dout.alloc(ctx, n_rows * T));
  SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  const size_t tot = n_rows * T;
  SB_REQUIRE((tot + 255) / 256 < (1ull << 31), SB_ERR_UNSUPPORTED, "predict_leaf: %zu outputs exceed one launch", tot);
  SB_LAUNCH(ctx, k_leaf_ids, (unsigned)((tot + 255) / 256), 256, 0, P, dX.p, n_rows, (int)n_cols, missing, dout.p);
  SB_CUDA(cudaMemcpyAsync(out, dout.p, dout.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_predict_interactions(sb_model* m, const float* X, size_t n_rows, size_t n_cols, float missing, float* out) {
  using namespace sb;
  SB_REQUIRE(m && (out || n_rows == 0) && (X || n_rows == 0), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_cols == (size_t)m->n_features, SB_ERR_DIMENSION,
             "dimension mismatch: expected %d features, got %zu", m->n_features, n_cols);
  if (n_rows == 0) return SB_OK;
  sb_ctx* ctx = m->ctx;
  SB_CUDA(cudaSetDevice(ctx->device));
  const int K = m->num_class >= 2 ? m->num_class : 1;
  const size_t WW = (n_cols + 1) * (n_cols + 1);
  DBuf<float> dX, dout;
  SB_TRY(dX.alloc(ctx, n_rows * n_cols));
  SB_TRY(dout.alloc(ctx, n_rows * K * WW));
  SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  SB_TRY(predict_interactions_device(m, dX.p, n_rows, n_cols, missing, dout.p));
  SB_CUDA(cudaMemcpyAsync(out, dout.p, dout.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

}  // extern "C"
