// sb_predict.cu — ensemble prediction (K9) and TreeSHAP (K10).
//
// Replaces BoostedModel::predict_margin_limited (learner/model.rs:231-285),
// predict (:291-300, with pred_transform of objective/classification.rs:
// :73-77 and multiclass.rs:93-99), and predict_contribs with tree_shap_cond,
// extend_path, unwind_path, unwound_path_sum, node_mean_value
// (learner/shap.rs:49-367).
//
// Margins: phase 1 routes every (row, tree) pair in parallel and stores the
// leaf value tree-major; phase 2 sums each (row, class) over its trees in
// tree order with separate f32 multiply and add, which is exactly the
// reference's accumulation, so margins are bit-identical.
// TreeSHAP: one thread per (row, tree) runs the path-dependent algorithm
// iteratively (explicit DFS, one path snapshot per depth, hot child first)
// in f64 and adds its contributions into a per-row f64 accumulator.
#include <cstring>
#include <functional>

#include "sb_internal.cuh"

namespace sb {
namespace {

constexpr uint32_t NF_DEFAULT_LEFT = 1u << 30;
constexpr uint32_t NF_CATEGORICAL = 1u << 31;
constexpr uint32_t NF_FEATURE = (1u << 30) - 1;
constexpr int SHAP_MAXD = 12;  // deepest tree TreeSHAP handles on the device

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

// RegTree::leaf_id_with over a dense row (regtree.rs:213-242): leaf value.
__device__ __forceinline__ float route(const PredDev& P, int t, const float* row, float missing,
                                       bool miss_nan) {
  const int4* nd = P.nodes + P.tree_off[t];
  int nid = 0;
  for (;;) {
    int4 x = __ldg(nd + nid);
    if (x.z < 0) return __int_as_float(x.y);
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

__global__ void k_margin_sum(PredDev P, const float* __restrict__ buf, size_t n, int K, int tree_limit,
                             float base, const float* __restrict__ base_margin, int bm_len_kind,
                             float* __restrict__ out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // (row, class)
  if (i >= n * K) return;
  size_t r = i / K;
  int c = (int)(i - r * K);
  float acc = base;
  if (bm_len_kind == 1) acc = base_margin[i];       // n*K
  else if (bm_len_kind == 2) acc = base_margin[r];  // n
  for (int t = c; t < tree_limit; t += K) {
    float w = P.weights ? P.weights[t] : 1.0f;
    acc = __fadd_rn(acc, __fmul_rn(w, buf[(size_t)t * n + r]));
  }
  out[i] = acc;
}

__global__ void k_transform(float* __restrict__ v, size_t n, int K, int objective) {
  size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  if (objective == SB_OBJ_LOGISTIC) {
    float x = v[r];
    float p;
    if (x >= 0.0f) p = __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-x)));
    else {
      float e = expf(x);
      p = __fdiv_rn(e, __fadd_rn(1.0f, e));
    }
    v[r] = p;
  } else if ((objective == SB_OBJ_SOFTMAX || objective == SB_OBJ_SOFTPROB) && K > 1) {
    float* row = v + r * K;
    float mx = -INFINITY;
    for (int c = 0; c < K; ++c)
      if (row[c] > mx) mx = row[c];
    float sum = 0.0f;
    for (int c = 0; c < K; ++c) {
      row[c] = expf(__fsub_rn(row[c], mx));
      sum = __fadd_rn(sum, row[c]);
    }
    float inv = __fdiv_rn(1.0f, sum);
    for (int c = 0; c < K; ++c) row[c] = __fmul_rn(row[c], inv);
  }
}

// ------------------------------------------------------------- TreeSHAP
struct PE {
  int f;
  double z, o, w;
};

__device__ void extend_path(PE* path, int& len, double z, double o, int f) {  // shap.rs:49-68
  const int ud = len;
  path[ud].f = f;
  path[ud].z = z;
  path[ud].o = o;
  path[ud].w = ud == 0 ? 1.0 : 0.0;
  const double denom = (double)(ud + 1);
  for (int i = ud - 1; i >= 0; --i) {
    double pw = path[i].w;
    path[i + 1].w += o * pw * (double)(i + 1) / denom;
    path[i].w = z * pw * (double)(ud - i) / denom;
  }
  len = ud + 1;
}
__device__ void unwind_path(PE* path, int& len, int pi) {  // shap.rs:72-94
  const int ud = len - 1;
  const double o = path[pi].o, z = path[pi].z;
  double next = path[ud].w;
  const double denom = (double)(ud + 1);
  for (int i = ud - 1; i >= 0; --i) {
    if (o != 0.0) {
      double tmp = path[i].w;
      path[i].w = next * denom / ((double)(i + 1) * o);
      next = tmp - path[i].w * z * (double)(ud - i) / denom;
    } else if (z != 0.0) {
      path[i].w = path[i].w * denom / (z * (double)(ud - i));
    }
  }
  for (int i = pi; i < ud; ++i) {
    path[i].f = path[i + 1].f;
    path[i].z = path[i + 1].z;
    path[i].o = path[i + 1].o;
  }
  len = ud;
}
__device__ double unwound_path_sum(const PE* path, int len, int pi) {  // shap.rs:98-116
  const int ud = len - 1;
  const double o = path[pi].o, z = path[pi].z;
  double next = path[ud].w;
  const double denom = (double)(ud + 1);
  double total = 0.0;
  for (int i = ud - 1; i >= 0; --i) {
    if (o != 0.0) {
      double tmp = next * denom / ((double)(i + 1) * o);
      total += tmp;
      next = path[i].w - tmp * z * (double)(ud - i) / denom;
    } else if (z != 0.0) {
      total += (path[i].w / z) / ((double)(ud - i) / denom);
    }
  }
  return total;
}

struct ShapDev {
  const sb_node* nodes;
  const int64_t* tree_off;
  int n_trees;
};

__global__ void k_shap(ShapDev P, const float* __restrict__ X, size_t n, int F, int K, float missing,
                       int trees_per_block, double* __restrict__ acc) {
  const bool miss_nan = isnan(missing);
  size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const float* row = X + r * F;
  const int width = F + 1;
  PE paths[SHAP_MAXD + 2][SHAP_MAXD + 2];
  int lens[SHAP_MAXD + 2];
  struct Item {
    int nid, d, f;
    double z, o;
  } stack[2 * SHAP_MAXD + 4];
  int t0 = blockIdx.y * trees_per_block;
  int t1 = min(P.n_trees, t0 + trees_per_block);
  for (int t = t0; t < t1; ++t) {
    const sb_node* nd = P.nodes + P.tree_off[t];
    double* phi = acc + (r * K + (t % K)) * (size_t)width;
    int sp = 0;
    stack[sp++] = Item{0, 0, -1, 1.0, 1.0};
    while (sp > 0) {
      Item it = stack[--sp];
      PE* path = paths[it.d];
      int len = 0;
      if (it.d > 0) {
        len = lens[it.d - 1];
        for (int i = 0; i < len; ++i) path[i] = paths[it.d - 1][i];
      }
      extend_path(path, len, it.z, it.o, it.f);
      const sb_node& node = nd[it.nid];
      const int ud = len - 1;
      if (node.left < 0) {
        const double leaf = (double)node.leaf_value;
        for (int i = 1; i <= ud; ++i) {
          double w = unwound_path_sum(path, len, i);
          atomicAdd(&phi[path[i].f], w * (path[i].o - path[i].z) * leaf * 1.0);
        }
        lens[it.d] = len;
        continue;
      }
      float v = row[node.split_feature];
      // the reference routes by `v < split_cond` here, categorical or not
      bool go_left = is_missing_d(v, missing, miss_nan) ? node.default_left != 0 : v < node.split_cond;
      int hot = go_left ? node.left : node.right, cold = go_left ? node.right : node.left;
      double cover = (double)node.sum_hess, hz = 0.0, cz = 0.0;
      if (cover > 0.0) {
        hz = (double)nd[hot].sum_hess / cover;
        cz = (double)nd[cold].sum_hess / cover;
      }
      int si = (int)node.split_feature;
      double iz = 1.0, io = 1.0;
      for (int i = 1; i <= ud; ++i)
        if (path[i].f == si) {
          iz = path[i].z;
          io = path[i].o;
          unwind_path(path, len, i);
          break;
        }
      lens[it.d] = len;
      if (it.d + 1 > SHAP_MAXD) continue;  // guarded by the host (depth check)
      stack[sp++] = Item{cold, it.d + 1, si, cz * iz, 0.0};
      stack[sp++] = Item{hot, it.d + 1, si, hz * iz, io};
    }
  }
}

__global__ void k_shap_finish(const double* __restrict__ acc, const double* __restrict__ bias, size_t n,
                              int K, int F, float* __restrict__ out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t width = (size_t)F + 1;
  if (i >= n * K * width) return;
  size_t j = i % width;
  size_t c = (i / width) % K;
  double v = acc[i];
  if (j == (size_t)F) v = bias[c];
  out[i] = (float)v;
}

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

}  // namespace

int model_upload(sb_model* m) {
  if (m->dev_valid) return SB_OK;
  sb_ctx* ctx = m->ctx;
  DevEnsemble& D = m->dev;
  const int T = (int)m->trees.size();
  std::vector<int64_t> off(T + 1, 0);
  for (int t = 0; t < T; ++t) off[t + 1] = off[t] + (int64_t)m->trees[t].nodes.size();
  std::vector<int4> packed(off[T]);
  std::vector<int> catend(off[T], 0);
  std::vector<sb_node> full(off[T]);
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
      full[off[t] + i] = nd;
    }
    maxd = std::max(maxd, tree_depth(tr));
  }
  SB_TRY(D.nodes.alloc(ctx, std::max<size_t>(packed.size(), 1)));
  SB_TRY(D.full.alloc(ctx, std::max<size_t>(full.size(), 1)));
  SB_TRY(D.tree_off.alloc(ctx, T + 1));
  SB_TRY(D.cats.alloc(ctx, std::max<size_t>(cats.size(), 1)));
  SB_TRY(D.weights.alloc(ctx, std::max(T, 1)));
  cudaStream_t st = ctx->stream;
  if (!packed.empty()) {
    SB_CUDA(cudaMemcpyAsync(D.nodes.p, packed.data(), packed.size() * 16, cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemcpyAsync(D.full.p, full.data(), full.size() * sizeof(sb_node), cudaMemcpyHostToDevice, st));
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
  // rows per batch so the tree-major leaf buffer stays <= 256 MB
  size_t batch = limit > 0 ? std::max<size_t>(1024, (size_t)(64ull << 20) / (size_t)limit) : n;
  batch = std::min(batch, n);
  DBuf<float> buf;
  if (limit > 0) SB_TRY(buf.alloc(ctx, (size_t)limit * std::max<size_t>(batch, 1)));
  for (size_t r0 = 0; r0 < n; r0 += batch) {
    size_t nb = std::min(batch, n - r0);
    if (limit > 0) {
      const int tpb = 8;
      dim3 grid((unsigned)((nb + 127) / 128), (unsigned)((limit + tpb - 1) / tpb));
      SB_LAUNCH(ctx, k_leaf_values, grid, 128, 0, P, d_X + r0 * F, nb, (int)F, missing, limit, tpb, buf.p);
    }
    const float* bm = d_base_margin ? d_base_margin + (bm_kind == 1 ? r0 * Kc : r0) : nullptr;
    size_t tot = nb * Kc;
    SB_LAUNCH(ctx, k_margin_sum, (unsigned)((tot + 255) / 256), 256, 0, P, buf.p, nb, Kc, limit,
              m->base_score, bm, bm ? bm_kind : 0, d_out + r0 * Kc);
  }
  return SB_OK;
}

int predict_contribs_device(sb_model* m, const float* d_X, size_t n, size_t F, float missing,
                            float* d_out) {
  sb_ctx* ctx = m->ctx;
  SB_TRY(model_upload(m));
  SB_REQUIRE(m->dev.max_depth <= SHAP_MAXD, SB_ERR_UNSUPPORTED,
             "TreeSHAP on the device supports trees up to depth %d (got %d)", SHAP_MAXD, m->dev.max_depth);
  const int K = m->num_class >= 2 ? m->num_class : 1;
  const int T = m->dev.n_trees;
  const size_t width = F + 1;
  // bias per class: base_score + sum of tree means in tree order (shap.rs:340-359)
  std::vector<double> means(T);
  if (T) {
    SB_CUDA(cudaMemcpyAsync(means.data(), m->dev.tree_mean.p, T * 8, cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  std::vector<double> bias(K, 0.0);
  for (int c = 0; c < K; ++c) bias[c] += (double)m->base_score;
  for (int t = 0; t < T; ++t) bias[t % K] += means[t];
  DBuf<double> d_bias, acc;
  SB_TRY(d_bias.alloc(ctx, K));
  SB_CUDA(cudaMemcpyAsync(d_bias.p, bias.data(), K * 8, cudaMemcpyHostToDevice, ctx->stream));
  SB_TRY(acc.alloc(ctx, n * K * width));
  SB_CUDA(cudaMemsetAsync(acc.p, 0, acc.bytes(), ctx->stream));
  ShapDev P;
  P.nodes = m->dev.full.p;
  P.tree_off = m->dev.tree_off.p;
  P.n_trees = T;
  if (T > 0 && n > 0) {
    const int tpb = 4;
    dim3 grid((unsigned)((n + 63) / 64), (unsigned)((T + tpb - 1) / tpb));
    SB_LAUNCH(ctx, k_shap, grid, 64, 0, P, d_X, n, (int)F, K, missing, tpb, acc.p);
  }
  size_t tot = n * K * width;
  if (tot) SB_LAUNCH(ctx, k_shap_finish, (unsigned)((tot + 255) / 256), 256, 0, acc.p, d_bias.p, n, K, (int)F, d_out);
  return SB_OK;
}

// ---- batch launchers on an explicit stream with caller-owned buffers (used
// by the serving loop; the model must be resident, see model_upload)

size_t margin_chunk_rows(const sb_model* m) {
  const size_t T = (size_t)std::max(m->dev.n_trees, 1);
  return std::max<size_t>(1024, (size_t)(64ull << 20) / (T * 4));  // leaf buffer <= 64 MB
}

int margin_batch(sb_model* m, cudaStream_t st, const float* d_X, size_t n, size_t F, float missing,
                 float* d_buf, size_t buf_rows, float* d_out) {
  sb_ctx* ctx = m->ctx;
  const int Kc = m->num_class >= 2 ? m->num_class : 1;
  const int T = m->dev.n_trees;
  PredDev P;
  P.nodes = m->dev.nodes.p;
  P.cat_end = m->dev.cat_end.p;
  P.tree_off = m->dev.tree_off.p;
  P.cats = m->dev.cats.p;
  P.weights = m->dev.weights.p;
  P.n_trees = T;
  for (size_t r0 = 0; r0 < n; r0 += buf_rows) {
    const size_t nb = std::min(buf_rows, n - r0);
    if (T > 0) {
      const int tpb = 8;
      dim3 grid((unsigned)((nb + 127) / 128), (unsigned)((T + tpb - 1) / tpb));
      SB_LAUNCH_ON(ctx, st, k_leaf_values, grid, 128, 0, P, d_X + r0 * F, nb, (int)F, missing, T, tpb, d_buf);
    }
    const size_t tot = nb * Kc;
    SB_LAUNCH_ON(ctx, st, k_margin_sum, (unsigned)((tot + 255) / 256), 256, 0, P, d_buf, nb, Kc, T,
                 m->base_score, (const float*)nullptr, 0, d_out + r0 * Kc);
  }
  return SB_OK;
}

int contribs_bias(sb_model* m, std::vector<double>* bias) {
  SB_TRY(model_upload(m));
  const int K = m->num_class >= 2 ? m->num_class : 1;
  bias->assign(K, (double)m->base_score);
  for (size_t t = 0; t < m->trees.size(); ++t) (*bias)[t % K] += node_mean_value(m->trees[t], 0);
  return SB_OK;
}

int contribs_batch(sb_model* m, cudaStream_t st, const float* d_X, size_t n, size_t F, float missing,
                   double* d_acc, const double* d_bias, float* d_out) {
  sb_ctx* ctx = m->ctx;
  SB_REQUIRE(m->dev.max_depth <= SHAP_MAXD, SB_ERR_UNSUPPORTED,
             "TreeSHAP on the device supports trees up to depth %d (got %d)", SHAP_MAXD, m->dev.max_depth);
  const int K = m->num_class >= 2 ? m->num_class : 1;
  const int T = m->dev.n_trees;
  const size_t tot = n * K * (F + 1);
  SB_CUDA(cudaMemsetAsync(d_acc, 0, tot * sizeof(double), st));
  ShapDev P;
  P.nodes = m->dev.full.p;
  P.tree_off = m->dev.tree_off.p;
  P.n_trees = T;
  if (T > 0 && n > 0) {
    const int tpb = 4;
    dim3 grid((unsigned)((n + 63) / 64), (unsigned)((T + tpb - 1) / tpb));
    SB_LAUNCH_ON(ctx, st, k_shap, grid, 64, 0, P, d_X, n, (int)F, K, missing, tpb, d_acc);
  }
  if (tot) SB_LAUNCH_ON(ctx, st, k_shap_finish, (unsigned)((tot + 255) / 256), 256, 0, d_acc, d_bias, n, K, (int)F, d_out);
  return SB_OK;
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
  SB_TRY(predict_margin_device(m, dX.p, n_rows, n_cols, missing, dbm.p, 1, 0, dout.p));
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

}  // extern "C"
