// sb_predict.cu — ensemble prediction (K9) and TreeSHAP (K10).
//
// Replaces BoostedModel::predict_margin_limited (learner/model.rs:231-285),
// predict (:291-300, with pred_transform of objective/classification.rs:
// :73-77 and multiclass.rs:93-99), predict_leaf (:330-341), predict_contribs
// with tree_shap_cond, extend_path, unwind_path, unwound_path_sum,
// node_mean_value (learner/shap.rs:49-367), and predict_interactions
// (learner/shap.rs:395-509).
//
// Margins: phase 1 routes every (row, tree) pair in parallel and stores the
// leaf value tree-major; phase 2 sums each (row, class) over its trees in
// tree order with separate f32 multiply and add, which is exactly the
// reference's accumulation, so margins are bit-identical.
// TreeSHAP: one thread per (row, tree) runs the path-dependent algorithm
// iteratively (explicit DFS, one path snapshot per depth, hot child first)
// in f64 and adds its contributions into a per-row f64 accumulator.
#include <cmath>
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

// ------------------------------------------------------------- TreeSHAP
// Path-dependent TreeSHAP (shap.rs:49-367) restated per root-to-leaf path.
// At a leaf, the recursive walk's path holds one element per feature split
// on the way (a repeated feature is unwound and extended again with the
// products of its fractions), with one-fraction o = [the row follows every
// such split] and zero-fraction z = the product of their cover fractions. So
// each leaf's contribution to a row is: EXTEND over its merged elements,
// then, per element, UNWOUND_SUM times (o - z) times the leaf value. The
// elements' order does not change the weights.
//
// A block takes SHAP_ROWS rows (one per thread) over one chunk of at most
// SHAP_CHUNK paths of one tree. Each thread adds its row's contributions
// into a feature-major f32 partial in shared memory (its own column: no
// conflicts, no atomics), flushed to the f64 accumulator at the end. The
// partial has a row only for the features the chunk's paths split on (their
// compact indices are precomputed per element), which keeps the block's
// shared memory small and more blocks resident. Blocks
// stay short (a few hundred microseconds at depth 8) and have the same 128
// threads as the margin kernels' blocks, so when a TreeSHAP block retires a
// waiting margin block (on a higher-priority stream) fits in its place.
constexpr int SHAP_ROWS = 128;
constexpr int SHAP_CHUNK = 64;  // paths per block

__constant__ double c_inv[32];  // 1 / k

struct ShapPathsDev {
  const PathEl* el;
  const int* off;
  const float* leaf;
  const int4* chunk;     // {class, first path, end path, -}
  const int* fc;         // per element: compact feature index within its chunk
  const int* chunk_fo;   // per chunk: offset of its feature list in chunk_f
  const int* chunk_f;    // the chunks' distinct features
};

template <int MAXL>
__global__ void __launch_bounds__(SHAP_ROWS) k_shap_paths(ShapPathsDev P, const float* __restrict__ X, size_t n,
                                                         int F, int K, float missing, unsigned row_blocks,
                                                         double* __restrict__ acc) {
  extern __shared__ float ph[];          // [chunk features][R] contributions of this block
  const int R = SHAP_ROWS;
  const int tid = threadIdx.x;
  const unsigned rb = blockIdx.x % row_blocks;  // 1-D grid over (path chunk, row block)
  const size_t r0 = (size_t)rb * R;
  const unsigned ci = blockIdx.x / row_blocks;
  const int4 ch = P.chunk[ci];
  const int c = ch.x;
  const int fo = P.chunk_fo[ci], nfc = P.chunk_fo[ci + 1] - fo;
  for (int i = tid; i < nfc * R; i += R) ph[i] = 0.0f;
  const float* row = X + (r0 + tid < n ? r0 + tid : r0) * (size_t)F;  // L1-resident while the block runs
  __syncwarp();
  const bool miss_nan = isnan(missing);
  {
    for (int p = ch.y; p < ch.z; ++p) {
      const int e0 = P.off[p], L = P.off[p + 1] - e0;
      const double leaf = (double)P.leaf[p];
      double w[MAXL], z[MAXL], iz[MAXL], o[MAXL];
      int fe[MAXL];  // the element's row of the block's partial
#pragma unroll
      for (int e = 0; e < MAXL; ++e) {
        fe[e] = -1;
        z[e] = 1.0;
        iz[e] = 1.0;
        o[e] = 1.0;
        if (e < L) {
          const PathEl el = P.el[e0 + e];
          fe[e] = P.fc[e0 + e];
          z[e] = el.z;
          iz[e] = el.inv_z;
          if (el.f >= 0) {
            const float v = __ldg(row + el.f);
            const bool mis = miss_nan ? isnan(v) : v == missing;
            o[e] = (mis ? el.miss_ok != 0 : (v >= el.lo && v < el.hi)) ? 1.0 : 0.0;
          }
        }
      }
      // EXTEND (extend_path, shap.rs:49-68) over every element
      w[0] = 1.0;
#pragma unroll
      for (int e = 1; e < MAXL; ++e) {
        w[e] = 0.0;
        if (e < L) {
          const double inv = c_inv[e + 1];
#pragma unroll
          for (int i = e - 1; i >= 0; --i) {
            const double pw = w[i];
            w[i + 1] += o[e] * pw * (double)(i + 1) * inv;
            w[i] = z[e] * pw * (double)(e - i) * inv;
          }
        }
      }
      const int ud = L - 1;
      double wl = 0.0;
#pragma unroll
      for (int e = 0; e < MAXL; ++e)
        if (e == ud) wl = w[e];
      const double dn = (double)(ud + 1), idn = c_inv[ud + 1];
      // UNWOUND_SUM (unwound_path_sum, shap.rs:98-116) per element
#pragma unroll
      for (int e = 1; e < MAXL; ++e) {
        if (e < L) {
          const double oo = o[e], zz = z[e];
          double next = wl, total = 0.0;
#pragma unroll
          for (int i = MAXL - 2; i >= 0; --i) {
            if (i < ud) {
              if (oo != 0.0) {
                const double tmp = next * dn * c_inv[i + 1];
                total += tmp;
                next = w[i] - tmp * zz * (double)(ud - i) * idn;
              } else if (zz != 0.0) {
                total += w[i] * iz[e] * dn * c_inv[ud - i];
              }
            }
          }
          ph[fe[e] * R + tid] += (float)(total * (oo - zz) * leaf);
        }
      }
    }
  }
  if (r0 + tid < n) {
    double* a = acc + ((r0 + tid) * K + c) * (size_t)(F + 1);
    for (int j = 0; j < nfc; ++j) {
      const float v = ph[j * R + tid];
      if (v != 0.0f) atomicAdd(a + P.chunk_f[fo + j], (double)v);
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

// ------------------------------------------------- TreeSHAP interactions
// predict_interactions (shap.rs:395-509) restated per root-to-leaf path, on
// the same merged path elements as k_shap_paths. Conditioning the walk on
// feature j (tree_shap_cond with condition +1 / -1) keeps j's splits off the
// path and multiplies a leaf's weight by the condition fraction: o_j (the
// row follows all of j's splits) when present, z_j (their cover fractions)
// when absent. Paths without j give the same value both ways. So for a path
// holding j as element m, the half-difference of the two runs is, for every
// other element i:
//     0.5 * (o_m - z_m) * UNWOUND_SUM(P \ m, i) * (o_i - z_i) * leaf,
// added to M[j][f_i] and subtracted from M[j][j]; M[f][f] also gets the
// ordinary contribution of the full path. A block takes IR rows (1 or 2)
// and INTER_TREES trees of one class, accumulates the rows' (F+1)^2 matrices
// in f32 shared memory (threads over (path, row), shared atomics), and adds
// the non-zero cells into the f64 accumulator.
constexpr int INTER_THREADS = 256;
constexpr int INTER_TREES = 16;

struct InterDev {
  const PathEl* el;
  const int* off;
  const float* leaf;
  const int* tree_path;  // [T + 1] first path of each tree
  int T, K, F;
  int rows_per_block;
  unsigned row_blocks;
  int groups_per_class;
};

// UNWOUND_SUM (unwound_path_sum, shap.rs:98-116) of an element with
// one-fraction oo, zero-fraction zz (izz = 1 / zz) over weights w of a path
// whose last index is ud. inv[k] = 1 / k: a shared-memory copy, because the
// threads of a warp walk paths of different lengths and a constant-bank
// read at divergent addresses is serialised.
template <int MAXL>
__device__ __forceinline__ double unwound_sum(const double* w, int ud, double oo, double zz, double izz,
                                              const double* inv) {
  double wl = 0.0;
#pragma unroll
  for (int e = 0; e < MAXL; ++e)
    if (e == ud) wl = w[e];
  const double dn = (double)(ud + 1), idn = inv[ud + 1];
  double next = wl, total = 0.0;
#pragma unroll
  for (int i = MAXL - 2; i >= 0; --i) {
    if (i < ud) {
      if (oo != 0.0) {
        const double tmp = next * dn * c_inv[i + 1];
        total += tmp;
        next = w[i] - tmp * zz * (double)(ud - i) * idn;
      } else if (zz != 0.0) {
        total += w[i] * izz * dn * inv[ud - i];
      }
    }
  }
  return total;
}

template <int MAXL>
__global__ void __launch_bounds__(INTER_THREADS) k_shap_inter(InterDev P, const float* __restrict__ X, size_t n,
                                                              float missing, double* __restrict__ acc) {
  extern __shared__ float mat[];  // [IR][W][W]
  __shared__ int s_tree[INTER_TREES];
  __shared__ int s_pre[INTER_TREES + 1];
  __shared__ double s_inv[32];
  const int F = P.F, W = F + 1, WW = W * W, IR = P.rows_per_block;
  const unsigned rb = blockIdx.x % P.row_blocks;
  const unsigned g = blockIdx.x / P.row_blocks;
  const int c = (int)(g / (unsigned)P.groups_per_class), gi = (int)(g % (unsigned)P.groups_per_class);
  const size_t r0 = (size_t)rb * IR;
  for (int i = threadIdx.x; i < IR * WW; i += blockDim.x) mat[i] = 0.0f;
  if (threadIdx.x < 32) s_inv[threadIdx.x] = c_inv[threadIdx.x];
  if (threadIdx.x == 0) {
    int nt = 0, tot = 0;
    s_pre[0] = 0;
    for (int j = 0; j < INTER_TREES; ++j) {
      const long long t = (long long)c + (long long)P.K * ((long long)gi * INTER_TREES + j);
      if (t < P.T) {
        s_tree[nt] = (int)t;
        tot += P.tree_path[t + 1] - P.tree_path[t];
        s_pre[++nt] = tot;
      }
    }
    for (int j = nt + 1; j <= INTER_TREES; ++j) s_pre[j] = tot;
  }
  __syncthreads();
  const int total = s_pre[INTER_TREES];
  const bool miss_nan = isnan(missing);
  for (int it = threadIdx.x; it < total * IR; it += blockDim.x) {
    const int q = it / IR, ri = it - q * IR;
    const size_t r = r0 + ri;
    if (r >= n) continue;
    int j = 0;
    while (q >= s_pre[j + 1]) ++j;
    const int p = P.tree_path[s_tree[j]] + (q - s_pre[j]);
    const int e0 = P.off[p], L = P.off[p + 1] - e0;
    const double leaf = (double)P.leaf[p];
    const float* row = X + r * (size_t)F;
    float* M = mat + ri * WW;
    double z[MAXL], iz[MAXL], o[MAXL], w[MAXL];
    int fe[MAXL];
#pragma unroll
    for (int e = 0; e < MAXL; ++e) {
      fe[e] = 0;
      z[e] = 1.0;
      iz[e] = 1.0;
      o[e] = 1.0;
      if (e < L) {
        const PathEl el = P.el[e0 + e];
        fe[e] = el.f < 0 ? 0 : el.f;
        z[e] = el.z;
        iz[e] = el.inv_z;
        if (el.f >= 0) {
          const float v = __ldg(row + el.f);
          const bool mis = miss_nan ? isnan(v) : v == missing;
          o[e] = (mis ? el.miss_ok != 0 : (v >= el.lo && v < el.hi)) ? 1.0 : 0.0;
        }
      }
    }
    // the full path: ordinary contributions on the diagonal
    w[0] = 1.0;
#pragma unroll
    for (int e = 1; e < MAXL; ++e) {
      w[e] = 0.0;
      if (e < L) {
        const double inv = c_inv[e + 1];
#pragma unroll
        for (int i = e - 1; i >= 0; --i) {
          const double pw = w[i];
          w[i + 1] += o[e] * pw * (double)(i + 1) * inv;
          w[i] = z[e] * pw * (double)(e - i) * inv;
        }
      }
    }
#pragma unroll
    for (int e = 1; e < MAXL; ++e)
      if (e < L) {
        const double v = unwound_sum<MAXL>(w, L - 1, o[e], z[e], iz[e], s_inv) * (o[e] - z[e]) * leaf;
        if (v != 0.0) atomicAdd(M + fe[e] * W + fe[e], (float)v);
      }
    // conditioned on element m's feature: the path without m. The m loop is
    // not unrolled: unrolling all three loop levels made the kernel larger
    // than the instruction cache (ncu: "no instruction" was the top stall).
    // Element m's values are picked with static indices, so the arrays stay
    // in registers.
#pragma unroll 1
    for (int m = 1; m < L; ++m) {
      double zm = 1.0, om = 1.0;
      int fm = 0;
#pragma unroll
      for (int e = 1; e < MAXL; ++e)
        if (e == m) {
          zm = z[e];
          om = o[e];
          fm = fe[e];
        }
      const double dm = om - zm;
      if (dm == 0.0) continue;
      double w2[MAXL];
      w2[0] = 1.0;
#pragma unroll
      for (int k = 1; k < MAXL - 1; ++k) {
        w2[k] = 0.0;
        if (k < L - 1) {
          const bool after = k >= m;  // reduced position k holds element k + 1
          const double ok = after ? o[k + 1] : o[k], zk = after ? z[k + 1] : z[k];
          const double inv = c_inv[k + 1];
#pragma unroll
          for (int i = k - 1; i >= 0; --i) {
            const double pw = w2[i];
            w2[i + 1] += ok * pw * (double)(i + 1) * inv;
            w2[i] = zk * pw * (double)(k - i) * inv;
          }
        }
      }
      w2[MAXL - 1] = 0.0;
      double dsum = 0.0;
      const int row_m = fm * W;
#pragma unroll
      for (int k = 1; k < MAXL - 1; ++k) {
        if (k < L - 1) {
          const bool after = k >= m;
          const double ok = after ? o[k + 1] : o[k], zk = after ? z[k + 1] : z[k];
          const double izk = after ? iz[k + 1] : iz[k];
          const int fk = after ? fe[k + 1] : fe[k];
          const double val = 0.5 * dm * unwound_sum<MAXL>(w2, L - 2, ok, zk, izk, s_inv) * (ok - zk) * leaf;
          if (val != 0.0) {
            atomicAdd(M + row_m + fk, (float)val);
            dsum += val;
          }
        }
      }
      if (dsum != 0.0) atomicAdd(M + row_m + fm, (float)(-dsum));
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < IR * WW; i += blockDim.x) {
    const int ri = i / WW;
    const size_t r = r0 + ri;
    const float v = mat[i];
    if (r < n && v != 0.0f) atomicAdd(acc + (r * P.K + c) * (size_t)WW + (i - ri * WW), (double)v);
  }
}

// f64 accumulator -> f32 output; the [F][F] cell of each (row, class) is the
// class's sum of tree expected values (no base score).
__global__ void k_inter_finish(const double* __restrict__ acc, const double* __restrict__ bias, size_t n, int K,
                               int F, float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t W = (size_t)F + 1, WW = W * W;
  if (i >= n * K * WW) return;
  const size_t cell = i % WW;
  const size_t c = (i / WW) % K;
  out[i] = cell == (size_t)F * W + F ? (float)bias[c] : (float)acc[i];
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
  // TreeSHAP paths: per leaf, its merged path elements
  std::vector<PathEl> pel;
  std::vector<int> poff(1, 0), tpath(1, 0);
  std::vector<float> pleaf;
  int maxlen = 1;
  for (int t = 0; t < T; ++t) {
    const HostTree& tr = m->trees[t];
    struct Frame {
      int nid;
      std::vector<PathEl> el;
    };
    std::vector<Frame> stack;
    PathEl bias{-1, 1, -INFINITY, INFINITY, 1.0, 1.0};
    stack.push_back(Frame{0, {bias}});
    while (!stack.empty() && !tr.nodes.empty()) {
      Frame fr = std::move(stack.back());
      stack.pop_back();
      const sb_node& nd = tr.nodes[fr.nid];
      if (nd.left < 0) {
        for (PathEl& e : fr.el) e.inv_z = e.z != 0.0 ? 1.0 / e.z : 0.0;
        pel.insert(pel.end(), fr.el.begin(), fr.el.end());
        poff.push_back((int)pel.size());
        pleaf.push_back(nd.leaf_value);
        maxlen = std::max(maxlen, (int)fr.el.size());
        continue;
      }
      const double cover = (double)nd.sum_hess;
      for (int side = 0; side < 2; ++side) {
        const int child = side == 0 ? nd.left : nd.right;
        const double zf = cover > 0.0 ? (double)tr.nodes[child].sum_hess / cover : 0.0;
        Frame nx{child, fr.el};
        size_t e = 1;
        while (e < nx.el.size() && nx.el[e].f != (int)nd.split_feature) ++e;
        if (e == nx.el.size()) nx.el.push_back(PathEl{(int)nd.split_feature, 1, -INFINITY, INFINITY, 1.0, 1.0});
        PathEl& el = nx.el[e];
        el.z *= zf;  // cover fraction of this split, times the earlier ones
        if (side == 0) {  // v < cond, or missing when default_left
          el.hi = std::min(el.hi, nd.split_cond);
          el.miss_ok = el.miss_ok && nd.default_left;
        } else {
          el.lo = std::max(el.lo, nd.split_cond);
          el.miss_ok = el.miss_ok && !nd.default_left;
        }
        stack.push_back(std::move(nx));
      }
    }
    tpath.push_back((int)pleaf.size());
  }
  SB_TRY(D.path_el.alloc(ctx, std::max<size_t>(pel.size(), 1)));
  SB_TRY(D.path_off.alloc(ctx, poff.size()));
  SB_TRY(D.path_leaf.alloc(ctx, std::max<size_t>(pleaf.size(), 1)));
  SB_TRY(D.tree_path.alloc(ctx, tpath.size()));
  if (!pel.empty())
    SB_CUDA(cudaMemcpyAsync(D.path_el.p, pel.data(), pel.size() * sizeof(PathEl), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(D.path_off.p, poff.data(), poff.size() * 4, cudaMemcpyHostToDevice, st));
  if (!pleaf.empty())
    SB_CUDA(cudaMemcpyAsync(D.path_leaf.p, pleaf.data(), pleaf.size() * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(D.tree_path.p, tpath.data(), tpath.size() * 4, cudaMemcpyHostToDevice, st));
  std::vector<int4> chunks;  // <= SHAP_CHUNK paths of one tree each
  const int Kc = m->num_class >= 2 ? m->num_class : 1;
  for (int t = 0; t < T; ++t)
    for (int p0 = tpath[t]; p0 < tpath[t + 1]; p0 += SHAP_CHUNK)
      chunks.push_back(make_int4(t % Kc, p0, std::min(p0 + SHAP_CHUNK, tpath[t + 1]), 0));
  SB_TRY(D.shap_chunk.alloc(ctx, std::max<size_t>(chunks.size(), 1)));
  if (!chunks.empty())
    SB_CUDA(cudaMemcpyAsync(D.shap_chunk.p, chunks.data(), chunks.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
  D.n_shap_chunks = (int)chunks.size();
  {  // per chunk, its paths' distinct features and each element's index among them
    std::vector<int> pfc(pel.size(), -1), cfo(1, 0), cf, slot(std::max(m->n_features, 1), -1);
    int maxfc = 1;
    for (const int4& chk : chunks) {
      const int first = (int)cf.size();
      for (int p = chk.y; p < chk.z; ++p)
        for (int e = poff[p]; e < poff[p + 1]; ++e) {
          const int f = pel[e].f;
          if (f < 0) continue;
          if (slot[f] < 0) {
            slot[f] = (int)cf.size() - first;
            cf.push_back(f);
          }
          pfc[e] = slot[f];
        }
      for (size_t j = first; j < cf.size(); ++j) slot[cf[j]] = -1;
      cfo.push_back((int)cf.size());
      maxfc = std::max(maxfc, (int)cf.size() - first);
    }
    SB_TRY(D.path_fc.alloc(ctx, std::max<size_t>(pfc.size(), 1)));
    SB_TRY(D.chunk_fo.alloc(ctx, cfo.size()));
    SB_TRY(D.chunk_f.alloc(ctx, std::max<size_t>(cf.size(), 1)));
    if (!pfc.empty())
      SB_CUDA(cudaMemcpyAsync(D.path_fc.p, pfc.data(), pfc.size() * 4, cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemcpyAsync(D.chunk_fo.p, cfo.data(), cfo.size() * 4, cudaMemcpyHostToDevice, st));
    if (!cf.empty()) SB_CUDA(cudaMemcpyAsync(D.chunk_f.p, cf.data(), cf.size() * 4, cudaMemcpyHostToDevice, st));
    D.shap_max_fc = maxfc;
  }
  {  // shared memory of the TreeSHAP blocks: f32 partials of SHAP_ROWS rows
    const int smem = (int)std::min<size_t>((size_t)m->n_features * SHAP_ROWS * 4, ctx->smem_optin);
    SB_TRY(raise_smem_limit((const void*)k_shap_paths<5>, (size_t)smem));
    SB_TRY(raise_smem_limit((const void*)k_shap_paths<9>, (size_t)smem));
    SB_TRY(raise_smem_limit((const void*)k_shap_paths<SHAP_MAXD + 1>, (size_t)smem));
  }
  D.max_path_len = maxlen;
  {
    double inv[32];
    inv[0] = 0.0;
    for (int k = 1; k < 32; ++k) inv[k] = 1.0 / (double)k;
    SB_CUDA(cudaMemcpyToSymbolAsync(c_inv, inv, sizeof(inv), 0, cudaMemcpyHostToDevice, st));
  }
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

// TreeSHAP contributions of n rows into d_acc ([n][K][F+1] doubles, zeroed
// here) on stream st.
int shap_paths(sb_model* m, cudaStream_t st, const float* d_X, size_t n, size_t F, float missing,
               double* d_acc) {
  sb_ctx* ctx = m->ctx;
  SB_REQUIRE(m->dev.max_depth <= SHAP_MAXD, SB_ERR_UNSUPPORTED,
             "TreeSHAP on the device supports trees up to depth %d (got %d)", SHAP_MAXD, m->dev.max_depth);
  const int K = m->num_class >= 2 ? m->num_class : 1;
  const int T = m->dev.n_trees;
  SB_CUDA(cudaMemsetAsync(d_acc, 0, n * K * (F + 1) * sizeof(double), st));
  if (T == 0 || n == 0) return SB_OK;
  const int R = SHAP_ROWS;
  const size_t smem = (size_t)m->dev.shap_max_fc * R * 4;
  SB_REQUIRE(smem <= ctx->smem_optin, SB_ERR_UNSUPPORTED,
             "TreeSHAP on the device supports up to %zu distinct features per %d paths of a tree",
             ctx->smem_optin / (4 * R), SHAP_CHUNK);
  ShapPathsDev P;
  P.el = m->dev.path_el.p;
  P.off = m->dev.path_off.p;
  P.leaf = m->dev.path_leaf.p;
  P.chunk = m->dev.shap_chunk.p;
  P.fc = m->dev.path_fc.p;
  P.chunk_fo = m->dev.chunk_fo.p;
  P.chunk_f = m->dev.chunk_f.p;
  const unsigned row_blocks = (unsigned)((n + R - 1) / R);
  SB_REQUIRE((uint64_t)row_blocks * m->dev.n_shap_chunks < (1ull << 31), SB_ERR_UNSUPPORTED,
             "TreeSHAP of %zu rows over %d path chunks exceeds one launch", n, m->dev.n_shap_chunks);
  const unsigned grid = row_blocks * (unsigned)m->dev.n_shap_chunks;
  const int L = m->dev.max_path_len;
  if (L <= 5)
    SB_LAUNCH_ON(ctx, st, k_shap_paths<5>, grid, R, smem, P, d_X, n, (int)F, K, missing, row_blocks, d_acc);
  else if (L <= 9)
    SB_LAUNCH_ON(ctx, st, k_shap_paths<9>, grid, R, smem, P, d_X, n, (int)F, K, missing, row_blocks, d_acc);
  else
    SB_LAUNCH_ON(ctx, st, k_shap_paths<SHAP_MAXD + 1>, grid, R, smem, P, d_X, n, (int)F, K, missing, row_blocks,
                 d_acc);
  return SB_OK;
}

int predict_contribs_device(sb_model* m, const float* d_X, size_t n, size_t F, float missing,
                            float* d_out) {
  sb_ctx* ctx = m->ctx;
  SB_TRY(model_upload(m));
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
  SB_TRY(acc.alloc(ctx, std::max<size_t>(n * K * width, 1)));
  SB_TRY(shap_paths(m, ctx->stream, d_X, n, F, missing, acc.p));
  size_t tot = n * K * width;
  if (tot) SB_LAUNCH(ctx, k_shap_finish, (unsigned)((tot + 255) / 256), 256, 0, acc.p, d_bias.p, n, K, (int)F, d_out);
  return SB_OK;
}

// Interaction values of n rows into d_out ([n][K][F+1][F+1] floats).
int predict_interactions_device(sb_model* m, const float* d_X, size_t n, size_t F, float missing,
                                float* d_out) {
  sb_ctx* ctx = m->ctx;
  SB_TRY(model_upload(m));
  SB_REQUIRE(m->dev.max_depth <= SHAP_MAXD, SB_ERR_UNSUPPORTED,
             "TreeSHAP on the device supports trees up to depth %d (got %d)", SHAP_MAXD, m->dev.max_depth);
  const int K = m->num_class >= 2 ? m->num_class : 1;
  const int T = m->dev.n_trees;
  const size_t W = F + 1, WW = W * W;
  const size_t room = ctx->smem_optin > 1024 ? ctx->smem_optin - 1024 : 0;  // less the static shared memory
  const int IR = 2 * WW * 4 <= room ? 2 : 1;
  SB_REQUIRE((size_t)IR * WW * 4 <= room, SB_ERR_UNSUPPORTED,
             "interaction values on the device support up to %d features",
             (int)std::sqrt((double)(room / 4)) - 1);
  const size_t smem = (size_t)IR * WW * 4;
  SB_TRY(raise_smem_limit((const void*)k_shap_inter<5>, smem));
  SB_TRY(raise_smem_limit((const void*)k_shap_inter<9>, smem));
  SB_TRY(raise_smem_limit((const void*)k_shap_inter<SHAP_MAXD + 1>, smem));
  // [F][F] cell per class: the sum of its trees' expected values (shap.rs:427-437)
  std::vector<double> bias(K, 0.0);
  for (int t = 0; t < T; ++t) bias[t % K] += node_mean_value(m->trees[t], 0);
  DBuf<double> d_bias, acc;
  SB_TRY(d_bias.alloc(ctx, K));
  SB_CUDA(cudaMemcpyAsync(d_bias.p, bias.data(), K * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (n == 0) return SB_OK;
  // rows per pass: the f64 accumulator stays <= 256 MB
  size_t chunk = std::max<size_t>((size_t)IR, (size_t)(256ull << 20) / ((size_t)K * WW * 8));
  chunk = std::min(chunk, n);
  SB_TRY(acc.alloc(ctx, chunk * K * WW));
  InterDev P;
  P.el = m->dev.path_el.p;
  P.off = m->dev.path_off.p;
  P.leaf = m->dev.path_leaf.p;
  P.tree_path = m->dev.tree_path.p;
  P.T = T;
  P.K = K;
  P.F = (int)F;
  P.rows_per_block = IR;
  const int per_class = (T + K - 1) / K;
  P.groups_per_class = std::max(1, (per_class + INTER_TREES - 1) / INTER_TREES);
  const int L = m->dev.max_path_len;
  for (size_t r0 = 0; r0 < n; r0 += chunk) {
    const size_t nb = std::min(chunk, n - r0);
    SB_CUDA(cudaMemsetAsync(acc.p, 0, nb * K * WW * 8, ctx->stream));
    P.row_blocks = (unsigned)((nb + IR - 1) / IR);
    const uint64_t blocks = (uint64_t)P.row_blocks * (uint64_t)K * (uint64_t)P.groups_per_class;
    SB_REQUIRE(blocks < (1ull << 31), SB_ERR_UNSUPPORTED, "interaction values: %llu blocks exceed one launch",
               (unsigned long long)blocks);
    if (T > 0) {
      const float* X = d_X + r0 * F;
      if (L <= 5)
        SB_LAUNCH(ctx, k_shap_inter<5>, (unsigned)blocks, INTER_THREADS, smem, P, X, nb, missing, acc.p);
      else if (L <= 9)
        SB_LAUNCH(ctx, k_shap_inter<9>, (unsigned)blocks, INTER_THREADS, smem, P, X, nb, missing, acc.p);
      else
        SB_LAUNCH(ctx, k_shap_inter<SHAP_MAXD + 1>, (unsigned)blocks, INTER_THREADS, smem, P, X, nb, missing,
                  acc.p);
    }
    const size_t tot = nb * K * WW;
    SB_LAUNCH(ctx, k_inter_finish, (unsigned)((tot + 255) / 256), 256, 0, acc.p, d_bias.p, nb, K, (int)F,
              d_out + r0 * K * WW);
  }
  return SB_OK;
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
  const int K = m->num_class >= 2 ? m->num_class : 1;
  const size_t tot = n * K * (F + 1);
  SB_TRY(shap_paths(m, st, d_X, n, F, missing, d_acc));
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
