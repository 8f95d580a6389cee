// sb_shap.cu — TreeSHAP on the device (K10): predict_contribs and
// predict_interactions.
//
// Replaces BoostedModel::predict_contribs with tree_shap_cond, extend_path,
// unwind_path and unwound_path_sum (learner/shap.rs:49-367) and
// predict_interactions (learner/shap.rs:395-509).
//
// This file is compiled with multiply-add contraction allowed: TreeSHAP's
// tolerance is 1e-4 and its additivity (contributions sum to the margin) is
// checked within that, while margins and split gains, which must round as the
// reference rounds, live in files compiled without contraction.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "sb_internal.cuh"

namespace sb {
namespace {

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
constexpr int SHAP_REG_MAXL = 13;  // longest path (elements) of the register forms
constexpr size_t SHAP_TABLE_BUDGET = 4ull << 30;  // most bytes of per-path tables
constexpr int SHAP_ROWS = 128;
constexpr int SHAP_CHUNK = 64;  // paths per block

constexpr int INV_N = 64;
__constant__ double c_inv[INV_N];  // 1 / k (0 at k = 0)

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
constexpr int SHAP_INTER_MAXL = 33;  // longest path (elements) of interaction values
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
  __shared__ double s_inv[INV_N];
  const int F = P.F, W = F + 1, WW = W * W, IR = P.rows_per_block;
  const unsigned rb = blockIdx.x % P.row_blocks;
  const unsigned g = blockIdx.x / P.row_blocks;
  const int c = (int)(g / (unsigned)P.groups_per_class), gi = (int)(g % (unsigned)P.groups_per_class);
  const size_t r0 = (size_t)rb * IR;
  for (int i = threadIdx.x; i < IR * WW; i += blockDim.x) mat[i] = 0.0f;
  for (int i = threadIdx.x; i < INV_N; i += blockDim.x) s_inv[i] = c_inv[i];
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

// ------------------------------------------------ per-path contribution tables
// For a path of L elements (the bias and D = L - 1 merged features), a row's
// contributions depend only on its pattern of one-fractions: bit e - 1 of the
// pattern m is o of element e. For paths with D <= SHAP_TABLE_MAXD the device
// precomputes, for every pattern, the f32 contribution of each element
// (UNWOUND_SUM * (o - z) * leaf, the value k_shap_paths adds), as a table
// [2^D][Dp] (Dp = D rounded up to a multiple of 4, zero padded). A row then
// costs its pattern and D table reads per path instead of O(L^2) f64 work:
// the precomputation of Fast TreeSHAP v2 (Yang, 2021), taken to the full
// per-pattern result.
constexpr int SHAP_TABLE_MAXD = 10;

struct ShapTableDev {
  const PathEl* el;
  const int* off;
  const float* leaf;
  const long long* tab_off;   // per path: first float of its table
  const long long* mask_off;  // per path: first (path, pattern) pair, [n_paths + 1]
  int n_paths;
  float* tab;
};

// One thread per (path, pattern) pair.
__global__ void __launch_bounds__(128) k_shap_table_build(ShapTableDev P, long long pairs) {
  constexpr int MAXL = SHAP_TABLE_MAXD + 1;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < pairs;
       q += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = P.n_paths;  // last path with mask_off <= q
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (P.mask_off[mid] <= q) lo = mid; else hi = mid;
    }
    const int p = lo;
    const unsigned m = (unsigned)(q - P.mask_off[p]);
    const int e0 = P.off[p], L = P.off[p + 1] - e0, D = L - 1, Dp = (D + 3) & ~3;
    const double leaf = (double)P.leaf[p];
    double w[MAXL], z[MAXL], iz[MAXL], o[MAXL];
#pragma unroll
    for (int e = 0; e < MAXL; ++e) {
      z[e] = 1.0;
      iz[e] = 1.0;
      o[e] = 1.0;
      if (e >= 1 && e < L) {
        const PathEl el = P.el[e0 + e];
        z[e] = el.z;
        iz[e] = el.inv_z;
        o[e] = ((m >> (e - 1)) & 1u) ? 1.0 : 0.0;
      }
    }
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
    float* out = P.tab + P.tab_off[p] + (long long)m * Dp;
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
        out[e - 1] = (float)(total * (oo - zz) * leaf);
      }
    }
    for (int j = D; j < Dp; ++j) out[j] = 0.0f;
  }
}

// The table form: a block takes TAB_ROWS rows (one per thread) over one
// table chunk, up to TAB_CHUNK_PATHS paths of several trees of one class,
// so that the block's partials go to the f64 accumulator once per many
// trees. The block first copies its rows' values of the chunk's features
// into shared memory, feature-major with a padded stride, so that the
// per-element reads of a warp (one feature, 32 rows) are one conflict-free
// shared access instead of 32 scattered row reads. Per path a row forms its
// pattern from the path's compact elements and adds the D table entries of
// it; four independent paths are in flight per step.
constexpr int TAB_ROWS = 64;
constexpr int TAB_STRIDE = TAB_ROWS + 1;  // words per feature in the row-value copy
constexpr int TAB_CHUNK_PATHS = 1024;
constexpr int TAB_CHUNK_FEATURES = 192;  // distinct features of a chunk (its partial's rows)
constexpr int TAB_TPR = 8;               // threads per row
constexpr int TAB_ILP = 1;               // paths in flight per thread

// Shared memory of one k_shap_table block for a chunk of `nfc` features:
// the f32 partials [nfc][TAB_ROWS] and the row values [nfc][TAB_STRIDE].
__host__ __device__ constexpr size_t shap_table_smem(int nfc) {
  return (size_t)nfc * (TAB_ROWS + TAB_STRIDE) * sizeof(float);
}

struct ShapTabDev {
  const int4* el;           // per element: {feature, lo bits, hi bits, (chunk feature index << 1) | miss_ok}
  const int4* head;         // per path: {first element, elements, table offset (two 32-bit halves)}
  const float* tab;
  const int* tree_path;     // [n_trees + 1]
  const int4* chunk;        // {class, first tree, number of trees, -}; trees t, t + K, t + 2K, ...
  const int* chunk_fo;      // [n_chunks + 1] offsets into chunk_f
  const int* chunk_f;       // each chunk's distinct features
  int K;
};

template <int TPR, int ILP>
__global__ void __launch_bounds__(TAB_ROWS * TPR, 2048 / (TAB_ROWS * TPR))
k_shap_table(ShapTabDev P, const float* __restrict__ X, size_t n, int F, float missing, unsigned row_blocks,
             double* __restrict__ acc) {
  extern __shared__ float ph[];  // [chunk features][TAB_ROWS], then xs
  const int R = TAB_ROWS;
  const int tid = threadIdx.x;
  const int row = tid % R, grp = tid / R;  // a row's TPR threads take every TPR-th group of paths
  const unsigned rb = blockIdx.x % row_blocks;
  const size_t r0 = (size_t)rb * R;
  const unsigned ci = blockIdx.x / row_blocks;
  const int4 ch = P.chunk[ci];
  const int c = ch.x;
  const int fo = P.chunk_fo[ci], nfc = P.chunk_fo[ci + 1] - fo;
  float* xs = ph + (size_t)nfc * R;  // [chunk features][TAB_STRIDE] row values
  for (int i = tid; i < nfc * R; i += blockDim.x) ph[i] = 0.0f;
  // consecutive threads read consecutive chunk features of one row
  const int rows_here = (int)min((size_t)R, n - r0);
  for (int i = tid; i < nfc * rows_here; i += blockDim.x) {
    const int r = i / nfc, j = i - r * nfc;
    xs[j * TAB_STRIDE + r] = __ldg(X + (r0 + r) * (size_t)F + P.chunk_f[fo + j]);
  }
  __syncthreads();
  const bool miss_nan = isnan(missing);
  const float* xr = xs + row;
  float* pr = ph + row;
  for (int ti = 0; ti < ch.z; ++ti) {
    const int t = ch.y + ti * P.K;
    const int pe = P.tree_path[t + 1];
    for (int p0 = P.tree_path[t] + grp * ILP; p0 < pe; p0 += TPR * ILP) {
      // ILP paths at a time, every element loop unrolled to the table depth
      // limit, so that all their element and table loads are in flight
      // together; each element's chunk-feature index stays in a register for
      // the partial updates.
      int4 hd[ILP];
#pragma unroll
      for (int u = 0; u < ILP; ++u) hd[u] = p0 + u < pe ? __ldg(P.head + p0 + u) : make_int4(0, 0, 0, 0);
      unsigned m[ILP];
      int fc[ILP][SHAP_TABLE_MAXD];
#pragma unroll
      for (int u = 0; u < ILP; ++u) m[u] = 0u;
#pragma unroll
      for (int e = 0; e < SHAP_TABLE_MAXD; ++e) {
#pragma unroll
        for (int u = 0; u < ILP; ++u) {
          fc[u][e] = 0;
          if (e < hd[u].y) {
            const int4 x = __ldg(P.el + hd[u].x + e);
            fc[u][e] = x.w >> 1;
            const float v = xr[(x.w >> 1) * TAB_STRIDE];
            const bool mis = miss_nan ? isnan(v) : v == missing;
            const bool o = mis ? (x.w & 1) != 0 : (v >= __int_as_float(x.y) && v < __int_as_float(x.z));
            m[u] |= (o ? 1u : 0u) << e;
          }
        }
      }
      float4 tv[ILP][3];
#pragma unroll
      for (int u = 0; u < ILP; ++u) {  // the table entries of the patterns
        const int dn = hd[u].y, dp = (dn + 3) & ~3;
        const long long toff = (long long)(((unsigned long long)(uint32_t)hd[u].w << 32) | (uint32_t)hd[u].z);
        const float4* t4 = reinterpret_cast<const float4*>(P.tab + toff + (long long)m[u] * dp);
#pragma unroll
        for (int j = 0; j < 3; ++j) tv[u][j] = 4 * j < dn ? __ldg(t4 + j) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < ILP; ++u) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const float vv[4] = {tv[u][j].x, tv[u][j].y, tv[u][j].z, tv[u][j].w};
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (4 * j + q < SHAP_TABLE_MAXD && 4 * j + q < hd[u].y) {
              if (TPR == 1) pr[fc[u][4 * j + q] * R] += vv[q];
              else atomicAdd(pr + fc[u][4 * j + q] * R, vv[q]);  // the row's other threads add too
            }
        }
      }
    }
  }
  __syncthreads();
  if (r0 + row < n) {
    const int Kc = P.K;
    double* a = acc + ((r0 + row) * Kc + c) * (size_t)(F + 1);
    for (int j = grp; j < nfc; j += TPR) {
      const float v = ph[j * R + row];
      if (v != 0.0f) atomicAdd(a + P.chunk_f[fo + j], (double)v);
    }
  }
}

// ------------------------------------------------------------- deep paths
// k_shap_paths for paths longer than its register forms hold: the same
// arithmetic with each thread's w, z, 1/z and o arrays in a global scratch
// buffer ([4][LM][threads], coalesced across a warp), and 1 / k computed. A
// persistent grid walks the (path chunk, row block) work items.
__global__ void __launch_bounds__(SHAP_ROWS) k_shap_deep(ShapPathsDev P, const float* __restrict__ X, size_t n,
                                                        int F, int K, float missing, unsigned row_blocks,
                                                        unsigned long long items, int LM,
                                                        double* __restrict__ scratch, double* __restrict__ acc) {
  extern __shared__ float ph[];
  const int R = SHAP_ROWS;
  const int tid = threadIdx.x;
  const size_t nthr = (size_t)gridDim.x * R;
  const size_t gt = (size_t)blockIdx.x * R + tid;
  double* w = scratch + gt;
  double* z = scratch + (size_t)LM * nthr + gt;
  double* iz = scratch + 2 * (size_t)LM * nthr + gt;
  double* o = scratch + 3 * (size_t)LM * nthr + gt;
#define SB_AT(a, e) a[(size_t)(e) * nthr]
  const bool miss_nan = isnan(missing);
  for (unsigned long long b = blockIdx.x; b < items; b += gridDim.x) {
    const unsigned rb = (unsigned)(b % row_blocks);
    const size_t r0 = (size_t)rb * R;
    const unsigned ci = (unsigned)(b / row_blocks);
    const int4 ch = P.chunk[ci];
    const int c = ch.x;
    const int fo = P.chunk_fo[ci], nfc = P.chunk_fo[ci + 1] - fo;
    __syncthreads();  // the previous item's partials are flushed
    for (int i = tid; i < nfc * R; i += R) ph[i] = 0.0f;
    __syncthreads();
    const float* row = X + (r0 + tid < n ? r0 + tid : r0) * (size_t)F;
    for (int p = ch.y; p < ch.z; ++p) {
      const int e0 = P.off[p], L = P.off[p + 1] - e0;
      const double leaf = (double)P.leaf[p];
      for (int e = 0; e < L; ++e) {
        const PathEl el = P.el[e0 + e];
        SB_AT(z, e) = el.z;
        SB_AT(iz, e) = el.inv_z;
        double oe = 1.0;
        if (el.f >= 0) {
          const float v = __ldg(row + el.f);
          const bool mis = miss_nan ? isnan(v) : v == missing;
          oe = (mis ? el.miss_ok != 0 : (v >= el.lo && v < el.hi)) ? 1.0 : 0.0;
        }
        SB_AT(o, e) = oe;
      }
      SB_AT(w, 0) = 1.0;
      for (int e = 1; e < L; ++e) {  // EXTEND, shap.rs:49-68
        SB_AT(w, e) = 0.0;
        const double inv = 1.0 / (double)(e + 1);
        const double oe = SB_AT(o, e), ze = SB_AT(z, e);
        for (int i = e - 1; i >= 0; --i) {
          const double pw = SB_AT(w, i);
          SB_AT(w, i + 1) += oe * pw * (double)(i + 1) * inv;
          SB_AT(w, i) = ze * pw * (double)(e - i) * inv;
        }
      }
      const int ud = L - 1;
      const double wl = SB_AT(w, ud);
      const double dn = (double)(ud + 1), idn = 1.0 / dn;
      for (int e = 1; e < L; ++e) {  // UNWOUND_SUM, shap.rs:98-116
        const double oo = SB_AT(o, e), zz = SB_AT(z, e), izz = SB_AT(iz, e);
        double next = wl, total = 0.0;
        for (int i = ud - 1; i >= 0; --i) {
          if (oo != 0.0) {
            const double tmp = next * dn / (double)(i + 1);
            total += tmp;
            next = SB_AT(w, i) - tmp * zz * (double)(ud - i) * idn;
          } else if (zz != 0.0) {
            total += SB_AT(w, i) * izz * dn / (double)(ud - i);
          }
        }
        ph[P.fc[e0 + e] * R + tid] += (float)(total * (oo - zz) * leaf);
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
#undef SB_AT
}

}  // namespace

// The TreeSHAP state of a model, built once: per leaf its merged path
// elements, path chunks with their distinct features, and, when every path
// has at most SHAP_TABLE_MAXD features and the tables fit the memory budget,
// the per-path contribution tables.
int shap_prepare(sb_model* m) {
  SB_TRY(model_upload(m));
  DevEnsemble& D = m->dev;
  if (D.shap_valid) return SB_OK;
  sb_ctx* ctx = m->ctx;
  cudaStream_t st = ctx->stream;
  const int T = (int)m->trees.size();
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
  const int n_paths = (int)pleaf.size();
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
  std::vector<int> pfc(pel.size(), -1), cfo(1, 0), cf;
  {  // per chunk, its paths' distinct features and each element's index among them
    std::vector<int> slot(std::max(m->n_features, 1), -1);
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
  D.max_path_len = maxlen;
  {
    double inv[INV_N];
    inv[0] = 0.0;
    for (int k = 1; k < INV_N; ++k) inv[k] = 1.0 / (double)k;
    SB_CUDA(cudaMemcpyToSymbolAsync(c_inv, inv, sizeof(inv), 0, cudaMemcpyHostToDevice, st));
  }
  {  // shared memory of the TreeSHAP blocks: f32 partials of SHAP_ROWS rows
    const size_t smem = std::min<size_t>((size_t)D.shap_max_fc * SHAP_ROWS * 4, ctx->smem_optin);
    SB_TRY(raise_smem_limit((const void*)k_shap_paths<5>, smem));
    SB_TRY(raise_smem_limit((const void*)k_shap_paths<9>, smem));
    SB_TRY(raise_smem_limit((const void*)k_shap_paths<SHAP_REG_MAXL>, smem));
    SB_TRY(raise_smem_limit((const void*)k_shap_deep, smem));
  }
  // per-path tables: 2^D patterns x Dp floats each
  D.shap_table = false;
  D.shap_tab.release();
  D.shap_tab_off.release();
  if (maxlen - 1 <= SHAP_TABLE_MAXD && n_paths > 0) {
    std::vector<long long> toff(n_paths), moff(n_paths + 1, 0);
    long long floats = 0;
    for (int p = 0; p < n_paths; ++p) {
      const int Dn = poff[p + 1] - poff[p] - 1, Dp = (Dn + 3) & ~3;
      toff[p] = floats;
      floats += (1ll << Dn) * Dp;
      moff[p + 1] = moff[p] + (1ll << Dn);
    }
    size_t free_b = 0, total_b = 0;
    SB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = std::min<size_t>(SHAP_TABLE_BUDGET, free_b / 4);
    if ((size_t)floats * 4 <= budget) {
      DBuf<long long> d_moff;
      SB_TRY(D.shap_tab.alloc(ctx, std::max<long long>(floats, 4)));
      SB_TRY(D.shap_tab_off.alloc(ctx, n_paths));
      SB_TRY(d_moff.alloc(ctx, n_paths + 1));
      SB_CUDA(cudaMemcpyAsync(D.shap_tab_off.p, toff.data(), n_paths * 8, cudaMemcpyHostToDevice, st));
      SB_CUDA(cudaMemcpyAsync(d_moff.p, moff.data(), (n_paths + 1) * 8, cudaMemcpyHostToDevice, st));
      ShapTableDev P;
      P.el = D.path_el.p;
      P.off = D.path_off.p;
      P.leaf = D.path_leaf.p;
      P.tab_off = D.shap_tab_off.p;
      P.mask_off = d_moff.p;
      P.n_paths = n_paths;
      P.tab = D.shap_tab.p;
      const long long pairs = moff[n_paths];
      const unsigned blocks = (unsigned)std::min<long long>((pairs + 127) / 128, (long long)ctx->num_sms * 64);
      SB_LAUNCH(ctx, k_shap_table_build, blocks, 128, 0, P, pairs);
      // table chunks: consecutive trees of one class, up to TAB_CHUNK_PATHS
      // paths and TAB_CHUNK_FEATURES distinct features
      std::vector<int4> tch;
      std::vector<int> tfo(1, 0), tf, tslot(std::max(m->n_features, 1), -1);
      std::vector<int4> tel(pel.size());
      int tmax = 1;
      for (int c = 0; c < Kc; ++c) {
        int t = c;
        while (t < T) {
          const int first = (int)tf.size();
          int nt = 0, np = 0;
          while (t < T) {
            const int tp = tpath[t + 1] - tpath[t];
            int fresh = 0;  // features of tree t not yet in the chunk
            for (int q = tpath[t]; q < tpath[t + 1]; ++q)
              for (int e = poff[q] + 1; e < poff[q + 1]; ++e)
                if (tslot[pel[e].f] == -1) {
                  tslot[pel[e].f] = -2;  // counted
                  ++fresh;
                }
            for (int q = tpath[t]; q < tpath[t + 1]; ++q)  // undo the counting marks
              for (int e = poff[q] + 1; e < poff[q + 1]; ++e)
                if (tslot[pel[e].f] == -2) tslot[pel[e].f] = -1;
            const int nf = (int)tf.size() - first;
            if (nt > 0 && (np + tp > TAB_CHUNK_PATHS || nf + fresh > TAB_CHUNK_FEATURES)) break;
            for (int q = tpath[t]; q < tpath[t + 1]; ++q)
              for (int e = poff[q]; e < poff[q + 1]; ++e) {
                const PathEl& el = pel[e];
                int fci = 0;
                if (el.f >= 0) {
                  if (tslot[el.f] < 0) {
                    tslot[el.f] = (int)tf.size() - first;
                    tf.push_back(el.f);
                  }
                  fci = tslot[el.f];
                }
                int lo, hi;
                std::memcpy(&lo, &el.lo, 4);
                std::memcpy(&hi, &el.hi, 4);
                tel[e] = make_int4(el.f < 0 ? 0 : el.f, lo, hi, (fci << 1) | (el.miss_ok ? 1 : 0));
              }
            np += tp;
            ++nt;
            t += Kc;
          }
          for (size_t j = first; j < tf.size(); ++j) tslot[tf[j]] = -1;
          tmax = std::max(tmax, (int)tf.size() - first);
          tch.push_back(make_int4(c, t - nt * Kc, nt, np));
          tfo.push_back((int)tf.size());
        }
      }
      std::vector<int4> thead(n_paths);
      for (int p = 0; p < n_paths; ++p)
        thead[p] = make_int4(poff[p] + 1, poff[p + 1] - poff[p] - 1, (int)(uint32_t)(toff[p] & 0xFFFFFFFFll),
                             (int)(toff[p] >> 32));
      SB_TRY(D.tab_head.alloc(ctx, std::max(n_paths, 1)));
      SB_CUDA(cudaMemcpyAsync(D.tab_head.p, thead.data(), n_paths * 16, cudaMemcpyHostToDevice, st));
      SB_TRY(D.tab_el.alloc(ctx, std::max<size_t>(tel.size(), 1)));
      SB_TRY(D.tab_chunk.alloc(ctx, std::max<size_t>(tch.size(), 1)));
      SB_TRY(D.tab_chunk_fo.alloc(ctx, tfo.size()));
      SB_TRY(D.tab_chunk_f.alloc(ctx, std::max<size_t>(tf.size(), 1)));
      if (!tel.empty()) SB_CUDA(cudaMemcpyAsync(D.tab_el.p, tel.data(), tel.size() * 16, cudaMemcpyHostToDevice, st));
      if (!tch.empty()) SB_CUDA(cudaMemcpyAsync(D.tab_chunk.p, tch.data(), tch.size() * 16, cudaMemcpyHostToDevice, st));
      SB_CUDA(cudaMemcpyAsync(D.tab_chunk_fo.p, tfo.data(), tfo.size() * 4, cudaMemcpyHostToDevice, st));
      if (!tf.empty()) SB_CUDA(cudaMemcpyAsync(D.tab_chunk_f.p, tf.data(), tf.size() * 4, cudaMemcpyHostToDevice, st));
      D.n_tab_chunks = (int)tch.size();
      D.tab_max_fc = tmax;
      // a tree with more distinct features than one block's partial can hold
      // keeps the f64 path kernels
      if (shap_table_smem(tmax) <= ctx->smem_optin) {
        SB_TRY(raise_smem_limit((const void*)k_shap_table<TAB_TPR, TAB_ILP>, shap_table_smem(tmax)));
        D.shap_table = true;
      }
      SB_CUDA(cudaStreamSynchronize(st));  // d_moff and the host vectors are released on return
    }
  }
  SB_CUDA(cudaStreamSynchronize(st));
  D.shap_valid = true;
  return SB_OK;
}

// TreeSHAP contributions of n rows into d_acc ([n][K][F+1] doubles, zeroed
// here) on stream st. The model must have been prepared (shap_prepare).
int shap_paths(sb_model* m, cudaStream_t st, const float* d_X, size_t n, size_t F, float missing,
               double* d_acc) {
  sb_ctx* ctx = m->ctx;
  SB_REQUIRE(m->dev.shap_valid, SB_ERR_INVALID_ARG, "internal: TreeSHAP state not prepared");
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
  const unsigned long long items = (unsigned long long)row_blocks * (unsigned long long)m->dev.n_shap_chunks;
  const int L = m->dev.max_path_len;
  if (L > SHAP_REG_MAXL) {  // deep paths: persistent grid, global scratch on this stream
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_shap_deep, R, smem);
    const size_t per_thread = 4 * (size_t)L * sizeof(double);
    size_t blocks = (size_t)ctx->num_sms * std::max(per_sm, 1);
    blocks = std::min(blocks, std::max<size_t>(1, (256ull << 20) / (per_thread * R)));
    blocks = std::min<size_t>(blocks, items);
    double* scratch = nullptr;
    SB_CUDA(cudaMallocAsync((void**)&scratch, blocks * R * per_thread, st));
    k_shap_deep<<<(unsigned)blocks, R, smem, st>>>(P, d_X, n, (int)F, K, missing, row_blocks, items, L, scratch,
                                                  d_acc);
    ctx->launches++;
    const cudaError_t le = cudaGetLastError();
    cudaFreeAsync(scratch, st);
    SB_CUDA(le);
    return SB_OK;
  }
  SB_REQUIRE(items < (1ull << 31), SB_ERR_UNSUPPORTED,
             "TreeSHAP of %zu rows over %d path chunks exceeds one launch", n, m->dev.n_shap_chunks);
  const unsigned grid = (unsigned)items;
  if (m->dev.shap_table) {
    ShapTabDev Q;
    Q.el = m->dev.tab_el.p;
    Q.head = m->dev.tab_head.p;
    Q.tab = m->dev.shap_tab.p;
    Q.tree_path = m->dev.tree_path.p;
    Q.chunk = m->dev.tab_chunk.p;
    Q.chunk_fo = m->dev.tab_chunk_fo.p;
    Q.chunk_f = m->dev.tab_chunk_f.p;
    Q.K = K;
    const unsigned trb = (unsigned)((n + TAB_ROWS - 1) / TAB_ROWS);
    const unsigned long long tb = (unsigned long long)trb * (unsigned long long)m->dev.n_tab_chunks;
    SB_REQUIRE(tb < (1ull << 31), SB_ERR_UNSUPPORTED, "TreeSHAP of %zu rows exceeds one launch", n);
    SB_LAUNCH_ON(ctx, st, (k_shap_table<TAB_TPR, TAB_ILP>), (unsigned)tb, TAB_ROWS * TAB_TPR,
                 shap_table_smem(m->dev.tab_max_fc), Q, d_X, n,
                 (int)F, missing, trb, d_acc);
  } else if (L <= 5) {
    SB_LAUNCH_ON(ctx, st, k_shap_paths<5>, grid, R, smem, P, d_X, n, (int)F, K, missing, row_blocks, d_acc);
  } else if (L <= 9) {
    SB_LAUNCH_ON(ctx, st, k_shap_paths<9>, grid, R, smem, P, d_X, n, (int)F, K, missing, row_blocks, d_acc);
  } else {
    SB_LAUNCH_ON(ctx, st, k_shap_paths<SHAP_REG_MAXL>, grid, R, smem, P, d_X, n, (int)F, K, missing, row_blocks,
                 d_acc);
  }
  return SB_OK;
}

int predict_contribs_device(sb_model* m, const float* d_X, size_t n, size_t F, float missing,
                            float* d_out) {
  sb_ctx* ctx = m->ctx;
  SB_TRY(shap_prepare(m));
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
  SB_TRY(shap_prepare(m));
  SB_REQUIRE(m->dev.max_path_len <= SHAP_INTER_MAXL, SB_ERR_UNSUPPORTED,
             "interaction values on the device support paths of up to %d distinct features (got %d)",
             SHAP_INTER_MAXL - 1, m->dev.max_path_len - 1);
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
  SB_TRY(raise_smem_limit((const void*)k_shap_inter<SHAP_REG_MAXL>, smem));
  SB_TRY(raise_smem_limit((const void*)k_shap_inter<SHAP_INTER_MAXL>, smem));
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
      else if (L <= SHAP_REG_MAXL)
        SB_LAUNCH(ctx, k_shap_inter<SHAP_REG_MAXL>, (unsigned)blocks, INTER_THREADS, smem, P, X, nb, missing,
                  acc.p);
      else
        SB_LAUNCH(ctx, k_shap_inter<SHAP_INTER_MAXL>, (unsigned)blocks, INTER_THREADS, smem, P, X, nb, missing,
                  acc.p);
    }
    const size_t tot = nb * K * WW;
    SB_LAUNCH(ctx, k_inter_finish, (unsigned)((tot + 255) / 256), 256, 0, acc.p, d_bias.p, nb, K, (int)F,
              d_out + r0 * K * WW);
  }
  return SB_OK;
}


int contribs_bias(sb_model* m, std::vector<double>* bias) {
  SB_TRY(shap_prepare(m));
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
