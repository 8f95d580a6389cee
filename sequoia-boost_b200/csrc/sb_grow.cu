// sb_grow.cu — depthwise tree growth and the boosting loop on the device.
//
// Replaces, for tree_method=hist:
//   train_impl's round loop        learner/train.rs:276-338
//   Objective::gradient            objective/regression.rs:18-85,
//                                  classification.rs:50-71, multiclass.rs:64-91
//   sample_rows / column sampling  train.rs:465-534, tree/sampler.rs:52-70
//   HistTreeBuilder::build         tree/builder/hist.rs:139-202
//   grow_depthwise / split         hist.rs:212-236, :280-411
//   evaluate / consider            hist.rs:418-706
//   leaf finalisation, scale_leaves and the margin update
//                                  hist.rs:193-200, regtree.rs:201-207,
//                                  train.rs:323-328
//
// One boosting round is a fixed sequence of kernels whose work sizes live in
// device memory (no host round trip inside a round):
//   k_gradient -> k_round_prep -> [k_quantize] -> root histograms ->
//   per level d: k_eval_scan -> k_eval_pick -> k_assign -> k_partition -> k_plan -> histograms
//   -> k_round_end.
// All frontier nodes of all K class trees are processed by each launch.
#include <algorithm>
#include <map>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>
#include <tuple>

#include "sb_internal.cuh"

namespace sb {
namespace {

constexpr double K_RT_EPS = 1e-6;  // hist.rs:22
constexpr int PART_TILE = 2048;    // rows per partition tile
constexpr int EVAL_THREADS = 256;

struct NodeSplit {
  double loss_chg;
  double lg, lh, rg, rh;
  double wl, wr;
  int feature;
  int bin;
  int default_left;
  int is_cat;
  int valid;
  int ncat;
  uint32_t cat_mask[MAX_CAT_BINS / 32];
  uint8_t cat_order[MAX_CAT_BINS];
};

// Rows a split node has sent to each child so far (the lists hold sampled
// rows only, so these are also the children's sampled counts). 8-byte
// aligned: the partition adds to both with one 64-bit atomic.
struct __align__(8) Fill {
  unsigned int left, right;
};

struct FeatRec;

// An entry of a lossguide tree's priority queue (NodeEntry ordered by
// loss_chg.total_cmp, hist.rs:79-95).
struct HeapEnt {
  long long key;  // total_cmp_key(loss_chg)
  int nid;
  int depth;
};

struct BState {
  // shapes
  int K, F, FW, HB, total_bins, max_depth, maxn, maxw, cat_cap;
  int cat_bins;             // most bins of a categorical feature (eval scratch entries)
  // lossguide growth (grow_lossguide, hist.rs:238-268)
  int lossguide;
  int max_leaves;           // leaf budget (2^max_depth when max_leaves is 0)
  int depth_limit;          // max_depth, or INT_MAX for 0
  char* nhist;              // [K][maxn][HB] x 16 B: every node's histogram
  HeapEnt* heap;            // [K][maxn]
  int* heap_size;           // [K]
  int* n_leaves;            // [K]
  int* ndepth;              // [K][maxn]
  int* prev_count;          // [K] frontier nodes expanded by the last k_assign
  size_t n, Fp;
  // binned data
  const uint16_t* bins;      // tile-relative codes, row-major (u16 codes)
  const uint8_t* bins8;      // the same with u8 codes (bins null)
  const uint16_t* bins_col;  // the same, feature-major
  const int* fbase;          // code of local bin 0, per feature
  const int* fmiss;          // code of a missing entry, per feature
  const int* rpos;           // row-major codes: position, code of local bin 0 and
  const int* rbase;          // code of a missing entry of each feature
  const int* rmiss;
  const uint32_t* foff;
  const float* cuts;
  const uint8_t* is_cat;
  // parameters
  RegP reg;
  double gamma;
  float eta;
  double subsample, bytree, bylevel, bynode;
  uint64_t seed;
  int objective, num_class;
  float spw;
  int fixed, bits;
  int constrained;
  const int8_t* mono;       // [F]
  int has_inter;
  const uint8_t* in_group;  // [F]
  const uint32_t* iset;     // [F][FW]
  int ext_gpair;            // gradients supplied by the caller
  int update_margin;
  // round counter (output tree slot) and the offset of the sampling keys
  unsigned long long* round;
  unsigned long long round_base;
  int k_base;
  // node state [K][maxn]
  double2* stats;
  double2* bounds;
  uint32_t* allowed;        // [K][maxn][FW]
  uint8_t* allowed_all;
  uint32_t* fmask;          // [K][maxn][FW]
  uint2* seg;
  uint32_t* nsamp;
  int* parent;
  uint8_t* built;
  NodeSplit* split;
  float* leafval;
  Fill* fill;
  // level bookkeeping [K]
  int* lvl_begin;
  int* lvl_count;
  int* prev_begin;
  int* num_nodes;
  int* cat_count;
  // rows
  uint32_t* rows0;          // [K][n]
  uint32_t* rows1;          // [K][n]
  unsigned int* kept;       // sampled rows this round (the root list's front)
  unsigned int* unkept;     // rows outside the subset (the root list's back)
  // gradients
  float* margin;            // [n][K]
  float* delta;             // [n][K] this round's leaf value of each row (pending add)
  int apply_delta;          // k_gradient first adds delta into margin
  const float* labels;
  const float* weights;
  float2* gpair;            // [K][n]
  unsigned long long* gpk;  // [K][n] packed fixed-point
  unsigned int* maxabs;     // [2K] float bits
  int* shifts;              // [2K]
  double* inv_scale;        // [2K]
  unsigned long long* qerr; // [2] float bits of max quantisation error
  // histograms
  char* hist0;
  char* hist1;              // [K][maxw][HB] x 16 B
  longlong2* root_total;    // [K] (double2 for FP32)
  HistItem* items;          // [K * maxw]
  uint64_t* prefix;         // [K * maxw + 1]
  int* item_count;
  // partition tiles
  int4* ptiles;
  int* ptile_count;
  int ptile_cap;
  FeatRec* frec;            // [K][maxw][F] phase-2a summaries
  // sampling
  uint32_t* pool;           // [K][F] the tree's colsample_bytree pool, ascending
  int* pool_len;            // [K]
  uint32_t* upool;          // [K][F] pool features with >= 2 bins, ascending
  int* upool_len;           // [K]
  uint32_t* pool_mask;      // [K][FW] bitmask of upool
  const uint32_t* usable;   // [FW] features with >= 2 bins
  uint32_t* samp_scratch;   // [max(1024, K)][F] when per-node sampling is on
  double* mbuf;             // [K][maxw][F] phase-1 best gain per (node, feature)
  // outputs
  sb_node* out_nodes;       // [tree_cap][maxn]
  uint32_t* out_cats;       // [tree_cap][cat_cap]
  int* out_nnodes;          // [tree_cap]
  int* out_ncats;           // [tree_cap]
  int32_t* row_leaf;        // [n] or null
};

__device__ __forceinline__ size_t NI(const BState& S, int k, int nid) { return (size_t)k * S.maxn + nid; }

__device__ __forceinline__ char* level_hist(const BState& S, int d, int k, int slot) {
  char* base = (d & 1) ? S.hist1 : S.hist0;
  return base + ((size_t)k * S.maxw + slot) * (size_t)S.HB * 16;
}

__device__ __forceinline__ char* node_hist(const BState& S, int k, int nid) {
  return S.nhist + NI(S, k, nid) * (size_t)S.HB * 16;
}

// Histogram of frontier slot `slot` of tree k at level d (lossguide: of the node).
__device__ __forceinline__ char* frontier_hist(const BState& S, int d, int k, int slot) {
  return S.lossguide ? node_hist(S, k, S.lvl_begin[k] + slot) : level_hist(S, d, k, slot);
}

// Histogram of the parent of node index ni (a node of frontier level d).
__device__ __forceinline__ const char* parent_hist(const BState& S, int d, int k, size_t ni) {
  return S.lossguide ? node_hist(S, k, S.parent[ni]) : level_hist(S, d - 1, k, S.parent[ni] - S.prev_begin[k]);
}

template <typename T>
__device__ T block_scan_excl(T v, T* total, T* sm) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T x = v;
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T w = lane < nw ? sm[lane] : T(0);
    T s = w;
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) sm[lane] = s - w;
    if (lane == 31) sm[32] = s;
  }
  __syncthreads();
  T r = sm[warp] + (x - v);
  if (total) *total = sm[32];
  __syncthreads();
  return r;
}

__device__ __forceinline__ float sigmoidf_ref(float x) {  // classification.rs:7-15
  if (x >= 0.0f) return __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-x)));
  float e = expf(x);
  return __fdiv_rn(e, __fadd_rn(1.0f, e));
}

// ---------------------------------------------------------------- K3
// Objective::gradient for one row's K margins `mr` (regression.rs:18-85,
// classification.rs:50-71, multiclass.rs:14-30 and :64-91), with explicit
// f32 rounding so that no multiply-add is contracted. `w0` is the row's
// weight (1 when the caller has none, `has_w` = 0). emit(c, g, h) receives
// the pair of output c.
template <typename Emit>
__device__ __forceinline__ void row_gradient(int objective, int K, float spw, const float* mr, float y,
                                             float w0, bool has_w, Emit emit) {
  if (K == 1) {
    const float m = mr[0];
    float g, h;
    if (objective == SB_OBJ_SQUARED_ERROR) {  // regression.rs:18-40
      const float d = __fsub_rn(m, y);
      g = has_w ? __fmul_rn(d, w0) : d;
      h = has_w ? w0 : 1.0f;
    } else if (objective == SB_OBJ_PSEUDOHUBER) {  // regression.rs:51-85
      const float d = __fsub_rn(m, y);
      const float s = __fadd_rn(1.0f, __fmul_rn(d, d));
      const float sq = __fsqrt_rn(s);
      g = __fmul_rn(__fdiv_rn(d, sq), w0);
      h = __fmul_rn(__fdiv_rn(1.0f, __fmul_rn(s, sq)), w0);
    } else {  // logistic, classification.rs:50-71
      const float p = sigmoidf_ref(m);
      float w = w0;
      if (y == 1.0f) w = __fmul_rn(w, spw);
      g = __fmul_rn(__fsub_rn(p, y), w);
      h = __fmul_rn(fmaxf(__fmul_rn(p, __fsub_rn(1.0f, p)), 1e-16f), w);
    }
    emit(0, g, h);
    return;
  }
  // softmax, multiclass.rs:14-30, :64-91
  float mx = -INFINITY;
  for (int c = 0; c < K; ++c)
    if (mr[c] > mx) mx = mr[c];
  float sum = 0.0f;
  for (int c = 0; c < K; ++c) sum = __fadd_rn(sum, expf(__fsub_rn(mr[c], mx)));
  const float inv = __fdiv_rn(1.0f, sum);
  const uint32_t label = f32_as_u32(y);  // `as usize` saturates: negative and NaN labels are class 0
  for (int c = 0; c < K; ++c) {
    const float p = __fmul_rn(expf(__fsub_rn(mr[c], mx)), inv);
    const float target = ((uint32_t)c == label) ? 1.0f : 0.0f;
    const float g = __fmul_rn(__fsub_rn(p, target), w0);
    const float h = fmaxf(__fmul_rn(__fmul_rn(__fmul_rn(2.0f, p), __fsub_rn(1.0f, p)), w0), 1e-16f);
    emit(c, g, h);
  }
}

// Batched launches over many boosters (sb_train_many): the x-blocks of one
// launch are every job's own grid laid end to end, block x belongs to job j
// when xoff[j] <= x < xoff[j + 1], and the kernel body runs with that job's
// state and its block index within its own grid. A job given no blocks has
// xoff[j] == xoff[j + 1].
struct JobGrid {
  const BState* states;  // [njobs]
  const unsigned* xoff;  // [njobs + 1]
  int njobs;
};

__device__ __forceinline__ int job_of(const JobGrid& J, unsigned x) {
  int lo = 0, hi = J.njobs;  // the last job whose first block is <= x
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (J.xoff[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// Gradients of every row (train.rs:297-302) and the round's row subset
// (sample_rows, train.rs:465-475). The subset goes to the root list compacted:
// each block owns a contiguous chunk of rows, reserves its places with one
// atomic per counter, and writes its sampled rows (ascending) to the front of
// rows0 and the others to the back, so the per-node lists hold sampled rows
// only; the rows left out get their leaf values from k_route_rest.
__device__ __forceinline__ void k_gradient_body(const BState& S, unsigned bx, unsigned gdx) {
  const unsigned long long round = *S.round + S.round_base;
  const uint64_t rk = sb_round_key(S.seed, round);
  float mg[16], mh[16];
  const int K = S.K;
  const size_t n = S.n;
  for (int c = 0; c < 16; ++c) mg[c] = mh[c] = 0.0f;
  __shared__ unsigned int s_base[2], s_wk[8], s_wu[8];
  __shared__ unsigned int s_max[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t per = (n + gdx - 1) / gdx;
  const size_t lo = min(n, (size_t)bx * per), hi = min(n, lo + per);
  // the caller's subset (flags in rows1), or the Bernoulli draw
  auto keep_of = [&](size_t r) -> bool {
    if (S.ext_gpair) return !(S.rows1[r] & UNSAMPLED);
    return S.subsample >= 1.0 || sb_u01(sb_row_draw(rk, r)) < S.subsample;
  };
  // each warp owns a contiguous part of the block's rows; the block's kept
  // rows go to the front of the root list and the others to its back, both in
  // row order (warp parts in order, ascending within a part)
  const int nw = blockDim.x >> 5;
  const size_t wper = (hi - lo + nw - 1) / nw;
  const size_t wlo = min(hi, lo + (size_t)warp * wper), whi = min(hi, wlo + wper);
  unsigned int c0 = 0;
  for (size_t r = wlo + lane; r < whi; r += 32) c0 += keep_of(r) ? 1u : 0u;
  for (int o = 16; o > 0; o >>= 1) c0 += __shfl_xor_sync(0xFFFFFFFFu, c0, o);
  if (tid < 32) s_max[tid] = 0u;
  if (lane == 0) {
    s_wk[warp] = c0;
    s_wu[warp] = (unsigned int)(whi - wlo) - c0;
  }
  __syncthreads();
  if (tid == 0) {  // one atomic per block and counter (same-address atomics serialise)
    unsigned int tk = 0, tu = 0;
    for (int w = 0; w < nw; ++w) {
      tk += s_wk[w];
      tu += s_wu[w];
    }
    s_base[0] = tk ? atomicAdd(S.kept, tk) : 0u;
    s_base[1] = tu ? atomicAdd(S.unkept, tu) : 0u;
  }
  __syncthreads();
  unsigned int front = s_base[0], back = s_base[1];
  for (int w = 0; w < warp; ++w) {
    front += s_wk[w];
    back += s_wu[w];
  }
  const unsigned lt = (1u << lane) - 1u;
  for (size_t base = wlo; base < whi; base += 32) {  // the same trip count in every lane
    const size_t r = base + lane;
    const bool valid = r < whi;
    bool keep = false;
    if (valid) {
      if (!S.ext_gpair) {
        const float w0 = S.weights ? S.weights[r] : 1.0f;
        const float y = S.labels[r];
        if (S.apply_delta)  // the previous tree's leaf values (train.rs:326-328)
          for (int c = 0; c < K; ++c) S.margin[r * K + c] = __fadd_rn(S.margin[r * K + c], S.delta[r * K + c]);
        row_gradient(S.objective, K, S.spw, S.margin + r * K, y, w0, S.weights != nullptr,
                     [&](int c, float g, float h) {
                       S.gpair[(size_t)c * n + r] = make_float2(g, h);
                       if (c < 16) {
                         mg[c] = fmaxf(mg[c], fabsf(g));
                         mh[c] = fmaxf(mh[c], fabsf(h));
                       }
                     });
      } else {
        for (int c = 0; c < K && c < 16; ++c) {
          float2 v = S.gpair[(size_t)c * n + r];
          mg[c] = fmaxf(mg[c], fabsf(v.x));
          mh[c] = fmaxf(mh[c], fabsf(v.y));
        }
      }
      keep = keep_of(r);
    }
    const unsigned km = __ballot_sync(0xFFFFFFFFu, keep), um = __ballot_sync(0xFFFFFFFFu, valid && !keep);
    if (keep) S.rows0[front + __popc(km & lt)] = (uint32_t)r;
    else if (valid) S.rows0[n - 1 - (back + __popc(um & lt))] = (uint32_t)r;
    front += __popc(km);
    back += __popc(um);
  }
  if (S.fixed) {
    for (int c = 0; c < K && c < 16; ++c) {
      float a2 = mg[c], b2 = mh[c];
      for (int o = 16; o > 0; o >>= 1) {
        a2 = fmaxf(a2, __shfl_xor_sync(0xFFFFFFFFu, a2, o));
        b2 = fmaxf(b2, __shfl_xor_sync(0xFFFFFFFFu, b2, o));
      }
      if (lane == 0) {
        atomicMax(&s_max[2 * c], __float_as_uint(a2));
        atomicMax(&s_max[2 * c + 1], __float_as_uint(b2));
      }
    }
  }
  __syncthreads();
  if (S.fixed && tid < 2 * K && tid < 32 && s_max[tid]) atomicMax(&S.maxabs[tid], s_max[tid]);
}
__global__ void __launch_bounds__(256) k_gradient(BState S) { k_gradient_body(S, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(256) k_gradient_jobs(JobGrid J) {
  const int j = job_of(J, blockIdx.x);
  k_gradient_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j]);
}

// Leaf values of the rows outside the round's subset (rows0[n - unkept, n)):
// each is routed through the round's K trees in bin space, as the partition
// routes sampled rows (missing -> default_left; categorical: the category
// set; numeric: local bin <= split bin).
__device__ __forceinline__ void k_route_rest_body(const BState& S, unsigned bx, unsigned gdx) {
  const size_t n = S.n;
  const size_t un = *S.unkept;
  const unsigned long long round = *S.round;
  for (size_t i = (size_t)bx * blockDim.x + threadIdx.x; i < un; i += (size_t)gdx * blockDim.x) {
    const uint32_t r = S.rows0[n - 1 - i];
    for (int k = 0; k < S.K; ++k) {
      const sb_node* out = S.out_nodes + ((size_t)round * S.K + k) * S.maxn;
      int nid = 0;
      while (out[nid].left != -1) {
        const NodeSplit& sp = S.split[NI(S, k, nid)];
        const int c = (int)S.bins_col[(size_t)sp.feature * n + r];
        bool go;
        if (c == (int)MISSING_BIN) go = sp.default_left != 0;
        else if (sp.is_cat) go = (sp.cat_mask[c >> 5] >> (c & 31)) & 1u;
        else go = c <= sp.bin;
        nid = go ? out[nid].left : out[nid].right;
      }
      if (S.update_margin) S.delta[(size_t)r * S.K + k] = S.leafval[NI(S, k, nid)];
    }
    if (S.row_leaf) S.row_leaf[r] = -1;
  }
}
__global__ void k_route_rest(BState S) { k_route_rest_body(S, blockIdx.x, gridDim.x); }
__global__ void k_route_rest_jobs(JobGrid J) {
  const int j = job_of(J, blockIdx.x);
  k_route_rest_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j]);
}

// Objective::gradient over caller-supplied margins (row-major [n][K]),
// writing the reference's row-major GradPair [n][K] layout.
__global__ void k_objective_gradient(int objective, int K, float spw, const float* __restrict__ preds,
                                     const float* __restrict__ labels, const float* __restrict__ weights,
                                     size_t n, float2* __restrict__ out) {
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (size_t)gridDim.x * blockDim.x) {
    const float w0 = weights ? weights[r] : 1.0f;
    row_gradient(objective, K, spw, preds + r * K, labels[r], w0, weights != nullptr,
                 [&](int c, float g, float h) { out[r * K + c] = make_float2(g, h); });
  }
}

// Column subset of node `nid` (sampler.rs:52-70 with sb_sampling.h keys),
// intersected with the tree's usable pool and the node's allowed set, as a
// bitmask written word by word.
__device__ void node_feature_mask(const BState& S, int k, int nid, uint64_t tkey, uint32_t* out,
                                  const uint32_t* allowed, bool allowed_all, uint32_t* scratch) {
  const uint32_t* pm = S.pool_mask + (size_t)k * S.FW;
  if (S.bylevel >= 1.0 && S.bynode >= 1.0) {
    for (int w = 0; w < S.FW; ++w) out[w] = pm[w] & (allowed_all ? 0xFFFFFFFFu : allowed[w]);
    return;
  }
  const uint32_t* pool = S.pool + (size_t)k * S.F;
  const int len = S.pool_len[k];
  for (int i = 0; i < len; ++i) scratch[i] = pool[i];
  sb_splitmix gen{sb_node_key(tkey, (uint64_t)nid)};
  int l1 = sb_subsample(scratch, len, S.bylevel, &gen);
  int l2 = sb_subsample(scratch, l1, S.bynode, &gen);
  int p = 0;
  for (int w = 0; w < S.FW; ++w) {
    uint32_t word = 0u;
    while (p < l2 && (int)(scratch[p] >> 5) == w) {
      word |= 1u << (scratch[p] & 31);
      ++p;
    }
    out[w] = word & pm[w] & (allowed_all ? 0xFFFFFFFFu : allowed[w]);
  }
}

// Per round, one CTA per class tree: quantisation scales, the sampled-row
// fallback, the tree's colsample_bytree pool (train.rs:479-489) and its root.
constexpr int PREP_THREADS = 128;
__device__ __forceinline__ void k_round_prep_body(const BState& S, unsigned bx, unsigned gdx) {
  __shared__ uint32_t s_a[4096];
  __shared__ uint32_t s_b[4096];
  __shared__ uint32_t s_mask[128];
  __shared__ int s_len;
  const unsigned long long round = *S.round + S.round_base;
  const int k = bx, tid = threadIdx.x;
  const int F = S.F;
  const uint64_t tkey = sb_tree_key(S.seed, round, (uint64_t)(k + S.k_base));
  // the subset's size; an empty draw takes one row (train.rs:472-474)
  const unsigned int kept0 = *S.kept;
  const bool fallback = kept0 == 0 && !S.ext_gpair && S.n > 0;
  const unsigned int kept = fallback ? 1u : kept0;
  if (k == 0 && tid == 0) {
    *S.qerr = 0ull;
    *S.ptile_count = 0;  // k_assign's blocks reserve the round's first tiles from 0
  }
  if (k == 0 && fallback) {  // every row is at the back: move the fallback row to the front
    __shared__ int s_at;
    if (tid == 0) s_at = -1;
    __syncthreads();
    const uint32_t fb = (uint32_t)sb_row_fallback(sb_round_key(S.seed, round), S.n);
    for (size_t i = tid; i < S.n; i += blockDim.x)
      if (S.rows0[i] == fb) s_at = (int)i;
    __syncthreads();
    if (tid == 0 && s_at >= 0) {
      S.rows0[s_at] = S.rows0[0];
      S.rows0[0] = fb;
      *S.unkept = (unsigned int)S.n - 1u;
      *S.kept = 1u;  // the other blocks took `kept` before this write
    }
  }
  for (int f = tid; f < F; f += blockDim.x) s_a[f] = (uint32_t)f;
  for (int w = tid; w < S.FW; w += blockDim.x) s_mask[w] = 0u;
  __syncthreads();
  if (tid == 0) {
    int len = F;
    if (S.bytree < 1.0) {
      sb_splitmix gen{tkey};
      len = sb_shuffle_truncate(s_a, F, S.bytree, &gen);
    }
    s_len = len;
  }
  __syncthreads();
  const int len = s_len;
  // sort the sample ascending: rank of each (distinct) feature id
  for (int i = tid; i < len; i += blockDim.x) {
    uint32_t v = s_a[i];
    int r = 0;
    for (int j = 0; j < len; ++j) r += s_a[j] < v ? 1 : 0;
    s_b[r] = v;
  }
  __syncthreads();
  uint32_t* pool = S.pool + (size_t)k * F;
  for (int i = tid; i < len; i += blockDim.x) {
    uint32_t f = s_b[i];
    pool[i] = f;
    if ((S.usable[f >> 5] >> (f & 31)) & 1u) atomicOr(&s_mask[f >> 5], 1u << (f & 31));
  }
  __syncthreads();
  for (int w = tid; w < S.FW; w += blockDim.x) S.pool_mask[(size_t)k * S.FW + w] = s_mask[w];
  if (tid == 0) {  // usable pool list, ascending
    int u = 0;
    uint32_t* up = S.upool + (size_t)k * F;
    for (int w = 0; w < S.FW; ++w) {
      uint32_t word = s_mask[w];
      while (word) {
        int b = __ffs(word) - 1;
        word &= word - 1;
        up[u++] = (uint32_t)(w * 32 + b);
      }
    }
    S.upool_len[k] = u;
    S.pool_len[k] = len;
    if (S.fixed) {
      int sg = quant_shift(__uint_as_float(S.maxabs[2 * k]), S.bits);
      int sh = quant_shift(__uint_as_float(S.maxabs[2 * k + 1]), S.bits);
      S.shifts[2 * k] = sg;
      S.shifts[2 * k + 1] = sh;
      S.inv_scale[2 * k] = ldexp(1.0, -sg);
      S.inv_scale[2 * k + 1] = ldexp(1.0, -sh);
    }
    S.num_nodes[k] = 1;
    S.lvl_begin[k] = 0;
    S.lvl_count[k] = 1;
    S.prev_begin[k] = 0;
    S.prev_count[k] = 0;
    S.cat_count[k] = 0;
    if (S.lossguide) S.ndepth[NI(S, k, 0)] = 0;
    const size_t r0 = NI(S, k, 0);
    S.seg[r0] = make_uint2(0u, kept);
    S.nsamp[r0] = kept;
    S.bounds[r0] = make_double2(-INFINITY, INFINITY);
    S.allowed_all[r0] = 1;
    S.built[r0] = 1;
    S.parent[r0] = -1;
    S.root_total[k] = make_longlong2(0, 0);
    HistItem it;
    it.rows = S.rows0;  // level 0 shares the root list of class 0 (sampled rows only)
    it.begin = 0;
    it.end = kept;
    it.k = (uint32_t)k;
    it.root = 1;
    it.out = S.lossguide ? node_hist(S, k, 0) : level_hist(S, 0, k, 0);
    it.total = &S.root_total[k];
    S.items[k] = it;
    S.prefix[k] = (uint64_t)k * kept;
    if (k == 0) {
      S.prefix[S.K] = (uint64_t)S.K * kept;
      *S.item_count = S.K;
    }
  }
  __syncthreads();
  if (tid == 0)  // after the pool mask is published
    node_feature_mask(S, k, 0, tkey, S.fmask + NI(S, k, 0) * S.FW, nullptr, true,
                      S.samp_scratch ? S.samp_scratch + (size_t)k * S.F : nullptr);
}
__global__ void __launch_bounds__(PREP_THREADS) k_round_prep(BState S) { k_round_prep_body(S, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(PREP_THREADS) k_round_prep_jobs(JobGrid J) {
  const int j = job_of(J, blockIdx.x);
  k_round_prep_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j]);
}

// FIXED: q = rint(x * 2^s), packed (q_g << 32) + q_h.
__device__ __forceinline__ void k_quantize_body(const BState& S, unsigned bx, unsigned gdx) {
  float eg = 0.0f, eh = 0.0f;
  const size_t total = (size_t)S.K * S.n;
  for (size_t i = (size_t)bx * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gdx * blockDim.x) {
    int k = (int)(i / S.n);
    float2 v = S.gpair[i];
    int sg = S.shifts[2 * k], sh = S.shifts[2 * k + 1];
    float xg = ldexpf(v.x, sg), xh = ldexpf(v.y, sh);
    int qg = __float2int_rn(xg), qh = __float2int_rn(xh);
    S.gpk[i] = ((unsigned long long)(uint32_t)qg << 32) + (unsigned long long)(uint32_t)qh;
    eg = fmaxf(eg, fabsf(__fsub_rn(v.x, ldexpf((float)qg, -sg))));
    eh = fmaxf(eh, fabsf(__fsub_rn(v.y, ldexpf((float)qh, -sh))));
  }
  __shared__ unsigned int s_e[2];
  if (threadIdx.x < 2) s_e[threadIdx.x] = 0u;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) {
    eg = fmaxf(eg, __shfl_xor_sync(0xFFFFFFFFu, eg, o));
    eh = fmaxf(eh, __shfl_xor_sync(0xFFFFFFFFu, eh, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&s_e[0], __float_as_uint(eg));
    atomicMax(&s_e[1], __float_as_uint(eh));
  }
  __syncthreads();
  if (threadIdx.x < 2 && s_e[threadIdx.x]) atomicMax((unsigned int*)&S.qerr[0] + threadIdx.x, s_e[threadIdx.x]);
}
__global__ void k_quantize(BState S) { k_quantize_body(S, blockIdx.x, gridDim.x); }
__global__ void k_quantize_jobs(JobGrid J) {
  const int j = job_of(J, blockIdx.x);
  k_quantize_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j]);
}

// ---------------------------------------------------------------- K6
struct EvalNode {
  double tg, th;      // node total
  double lo, hi;      // monotone bounds
  double parent_gain;
};

__device__ __forceinline__ double2 hist_entry(const BState& S, const char* H, int i, int k) {
  if (S.fixed) {
    longlong2 q = reinterpret_cast<const longlong2*>(H)[i];
    return make_double2(dmul((double)q.x, S.inv_scale[2 * k]), dmul((double)q.y, S.inv_scale[2 * k + 1]));
  }
  return reinterpret_cast<const double2*>(H)[i];
}

// Gain of one candidate (consider, hist.rs:549-596). -inf when the candidate
// is not eligible (min_child_weight or a monotone violation).
__device__ __forceinline__ double cand_gain(const BState& S, const EvalNode& E, int dir, double lg,
                                            double lh, double rg, double rh, double* wl, double* wr) {
  if (!(lh >= S.reg.mcw && rh >= S.reg.mcw)) return -INFINITY;
  if (S.constrained) {
    double a = calc_weight_bounded(lg, lh, S.reg, E.lo, E.hi);
    double b = calc_weight_bounded(rg, rh, S.reg, E.lo, E.hi);
    *wl = a;
    *wr = b;
    if (!satisfies(dir, a, b)) return -INFINITY;
    return dsub(dadd(gain_at_weight(lg, lh, S.reg, a), gain_at_weight(rg, rh, S.reg, b)), E.parent_gain);
  }
  *wl = 0.0;
  *wr = 0.0;
  return dsub(dadd(calc_gain(lg, lh, S.reg), calc_gain(rg, rh, S.reg)), E.parent_gain);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
  return v;
}
__device__ __forceinline__ double warp_incl_sum(double v) {
  const int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    double y = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if (lane >= o) v += y;
  }
  return v;
}
__device__ __forceinline__ double warp_excl_max(double v, double init) {
  const int lane = threadIdx.x & 31;
  double x = v;
  for (int o = 1; o < 32; o <<= 1) {
    double y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x = fmax(x, y);
  }
  double e = __shfl_up_sync(0xFFFFFFFFu, x, 1);
  return lane == 0 ? init : fmax(init, e);
}

// Scratch of one warp for a categorical feature.
// One warp's categorical scratch: arrays of `cap` entries (the most bins of
// a categorical feature of the index), carved from the block's dynamic
// shared memory so that the eval kernels' occupancy follows the data.
struct CatScratch {
  double* g;
  double* h;
  long long* key;
  uint16_t* ne;      // non-empty bins, ascending
  uint16_t* order;   // positions into ne/g/h, sorted by ratio (stable)
};

__host__ __device__ constexpr size_t cat_scratch_bytes(int cap) {
  return ((size_t)cap * (8 + 8 + 8 + 2 + 2) + 7) / 8 * 8;
}

__device__ __forceinline__ CatScratch cat_scratch(double* base, int warp, int cap) {
  double* b = base + (size_t)warp * (cat_scratch_bytes(cap) / 8);
  CatScratch c;
  c.g = b;
  c.h = b + cap;
  c.key = reinterpret_cast<long long*>(b + 2 * cap);
  c.ne = reinterpret_cast<uint16_t*>(b + 3 * cap);
  c.order = c.ne + cap;
  return c;
}

constexpr int AMB_MAX = 6;  // ambiguous records kept per (node, feature)

// Phase-2 summary of one feature of one node (see k_eval_records).
struct FeatRec {
  double def_gain;          // gain of the last certain record
  int def_idx;              // its candidate index, -1 none
  int namb;                 // ambiguous records after it (AMB_MAX + 1 = overflow)
  double amb_gain[AMB_MAX];
  int amb_idx[AMB_MAX];
};

struct Chosen {
  double gain;
  int cand;    // candidate index within the feature, -1 none
};

enum { SCAN_MAX = 0, SCAN_REPLAY = 1, SCAN_RECORDS = 2, SCAN_EXTRACT = 3 };

// Warp-parallel walk over one feature's candidates in the reference's order:
//   numeric  : bins ascending, direction A (missing right) before direction B
//              (missing left, only when the node has missing values);
//              candidate index 2*i + dir
//   category : prefixes of the non-empty bins sorted by G/(H+lambda)
//              (evaluate_categorical, hist.rs:607-653); candidate index = prefix
// Modes:
//   SCAN_MAX     the feature's best candidate gain
//   SCAN_RECORDS with the prefix maximum P started at `b_in` (the best gain of
//                earlier features, or 0): the last candidate with g > P + eps
//                (certainly taken by consider's rule g > best + 1e-6) and the
//                ambiguous records after it (P < g <= P + eps)
//   SCAN_REPLAY  consider's sequential rule from state b_in (exact fallback)
//   SCAN_EXTRACT statistics of candidate `want` into *out
template <int MODE>
__device__ Chosen scan_feature(const BState& S, const char* H, int k, int f, const EvalNode& E,
                               double b_in, CatScratch* cs, double* s_gains, NodeSplit* out,
                               FeatRec* rec = nullptr, int want = -1) {
  const int lane = threadIdx.x & 31;
  const int fs = (int)S.foff[f], nb = (int)S.foff[f + 1] - fs;
  const int dir = S.mono ? S.mono[f] : 0;
  const bool cat = S.is_cat[f] != 0;
  double2 miss = make_double2(0.0, 0.0);
  double pg = 0.0, ph = 0.0;
  int ncand;   // candidate positions (bins or prefixes)
  bool has_missing = false;
  if (!cat) {
    miss = hist_entry(S, H, S.total_bins + f, k);  // missing statistics: the missing bin
    for (int c0 = 0; c0 < nb; c0 += 32) {
      const int i = c0 + lane;
      const double2 v = i < nb ? hist_entry(S, H, fs + i, k) : make_double2(0.0, 0.0);
      pg += v.x;
      ph += v.y;
    }
    pg = warp_sum(pg);
    ph = warp_sum(ph);
    has_missing = miss.y > 1e-6;
    ncand = nb - 1;
  } else {
    const double lam = S.reg.lambda;
    int nne = 0;
    for (int c0 = 0; c0 < nb; c0 += 32) {
      const int i = c0 + lane;
      const double2 v = i < nb ? hist_entry(S, H, fs + i, k) : make_double2(0.0, -1.0);
      const bool ne = i < nb && v.y > 0.0;
      const unsigned m = __ballot_sync(0xFFFFFFFFu, ne);
      if (ne) {
        const int pos = nne + __popc(m & ((1u << lane) - 1u));
        cs->ne[pos] = (uint16_t)i;
        cs->g[pos] = v.x;
        cs->h[pos] = v.y;
        cs->key[pos] = total_cmp_key(ddiv(v.x, dadd(v.y, lam)));
      }
      nne += __popc(m);
    }
    __syncwarp();
    for (int i = lane; i < nne; i += 32) {  // stable rank by key
      const long long ki = cs->key[i];
      int r = 0;
      for (int j = 0; j < nne; ++j) {
        const long long kj = cs->key[j];
        r += (kj < ki || (kj == ki && j < i)) ? 1 : 0;
      }
      cs->order[r] = (uint16_t)i;
    }
    __syncwarp();
    ncand = nne - 1;  // prefixes leaving at least one category right
  }
  Chosen res{MODE == SCAN_MAX ? -INFINITY : b_in, -1};
  if (ncand <= 0) {
    if (MODE == SCAN_RECORDS && lane == 0) {
      rec->def_idx = -1;
      rec->namb = 0;
    }
    return res;
  }

  double run_max = -INFINITY;  // SCAN_MAX
  double P = b_in;             // prefix maximum (RECORDS / REPLAY)
  int def_idx = -1;            // RECORDS: last certain record
  double def_gain = 0.0;
  int namb = 0;                // RECORDS: ambiguous records after def_idx (lane 0's copy)
  double bstate = b_in;        // REPLAY
  int chosen = -1;
  double cg = 0.0, ch = 0.0;   // running prefix of the bins walked so far
  for (int c0 = 0; c0 < ncand; c0 += 32) {
    const int i = c0 + lane;   // candidate position
    double vg = 0.0, vh = 0.0;
    if (!cat) {
      if (i < nb) {
        const double2 v = hist_entry(S, H, fs + i, k);
        vg = v.x;
        vh = v.y;
      }
    } else if (i <= ncand) {
      const int o = cs->order[i];
      vg = cs->g[o];
      vh = cs->h[o];
    }
    const double ag = cg + warp_incl_sum(vg), ah = ch + warp_incl_sum(vh);
    const double tg = __shfl_sync(0xFFFFFFFFu, ag - cg, 31), th = __shfl_sync(0xFFFFFFFFu, ah - ch, 31);
    double gA = -INFINITY, gB = -INFINITY, wlA = 0, wrA = 0, wlB = 0, wrB = 0;
    if (i < ncand) {
      gA = cand_gain(S, E, dir, ag, ah, dsub(E.tg, ag), dsub(E.th, ah), &wlA, &wrA);
      if (!cat && has_missing)
        gB = cand_gain(S, E, dir, dadd(ag, miss.x), dadd(ah, miss.y), dsub(pg, ag), dsub(ph, ah), &wlB, &wrB);
    }
    const double lm = fmax(gA, gB);
    if (MODE == SCAN_MAX) {
      run_max = fmax(run_max, lm);
    } else if (MODE == SCAN_EXTRACT) {
      if (out && (want >> (cat ? 0 : 1)) == i) {
        const bool isB = !cat && (want & 1);
        out->feature = f;
        out->bin = cat ? 0 : i;
        out->default_left = isB ? 1 : 0;
        out->is_cat = cat ? 1 : 0;
        out->ncat = cat ? i + 1 : 0;
        out->lg = isB ? dadd(ag, miss.x) : ag;
        out->lh = isB ? dadd(ah, miss.y) : ah;
        out->rg = isB ? dsub(pg, ag) : dsub(E.tg, ag);
        out->rh = isB ? dsub(ph, ah) : dsub(E.th, ah);
        out->wl = isB ? wlB : wlA;
        out->wr = isB ? wrB : wrA;
      }
      if ((want >> (cat ? 0 : 1)) < c0 + 32) break;
    } else {
      const double PA = warp_excl_max(lm, P);  // prefix max before candidate 2i (or i)
      const double PB = fmax(PA, gA);          // before candidate 2i+1
      const int step = cat ? 1 : 2;
      if (MODE == SCAN_RECORDS) {
        int ci = -1;
        double cgain = 0.0;
        if (!cat && gB > PB + K_RT_EPS) { ci = 2 * i + 1; cgain = gB; }
        else if (gA > PA + K_RT_EPS) { ci = step * i; cgain = gA; }
        int best_ci = ci;
        for (int o = 16; o > 0; o >>= 1) best_ci = max(best_ci, __shfl_xor_sync(0xFFFFFFFFu, best_ci, o));
        if (best_ci >= 0) {
          const int owner = cat ? best_ci - c0 : (best_ci >> 1) - c0;
          def_gain = __shfl_sync(0xFFFFFFFFu, cgain, owner);
          def_idx = best_ci;
          namb = 0;  // earlier ambiguous records are no longer after the last certain one
        }
        const bool ambA = step * i > def_idx && gA > PA && !(gA > PA + K_RT_EPS);
        const bool ambB = !cat && 2 * i + 1 > def_idx && gB > PB && !(gB > PB + K_RT_EPS);
        const unsigned ma = __ballot_sync(0xFFFFFFFFu, ambA), mb = __ballot_sync(0xFFFFFFFFu, ambB);
        if (ma | mb) {
          s_gains[lane] = gA;
          s_gains[32 + lane] = gB;
          __syncwarp();
          if (lane == 0) {
            for (int L = 0; L < 32; ++L) {
              for (int d2 = 0; d2 < 2; ++d2) {
                if (!(((d2 ? mb : ma) >> L) & 1u)) continue;
                if (namb < AMB_MAX) {
                  rec->amb_gain[namb] = s_gains[d2 * 32 + L];
                  rec->amb_idx[namb] = cat ? c0 + L : 2 * (c0 + L) + d2;
                }
                namb++;
              }
            }
          }
          __syncwarp();
        }
      } else {  // SCAN_REPLAY: consider's rule, candidates in order, from bstate
        const bool rA = gA > PA, rB = !cat && gB > PB;  // only records can be taken
        const unsigned ma = __ballot_sync(0xFFFFFFFFu, rA), mb = __ballot_sync(0xFFFFFFFFu, rB);
        if (ma | mb) {
          s_gains[lane] = gA;
          s_gains[32 + lane] = gB;
          __syncwarp();
          if (lane == 0) {
            for (int L = 0; L < 32; ++L)
              for (int d2 = 0; d2 < 2; ++d2) {
                if (!(((d2 ? mb : ma) >> L) & 1u)) continue;
                const double gv = s_gains[d2 * 32 + L];
                if (gv > bstate + K_RT_EPS) {
                  bstate = gv;
                  chosen = cat ? c0 + L : 2 * (c0 + L) + d2;
                }
              }
          }
          bstate = __shfl_sync(0xFFFFFFFFu, bstate, 0);
          chosen = __shfl_sync(0xFFFFFFFFu, chosen, 0);
          __syncwarp();
        }
      }
      P = fmax(P, warp_max(lm));
    }
    cg += tg;
    ch += th;
  }
  if (MODE == SCAN_MAX) res.gain = warp_max(run_max);
  if (MODE == SCAN_RECORDS && lane == 0) {
    rec->def_idx = def_idx;
    rec->def_gain = def_gain;
    rec->namb = namb > AMB_MAX ? AMB_MAX + 1 : namb;
  }
  if (MODE == SCAN_REPLAY) {
    res.gain = bstate;
    res.cand = chosen;
  }
  if (MODE == SCAN_EXTRACT && cat && out) {
    // categories routed left, in sweep order (cats_left, hist.rs:630-636)
    for (int i = lane; i < MAX_CAT_BINS / 32; i += 32) out->cat_mask[i] = 0u;
    __syncwarp();
    for (int p = lane; p <= want; p += 32) {
      const int b = cs->ne[cs->order[p]];
      out->cat_order[p] = (uint8_t)b;
      atomicOr(&out->cat_mask[b >> 5], 1u << (b & 31));
    }
    __syncwarp();
  }
  return res;
}

// Evaluation context of a frontier node: its total, monotone bounds and the
// parent gain of evaluate() (hist.rs:445-457).
__device__ EvalNode eval_node(const BState& S, int k, size_t ni, int d) {
  double2 st;
  if (d == 0) {  // root statistics, summed by the root histogram launch
    if (S.fixed) {
      longlong2 q = S.root_total[k];
      st = make_double2(dmul((double)q.x, S.inv_scale[2 * k]), dmul((double)q.y, S.inv_scale[2 * k + 1]));
    } else {
      st = reinterpret_cast<const double2*>(S.root_total)[k];
    }
  } else {
    st = S.stats[ni];
  }
  const double2 bd = S.bounds[ni];
  EvalNode E;
  E.tg = st.x;
  E.th = st.y;
  E.lo = bd.x;
  E.hi = bd.y;
  E.parent_gain = S.constrained
      ? gain_at_weight(st.x, st.y, S.reg, calc_weight_bounded(st.x, st.y, S.reg, bd.x, bd.y))
      : calc_gain(st.x, st.y, S.reg);
  return E;
}

constexpr int SCAN_WARPS = EVAL_THREADS / 32;

__device__ __forceinline__ bool in_mask(const uint32_t* m, int f) { return (m[f >> 5] >> (f & 31)) & 1u; }

// Phase 1, one warp per (frontier node, usable pool feature): materialise the
// feature's bins of a node whose histogram is the parent's minus the built
// sibling's (the subtraction trick, K5), then record the feature's best
// candidate gain (-inf when the node may not use the feature).
__device__ __forceinline__ void k_eval_scan_body(const BState& S, unsigned bx, unsigned gdx, int d) {
  extern __shared__ double ev_sm[];
  const int slot = bx, k = blockIdx.z;
  if (k >= S.K || slot >= S.lvl_count[k]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pi = blockIdx.y * SCAN_WARPS + warp;
  if (pi >= S.upool_len[k]) return;
  const int f = (int)S.upool[(size_t)k * S.F + pi];
  const int nid = S.lvl_begin[k] + slot;
  const size_t ni = NI(S, k, nid);
  char* H = frontier_hist(S, d, k, slot);
  if (d > 0 && !S.built[ni]) {
    const char* P = parent_hist(S, d, k, ni);
    const char* B = frontier_hist(S, d, k, slot ^ 1);
    const int fs = (int)S.foff[f], nb = (int)S.foff[f + 1] - fs;
    for (int i = lane; i <= nb; i += 32) {
      const int e = i < nb ? fs + i : S.total_bins + f;  // bins, then the missing bin
      if (S.fixed) {
        longlong2 x = reinterpret_cast<const longlong2*>(P)[e], y = reinterpret_cast<const longlong2*>(B)[e];
        reinterpret_cast<longlong2*>(H)[e] = make_longlong2(x.x - y.x, x.y - y.y);
      } else {
        double2 x = reinterpret_cast<const double2*>(P)[e], y = reinterpret_cast<const double2*>(B)[e];
        reinterpret_cast<double2*>(H)[e] = make_double2(dsub(x.x, y.x), dsub(x.y, y.y));
      }
    }
    __syncwarp();
  }
  double m = -INFINITY;
  if (in_mask(S.fmask + ni * S.FW, f)) {
    const EvalNode E = eval_node(S, k, ni, d);
    CatScratch csv{};
  if (S.cat_cap > 0) csv = cat_scratch(ev_sm, warp, S.cat_bins);
  CatScratch* cs = S.cat_cap > 0 ? &csv : nullptr;
    m = scan_feature<SCAN_MAX>(S, H, k, f, E, 0.0, cs, nullptr, nullptr).gain;
  }
  if (lane == 0) S.mbuf[((size_t)k * S.maxw + slot) * S.F + f] = m;
}
__global__ void __launch_bounds__(EVAL_THREADS) k_eval_scan(BState S, int d) { k_eval_scan_body(S, blockIdx.x, gridDim.x, d); }
__global__ void __launch_bounds__(EVAL_THREADS) k_eval_scan_jobs(JobGrid J, int d) {
  const int j = job_of(J, blockIdx.x);
  k_eval_scan_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j], d);
}

// Phase 2a, one warp per (frontier node, usable pool feature): with Q = the
// best gain of the node's earlier features (or 0), find this feature's last
// certain record and its ambiguous records (FeatRec).
__device__ __forceinline__ void k_eval_records_body(const BState& S, unsigned bx, unsigned gdx, int d) {
  extern __shared__ double ev_sm[];
  __shared__ double s_gains[SCAN_WARPS][64];
  const int slot = bx, k = blockIdx.z;
  if (k >= S.K || slot >= S.lvl_count[k]) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pi = blockIdx.y * SCAN_WARPS + warp;
  if (pi >= S.upool_len[k]) return;
  const int f = (int)S.upool[(size_t)k * S.F + pi];
  const int nid = S.lvl_begin[k] + slot;
  const size_t ni = NI(S, k, nid);
  const size_t ri = ((size_t)k * S.maxw + slot) * S.F + f;
  FeatRec* rec = S.frec + ri;
  const double* M = S.mbuf + ((size_t)k * S.maxw + slot) * S.F;
  if (!(M[f] > K_RT_EPS)) {  // no candidate can be taken from any state >= 0
    if (lane == 0) {
      rec->def_idx = -1;
      rec->namb = 0;
    }
    return;
  }
  const uint32_t* fm = S.fmask + ni * S.FW;
  double q = 0.0;  // max over the node's earlier features (only masked slots are current)
  for (int j = lane; j < f; j += 32)
    if (in_mask(fm, j)) q = fmax(q, M[j]);
  q = warp_max(q);
  // every record of this feature needs a gain above the running best, which
  // starts at q: a feature whose best gain is not above q has none
  if (!(M[f] > q)) {
    if (lane == 0) {
      rec->def_idx = -1;
      rec->namb = 0;
    }
    return;
  }
  const EvalNode E = eval_node(S, k, ni, d);
  CatScratch csv{};
  if (S.cat_cap > 0) csv = cat_scratch(ev_sm, warp, S.cat_bins);
  CatScratch* cs = S.cat_cap > 0 ? &csv : nullptr;
  scan_feature<SCAN_RECORDS>(S, frontier_hist(S, d, k, slot), k, f, E, q, cs, s_gains[warp], nullptr, rec);
}
__global__ void __launch_bounds__(EVAL_THREADS) k_eval_records(BState S, int d) { k_eval_records_body(S, blockIdx.x, gridDim.x, d); }
__global__ void __launch_bounds__(EVAL_THREADS) k_eval_records_jobs(JobGrid J, int d) {
  const int j = job_of(J, blockIdx.x);
  k_eval_records_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j], d);
}

// Phase 2b, one warp per frontier node: the winner of consider's sequential
// rule is the last certain record over all features, followed by a short
// sequential resolution over the ambiguous records after it.
__device__ __forceinline__ void k_eval_pick_body(const BState& S, unsigned bx, unsigned gdx, int d) {
  extern __shared__ double ev_sm[];
  __shared__ NodeSplit s_best[SCAN_WARPS];
  __shared__ double s_gains[SCAN_WARPS][64];
  const int k = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= S.K) return;
  const int slot = bx * SCAN_WARPS + warp;
  if (slot >= S.lvl_count[k]) return;
  const int nid = S.lvl_begin[k] + slot;
  const size_t ni = NI(S, k, nid);
  const char* H = frontier_hist(S, d, k, slot);
  const EvalNode E = eval_node(S, k, ni, d);
  NodeSplit* best = &s_best[warp];
  const double* M = S.mbuf + ((size_t)k * S.maxw + slot) * S.F;
  const FeatRec* R = S.frec + ((size_t)k * S.maxw + slot) * S.F;
  const uint32_t* fm = S.fmask + ni * S.FW;
  CatScratch csv{};
  if (S.cat_cap > 0) csv = cat_scratch(ev_sm, warp, S.cat_bins);
  CatScratch* cs = S.cat_cap > 0 ? &csv : nullptr;
  // last feature holding a certain record
  int fstar = -1;
  for (int j = lane; j < S.F; j += 32)
    if (in_mask(fm, j) && M[j] > K_RT_EPS && R[j].def_idx >= 0) fstar = j;
  for (int o = 16; o > 0; o >>= 1) fstar = max(fstar, __shfl_xor_sync(0xFFFFFFFFu, fstar, o));
  double b = 0.0;
  int cf = -1, cidx = -1;
  if (fstar >= 0) {
    b = R[fstar].def_gain;
    cf = fstar;
    cidx = R[fstar].def_idx;
  }
  // ambiguous records after the winner, in candidate order: 32 features are
  // tested at a time, and the (rare) features holding any are walked in order
  for (int f0 = fstar < 0 ? 0 : fstar; f0 < S.F; f0 += 32) {
    const int fl = f0 + lane;
    const bool has = fl < S.F && in_mask(fm, fl) && M[fl] > K_RT_EPS && R[fl].namb > 0;
    unsigned hm = __ballot_sync(0xFFFFFFFFu, has);
    while (hm) {
      const int f = f0 + __ffs(hm) - 1;
      hm &= hm - 1;
      const FeatRec& r = R[f];
      if (r.namb > AMB_MAX) {  // overflow: exact replay of this feature from b
        Chosen c = scan_feature<SCAN_REPLAY>(S, H, k, f, E, b, cs, s_gains[warp], nullptr);
        if (c.cand >= 0) {
          b = c.gain;
          cf = f;
          cidx = c.cand;
        }
        continue;
      }
      for (int a = 0; a < r.namb; ++a)
        if (r.amb_gain[a] > b + K_RT_EPS) {
          b = r.amb_gain[a];
          cf = f;
          cidx = r.amb_idx[a];
        }
    }
  }
  if (lane == 0) {
    best->feature = -1;
    best->is_cat = 0;
    best->ncat = 0;
    best->default_left = 1;
    best->bin = 0;
    best->lg = best->lh = best->rg = best->rh = 0.0;
    best->wl = best->wr = 0.0;
    if (d == 0) S.stats[ni] = make_double2(E.tg, E.th);
  }
  __syncwarp();
  if (cf >= 0) scan_feature<SCAN_EXTRACT>(S, H, k, cf, E, 0.0, cs, nullptr, best, nullptr, cidx);
  __syncwarp();
  NodeSplit& o = S.split[ni];
  if (lane == 0) {
    const bool found = cf >= 0 && b > K_RT_EPS;
    const bool valid = found && b > S.gamma && best->lh >= S.reg.mcw && best->rh >= S.reg.mcw;
    o.loss_chg = found ? b : 0.0;
    o.lg = best->lg;
    o.lh = best->lh;
    o.rg = best->rg;
    o.rh = best->rh;
    o.wl = best->wl;
    o.wr = best->wr;
    o.feature = best->feature;
    o.bin = best->bin;
    o.default_left = best->default_left;
    o.is_cat = best->is_cat;
    o.ncat = best->is_cat ? best->ncat : 0;
    o.valid = valid ? 1 : 0;
  }
  if (cf >= 0 && best->is_cat) {
    for (int i = lane; i < MAX_CAT_BINS / 32; i += 32) o.cat_mask[i] = best->cat_mask[i];
    for (int i = lane; i < best->ncat; i += 32) o.cat_order[i] = best->cat_order[i];
  }
}
__global__ void __launch_bounds__(EVAL_THREADS) k_eval_pick(BState S, int d) { k_eval_pick_body(S, blockIdx.x, gridDim.x, d); }
__global__ void __launch_bounds__(EVAL_THREADS) k_eval_pick_jobs(JobGrid J, int d) {
  const int j = job_of(J, blockIdx.x);
  k_eval_pick_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j], d);
}

__device__ sb_node make_leaf(float value, float sum_hess) {  // Node::leaf, regtree.rs:51-65
  sb_node nd;
  nd.left = -1;
  nd.right = -1;
  nd.split_feature = 0;
  nd.split_cond = 0.0f;
  nd.leaf_value = value;
  nd.sum_hess = sum_hess;
  nd.split_gain = 0.0f;
  nd.default_left = 1;
  nd.is_categorical = 0;
  nd.reserved = 0;
  nd.cat_begin = 0;
  nd.cat_end = 0;
  return nd;
}

// Expand the frontier of level d: child ids in the reference's order
// (left = num_nodes + 2 * rank among split nodes), child state, final leaf
// values, and the level's partition tiles.
__device__ __forceinline__ void k_assign_body(const BState& S, unsigned bx, unsigned gdx, int d, int write_tiles) {
  __shared__ int sm_i[33];
  __shared__ int s_tile_carry;
  __shared__ int s_toff[1024], s_nid[1024];
  __shared__ uint2 s_seg[1024];
  const unsigned long long round = *S.round;
  const int tid = threadIdx.x;
  const bool last = !S.lossguide && (d + 1 == S.max_depth);
  for (int k = bx; k < S.K; k += gdx) {  // one class tree per block
    const int begin = S.lvl_begin[k], cnt = S.lvl_count[k], nn0 = S.num_nodes[k];
    if (write_tiles) {  // reserve the tree's partition tiles (their order in the list is free)
      int mine = 0;
      for (int q = tid; q < cnt; q += blockDim.x) {
        const uint2 sg = S.seg[NI(S, k, begin + q)];
        mine += (int)((sg.y - sg.x + PART_TILE - 1) / PART_TILE);
      }
      int all;
      block_scan_excl<int>(mine, &all, sm_i);
      if (tid == 0) s_tile_carry = all ? atomicAdd(S.ptile_count, all) : 0;
      __syncthreads();
    }
    const size_t t = (size_t)round * S.K + k;
    sb_node* out = S.out_nodes + t * S.maxn;
    uint32_t* ocats = S.out_cats ? S.out_cats + t * S.cat_cap : nullptr;
    const uint64_t tkey = sb_tree_key(S.seed, round + S.round_base, (uint64_t)(k + S.k_base));
    int carry_v = 0, carry_c = S.cat_count[k];
    for (int c0 = 0; c0 < cnt; c0 += blockDim.x) {
      const int slot = c0 + tid;
      const bool act = slot < cnt;
      const int nid = begin + slot;
      const size_t ni = act ? NI(S, k, nid) : 0;
      const NodeSplit* sp = act ? &S.split[ni] : nullptr;
      const int v = (act && sp->valid) ? 1 : 0;
      const int nc = (v && sp->is_cat) ? sp->ncat : 0;
      int tot_v, tot_c;
      const int rank = carry_v + block_scan_excl<int>(v, &tot_v, sm_i);
      const int coff = carry_c + block_scan_excl<int>(nc, &tot_c, sm_i);
      int tiles = 0;
      if (act) {
        const double2 st = S.stats[ni];
        const double2 bd = S.bounds[ni];
        if (d == 0) out[0] = make_leaf(0.0f, (float)st.y);  // RegTree::with_root
        const uint2 sg = S.seg[ni];
        tiles = (int)((sg.y - sg.x + PART_TILE - 1) / PART_TILE);
        S.fill[ni] = Fill{0u, 0u};
        if (v) {
          const int left = nn0 + 2 * rank, right = left + 1;
          const int f = sp->feature;
          const int dr = S.mono ? S.mono[f] : 0;
          double2 lb = bd, rb = bd;  // child_bounds, constraints.rs:94-124
          if (dr != 0) {
            double mid = dmul(0.5, dadd(sp->wl, sp->wr));
            if (dr > 0) { lb = make_double2(bd.x, mid); rb = make_double2(mid, bd.y); }
            else { lb = make_double2(mid, bd.y); rb = make_double2(bd.x, mid); }
          }
          sb_node& pn = out[nid];  // expand / expand_categorical, regtree.rs:129-186
          pn.split_feature = (uint32_t)f;
          pn.default_left = (uint8_t)sp->default_left;
          pn.left = left;
          pn.right = right;
          pn.split_gain = (float)sp->loss_chg;
          if (sp->is_cat) {
            pn.is_categorical = 1;
            pn.cat_begin = (uint32_t)coff;
            pn.cat_end = (uint32_t)(coff + sp->ncat);
            const uint32_t fs = S.foff[f];
            for (int c = 0; c < sp->ncat; ++c)
              if (ocats && coff + c < S.cat_cap) ocats[coff + c] = f32_as_u32(S.cuts[fs + sp->cat_order[c]]);
          } else {
            pn.split_cond = S.cuts[S.foff[f] + sp->bin];
          }
          out[left] = make_leaf((float)sp->wl, (float)sp->lh);
          out[right] = make_leaf((float)sp->wr, (float)sp->rh);
          // interaction constraints (intersect_allowed, hist.rs:736-747)
          const size_t li = NI(S, k, left), ri = NI(S, k, right);
          const bool pall = S.allowed_all[ni];
          const bool fall = !S.has_inter || !S.in_group[f];
          const bool call = pall && fall;
          for (int w = 0; w < S.FW; ++w) {
            uint32_t a = pall ? 0xFFFFFFFFu : S.allowed[ni * S.FW + w];
            uint32_t b = fall ? 0xFFFFFFFFu : S.iset[(size_t)f * S.FW + w];
            uint32_t x = a & b;
            S.allowed[li * S.FW + w] = x;
            S.allowed[ri * S.FW + w] = x;
          }
          S.allowed_all[li] = call;
          S.allowed_all[ri] = call;
          S.stats[li] = make_double2(sp->lg, sp->lh);
          S.stats[ri] = make_double2(sp->rg, sp->rh);
          S.bounds[li] = lb;
          S.bounds[ri] = rb;
          S.parent[li] = nid;
          S.parent[ri] = nid;
          S.built[li] = 0;
          S.built[ri] = 0;
          S.split[li].valid = 0;
          S.split[ri].valid = 0;
          // the launch has at most 1024 threads in all when per-node sampling is on
          uint32_t* scratch =
              S.samp_scratch ? S.samp_scratch + ((size_t)bx * blockDim.x + tid) * S.F : nullptr;
          if (!last) {
            node_feature_mask(S, k, left, tkey, S.fmask + li * S.FW, S.allowed + li * S.FW, call, scratch);
            node_feature_mask(S, k, right, tkey, S.fmask + ri * S.FW, S.allowed + ri * S.FW, call, scratch);
          } else {  // children at max_depth are final leaves
            float lv = __fmul_rn((float)calc_weight_bounded(sp->lg, sp->lh, S.reg, lb.x, lb.y), S.eta);
            float rv = __fmul_rn((float)calc_weight_bounded(sp->rg, sp->rh, S.reg, rb.x, rb.y), S.eta);
            out[left].leaf_value = lv;
            out[right].leaf_value = rv;
            S.leafval[li] = lv;
            S.leafval[ri] = rv;
          }
        } else {  // final leaf (hist.rs:193-200 then scale_leaves)
          float lv = __fmul_rn((float)calc_weight_bounded(st.x, st.y, S.reg, bd.x, bd.y), S.eta);
          out[nid].leaf_value = lv;
          S.leafval[ni] = lv;
        }
      }
      // partition tiles of this chunk's frontier nodes: one thread per tile,
      // its node found by a binary search over the chunk's tile offsets
      int tot_t;
      const int toff = block_scan_excl<int>(tiles, &tot_t, sm_i);
      if (write_tiles) {
        s_toff[tid] = toff + tiles;  // inclusive end
        if (act) {
          s_seg[tid] = S.seg[ni];
          s_nid[tid] = nid;
        }
        __syncthreads();
        const int nact = min(cnt - c0, (int)blockDim.x);
        for (int q = tid; q < tot_t; q += blockDim.x) {
          int lo = 0, hi = nact - 1;  // first node whose end exceeds q
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s_toff[mid] > q) hi = mid; else lo = mid + 1;
          }
          const int qi = q - (s_toff[lo] - (int)((s_seg[lo].y - s_seg[lo].x + PART_TILE - 1) / PART_TILE));
          const unsigned b = s_seg[lo].x + (unsigned)qi * PART_TILE;
          const unsigned e = min(s_seg[lo].y, b + PART_TILE);
          const int slot_t = s_tile_carry + q;
          if (slot_t < S.ptile_cap) S.ptiles[slot_t] = make_int4(k, s_nid[lo], (int)b, (int)e);
        }
      }
      __syncthreads();
      if (tid == 0) s_tile_carry += tot_t;
      carry_v += tot_v;
      carry_c += tot_c;
      __syncthreads();
    }
    __syncthreads();
    if (tid == 0) {
      S.prev_begin[k] = begin;
      S.prev_count[k] = cnt;
      S.lvl_begin[k] = nn0;
      S.lvl_count[k] = 2 * carry_v;
      S.num_nodes[k] = nn0 + 2 * carry_v;
      S.cat_count[k] = carry_c;
    }
    __syncthreads();
  }
}
__global__ void __launch_bounds__(1024) k_assign(BState S, int d, int write_tiles) { k_assign_body(S, blockIdx.x, gridDim.x, d, write_tiles); }
__global__ void __launch_bounds__(1024) k_assign_jobs(JobGrid J, int d, int write_tiles) {
  const int j = job_of(J, blockIdx.x);
  k_assign_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j], d, write_tiles);
}

// K7 + K8: partition every split node's rows into its two children (left rows
// fill the segment from its start, right rows from its end), and the margin
// update (train.rs:326-328) for rows whose node is final. A warp walks 32
// consecutive positions per step (coalesced row-id loads); ballots compact the
// left / right rows into contiguous runs (coalesced stores); the split
// feature's codes come from the feature-major copy, read in ascending row
// order within each run so shallow levels share DRAM sectors.
constexpr int PART_THREADS = 256;
constexpr int PART_WARPS = PART_THREADS / 32;
constexpr int PART_STEPS = PART_TILE / PART_THREADS;  // 32-row steps per warp
__device__ __forceinline__ void k_partition_body(const BState& S, unsigned bx, unsigned gdx, int d) {
  __shared__ unsigned int s_wl[PART_WARPS], s_wa[PART_WARPS];
  __shared__ unsigned int s_base[2];
  const bool last = !S.lossguide && (d + 1 == S.max_depth);
  const int ntiles = min(*S.ptile_count, S.ptile_cap);
  // lossguide: from the tree's list into the scratch list (k_lg_copy moves it back)
  const uint32_t* rows_cur_all = (!S.lossguide && (d & 1)) ? S.rows1 : S.rows0;
  uint32_t* rows_nxt_all = (!S.lossguide && (d & 1)) ? S.rows0 : S.rows1;
  const int K = S.K;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (int t = bx; t < ntiles; t += gdx) {
    const int4 tile = S.ptiles[t];
    const int k = tile.x, nid = tile.y;
    const size_t ni = NI(S, k, nid);
    const uint32_t* rows_cur = rows_cur_all + (d == 0 ? 0 : (size_t)k * S.n);
    uint32_t* rows_nxt = rows_nxt_all + (size_t)k * S.n;
    if (!S.split[ni].valid) {  // a final leaf: its rows take the leaf value
      const float lv = S.leafval[ni];
      for (int p = tile.z + threadIdx.x; p < tile.w; p += PART_THREADS) {
        const uint32_t rv = rows_cur[p];
        const uint32_t id = rv & ~UNSAMPLED;
        if (S.update_margin) S.delta[(size_t)id * K + k] = lv;
        if (S.row_leaf) S.row_leaf[id] = (rv & UNSAMPLED) ? -1 : nid;
      }
      continue;
    }
    const NodeSplit& sp = S.split[ni];
    const int f = sp.feature, dl = sp.default_left, isc = sp.is_cat;
    const int fb = S.fbase[f], fmc = S.fmiss[f];
    const int sbin_code = fb + sp.bin;  // numeric: left iff code <= fbase + split bin
    const uint16_t* col = S.bins_col + (size_t)f * S.n;
    const int wbeg = tile.z + warp * (PART_STEPS * 32);
    uint32_t rv[PART_STEPS];
    unsigned lm[PART_STEPS];
    unsigned nl = 0, na = 0;  // lane-uniform warp totals
#pragma unroll
    for (int i = 0; i < PART_STEPS; ++i) {
      const int p = wbeg + i * 32 + lane;
      const bool valid = p < tile.w;
      rv[i] = valid ? rows_cur[p] : UNSAMPLED;
    }
    int code[PART_STEPS];
#pragma unroll
    for (int i = 0; i < PART_STEPS; ++i)
      code[i] = (wbeg + i * 32 + lane < tile.w) ? (int)col[rv[i] & ~UNSAMPLED] : 0;
#pragma unroll
    for (int i = 0; i < PART_STEPS; ++i) {
      const bool valid = wbeg + i * 32 + lane < tile.w;
      const int c = code[i];
      bool go;
      if (c == fmc) go = dl != 0;
      else if (isc) {
        const int b = c - fb;
        go = (sp.cat_mask[b >> 5] >> (b & 31)) & 1u;
      } else go = c <= sbin_code;
      lm[i] = __ballot_sync(0xFFFFFFFFu, valid && go);
      const unsigned vm = __ballot_sync(0xFFFFFFFFu, valid);
      nl += __popc(lm[i]);
      na += __popc(vm);
    }
    if (last) {  // children are final leaves: margins only
      const int left_id = S.out_nodes[((size_t)(*S.round) * K + k) * S.maxn + nid].left;
      const size_t li = NI(S, k, left_id);
      const float lv = S.leafval[li], rvv = S.leafval[li + 1];
#pragma unroll
      for (int i = 0; i < PART_STEPS; ++i) {
        if (wbeg + i * 32 + lane >= tile.w) continue;
        const uint32_t id = rv[i] & ~UNSAMPLED;
        const bool go = (lm[i] >> lane) & 1u;
        if (S.update_margin) S.delta[(size_t)id * K + k] = go ? lv : rvv;
        if (S.row_leaf) S.row_leaf[id] = (rv[i] & UNSAMPLED) ? -1 : (go ? left_id : left_id + 1);
      }
      continue;
    }
    if (lane == 0) {
      s_wl[warp] = nl;
      s_wa[warp] = na;
    }
    Fill* fl = &S.fill[ni];
    __syncthreads();
    if (threadIdx.x == 0) {  // one 64-bit atomic per tile reserves both children's places
      unsigned tl = 0, ta = 0;
      for (int w = 0; w < PART_WARPS; ++w) {
        tl += s_wl[w];
        ta += s_wa[w];
      }
      const unsigned long long old = atomicAdd(reinterpret_cast<unsigned long long*>(fl),
                                               ((unsigned long long)(ta - tl) << 32) | tl);
      s_base[0] = (unsigned)old;
      s_base[1] = (unsigned)(old >> 32) + (ta - tl);  // right rows fill downwards
    }
    __syncthreads();
    unsigned wl = 0, wa = 0;  // rows of earlier warps of this tile
    for (int w = 0; w < warp; ++w) {
      wl += s_wl[w];
      wa += s_wa[w];
    }
    const uint2 sg = S.seg[ni];
    unsigned lpos = sg.x + s_base[0] + wl;            // next left slot of this warp
    unsigned rpos = sg.y - s_base[1] + (wa - wl);     // next right slot of this warp
#pragma unroll
    for (int i = 0; i < PART_STEPS; ++i) {
      const bool valid = wbeg + i * 32 + lane < tile.w;
      const unsigned vm = __ballot_sync(0xFFFFFFFFu, valid);
      const unsigned rm = vm & ~lm[i];
      if ((lm[i] >> lane) & 1u) rows_nxt[lpos + __popc(lm[i] & lt)] = rv[i];
      else if (valid) rows_nxt[rpos + __popc(rm & lt)] = rv[i];
      lpos += __popc(lm[i]);
      rpos += __popc(rm);
    }
    __syncthreads();
  }
}
__global__ void __launch_bounds__(PART_THREADS, 4) k_partition(BState S, int d) { k_partition_body(S, blockIdx.x, gridDim.x, d); }
__global__ void __launch_bounds__(PART_THREADS, 4) k_partition_jobs(JobGrid J, int d) {
  const int j = job_of(J, blockIdx.x);
  k_partition_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j], d);
}

// After the partition: children segments and sampled counts, the smaller
// child to build (hist.rs:352-362: left when left_rows <= right_rows), and
// the histogram work list of level d + 1.
__device__ __forceinline__ void k_plan_body(const BState& S, unsigned bx, unsigned gdx, int d) {
  constexpr int GROUP = 1024;  // class trees per pass over the (tree, node) pairs
  __shared__ int sm_i[33];
  __shared__ unsigned long long sm_u[33];
  __shared__ int s_items;
  __shared__ unsigned long long s_pos;
  __shared__ int s_off[GROUP + 1];
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_items = 0;
    s_pos = 0;
  }
  __syncthreads();
  const unsigned long long round = *S.round;
  const int dn = d + 1;
  for (int k0 = 0; k0 < S.K; k0 += GROUP) {
    const int nk = min(GROUP, S.K - k0);
    // offsets of the group's frontiers in its list of (tree, node) pairs
    int base = 0;  // the same in every thread
    for (int j0 = 0; j0 < nk; j0 += blockDim.x) {
      const int j = j0 + tid;
      int tot;
      const int o = block_scan_excl<int>(j < nk ? S.prev_count[k0 + j] : 0, &tot, sm_i);
      if (j < nk) s_off[j] = base + o;
      base += tot;
    }
    if (tid == 0) s_off[nk] = base;
    __syncthreads();
    const int pairs = s_off[nk];
    for (int c0 = 0; c0 < pairs; c0 += blockDim.x) {
      const int q = c0 + tid;
      int v = 0, k = k0, bchild = -1;
      unsigned long long len = 0;
      uint2 bseg = make_uint2(0, 0);
      if (q < pairs) {
        int lo = 0, hi = nk;  // the last tree whose offset is <= q
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (s_off[mid] <= q) lo = mid; else hi = mid;
        }
        k = k0 + lo;
        const int nid = S.prev_begin[k] + (q - s_off[lo]);
        const size_t ni = NI(S, k, nid);
        if (S.split[ni].valid) {
          const sb_node* out = S.out_nodes + ((size_t)round * S.K + k) * S.maxn;
          const Fill fl = S.fill[ni];
          const uint2 sg = S.seg[ni];
          const int l = out[nid].left, r = l + 1;
          const size_t li = NI(S, k, l), ri = NI(S, k, r);
          S.seg[li] = make_uint2(sg.x, sg.x + fl.left);
          S.seg[ri] = make_uint2(sg.x + fl.left, sg.y);
          S.nsamp[li] = fl.left;
          S.nsamp[ri] = fl.right;
          const bool build_left = fl.left <= fl.right;
          S.built[li] = build_left ? 1 : 0;
          S.built[ri] = build_left ? 0 : 1;
          bchild = build_left ? l : r;
          bseg = build_left ? S.seg[li] : S.seg[ri];
          v = 1;
          len = bseg.y - bseg.x;
        }
      }
      int tot_v;
      const int idx = s_items + block_scan_excl<int>(v, &tot_v, sm_i);
      unsigned long long tot_len;
      const unsigned long long pos = s_pos + block_scan_excl<unsigned long long>(len, &tot_len, sm_u);
      if (v) {
        HistItem it;
        it.rows = ((!S.lossguide && (dn & 1)) ? S.rows1 : S.rows0) + (size_t)k * S.n;
        it.begin = bseg.x;
        it.end = bseg.y;
        it.k = (uint32_t)k;
        it.root = 0;
        it.out = S.lossguide ? node_hist(S, k, bchild) : level_hist(S, dn, k, bchild - S.lvl_begin[k]);
        it.total = nullptr;
        S.items[idx] = it;
        S.prefix[idx] = pos;
      }
      __syncthreads();
      if (tid == 0) {
        s_items += tot_v;
        s_pos += tot_len;
      }
      __syncthreads();
    }
  }
  if (tid == 0) {
    *S.item_count = s_items;
    S.prefix[s_items] = s_pos;
    *S.ptile_count = 0;  // the partition has consumed this level's tiles
  }
}
__global__ void __launch_bounds__(1024) k_plan(BState S, int d) { k_plan_body(S, blockIdx.x, gridDim.x, d); }
__global__ void __launch_bounds__(1024) k_plan_jobs(JobGrid J, int d) {
  const int j = job_of(J, blockIdx.x);
  k_plan_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j], d);
}

// ------------------------------------------------------- lossguide growth
// grow_lossguide (hist.rs:238-268): per class tree, a max-heap of evaluated
// nodes keyed by loss_chg; each step pops the next node to expand, and the
// step's kernels (assign, partition, histogram of the smaller child,
// evaluation of both children) run for all K trees at once.

// One block per class tree. Pushes the children evaluated by the last step
// (or the root, `init`), then pops until a node that may be split: the steps
// of Rust's BinaryHeap (sift_up on push; swap with the last entry,
// sift_down_to_bottom and sift_up on pop), run by one thread on a
// shared-memory copy of the queue, so equal keys leave in the same order.
__global__ void __launch_bounds__(256) k_lg_heap(BState S, int init) {
  extern __shared__ HeapEnt sh_heap[];  // [maxn]
  __shared__ int s_size;
  const int k = blockIdx.x, tid = threadIdx.x;
  HeapEnt* gh = S.heap + (size_t)k * S.maxn;
  if (tid == 0) s_size = init ? 0 : S.heap_size[k];
  __syncthreads();
  const int size0 = s_size;
  for (int i = tid; i < size0; i += blockDim.x) sh_heap[i] = gh[i];
  __syncthreads();
  if (tid == 0) {
    HeapEnt* h = sh_heap;
    int size = size0;
    auto sift_up = [&](int start, int pos) {
      const HeapEnt hole = h[pos];
      while (pos > start) {
        const int par = (pos - 1) / 2;
        if (hole.key <= h[par].key) break;
        h[pos] = h[par];
        pos = par;
      }
      h[pos] = hole;
    };
    auto push = [&](HeapEnt e) {
      h[size] = e;
      size++;
      sift_up(0, size - 1);
    };
    auto pop = [&]() {
      HeapEnt item = h[size - 1];
      size--;
      if (size > 0) {
        const HeapEnt top = h[0];
        h[0] = item;
        item = top;
        // sift_down_to_bottom(0)
        const int end = size;
        int pos = 0;
        const HeapEnt hole = h[0];
        int child = 1;
        while (end >= 2 && child <= end - 2) {
          child += (h[child].key <= h[child + 1].key) ? 1 : 0;
          h[pos] = h[child];
          pos = child;
          child = 2 * pos + 1;
        }
        if (child == end - 1) {
          h[pos] = h[child];
          pos = child;
        }
        h[pos] = hole;
        sift_up(0, pos);
      }
      return item;
    };
    sb_node* out = S.out_nodes + ((size_t)(*S.round) * S.K + k) * S.maxn;
    if (init) {
      const size_t r = NI(S, k, 0);
      out[0] = make_leaf(0.0f, (float)S.stats[r].y);  // RegTree::with_root
      push(HeapEnt{total_cmp_key(S.split[r].loss_chg), 0, 0});
      S.n_leaves[k] = 1;
    } else if (S.prev_count[k] > 0) {  // heap.push(l); heap.push(r)
      for (int c = 0; c < S.lvl_count[k]; ++c) {
        const int nid = S.lvl_begin[k] + c;
        const size_t ni = NI(S, k, nid);
        const int dep = S.ndepth[NI(S, k, S.parent[ni])] + 1;
        S.ndepth[ni] = dep;
        push(HeapEnt{total_cmp_key(S.split[ni].loss_chg), nid, dep});
      }
    }
    int expand = -1, nl = S.n_leaves[k];
    while (size > 0) {
      const HeapEnt e = pop();
      if (nl >= S.max_leaves) {
        size = 0;
        break;
      }
      if (e.depth >= S.depth_limit || !S.split[NI(S, k, e.nid)].valid) continue;  // permanent leaf
      expand = e.nid;
      nl++;  // one leaf becomes two
      break;
    }
    S.n_leaves[k] = nl;
    S.lvl_begin[k] = expand >= 0 ? expand : S.num_nodes[k];
    S.lvl_count[k] = expand >= 0 ? 1 : 0;
    s_size = size;
  }
  __syncthreads();
  const int size1 = s_size;
  for (int i = tid; i < size1; i += blockDim.x) gh[i] = sh_heap[i];
  if (tid == 0) S.heap_size[k] = size1;
}

// The expanded node's partitioned rows back into the tree's row list.
__global__ void k_lg_copy(BState S) {
  const int ntiles = min(*S.ptile_count, S.ptile_cap);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tile = S.ptiles[t];
    const size_t base = (size_t)tile.x * S.n;
    for (int p = tile.z + threadIdx.x; p < tile.w; p += blockDim.x) S.rows0[base + p] = S.rows1[base + p];
  }
}

// Leaf values of every leaf (hist.rs:193-200 then scale_leaves) and the
// leaf value of each of its rows (the margin update, train.rs:326-328).
__global__ void k_lg_finalize(BState S) {
  const int k = blockIdx.y, nid = blockIdx.x;
  if (nid >= S.num_nodes[k]) return;
  const size_t ni = NI(S, k, nid);
  sb_node* out = S.out_nodes + ((size_t)(*S.round) * S.K + k) * S.maxn;
  if (out[nid].left != -1) return;
  const double2 st = S.stats[ni], bd = S.bounds[ni];
  const float lv = __fmul_rn((float)calc_weight_bounded(st.x, st.y, S.reg, bd.x, bd.y), S.eta);
  if (threadIdx.x == 0) {
    out[nid].leaf_value = lv;
    S.leafval[ni] = lv;
  }
  if (!S.row_leaf) return;  // k_lg_route gives every row its leaf values
  const uint2 sg = S.seg[ni];
  const uint32_t* rows = S.rows0 + (nid == 0 ? 0 : (size_t)k * S.n);  // an unsplit root keeps the shared list
  for (uint32_t p = sg.x + threadIdx.x; p < sg.y; p += blockDim.x) {
    const uint32_t rv = rows[p];
    const uint32_t id = rv & ~UNSAMPLED;
    if (S.update_margin) S.delta[(size_t)id * S.K + k] = lv;
    if (S.row_leaf) S.row_leaf[id] = (rv & UNSAMPLED) ? -1 : nid;
  }
}

// Every row's leaf value in each class tree of the round (the margin update,
// train.rs:326-328), sampled or not: the row is routed through the finished
// tree with its row-major codes, whose few sectors stay in cache for all K
// trees, and its K values are stored together. This replaces per-leaf writes
// scattered over the whole delta array (and routing the unsampled rows alone).
// The decisions are the partition's: missing -> default direction,
// categorical -> the node's category set, numeric -> local bin <= split bin.
__global__ void k_lg_route(BState S) {
  const unsigned long long round = *S.round;
  const int K = S.K;
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < S.n; r += (size_t)gridDim.x * blockDim.x) {
    const uint16_t* row = S.bins ? S.bins + r * S.Fp : nullptr;
    const uint8_t* row8 = S.bins8 ? S.bins8 + r * S.Fp : nullptr;
    for (int k = 0; k < K; ++k) {
      const sb_node* out = S.out_nodes + ((size_t)round * K + k) * S.maxn;
      int nid = 0;
      while (out[nid].left != -1) {
        const NodeSplit& sp = S.split[NI(S, k, nid)];
        const int f = sp.feature;
        const int code = row8 ? (int)row8[S.rpos[f]] : (int)row[S.rpos[f]];
        bool go;
        if (code == S.rmiss[f]) go = sp.default_left != 0;
        else {
          const int c = code - S.rbase[f];
          go = sp.is_cat ? ((sp.cat_mask[c >> 5] >> (c & 31)) & 1u) != 0 : c <= sp.bin;
        }
        nid = go ? out[nid].left : out[nid].right;
      }
      S.delta[r * K + k] = S.leafval[NI(S, k, nid)];
    }
  }
}

// margin += the last tree's leaf values, when no further round folds them in
__global__ void k_apply_delta(float* __restrict__ margin, const float* __restrict__ delta, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    margin[i] = __fadd_rn(margin[i], delta[i]);
}

__device__ __forceinline__ void k_round_end_body(const BState& S, unsigned bx, unsigned gdx) {
  const unsigned long long round = *S.round;
  for (int k = threadIdx.x; k < S.K; k += blockDim.x) {
    size_t t = (size_t)round * S.K + k;
    S.out_nnodes[t] = S.num_nodes[k];
    S.out_ncats[t] = S.cat_count[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *S.round = round + 1;
    *S.kept = 0;
    *S.unkept = 0;
    if (S.fixed)
      for (int i = 0; i < 2 * S.K; ++i) S.maxabs[i] = 0u;
  }
}
__global__ void k_round_end(BState S) { k_round_end_body(S, blockIdx.x, gridDim.x); }
__global__ void k_round_end_jobs(JobGrid J) {
  const int j = job_of(J, blockIdx.x);
  k_round_end_body(J.states[j], blockIdx.x - J.xoff[j], J.xoff[j + 1] - J.xoff[j]);
}

}  // namespace

// Packs f32 pairs to fixed point with the power-of-two scales of their max.
int quantize_pairs(sb_ctx* ctx, const float2* d_gp, size_t n, int bits, unsigned long long* d_packed,
                   int* h_shift_g, int* h_shift_h);

}  // namespace sb

// ===================================================================== booster
struct sb_booster {
  sb_ctx* ctx = nullptr;
  const sb_ghist* g = nullptr;
  sb_train_params p{};
  std::vector<int8_t> mono;
  std::vector<uint32_t> ioff, ifeat;
  int K = 1;
  int D = 0;
  size_t n = 0;
  int maxn = 0, maxw = 0;
  int tree_cap = 0;
  int rounds_done = 0;
  float base_score = 0.0f;
  bool ext = false;
  int timing = 0;
  sb_booster_stats stats{};
  sb::BState S{};
  // owned device buffers
  sb::DBuf<int8_t> d_mono;
  sb::DBuf<uint8_t> d_in_group;
  sb::DBuf<uint32_t> d_iset;
  sb::DBuf<unsigned long long> d_round;
  sb::DBuf<double2> d_stats, d_bounds;
  sb::DBuf<uint32_t> d_allowed, d_fmask;
  sb::DBuf<uint8_t> d_allowed_all, d_built;
  sb::DBuf<uint2> d_seg;
  sb::DBuf<uint32_t> d_nsamp;
  sb::DBuf<int> d_parent;
  sb::DBuf<sb::NodeSplit> d_split;
  sb::DBuf<float> d_leafval;
  sb::DBuf<sb::Fill> d_fill;
  sb::DBuf<int> d_lvl;  // 5*K ints
  sb::DBuf<uint32_t> d_rows0, d_rows1;
  sb::DBuf<unsigned int> d_kept;
  sb::DBuf<float> d_margin, d_labels, d_weights;
  sb::DBuf<float> d_delta;   // [n][K] leaf values of the last tree, not yet in d_margin
  mutable bool delta_pending = false;  // margins are read through const handles
  bool use_graphs = true;              // replay steady-state rounds as a CUDA graph
  cudaGraphExec_t graph_exec = nullptr;
  uint64_t graph_nodes = 0;            // kernels in the recorded round
  sb::BState prev_key;                 // device state of the previous round
  bool have_prev_key = false;
  sb::DBuf<float2> d_gpair;
  sb::DBuf<unsigned long long> d_gpk;
  sb::DBuf<unsigned int> d_maxabs;
  sb::DBuf<int> d_shifts;
  sb::DBuf<double> d_inv_scale;
  sb::DBuf<unsigned long long> d_qerr;
  sb::DBuf<char> d_hist0, d_hist1;
  bool lossguide = false;
  int leaves = 0, steps = 0;              // lossguide: leaf budget, expansions per tree
  sb::DBuf<char> d_nhist;                 // lossguide: [K][maxn][HB] node histograms
  sb::DBuf<sb::HeapEnt> d_heap;           // lossguide: [K][maxn] queues
  sb::DBuf<int> d_heap_size;              // lossguide: [K] sizes, then [K] leaf counts
  sb::DBuf<int> d_ndepth;                 // lossguide: [K][maxn] node depths
  sb::DBuf<longlong2> d_root_total;
  sb::DBuf<sb::HistItem> d_items;
  sb::DBuf<uint64_t> d_prefix;
  sb::DBuf<int> d_item_count;
  sb::DBuf<int4> d_ptiles;
  sb::DBuf<int> d_ptile_count;
  sb::DBuf<uint32_t> d_pool, d_upool, d_pool_mask, d_usable;
  sb::DBuf<int> d_pool_len, d_upool_len;
  sb::DBuf<double> d_mbuf;
  sb::DBuf<sb::FeatRec> d_frec;
  sb::DBuf<uint32_t> d_samp;
  sb::DBuf<sb_node> d_out_nodes;
  sb::DBuf<uint32_t> d_out_cats;
  sb::DBuf<int> d_out_nnodes, d_out_ncats;
  sb::DBuf<sb::FeatureTile> d_tiles;
  sb::DBuf<int32_t> d_row_leaf;
  sb::DBuf<unsigned long long> d_hist_rows;  // sampled rows seen by timed histogram launches
  std::vector<cudaEvent_t> ev;
  std::vector<int> ev_kind;  // 0 = hist pair, 1 = round pair
  std::vector<double> ev_bytes;
  std::vector<std::unique_ptr<sb::EvalSet>> evals;  // eval sets (sb_booster_eval_add)
};

namespace sb {

__global__ void k_pack(const float2* __restrict__ gp, size_t n, const unsigned int* __restrict__ maxabs,
                       int bits, unsigned long long* __restrict__ out, int* __restrict__ shifts) {
  int sg = quant_shift(__uint_as_float(maxabs[0]), bits);
  int sh = quant_shift(__uint_as_float(maxabs[1]), bits);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    shifts[0] = sg;
    shifts[1] = sh;
  }
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    float2 v = gp[i];
    int qg = __float2int_rn(ldexpf(v.x, sg)), qh = __float2int_rn(ldexpf(v.y, sh));
    out[i] = ((unsigned long long)(uint32_t)qg << 32) + (unsigned long long)(uint32_t)qh;
  }
}
__global__ void k_maxabs(const float2* __restrict__ gp, size_t n, unsigned int* __restrict__ maxabs) {
  float a = 0.f, b = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    a = fmaxf(a, fabsf(gp[i].x));
    b = fmaxf(b, fabsf(gp[i].y));
  }
  for (int o = 16; o > 0; o >>= 1) {
    a = fmaxf(a, __shfl_xor_sync(0xFFFFFFFFu, a, o));
    b = fmaxf(b, __shfl_xor_sync(0xFFFFFFFFu, b, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&maxabs[0], __float_as_uint(a));
    atomicMax(&maxabs[1], __float_as_uint(b));
  }
}

int quantize_pairs(sb_ctx* ctx, const float2* d_gp, size_t n, int bits, unsigned long long* d_packed,
                   int* h_shift_g, int* h_shift_h) {
  DBuf<unsigned int> mx;
  DBuf<int> sh;
  SB_TRY(mx.alloc(ctx, 2));
  SB_TRY(sh.alloc(ctx, 2));
  SB_CUDA(cudaMemsetAsync(mx.p, 0, 8, ctx->stream));
  unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8);
  if (blocks == 0) blocks = 1;
  SB_LAUNCH(ctx, k_maxabs, blocks, 256, 0, d_gp, n, mx.p);
  SB_LAUNCH(ctx, k_pack, blocks, 256, 0, d_gp, n, mx.p, bits, d_packed, sh.p);
  int hs[2];
  SB_CUDA(cudaMemcpyAsync(hs, sh.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  *h_shift_g = hs[0];
  *h_shift_h = hs[1];
  return SB_OK;
}

namespace {

// Objective::base_margin / prob_to_margin with TrainingParams::base_score
// (learner/train.rs:203-210) from host labels and weights.
float base_margin_of(const sb_train_params* p, const float* labels, const float* weights, size_t n, int K) {
  float base;
  if (K > 1) base = 0.0f;
  else if (p->has_base_score) {
    float bs = (float)p->base_score;
    if (p->objective == SB_OBJ_LOGISTIC) {
      float pp = bs < 1e-6f ? 1e-6f : (bs > 1.0f - 1e-6f ? 1.0f - 1e-6f : bs);
      base = logf(pp / (1.0f - pp));
    } else {
      base = bs;
    }
  } else {
    double mean = 0.0;
    if (weights) {
      double num = 0.0, den = 0.0;
      for (size_t i = 0; i < n; ++i) {
        num += (double)labels[i] * (double)weights[i];
        den += (double)weights[i];
      }
      mean = den > 0.0 ? num / den : 0.0;
    } else {
      double sum = 0.0;
      for (size_t i = 0; i < n; ++i) sum += (double)labels[i];
      mean = sum / (double)n;
    }
    if (p->objective == SB_OBJ_LOGISTIC) {
      double pp = mean < 1e-6 ? 1e-6 : (mean > 1.0 - 1e-6 ? 1.0 - 1e-6 : mean);
      base = (float)log(pp / (1.0 - pp));
    } else {
      base = (float)mean;
    }
  }
  return base;
}

// ----------------------------------------------------- tree_method=approx
// Row subset of round `round` with the hist path's keys (sample_rows,
// train.rs:465-475): rows[r] = r, flagged UNSAMPLED when not drawn.
__global__ void k_approx_rows(uint64_t seed, unsigned long long round, double subsample, size_t n,
                              uint32_t* __restrict__ rows, unsigned int* __restrict__ kept) {
  const uint64_t rk = sb_round_key(seed, round);
  unsigned int c = 0;
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    const bool keep = subsample >= 1.0 || sb_u01(sb_row_draw(rk, r)) < subsample;
    rows[r] = (uint32_t)r | (keep ? 0u : UNSAMPLED);
    c += keep ? 1u : 0u;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(kept, c);
}

__global__ void k_approx_fallback(uint64_t seed, unsigned long long round, size_t n, uint32_t* __restrict__ rows,
                                  const unsigned int* __restrict__ kept) {
  if (*kept == 0) rows[sb_row_fallback(sb_round_key(seed, round), n)] &= ~UNSAMPLED;  // train.rs:472-474
}

// Class k's gradient pairs and hessians out of the row-major [n][K] pairs.
__global__ void k_class_column(const float2* __restrict__ gp, size_t n, int K, int k, float2* __restrict__ out,
                               float* __restrict__ hess) {
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    const float2 v = gp[r * K + k];
    out[r] = v;
    hess[r] = v.y;
  }
}

// margin[r][k] += f32(leaf * eta) of the row's leaf in one tree, routed on
// the raw values (RegTree::predict_row, regtree.rs:213-242; train.rs:323-328).
__global__ void k_add_tree(const sb_node* __restrict__ nodes, const uint32_t* __restrict__ cats,
                           const float* __restrict__ X, size_t n, int F, float missing, int K, int k, float eta,
                           float* __restrict__ margin) {
  const bool miss_nan = isnan(missing);
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x) {
    int nid = 0;
    while (nodes[nid].left >= 0) {
      const sb_node nd = nodes[nid];
      const float v = X[r * F + nd.split_feature];
      bool left;
      if (miss_nan ? isnan(v) : v == missing) left = nd.default_left != 0;
      else if (nd.is_categorical) {
        const uint32_t c = f32_as_u32(v);
        left = false;
        for (uint32_t i = nd.cat_begin; i < nd.cat_end; ++i)
          if (cats[i] == c) {
            left = true;
            break;
          }
      } else {
        left = v < nd.split_cond;
      }
      nid = left ? nd.left : nd.right;
    }
    float* m = margin + r * K + k;
    *m = __fadd_rn(*m, __fmul_rn(nodes[nid].leaf_value, eta));
  }
}

int booster_alloc_trees(sb_booster* b, int need) {
  if (need <= b->tree_cap) return SB_OK;
  int cap = std::max(need, b->tree_cap * 2);
  cap = std::max(cap, 16);
  sb_ctx* ctx = b->ctx;
  DBuf<sb_node> nodes;
  DBuf<uint32_t> cats;
  DBuf<int> nn, nc;
  SB_TRY(nodes.alloc(ctx, (size_t)cap * b->maxn));
  if (b->S.cat_cap) SB_TRY(cats.alloc(ctx, (size_t)cap * b->S.cat_cap));
  SB_TRY(nn.alloc(ctx, cap));
  SB_TRY(nc.alloc(ctx, cap));
  if (b->tree_cap) {
    SB_CUDA(cudaMemcpyAsync(nodes.p, b->d_out_nodes.p, b->d_out_nodes.bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
    if (b->S.cat_cap)
      SB_CUDA(cudaMemcpyAsync(cats.p, b->d_out_cats.p, b->d_out_cats.bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
    SB_CUDA(cudaMemcpyAsync(nn.p, b->d_out_nnodes.p, b->d_out_nnodes.bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
    SB_CUDA(cudaMemcpyAsync(nc.p, b->d_out_ncats.p, b->d_out_ncats.bytes(), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  std::swap(b->d_out_nodes.p, nodes.p);
  std::swap(b->d_out_nodes.n, nodes.n);
  std::swap(b->d_out_cats.p, cats.p);
  std::swap(b->d_out_cats.n, cats.n);
  b->d_out_cats.ctx = ctx;
  std::swap(b->d_out_nnodes.p, nn.p);
  std::swap(b->d_out_nnodes.n, nn.n);
  std::swap(b->d_out_ncats.p, nc.p);
  std::swap(b->d_out_ncats.n, nc.n);
  b->d_out_nodes.ctx = b->d_out_nnodes.ctx = b->d_out_ncats.ctx = ctx;
  b->tree_cap = cap;
  b->S.out_nodes = b->d_out_nodes.p;
  b->S.out_cats = b->d_out_cats.p;
  b->S.out_nnodes = b->d_out_nnodes.p;
  b->S.out_ncats = b->d_out_ncats.p;
  return SB_OK;
}

int booster_init(sb_booster* b, sb_ctx* ctx, const sb_ghist* g, const sb_train_params* p, int K,
                 bool ext) {
  b->ctx = ctx;
  b->g = g;
  b->p = *p;
  b->K = K;
  b->ext = ext;
  b->n = g->n;
  const int F = (int)g->F;
  const int FW = (F + 31) / 32;
  SB_REQUIRE(K >= 1 && K <= 16, SB_ERR_UNSUPPORTED, "at most 16 outputs per round on the GPU");
  b->lossguide = p->grow_policy == SB_GROW_LOSSGUIDE;
  b->D = p->max_depth;
  if (b->lossguide) {  // one node expanded per tree and step
    b->leaves = p->max_leaves > 0 ? p->max_leaves : (1 << p->max_depth);
    b->steps = b->leaves - 1;
    if (p->max_depth > 0 && p->max_depth < 31) b->steps = std::min(b->steps, (1 << p->max_depth) - 1);
    b->maxn = 2 * b->leaves - 1;
    b->maxw = 2;
  } else {
    b->maxn = (1 << (b->D + 1)) - 1;
    b->maxw = 1 << (b->D - 1);
  }
  if (p->n_monotone > 0 && p->monotone) b->mono.assign(p->monotone, p->monotone + p->n_monotone);
  bool constrained = false;
  for (int8_t m : b->mono) constrained |= m != 0;
  std::vector<int8_t> mono_full(F, 0);
  for (int i = 0; i < F && i < (int)b->mono.size(); ++i) mono_full[i] = b->mono[i];
  std::vector<uint8_t> in_group(F, 0);
  std::vector<uint32_t> iset((size_t)F * FW, 0u);
  const bool has_inter = p->n_interaction_groups > 0;
  if (has_inter) {  // build_interaction_sets, hist.rs:715-731
    for (int gi = 0; gi < p->n_interaction_groups; ++gi) {
      uint32_t s = p->interaction_offsets[gi], e = p->interaction_offsets[gi + 1];
      for (uint32_t a = s; a < e; ++a) {
        uint32_t f = p->interaction_features[a];
        if ((int)f >= F) continue;
        in_group[f] = 1;
        for (uint32_t c = s; c < e; ++c) {
          uint32_t h = p->interaction_features[c];
          if ((int)h < F) iset[(size_t)f * FW + (h >> 5)] |= 1u << (h & 31);
        }
      }
    }
  }
  const size_t KN = (size_t)K * b->maxn;
  const size_t HB = g->total_bins + g->F;
  cudaStream_t st = ctx->stream;
  SB_TRY(b->d_mono.alloc_zero(ctx, F));
  SB_TRY(b->d_in_group.alloc_zero(ctx, F));
  SB_TRY(b->d_iset.alloc_zero(ctx, (size_t)F * FW));
  SB_CUDA(cudaMemcpyAsync(b->d_mono.p, mono_full.data(), F, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(b->d_in_group.p, in_group.data(), F, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(b->d_iset.p, iset.data(), iset.size() * 4, cudaMemcpyHostToDevice, st));
  SB_TRY(b->d_round.alloc_zero(ctx, 1));
  SB_CUDA(cudaMemsetAsync(b->d_round.p, 0, 8, st));
  SB_TRY(b->d_stats.alloc_zero(ctx, KN));
  SB_TRY(b->d_bounds.alloc_zero(ctx, KN));
  SB_TRY(b->d_allowed.alloc_zero(ctx, KN * FW));
  SB_TRY(b->d_fmask.alloc_zero(ctx, KN * FW));
  SB_TRY(b->d_allowed_all.alloc_zero(ctx, KN));
  SB_TRY(b->d_built.alloc_zero(ctx, KN));
  SB_TRY(b->d_seg.alloc_zero(ctx, KN));
  SB_TRY(b->d_nsamp.alloc_zero(ctx, KN));
  SB_TRY(b->d_parent.alloc_zero(ctx, KN));
  SB_TRY(b->d_split.alloc_zero(ctx, KN));
  SB_CUDA(cudaMemsetAsync(b->d_split.p, 0, b->d_split.bytes(), st));
  SB_TRY(b->d_leafval.alloc_zero(ctx, KN));
  SB_TRY(b->d_fill.alloc_zero(ctx, KN));
  SB_TRY(b->d_lvl.alloc_zero(ctx, 6 * K));
  SB_TRY(b->d_rows0.alloc_zero(ctx, (size_t)K * b->n));
  SB_TRY(b->d_rows1.alloc_zero(ctx, (size_t)K * b->n));
  SB_TRY(b->d_kept.alloc_zero(ctx, 2));  // kept, unkept
  SB_TRY(b->d_margin.alloc_zero(ctx, b->n * K));
  SB_TRY(b->d_delta.alloc_zero(ctx, b->n * K));
  SB_TRY(b->d_gpair.alloc_zero(ctx, (size_t)K * b->n));
  const bool fixed = p->hist_precision == SB_HIST_FIXED;
  if (fixed) SB_TRY(b->d_gpk.alloc_zero(ctx, (size_t)K * b->n));
  SB_TRY(b->d_maxabs.alloc_zero(ctx, 2 * K));
  SB_CUDA(cudaMemsetAsync(b->d_maxabs.p, 0, 8 * K, st));
  SB_TRY(b->d_shifts.alloc_zero(ctx, 2 * K));
  SB_CUDA(cudaMemsetAsync(b->d_shifts.p, 0, 8 * K, st));
  SB_TRY(b->d_inv_scale.alloc_zero(ctx, 2 * K));
  SB_TRY(b->d_qerr.alloc_zero(ctx, 1));
  SB_CUDA(cudaMemsetAsync(b->d_qerr.p, 0, 8, st));
  if (b->lossguide) {  // every node keeps its histogram until its children are evaluated
    SB_TRY(b->d_nhist.alloc_zero(ctx, KN * HB * 16));
    SB_TRY(b->d_heap.alloc_zero(ctx, KN));
    SB_TRY(b->d_heap_size.alloc_zero(ctx, 2 * K));
    SB_TRY(b->d_ndepth.alloc_zero(ctx, KN));
  } else {
    const size_t hist_bytes = (size_t)K * b->maxw * HB * 16;
    SB_TRY(b->d_hist0.alloc_zero(ctx, hist_bytes));
    SB_TRY(b->d_hist1.alloc_zero(ctx, hist_bytes));
  }
  SB_TRY(b->d_root_total.alloc_zero(ctx, K));
  SB_TRY(b->d_items.alloc_zero(ctx, (size_t)K * b->maxw + K));
  SB_TRY(b->d_prefix.alloc_zero(ctx, (size_t)K * b->maxw + K + 1));
  SB_TRY(b->d_item_count.alloc_zero(ctx, 1));
  const int ptile_cap = (int)((size_t)K * ((b->n + PART_TILE - 1) / PART_TILE + b->maxn + 1));
  SB_TRY(b->d_ptiles.alloc_zero(ctx, ptile_cap));
  SB_TRY(b->d_ptile_count.alloc_zero(ctx, 1));
  SB_TRY(b->d_pool.alloc_zero(ctx, (size_t)K * F));
  SB_TRY(b->d_pool_len.alloc_zero(ctx, K));
  SB_TRY(b->d_upool.alloc_zero(ctx, (size_t)K * F));
  SB_TRY(b->d_upool_len.alloc_zero(ctx, K));
  SB_TRY(b->d_pool_mask.alloc_zero(ctx, (size_t)K * FW));
  SB_TRY(b->d_mbuf.alloc_zero(ctx, (size_t)K * b->maxw * F));
  SB_TRY(b->d_frec.alloc_zero(ctx, (size_t)K * b->maxw * F));
  {
    std::vector<uint32_t> usable(FW, 0u);
    for (int f = 0; f < F; ++f)
      if (g->h_foff[f + 1] - g->h_foff[f] >= 2) usable[f >> 5] |= 1u << (f & 31);
    SB_TRY(b->d_usable.alloc_zero(ctx, FW));
    SB_CUDA(cudaMemcpyAsync(b->d_usable.p, usable.data(), FW * 4, cudaMemcpyHostToDevice, st));
  }
  // per-node sampling scratch: one row per k_assign thread (1024 in all) and per class tree (k_round_prep)
  if (p->colsample_bylevel < 1.0 || p->colsample_bynode < 1.0)
    SB_TRY(b->d_samp.alloc_zero(ctx, (size_t)std::max(1024, K) * F));
  SB_TRY(b->d_tiles.alloc_zero(ctx, g->tiles.size()));
  SB_CUDA(cudaMemcpyAsync(b->d_tiles.p, g->tiles.data(), g->tiles.size() * sizeof(FeatureTile),
                          cudaMemcpyHostToDevice, st));

  BState& S = b->S;
  S.K = K;
  S.F = F;
  S.FW = FW;
  S.HB = (int)HB;
  S.total_bins = (int)g->total_bins;
  S.max_depth = b->D;
  S.maxn = b->maxn;
  S.maxw = b->maxw;
  S.lossguide = b->lossguide ? 1 : 0;
  S.max_leaves = b->lossguide ? b->leaves : 0;
  S.depth_limit = p->max_depth > 0 ? p->max_depth : 0x7FFFFFFF;
  S.nhist = b->d_nhist.p;
  S.heap = b->d_heap.p;
  S.heap_size = b->d_heap_size.p;
  S.n_leaves = b->d_heap_size.p ? b->d_heap_size.p + K : nullptr;
  S.ndepth = b->d_ndepth.p;
  S.cat_cap = g->has_categorical ? (b->maxn / 2 + 1) * g->max_feature_bins : 0;
  S.cat_bins = 1;
  for (size_t f = 0; f < g->F; ++f)
    if (g->h_is_cat[f]) S.cat_bins = std::max(S.cat_bins, (int)(g->h_foff[f + 1] - g->h_foff[f]));
  S.n = b->n;
  S.Fp = g->Fp;
  S.bins = g->code_bytes == 1 ? nullptr : g->bins.p;
  S.bins8 = g->code_bytes == 1 ? g->bins8.p : nullptr;
  S.bins_col = g->bins_col.p;
  S.fbase = g->fbase.p;
  S.fmiss = g->fmiss.p;
  S.rpos = g->rpos.p;
  S.rbase = g->rbase.p;
  S.rmiss = g->rmiss.p;
  S.foff = g->foff.p;
  S.cuts = g->cuts.p;
  S.is_cat = g->is_cat.p;
  S.reg = RegP{p->lambda, p->alpha, p->max_delta_step, p->min_child_weight};
  S.gamma = p->gamma;
  S.eta = ext ? 1.0f : (float)p->eta;
  S.subsample = p->subsample;
  S.bytree = p->colsample_bytree;
  S.bylevel = p->colsample_bylevel;
  S.bynode = p->colsample_bynode;
  S.seed = p->seed;
  S.objective = p->objective;
  S.num_class = p->num_class;
  S.spw = (float)p->scale_pos_weight;
  S.fixed = fixed ? 1 : 0;
  S.bits = p->quantize_bits ? p->quantize_bits : 16;
  S.constrained = constrained ? 1 : 0;
  S.mono = b->d_mono.p;
  S.has_inter = has_inter ? 1 : 0;
  S.in_group = b->d_in_group.p;
  S.iset = b->d_iset.p;
  S.ext_gpair = ext ? 1 : 0;
  S.update_margin = ext ? 0 : 1;
  S.round = b->d_round.p;
  S.round_base = 0;
  S.k_base = 0;
  S.stats = b->d_stats.p;
  S.bounds = b->d_bounds.p;
  S.allowed = b->d_allowed.p;
  S.allowed_all = b->d_allowed_all.p;
  S.fmask = b->d_fmask.p;
  S.seg = b->d_seg.p;
  S.nsamp = b->d_nsamp.p;
  S.parent = b->d_parent.p;
  S.built = b->d_built.p;
  S.split = b->d_split.p;
  S.leafval = b->d_leafval.p;
  S.fill = b->d_fill.p;
  S.lvl_begin = b->d_lvl.p;
  S.lvl_count = b->d_lvl.p + K;
  S.prev_begin = b->d_lvl.p + 2 * K;
  S.num_nodes = b->d_lvl.p + 3 * K;
  S.cat_count = b->d_lvl.p + 4 * K;
  S.prev_count = b->d_lvl.p + 5 * K;
  S.rows0 = b->d_rows0.p;
  S.rows1 = b->d_rows1.p;
  S.kept = b->d_kept.p;
  S.unkept = b->d_kept.p + 1;
  S.margin = b->d_margin.p;
  S.delta = b->d_delta.p;
  S.apply_delta = 0;
  S.labels = b->d_labels.p;
  S.weights = b->d_weights.p;
  S.gpair = b->d_gpair.p;
  S.gpk = b->d_gpk.p;
  S.maxabs = b->d_maxabs.p;
  S.shifts = b->d_shifts.p;
  S.inv_scale = b->d_inv_scale.p;
  S.qerr = b->d_qerr.p;
  S.hist0 = b->d_hist0.p;
  S.hist1 = b->d_hist1.p;
  S.root_total = b->d_root_total.p;
  S.items = b->d_items.p;
  S.prefix = b->d_prefix.p;
  S.item_count = b->d_item_count.p;
  S.ptiles = b->d_ptiles.p;
  S.ptile_count = b->d_ptile_count.p;
  S.ptile_cap = ptile_cap;
  S.pool = b->d_pool.p;
  S.pool_len = b->d_pool_len.p;
  S.upool = b->d_upool.p;
  S.upool_len = b->d_upool_len.p;
  S.pool_mask = b->d_pool_mask.p;
  S.usable = b->d_usable.p;
  S.mbuf = b->d_mbuf.p;
  S.frec = b->d_frec.p;
  S.samp_scratch = b->d_samp.p;
  S.row_leaf = nullptr;
  SB_TRY(booster_alloc_trees(b, K * 16));
  return SB_OK;
}

size_t eval_smem(const sb_booster* b) {
  return b->S.cat_cap ? (EVAL_THREADS / 32) * cat_scratch_bytes(b->S.cat_bins) : 0;
}

// The launches of one boosting round on the context stream (also recorded into
// a CUDA graph by booster_round). Work sizes live in device memory, so the
// sequence depends only on the booster's shape.
// Blocks of a partition launch: its tiles (PART_TILE rows of one node; the
// nodes' rows are at most n per class tree) up to eight per SM.
static unsigned part_blocks(sb_ctx* ctx, size_t n, int K, size_t nodes) {
  const size_t tiles = (n * (size_t)K + PART_TILE - 1) / PART_TILE + nodes;
  return (unsigned)std::min<size_t>(tiles, (size_t)ctx->num_sms * 8);
}

// Blocks of a k_assign launch: one per class tree, and no more than 1024
// threads in all when per-node sampling gives every thread a scratch row.
static unsigned assign_blocks(const sb_booster* b, unsigned threads) {
  const unsigned k = (unsigned)b->K;
  return b->S.samp_scratch ? std::max(1u, std::min(k, 1024u / threads)) : k;
}

int booster_round_body(sb_booster* b, int apply_delta) {
  sb_ctx* ctx = b->ctx;
  BState& S = b->S;
  cudaEvent_t r0 = nullptr, r1 = nullptr;
  if (b->timing) {
    if (!b->d_hist_rows.p) {
      SB_TRY(b->d_hist_rows.alloc_zero(ctx, 1));
      SB_CUDA(cudaMemsetAsync(b->d_hist_rows.p, 0, 8, ctx->stream));
    }
    SB_CUDA(cudaEventCreate(&r0));
    SB_CUDA(cudaEventCreate(&r1));
    SB_CUDA(cudaEventRecord(r0, ctx->stream));
  }
  const unsigned gblocks = (unsigned)std::min<size_t>((b->n + 255) / 256, (size_t)ctx->num_sms * 16);
  S.apply_delta = apply_delta;
  SB_LAUNCH(ctx, k_gradient, gblocks, 256, 0, S);
  S.apply_delta = 0;
  SB_LAUNCH(ctx, k_round_prep, (unsigned)b->K, PREP_THREADS, 0, S);
  if (S.fixed) SB_LAUNCH(ctx, k_quantize, gblocks, 256, 0, S);
  HistLaunch L;
  L.g = b->g;
  L.gpair = S.fixed ? (const void*)S.gpk : (const void*)S.gpair;
  L.fixed = S.fixed;
  L.quant_bits = S.bits;
  L.items = S.items;
  L.prefix = S.prefix;
  L.count = S.item_count;
  L.tiles = b->d_tiles.p;
  L.ntiles = (int)b->g->tiles.size();
  L.rows_done = b->timing ? b->d_hist_rows.p : nullptr;
  L.pool_mask = S.pool_mask;
  L.rows_bound = b->n * (size_t)b->K;  // each class tree's rows at most once per level
  const size_t esm = eval_smem(b);
  auto hist = [&](int max_items) -> int {
    L.max_items = max_items;
    SB_TRY(launch_zero_items(ctx, b->g, S.items, S.item_count, max_items));
    if (b->timing) {
      cudaEvent_t e0, e1;
      SB_CUDA(cudaEventCreate(&e0));
      SB_CUDA(cudaEventCreate(&e1));
      SB_CUDA(cudaEventRecord(e0, ctx->stream));
      SB_TRY(launch_hist(ctx, L));
      SB_CUDA(cudaEventRecord(e1, ctx->stream));
      b->ev.push_back(e0);
      b->ev.push_back(e1);
      b->ev_kind.push_back(0);
    } else {
      SB_TRY(launch_hist(ctx, L));
    }
    return SB_OK;
  };
  SB_TRY(hist(b->K));
  if (b->lossguide) {
    const unsigned fy = (unsigned)((b->g->F + SCAN_WARPS - 1) / SCAN_WARPS);
    const size_t heap_smem = (size_t)b->maxn * sizeof(HeapEnt);
    auto eval = [&](int d, unsigned width) -> int {
      dim3 sg(width, fy, (unsigned)b->K);
      SB_LAUNCH(ctx, k_eval_scan, sg, EVAL_THREADS, esm, S, d);
      SB_LAUNCH(ctx, k_eval_records, sg, EVAL_THREADS, esm, S, d);
      dim3 pg(1, (unsigned)b->K);
      SB_LAUNCH(ctx, k_eval_pick, pg, EVAL_THREADS, esm, S, d);
      return SB_OK;
    };
    SB_TRY(eval(0, 1));  // the root
    SB_LAUNCH(ctx, k_lg_heap, (unsigned)b->K, 256, heap_smem, S, 1);
    // a step partitions one node per class tree: its tiles, at most
    const unsigned pblocks = part_blocks(ctx, b->n, b->K, b->K);
    for (int step = 0; step < b->steps; ++step) {
      const int d = step == 0 ? 0 : 1;  // only the first expansion reads the shared root list
      SB_LAUNCH(ctx, k_assign, assign_blocks(b, 256), 256, 0, S, d, 1);  // one frontier node per tree
      SB_LAUNCH(ctx, k_partition, pblocks, PART_THREADS, 0, S, d);
      SB_LAUNCH(ctx, k_lg_copy, pblocks, 256, 0, S);
      SB_LAUNCH(ctx, k_plan, 1, 1024, 0, S, d);
      SB_TRY(hist(b->K));
      SB_TRY(eval(1, 2));
      SB_LAUNCH(ctx, k_lg_heap, (unsigned)b->K, 256, heap_smem, S, 0);
    }
    SB_LAUNCH(ctx, k_lg_finalize, dim3((unsigned)b->maxn, (unsigned)b->K), 256, 0, S);
    if (!S.row_leaf && S.update_margin) SB_LAUNCH(ctx, k_lg_route, gblocks, 256, 0, S);
  }
  for (int d = 0; d < b->D && !b->lossguide; ++d) {
    const unsigned width = (unsigned)std::min(1 << d, b->maxw);
    dim3 sg(width, (unsigned)((b->g->F + SCAN_WARPS - 1) / SCAN_WARPS), (unsigned)b->K);
    SB_LAUNCH(ctx, k_eval_scan, sg, EVAL_THREADS, esm, S, d);
    SB_LAUNCH(ctx, k_eval_records, sg, EVAL_THREADS, esm, S, d);
    dim3 pg((width + SCAN_WARPS - 1) / SCAN_WARPS, (unsigned)b->K);
    SB_LAUNCH(ctx, k_eval_pick, pg, EVAL_THREADS, esm, S, d);
    // 1024 threads: the threads also write the level's partition tiles (about
    // n / PART_TILE at the root), one binary search each
    SB_LAUNCH(ctx, k_assign, assign_blocks(b, 1024), 1024, 0, S, d, 1);
    const unsigned pblocks = part_blocks(ctx, b->n, b->K, (size_t)b->K * width);
    SB_LAUNCH(ctx, k_partition, pblocks, PART_THREADS, 0, S, d);
    if (d + 1 < b->D) {
      SB_LAUNCH(ctx, k_plan, 1, 1024, 0, S, d);
      SB_TRY(hist(b->K * (1 << d)));
    }
  }
  // the rows outside the subset take their leaf values by routing (lossguide
  // rounds without row -> leaf output routed every row above)
  if (!b->lossguide || S.row_leaf) SB_LAUNCH(ctx, k_route_rest, gblocks, 256, 0, S);
  SB_LAUNCH(ctx, k_round_end, 1, 32, 0, S);
  if (b->timing) {
    SB_CUDA(cudaEventRecord(r1, ctx->stream));
    b->ev.push_back(r0);
    b->ev.push_back(r1);
    b->ev_kind.push_back(1);
  }
  return SB_OK;
}

// One boosting round. Once two consecutive rounds see the same device state
// (buffers, shapes, whether the previous tree's leaf values are pending), the
// round is recorded as a CUDA graph and replayed with one launch per round
// until that state changes (for instance when the tree buffers grow).
int booster_round(sb_booster* b) {
  sb_ctx* ctx = b->ctx;
  const int apply = b->delta_pending ? 1 : 0;
  BState key;
  std::memcpy(&key, &b->S, sizeof(BState));
  key.apply_delta = apply;
  const bool same = b->have_prev_key && std::memcmp(&key, &b->prev_key, sizeof(BState)) == 0;
  std::memcpy(&b->prev_key, &key, sizeof(BState));
  b->have_prev_key = true;
  if (!b->use_graphs || b->timing || !same) {
    if (b->graph_exec && !same) {
      cudaGraphExecDestroy(b->graph_exec);
      b->graph_exec = nullptr;
    }
    SB_TRY(booster_round_body(b, apply));
  } else {
    if (!b->graph_exec) {
      const uint64_t l0 = ctx->launches;
      SB_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = booster_round_body(b, apply);
      cudaGraph_t graph = nullptr;
      const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
      b->graph_nodes = ctx->launches - l0;
      ctx->launches = l0;  // recorded, not launched
      if (rc != SB_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      SB_CUDA(e);
      const cudaError_t ei = cudaGraphInstantiate(&b->graph_exec, graph, 0);
      cudaGraphDestroy(graph);
      SB_CUDA(ei);
    }
    SB_CUDA(cudaGraphLaunch(b->graph_exec, ctx->stream));
    ctx->launches += b->graph_nodes;
  }
  b->delta_pending = b->S.update_margin != 0;
  return SB_OK;
}

int booster_collect_timing(sb_booster* b) {
  if (b->ev.empty()) return SB_OK;
  SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
  for (size_t i = 0; i + 1 < b->ev.size(); i += 2) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, b->ev[i], b->ev[i + 1]);
    if (b->ev_kind[i / 2] == 0) {
      b->stats.hist_ms += ms;
      b->stats.hist_launches++;
    } else {
      b->stats.round_ms += ms;
    }
  }
  for (auto e : b->ev) cudaEventDestroy(e);
  b->ev.clear();
  b->ev_kind.clear();
  if (b->d_hist_rows.p) {  // algorithmic bytes: row id + gradient pair + F u16 bins per sampled row
    unsigned long long rows = 0;
    SB_CUDA(cudaMemcpy(&rows, b->d_hist_rows.p, 8, cudaMemcpyDeviceToHost));
    SB_CUDA(cudaMemsetAsync(b->d_hist_rows.p, 0, 8, b->ctx->stream));
    SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
    b->stats.hist_bytes += (double)rows * (4.0 + 8.0 + 2.0 * (double)b->g->F);
  }
  return SB_OK;
}

}  // namespace

int booster_set_eval_smem(sb_booster* b) {
  int esm = (int)eval_smem(b);
  SB_TRY(raise_smem_limit((const void*)k_eval_scan, (size_t)esm));
  SB_TRY(raise_smem_limit((const void*)k_eval_pick, (size_t)esm));
  SB_TRY(raise_smem_limit((const void*)k_eval_records, (size_t)esm));
  if (b->lossguide) {
    const size_t heap_smem = (size_t)b->maxn * sizeof(HeapEnt);
    SB_REQUIRE(heap_smem <= b->ctx->smem_optin, SB_ERR_UNSUPPORTED, "lossguide queue of %d nodes exceeds shared memory",
               b->maxn);
    SB_TRY(raise_smem_limit((const void*)k_lg_heap, (size_t)heap_smem));
  }
  return SB_OK;
}

// Appends to `m` the booster's trees it does not hold yet: m holds the
// booster's first m->trees.size() trees (none, or what an earlier export or
// append left), and only the trees after them cross to the host. New trees
// get weight 1.
int booster_export_append(const sb_booster* b, sb_model* m) {
  sb_ctx* ctx = b->ctx;
  const int ntrees = b->rounds_done * b->K;
  const int t0 = (int)m->trees.size();
  SB_REQUIRE(t0 <= ntrees, SB_ERR_INVALID_ARG, "internal: the model holds %d trees, the booster %d", t0, ntrees);
  const int cnt = ntrees - t0;
  const size_t cc = b->S.cat_cap;
  std::vector<int> nn(cnt), nc(cnt);
  std::vector<sb_node> nodes((size_t)cnt * b->maxn);
  std::vector<uint32_t> cats(cc ? (size_t)cnt * cc : 0);
  if (cnt) {
    SB_CUDA(cudaMemcpyAsync(nn.data(), b->d_out_nnodes.p + t0, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(cudaMemcpyAsync(nc.data(), b->d_out_ncats.p + t0, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(cudaMemcpyAsync(nodes.data(), b->d_out_nodes.p + (size_t)t0 * b->maxn, nodes.size() * sizeof(sb_node),
                            cudaMemcpyDeviceToHost, ctx->stream));
    if (!cats.empty())
      SB_CUDA(cudaMemcpyAsync(cats.data(), b->d_out_cats.p + (size_t)t0 * cc, cats.size() * 4,
                              cudaMemcpyDeviceToHost, ctx->stream));
  }
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  m->trees.resize(ntrees);
  m->weights.resize(ntrees, 1.0f);
  for (int i = 0; i < cnt; ++i) {
    const int t = t0 + i;
    m->trees[t].nodes.assign(nodes.begin() + (size_t)i * b->maxn, nodes.begin() + (size_t)i * b->maxn + nn[i]);
    if (!cats.empty())
      m->trees[t].cats.assign(cats.begin() + (size_t)i * cc, cats.begin() + (size_t)i * cc + nc[i]);
  }
  m->base_score = b->base_score;
  m->num_class = b->p.num_class;
  m->n_features = (int)b->g->F;
  m->objective = b->p.objective;
  m->dev_valid = false;
  return SB_OK;
}

int booster_export(const sb_booster* b, sb_model* m) {
  m->trees.clear();
  m->weights.clear();
  return booster_export_append(b, m);
}

int booster_trees(const sb_booster* b, BoosterTrees* v) {
  v->ctx = b->ctx;
  v->nodes = b->d_out_nodes.p;
  v->cats = b->S.cat_cap ? b->d_out_cats.p : nullptr;
  v->maxn = b->maxn;
  v->cat_cap = b->S.cat_cap;
  v->K = b->K;
  v->rounds_done = b->rounds_done;
  v->base_score = b->base_score;
  v->objective = b->p.objective;
  v->num_class = b->p.num_class;
  v->n_features = b->g->F;
  return SB_OK;
}

std::vector<std::unique_ptr<EvalSet>>& booster_evals(sb_booster* b) { return b->evals; }

// Folds a pending tree's leaf values into the margins before the host reads them.
int booster_flush_delta(const sb_booster* b) {
  if (!b->delta_pending) return SB_OK;
  sb_ctx* ctx = b->ctx;
  const size_t nk = b->n * (size_t)b->K;
  const unsigned blocks = (unsigned)std::min<size_t>((nk + 255) / 256, (size_t)ctx->num_sms * 16);
  SB_LAUNCH(ctx, k_apply_delta, blocks, 256, 0, b->d_margin.p, b->d_delta.p, nk);
  b->delta_pending = false;
  return SB_OK;
}

int booster_run(sb_booster* b, int n_rounds) {
  SB_TRY(booster_alloc_trees(b, (b->rounds_done + n_rounds) * b->K));
  SB_TRY(booster_set_eval_smem(b));
  for (int r = 0; r < n_rounds; ++r) {
    SB_TRY(booster_round(b));
    b->rounds_done++;
  }
  return SB_OK;
}

// ------------------------------------------------------------ batched jobs
// Depthwise boosters of one device trained together (sb_train_many): every
// round is one launch per kernel step over all jobs, whose grids are laid end
// to end (JobGrid), recorded once as a CUDA graph and replayed. A job runs
// the same kernel bodies on its own state as when it trains alone, so its
// model is the same; a job deeper than others simply gets no blocks in the
// launches of the levels it does not have.
bool booster_batchable(const sb_booster* b) {
  return b && !b->lossguide && !b->ext && !b->timing && b->evals.empty() && b->S.row_leaf == nullptr &&
         b->g->layout == HIST_LAYOUT_TILED;
}

// Before batched rounds: each job's own stream drained and its tree buffers
// sized for `rounds` more rounds. Done before any batch records a graph: a
// job's stream may be the stream another batch records on.
int boosters_batch_prepare(sb_booster* b, int rounds) {
  SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
  SB_TRY(booster_alloc_trees(b, (b->rounds_done + rounds) * b->K));
  SB_TRY(booster_set_eval_smem(b));
  SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
  return SB_OK;
}

int boosters_train_batched(sb_ctx* ctx, sb_booster* const* bs, int nb, int rounds) {
  if (nb <= 0 || rounds <= 0) return SB_OK;
  const int fixed = bs[0]->S.fixed;
  int maxD = 0, maxK = 1;
  size_t esm = 0;
  for (int j = 0; j < nb; ++j) {
    sb_booster* b = bs[j];
    SB_REQUIRE(booster_batchable(b) && b->S.fixed == fixed, SB_ERR_INVALID_ARG, "internal: job %d not batchable", j);
    SB_REQUIRE(b->tree_cap >= (b->rounds_done + rounds) * b->K, SB_ERR_INVALID_ARG,
               "internal: job %d: tree buffers not prepared", j);
    maxD = std::max(maxD, b->D);
    maxK = std::max(maxK, b->K);
    esm = std::max(esm, eval_smem(b));
  }
  SB_TRY(raise_smem_limit((const void*)k_eval_scan_jobs, esm));
  SB_TRY(raise_smem_limit((const void*)k_eval_records_jobs, esm));
  SB_TRY(raise_smem_limit((const void*)k_eval_pick_jobs, esm));
  // the histogram launches' per-job descriptions
  std::vector<HistLaunch> Ls(nb);
  for (int j = 0; j < nb; ++j) {
    const sb_booster* b = bs[j];
    const BState& S = b->S;
    HistLaunch& L = Ls[j];
    L.g = b->g;
    L.gpair = S.fixed ? (const void*)S.gpk : (const void*)S.gpair;
    L.fixed = S.fixed;
    L.quant_bits = S.bits;
    L.items = S.items;
    L.prefix = S.prefix;
    L.count = S.item_count;
    L.max_items = 0;
    L.tiles = b->d_tiles.p;
    L.ntiles = (int)b->g->tiles.size();
    L.rows_done = nullptr;
    L.pool_mask = S.pool_mask;
    L.rows_bound = b->n * (size_t)b->K;
    L.min_units = 2048;  // the batches' launches overlap: fewer, fuller CTAs for small nodes
  }
  HistJobsPlan hp;
  SB_TRY(hist_jobs_prepare(ctx, Ls, &hp));
  // block offsets of every launch step, in one device table
  struct Step {
    size_t off = 0;
    unsigned blocks = 0;
  };
  std::vector<unsigned> tab;
  auto step = [&](auto blocks_of) {
    Step st;
    st.off = tab.size();
    tab.push_back(0);
    for (int j = 0; j < nb; ++j) {
      st.blocks += (unsigned)blocks_of(j);
      tab.push_back(st.blocks);
    }
    return st;
  };
  auto gblocks = [&](int j) { return std::min<size_t>((bs[j]->n + 255) / 256, (size_t)ctx->num_sms * 16); };
  const Step s_grad = step(gblocks);
  const Step s_prep = step([&](int j) { return bs[j]->K; });
  const Step s_quant = step([&](int j) { return fixed ? gblocks(j) : 0; });
  const Step s_hist0 = step([&](int j) { return hp.hist_grid[j]; });
  const Step s_zero0 = step([&](int j) { return hp.zero_grid[j]; });
  std::vector<Step> s_scan(maxD), s_pick(maxD), s_assign(maxD), s_part(maxD), s_plan(maxD), s_hist(maxD),
      s_zero(maxD);
  std::vector<unsigned> fy(maxD, 1);
  std::vector<int> items(maxD, 0);
  for (int d = 0; d < maxD; ++d) {
    auto width = [&](int j) { return (unsigned)std::min(1 << d, bs[j]->maxw); };
    auto act = [&](int j) { return d < bs[j]->D; };
    auto build = [&](int j) { return d + 1 < bs[j]->D; };
    s_scan[d] = step([&](int j) { return act(j) ? width(j) : 0u; });
    s_pick[d] = step([&](int j) { return act(j) ? (width(j) + SCAN_WARPS - 1) / SCAN_WARPS : 0u; });
    s_assign[d] = step([&](int j) { return act(j) ? assign_blocks(bs[j], 1024) : 0u; });
    s_part[d] = step([&](int j) {
      return act(j) ? part_blocks(ctx, bs[j]->n, bs[j]->K, (size_t)bs[j]->K * width(j)) : 0u;
    });
    s_plan[d] = step([&](int j) { return build(j) ? 1u : 0u; });
    s_hist[d] = step([&](int j) { return build(j) ? hp.hist_grid[j] : 0u; });
    s_zero[d] = step([&](int j) { return build(j) ? hp.zero_grid[j] : 0u; });
    for (int j = 0; j < nb; ++j) {
      if (act(j)) fy[d] = std::max(fy[d], (unsigned)((bs[j]->g->F + SCAN_WARPS - 1) / SCAN_WARPS));
      if (build(j)) items[d] = std::max(items[d], bs[j]->K * (1 << d));
    }
  }
  const Step s_route = step(gblocks);
  const Step s_end = step([&](int) { return 1; });
  DBuf<unsigned> d_tab;
  DBuf<BState> d_states, d_states_g;
  SB_TRY(d_tab.alloc(ctx, tab.size()));
  SB_TRY(d_states.alloc(ctx, nb));
  SB_TRY(d_states_g.alloc(ctx, nb));
  SB_CUDA(cudaMemcpyAsync(d_tab.p, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
  auto J = [&](const BState* states, const Step& st) { return JobGrid{states, d_tab.p + st.off, nb}; };
  auto body = [&]() -> int {
    SB_LAUNCH(ctx, k_gradient_jobs, s_grad.blocks, 256, 0, J(d_states_g.p, s_grad));
    SB_LAUNCH(ctx, k_round_prep_jobs, s_prep.blocks, PREP_THREADS, 0, J(d_states.p, s_prep));
    if (fixed) SB_LAUNCH(ctx, k_quantize_jobs, s_quant.blocks, 256, 0, J(d_states.p, s_quant));
    SB_TRY(launch_hist_jobs(ctx, hp, d_tab.p + s_hist0.off, s_hist0.blocks, d_tab.p + s_zero0.off, s_zero0.blocks,
                            maxK));
    for (int d = 0; d < maxD; ++d) {
      if (s_scan[d].blocks == 0) break;
      const dim3 sg(s_scan[d].blocks, fy[d], (unsigned)maxK);
      SB_LAUNCH(ctx, k_eval_scan_jobs, sg, EVAL_THREADS, esm, J(d_states.p, s_scan[d]), d);
      SB_LAUNCH(ctx, k_eval_records_jobs, sg, EVAL_THREADS, esm, J(d_states.p, s_scan[d]), d);
      SB_LAUNCH(ctx, k_eval_pick_jobs, dim3(s_pick[d].blocks, (unsigned)maxK), EVAL_THREADS, esm,
                J(d_states.p, s_pick[d]), d);
      SB_LAUNCH(ctx, k_assign_jobs, s_assign[d].blocks, 1024, 0, J(d_states.p, s_assign[d]), d, 1);
      SB_LAUNCH(ctx, k_partition_jobs, s_part[d].blocks, PART_THREADS, 0, J(d_states.p, s_part[d]), d);
      if (s_plan[d].blocks) {
        SB_LAUNCH(ctx, k_plan_jobs, s_plan[d].blocks, 1024, 0, J(d_states.p, s_plan[d]), d);
        SB_TRY(launch_hist_jobs(ctx, hp, d_tab.p + s_hist[d].off, s_hist[d].blocks, d_tab.p + s_zero[d].off,
                                s_zero[d].blocks, items[d]));
      }
    }
    SB_LAUNCH(ctx, k_route_rest_jobs, s_route.blocks, 256, 0, J(d_states.p, s_route));
    SB_LAUNCH(ctx, k_round_end_jobs, s_end.blocks, 32, 0, J(d_states.p, s_end));
    return SB_OK;
  };
  // the jobs' states: the gradient pass folds in the last tree's leaf values
  // from the second round of a fresh booster on
  std::vector<BState> hs(nb), hg(nb), ug(nb);
  for (int j = 0; j < nb; ++j) {
    std::memcpy(&hs[j], &bs[j]->S, sizeof(BState));
    hs[j].apply_delta = 0;
  }
  SB_CUDA(cudaMemcpyAsync(d_states.p, hs.data(), nb * sizeof(BState), cudaMemcpyHostToDevice, ctx->stream));
  cudaGraphExec_t exec = nullptr;
  uint64_t graph_nodes = 0;
  int rc = SB_OK;
  bool uploaded = false;
  for (int r = 0; r < rounds && rc == SB_OK; ++r) {
    for (int j = 0; j < nb; ++j) {
      std::memcpy(&hg[j], &hs[j], sizeof(BState));
      hg[j].apply_delta = bs[j]->delta_pending ? 1 : 0;
    }
    if (!uploaded || std::memcmp(hg.data(), ug.data(), nb * sizeof(BState)) != 0) {
      const cudaError_t e = cudaMemcpyAsync(d_states_g.p, hg.data(), nb * sizeof(BState), cudaMemcpyHostToDevice,
                                            ctx->stream);
      if (e != cudaSuccess) {
        rc = cuda_status(e, "cudaMemcpyAsync", __FILE__, __LINE__);
        break;
      }
      std::memcpy(ug.data(), hg.data(), nb * sizeof(BState));
      uploaded = true;
    }
    if (!exec) {  // record the round once; it reads the jobs' states from device memory
      const uint64_t l0 = ctx->launches;
      cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) {
        rc = cuda_status(e, "cudaStreamBeginCapture", __FILE__, __LINE__);
        break;
      }
      rc = body();
      cudaGraph_t graph = nullptr;
      e = cudaStreamEndCapture(ctx->stream, &graph);
      graph_nodes = ctx->launches - l0;
      ctx->launches = l0;  // recorded, not launched
      if (rc == SB_OK && e != cudaSuccess) rc = cuda_status(e, "cudaStreamEndCapture", __FILE__, __LINE__);
      if (rc == SB_OK) {
        e = cudaGraphInstantiate(&exec, graph, 0);
        if (e != cudaSuccess) rc = cuda_status(e, "cudaGraphInstantiate", __FILE__, __LINE__);
      }
      if (graph) cudaGraphDestroy(graph);
      if (rc != SB_OK) break;
    }
    const cudaError_t e = cudaGraphLaunch(exec, ctx->stream);
    if (e != cudaSuccess) {
      rc = cuda_status(e, "cudaGraphLaunch", __FILE__, __LINE__);
      break;
    }
    ctx->launches += graph_nodes;
    for (int j = 0; j < nb; ++j) {
      bs[j]->rounds_done++;
      bs[j]->delta_pending = bs[j]->S.update_margin != 0;
    }
  }
  const cudaError_t se = cudaStreamSynchronize(ctx->stream);
  if (exec) cudaGraphExecDestroy(exec);
  if (rc == SB_OK && se != cudaSuccess) rc = cuda_status(se, "cudaStreamSynchronize", __FILE__, __LINE__);
  for (int j = 0; j < nb; ++j) bs[j]->stats.rounds = bs[j]->rounds_done;
  return rc;
}

int boosters_train_many(sb_ctx* const* ctxs, int nctx, sb_booster* const* bs, const int* rounds, int nb,
                        int* status) {
  // batchable boosters train in groups that share one histogram kernel: the
  // same precision, rows per warp instruction and code width
  // (SB_JOBS_BATCH=0: none, every job goes through the stream pool)
  const char* eb = std::getenv("SB_JOBS_BATCH");
  const bool batching = !(eb && std::strcmp(eb, "0") == 0);
  std::map<std::tuple<int, int, int>, std::vector<int>> groups;
  std::vector<int> rest;
  for (int j = 0; j < nb; ++j) {
    if (status[j] != SB_OK || !bs[j] || rounds[j] <= 0) continue;
    if (batching && booster_batchable(bs[j])) groups[{bs[j]->S.fixed, bs[j]->g->tiled_rl, bs[j]->g->code_bytes}].push_back(j);
    else rest.push_back(j);
  }
  // a group becomes up to nctx batches of jobs of similar size (each batched
  // launch waits for its largest job's part), one per stream, run by host
  // threads at once so that the batches' launches overlap
  std::vector<std::vector<int>> batches;
  for (auto& kv : groups) {
    std::vector<int>& v = kv.second;
    if (v.size() < 2) {
      rest.insert(rest.end(), v.begin(), v.end());
      continue;
    }
    std::stable_sort(v.begin(), v.end(), [&](int a, int b) { return bs[a]->n > bs[b]->n; });
    const int parts = std::max(1, std::min(nctx, (int)v.size() / 2));
    for (int q = 0; q < parts; ++q)
      batches.emplace_back(v.begin() + (size_t)v.size() * q / parts, v.begin() + (size_t)v.size() * (q + 1) / parts);
  }
  for (const std::vector<int>& batch : batches)
    for (int j : batch)
      if (status[j] == SB_OK) status[j] = boosters_batch_prepare(bs[j], rounds[j]);
  // the others: round r of each before round r + 1 of any, on their own streams
  int max_rest = 0;
  for (int j : rest) max_rest = std::max(max_rest, rounds[j]);
  for (int r = 0; r < max_rest; ++r)
    for (int j : rest)
      if (status[j] == SB_OK && r < rounds[j]) {
        status[j] = booster_run(bs[j], 1);
        bs[j]->stats.rounds = bs[j]->rounds_done;
      }
  // each batch in segments of rounds that all its remaining jobs still have
  auto run_batch = [&](std::vector<int> batch, sb_ctx* ctx) {
    cudaSetDevice(ctx->device);
    batch.erase(std::remove_if(batch.begin(), batch.end(), [&](int j) { return status[j] != SB_OK; }), batch.end());
    int done = 0;
    while (!batch.empty()) {
      int seg = INT32_MAX;
      for (int j : batch) seg = std::min(seg, rounds[j] - done);
      std::vector<sb_booster*> part;
      for (int j : batch) part.push_back(bs[j]);
      const int rc = boosters_train_batched(ctx, part.data(), (int)part.size(), seg);
      if (rc != SB_OK) {
        for (int j : batch) status[j] = rc;
        return;
      }
      done += seg;
      std::vector<int> next;
      for (int j : batch)
        if (rounds[j] > done) next.push_back(j);
      batch.swap(next);
    }
  };
  for (size_t b0 = 0; b0 < batches.size(); b0 += (size_t)nctx) {
    std::vector<std::thread> pool;
    const size_t b1 = std::min(batches.size(), b0 + (size_t)nctx);
    for (size_t b = b0 + 1; b < b1; ++b) pool.emplace_back(run_batch, batches[b], ctxs[b - b0]);
    run_batch(batches[b0], ctxs[0]);
    for (std::thread& th : pool) th.join();
  }
  for (int j = 0; j < nb; ++j)
    if (status[j] != SB_OK) return status[j];
  return SB_OK;
}

}  // namespace sb

namespace sb {

// train_impl for tree_method=approx (learner/train.rs:46-53, 276-338): each
// round, per class, hessian-weighted cuts of that class's hessians, the
// matrix re-binned with them, one tree grown by the hist builder on it, and
// the margins updated on the raw values.
int approx_train(sb_ctx* ctx, const float* d_X, size_t n, size_t F, const uint8_t* ftypes, float missing,
                 const float* labels, const float* weights, const float* base_margin, const sb_train_params* p,
                 int rounds, sb_model** out) {
  cudaStream_t st = ctx->stream;
  const int K = n_outputs(p->objective, p->num_class);
  if (weights)
    for (size_t i = 0; i < n; ++i)
      SB_REQUIRE(weights[i] >= 0.0f, SB_ERR_UNSUPPORTED, "tree_method=approx needs non-negative weights");
  ApproxState* A = approx_state_new();
  std::unique_ptr<ApproxState, void (*)(ApproxState*)> own(A, approx_state_free);
  SB_TRY(approx_prepare(ctx, d_X, n, F, ftypes, missing, p->max_bin, A));
  const float base = base_margin_of(p, labels, weights, n, K);
  std::vector<float> m0(n * K, base);
  if (base_margin) std::memcpy(m0.data(), base_margin, n * K * sizeof(float));
  DBuf<float> d_y, d_w, d_margin, d_hess;
  DBuf<float2> d_gp, d_gk;
  DBuf<unsigned int> d_kept;
  SB_TRY(d_y.alloc(ctx, n));
  if (weights) SB_TRY(d_w.alloc(ctx, n));
  SB_TRY(d_margin.alloc(ctx, n * K));
  SB_TRY(d_hess.alloc(ctx, n));
  SB_TRY(d_gp.alloc(ctx, n * K));
  SB_TRY(d_gk.alloc(ctx, n));
  SB_TRY(d_kept.alloc(ctx, 1));
  SB_CUDA(cudaMemcpyAsync(d_y.p, labels, n * 4, cudaMemcpyHostToDevice, st));
  if (weights) SB_CUDA(cudaMemcpyAsync(d_w.p, weights, n * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_margin.p, m0.data(), n * K * 4, cudaMemcpyHostToDevice, st));
  std::unique_ptr<sb_model> mdl(new sb_model);
  mdl->ctx = ctx;
  mdl->base_score = base;
  mdl->num_class = p->num_class;
  mdl->n_features = (int)F;
  mdl->objective = p->objective;
  sb_train_params q = *p;  // the trees' builder params (its gradients come from here)
  q.objective = SB_OBJ_SQUARED_ERROR;
  q.num_class = 0;
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 16);
  const float eta = (float)p->eta;
  for (int r = 0; r < rounds; ++r) {
    SB_LAUNCH(ctx, k_objective_gradient, blocks, 256, 0, p->objective, K, (float)p->scale_pos_weight, d_margin.p,
              d_y.p, d_w.p, n, d_gp.p);
    for (int k = 0; k < K; ++k) {
      SB_LAUNCH(ctx, k_class_column, blocks, 256, 0, d_gp.p, n, K, k, d_gk.p, d_hess.p);
      sb_ghist g;
      g.ctx = ctx;
      g.n = n;
      g.F = F;
      g.max_bin = p->max_bin;
      g.missing = missing;
      SB_TRY(approx_cuts(A, d_hess.p, &g));  // HistCuts::from_dmatrix_weighted
      SB_TRY(ghist_bin(ctx, d_X, &g));       // GHistIndex::from_dmatrix
      sb_booster b;
      SB_TRY(booster_init(&b, ctx, &g, &q, 1, true));
      SB_CUDA(cudaMemsetAsync(d_kept.p, 0, 4, st));
      SB_LAUNCH(ctx, k_approx_rows, blocks, 256, 0, p->seed, (unsigned long long)r, p->subsample, n, b.d_rows1.p,
                d_kept.p);  // the subset's flags, which the round's gradient pass compacts
      SB_LAUNCH(ctx, k_approx_fallback, 1, 1, 0, p->seed, (unsigned long long)r, n, b.d_rows1.p, d_kept.p);
      SB_CUDA(cudaMemcpyAsync(b.d_gpair.p, d_gk.p, n * 8, cudaMemcpyDeviceToDevice, st));
      b.S.round_base = (unsigned long long)r;  // column sampling of class k in round r
      b.S.k_base = k;
      SB_TRY(booster_set_eval_smem(&b));
      SB_TRY(booster_round(&b));
      SB_LAUNCH(ctx, k_add_tree, blocks, 256, 0, b.d_out_nodes.p, b.d_out_cats.p, d_X, n, (int)F, missing, K, k,
                eta, d_margin.p);
      int nn = 0, nc = 0;
      std::vector<sb_node> nodes(b.maxn);
      SB_CUDA(cudaMemcpyAsync(&nn, b.d_out_nnodes.p, 4, cudaMemcpyDeviceToHost, st));
      SB_CUDA(cudaMemcpyAsync(&nc, b.d_out_ncats.p, 4, cudaMemcpyDeviceToHost, st));
      SB_CUDA(cudaMemcpyAsync(nodes.data(), b.d_out_nodes.p, b.maxn * sizeof(sb_node), cudaMemcpyDeviceToHost, st));
      std::vector<uint32_t> cats(b.S.cat_cap);
      if (b.S.cat_cap)
        SB_CUDA(cudaMemcpyAsync(cats.data(), b.d_out_cats.p, b.S.cat_cap * 4, cudaMemcpyDeviceToHost, st));
      SB_CUDA(cudaStreamSynchronize(st));
      HostTree t;
      t.nodes.assign(nodes.begin(), nodes.begin() + nn);
      t.cats.assign(cats.begin(), cats.begin() + nc);
      for (sb_node& nd : t.nodes)  // scale_leaves(eta), regtree.rs:201-207
        if (nd.left < 0) nd.leaf_value = nd.leaf_value * eta;
      mdl->trees.push_back(std::move(t));
      mdl->weights.push_back(1.0f);
    }
  }
  SB_CUDA(cudaStreamSynchronize(st));
  *out = mdl.release();
  return SB_OK;
}

}  // namespace sb

namespace sb {

// DART's dropout set of round `rnd` over the `existing` trees (train.rs:
// 397-425): none with probability skip_drop, else each tree with probability
// rate_drop, and at least one. Draws: a sequential stream from sb_dart_key,
// each draw the SplitMix64 mix of the state before the state advances.
std::vector<int> dart_dropout(uint64_t seed, uint64_t rnd, int existing, double rate_drop,
                                     double skip_drop) {
  uint64_t st = sb_dart_key(seed, rnd);
  auto next = [&]() {
    const uint64_t x = sb_mix64(st);
    st += 0x9E3779B97F4A7C15ULL;
    return x;
  };
  std::vector<int> dropped;
  if (sb_u01(next()) < skip_drop || existing == 0) return dropped;
  for (int i = 0; i < existing; ++i)
    if (sb_u01(next()) < rate_drop) dropped.push_back(i);
  if (dropped.empty())
    dropped.push_back((int)(((unsigned __int128)next() * (unsigned __int128)existing) >> 64));
  return dropped;
}

}  // namespace sb

extern "C" {

int sb_booster_create(sb_ctx* ctx, const sb_ghist* g, const sb_train_params* p, const float* labels,
                      const float* weights, const float* base_margin, sb_booster** out) {
  using namespace sb;
  SB_REQUIRE(ctx && g && p && labels && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_SAME_DEVICE(ctx, g);
  *out = nullptr;
  SB_TRY(sb_train_params_validate(p));
  SB_REQUIRE(p->tree_method == SB_TREE_HIST, SB_ERR_UNSUPPORTED,
             "a booster trains tree_method=hist; tree_method=approx trains through sb_train");
  SB_CUDA(cudaSetDevice(ctx->device));
  const int K = n_outputs(p->objective, p->num_class);
  const size_t n = g->n;
  if (p->hist_precision == SB_HIST_FIXED && weights)
    for (size_t i = 0; i < n; ++i)
      SB_REQUIRE(weights[i] >= 0.0f, SB_ERR_UNSUPPORTED,
                 "the fixed-point form needs non-negative weights (hessians)");
  sb_booster* b = new sb_booster;
  int s = booster_init(b, ctx, g, p, K, false);
  if (s != SB_OK) {
    delete b;
    return s;
  }
  const float base = base_margin_of(p, labels, weights, n, K);
  b->base_score = base;
  std::vector<float> m(n * K, base);  // init_margin, train.rs:496-511
  if (base_margin) std::memcpy(m.data(), base_margin, n * K * sizeof(float));
  cudaStream_t st = ctx->stream;
  if ((s = b->d_labels.alloc(ctx, n)) != SB_OK) { delete b; return s; }
  cudaMemcpyAsync(b->d_labels.p, labels, n * 4, cudaMemcpyHostToDevice, st);
  if (weights) {
    if ((s = b->d_weights.alloc(ctx, n)) != SB_OK) { delete b; return s; }
    cudaMemcpyAsync(b->d_weights.p, weights, n * 4, cudaMemcpyHostToDevice, st);
  }
  cudaMemcpyAsync(b->d_margin.p, m.data(), n * K * 4, cudaMemcpyHostToDevice, st);
  b->S.labels = b->d_labels.p;
  b->S.weights = b->d_weights.p;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    delete b;
    return sb::cuda_status(e, "booster upload", __FILE__, __LINE__);
  }
  *out = b;
  return SB_OK;
}

int sb_booster_update(sb_booster* b, int n_rounds) {
  SB_REQUIRE(b != nullptr && n_rounds >= 0, SB_ERR_INVALID_ARG, "invalid argument");
  SB_CUDA(cudaSetDevice(b->ctx->device));
  SB_TRY(sb::booster_run(b, n_rounds));
  b->stats.rounds = b->rounds_done;
  return SB_OK;
}

int sb_booster_margins(const sb_booster* b, float* out) {
  SB_REQUIRE(b && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_TRY(sb::booster_flush_delta(b));
  SB_CUDA(cudaMemcpyAsync(out, b->d_margin.p, b->d_margin.bytes(), cudaMemcpyDeviceToHost, b->ctx->stream));
  SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
  return SB_OK;
}

int sb_booster_set_margins(sb_booster* b, const float* margins) {
  SB_REQUIRE(b && margins, SB_ERR_INVALID_ARG, "NULL argument");
  SB_CUDA(cudaSetDevice(b->ctx->device));
  SB_CUDA(cudaMemcpyAsync(b->d_margin.p, margins, b->d_margin.bytes(), cudaMemcpyHostToDevice, b->ctx->stream));
  SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
  b->delta_pending = false;  // the last tree's leaf values are not added on top
  return SB_OK;
}

int sb_booster_gradients(const sb_booster* b, sb_gradpair* out) {
  SB_REQUIRE(b && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_CUDA(cudaMemcpyAsync(out, b->d_gpair.p, b->d_gpair.bytes(), cudaMemcpyDeviceToHost, b->ctx->stream));
  SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
  return SB_OK;
}

int sb_booster_row_mask(const sb_booster* b, uint64_t round, uint8_t* out) {
  SB_REQUIRE(b && out, SB_ERR_INVALID_ARG, "NULL argument");
  const size_t n = b->n;
  if (b->p.subsample >= 1.0) {
    std::memset(out, 1, n);
    return SB_OK;
  }
  uint64_t rk = sb_round_key(b->p.seed, round);
  size_t kept = 0;
  for (size_t r = 0; r < n; ++r) {
    out[r] = sb_u01(sb_row_draw(rk, r)) < b->p.subsample ? 1 : 0;
    kept += out[r];
  }
  if (!kept) out[sb_row_fallback(rk, n)] = 1;
  return SB_OK;
}

int sb_booster_model(const sb_booster* b, sb_model** out) {
  SB_REQUIRE(b && out, SB_ERR_INVALID_ARG, "NULL argument");
  sb_model* m = new sb_model;
  m->ctx = b->ctx;
  int s = sb::booster_export(b, m);
  if (s != SB_OK) {
    delete m;
    return s;
  }
  *out = m;
  return SB_OK;
}

int sb_booster_destroy(sb_booster* b) {
  if (b) {
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    for (auto e : b->ev) cudaEventDestroy(e);
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    delete b;
  }
  return SB_OK;
}

int sb_booster_set_graphs(sb_booster* b, int enable) {
  SB_REQUIRE(b != nullptr, SB_ERR_INVALID_ARG, "booster is NULL");
  b->use_graphs = enable != 0;
  if (!b->use_graphs && b->graph_exec) {
    cudaGraphExecDestroy(b->graph_exec);
    b->graph_exec = nullptr;
  }
  return SB_OK;
}

int sb_booster_set_timing(sb_booster* b, int timing) {
  SB_REQUIRE(b != nullptr, SB_ERR_INVALID_ARG, "booster is NULL");
  b->timing = timing;
  return SB_OK;
}

int sb_booster_stats_get(const sb_booster* b, sb_booster_stats* out) {
  SB_REQUIRE(b && out, SB_ERR_INVALID_ARG, "NULL argument");
  sb_booster* mb = const_cast<sb_booster*>(b);
  SB_TRY(sb::booster_collect_timing(mb));
  *out = b->stats;
  if (b->S.fixed) {
    unsigned int q[2];
    int sh[2];
    SB_CUDA(cudaMemcpyAsync(q, b->d_qerr.p, 8, cudaMemcpyDeviceToHost, b->ctx->stream));
    SB_CUDA(cudaMemcpyAsync(sh, b->d_shifts.p, 8, cudaMemcpyDeviceToHost, b->ctx->stream));
    SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
    float fq[2];
    std::memcpy(fq, q, 8);
    out->quant_err_grad = fq[0];
    out->quant_err_hess = fq[1];
    out->quant_shift_grad = sh[0];
    out->quant_shift_hess = sh[1];
  }
  return SB_OK;
}

int sb_booster_stats_reset(sb_booster* b) {
  SB_REQUIRE(b != nullptr, SB_ERR_INVALID_ARG, "booster is NULL");
  SB_TRY(sb::booster_collect_timing(b));
  b->stats = sb_booster_stats{};
  b->stats.rounds = b->rounds_done;
  return SB_OK;
}

int sb_objective_gradient(sb_ctx* ctx, int objective, int num_class, double scale_pos_weight,
                          const float* preds, const float* labels, const float* weights, size_t n_rows,
                          sb_gradpair* out) {
  using namespace sb;
  SB_REQUIRE(ctx && labels && out && (n_rows == 0 || preds), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(objective >= SB_OBJ_SQUARED_ERROR && objective <= SB_OBJ_SOFTPROB, SB_ERR_INVALID_ARG,
             "unknown objective %d", objective);
  const bool multi = objective == SB_OBJ_SOFTMAX || objective == SB_OBJ_SOFTPROB;
  SB_REQUIRE(!multi || num_class >= 2, SB_ERR_INVALID_ARG,
             "invalid parameter `num_class`: multiclass objectives require num_class >= 2");
  SB_REQUIRE(scale_pos_weight > 0.0, SB_ERR_INVALID_ARG, "invalid parameter `scale_pos_weight`: must be > 0");
  if (n_rows == 0) return SB_OK;
  SB_CUDA(cudaSetDevice(ctx->device));
  const int K = n_outputs(objective, num_class);
  const size_t nk = n_rows * (size_t)K;
  cudaStream_t st = ctx->stream;
  DBuf<float> d_p, d_y, d_w;
  DBuf<float2> d_out;
  SB_TRY(d_p.alloc(ctx, nk));
  SB_TRY(d_y.alloc(ctx, n_rows));
  if (weights) SB_TRY(d_w.alloc(ctx, n_rows));
  SB_TRY(d_out.alloc(ctx, nk));
  SB_CUDA(cudaMemcpyAsync(d_p.p, preds, nk * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_y.p, labels, n_rows * 4, cudaMemcpyHostToDevice, st));
  if (weights) SB_CUDA(cudaMemcpyAsync(d_w.p, weights, n_rows * 4, cudaMemcpyHostToDevice, st));
  const unsigned blocks = (unsigned)std::min<size_t>((n_rows + 255) / 256, (size_t)ctx->num_sms * 16);
  SB_LAUNCH(ctx, k_objective_gradient, blocks, 256, 0, objective, K, (float)scale_pos_weight, d_p.p, d_y.p,
            d_w.p, n_rows, d_out.p);
  SB_CUDA(cudaMemcpyAsync(out, d_out.p, nk * 8, cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  return SB_OK;
}

int sb_tree_build(sb_ctx* ctx, const sb_ghist* g, const sb_train_params* p, const sb_gradpair* gpair,
                  size_t n, const uint32_t* rows, size_t m, uint64_t round, uint32_t k,
                  int32_t* row_leaf, sb_model** out) {
  using namespace sb;
  SB_REQUIRE(ctx && g && p && gpair && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_SAME_DEVICE(ctx, g);
  SB_REQUIRE(m == 0 || rows, SB_ERR_INVALID_ARG, "rows is NULL");
  SB_REQUIRE(n == g->n, SB_ERR_DIMENSION, "dimension mismatch: gpair length expected %zu, got %zu",
             g->n, n);
  SB_TRY(sb_train_params_validate(p));
  SB_CUDA(cudaSetDevice(ctx->device));
  *out = nullptr;
  sb_train_params q = *p;
  q.objective = SB_OBJ_SQUARED_ERROR;
  q.num_class = 0;
  sb_booster b;
  SB_TRY(booster_init(&b, ctx, g, &q, 1, true));
  b.p.objective = p->objective;
  b.p.num_class = p->num_class;
  std::vector<uint32_t> rl(n, UNSAMPLED);
  for (size_t i = 0; i < n; ++i) rl[i] = (uint32_t)i | UNSAMPLED;
  for (size_t i = 0; i < m; ++i) {
    SB_REQUIRE(rows[i] < n, SB_ERR_INVALID_ARG, "row %u out of range", rows[i]);
    rl[rows[i]] &= ~UNSAMPLED;
  }
  cudaStream_t st = ctx->stream;
  SB_CUDA(cudaMemcpyAsync(b.d_rows1.p, rl.data(), n * 4, cudaMemcpyHostToDevice, st));  // subset flags
  SB_CUDA(cudaMemcpyAsync(b.d_gpair.p, gpair, n * 8, cudaMemcpyHostToDevice, st));
  b.S.round_base = round;  // column sampling of class k in round `round`
  b.S.k_base = (int)k;
  if (row_leaf) {
    SB_TRY(b.d_row_leaf.alloc(ctx, n));
    b.S.row_leaf = b.d_row_leaf.p;
  }
  SB_TRY(booster_set_eval_smem(&b));
  SB_TRY(booster_round(&b));
  sb_model* mdl = new sb_model;
  mdl->ctx = ctx;
  // export tree `round`
  int nn = 0, nc = 0;
  std::vector<sb_node> nodes(b.maxn);
  SB_CUDA(cudaMemcpyAsync(&nn, b.d_out_nnodes.p, 4, cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaMemcpyAsync(&nc, b.d_out_ncats.p, 4, cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaMemcpyAsync(nodes.data(), b.d_out_nodes.p, b.maxn * sizeof(sb_node),
                          cudaMemcpyDeviceToHost, st));
  std::vector<uint32_t> cats(b.S.cat_cap);
  if (b.S.cat_cap)
    SB_CUDA(cudaMemcpyAsync(cats.data(), b.d_out_cats.p, b.S.cat_cap * 4,
                            cudaMemcpyDeviceToHost, st));
  if (row_leaf) SB_CUDA(cudaMemcpyAsync(row_leaf, b.d_row_leaf.p, n * 4, cudaMemcpyDeviceToHost, st));
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    delete mdl;
    return sb::cuda_status(e, "tree build", __FILE__, __LINE__);
  }
  mdl->trees.resize(1);
  mdl->trees[0].nodes.assign(nodes.begin(), nodes.begin() + nn);
  mdl->trees[0].cats.assign(cats.begin(), cats.begin() + nc);
  mdl->weights.assign(1, 1.0f);
  mdl->base_score = 0.0f;
  mdl->num_class = p->num_class;
  mdl->n_features = (int)g->F;
  mdl->objective = p->objective;
  *out = mdl;
  return SB_OK;
}

int sb_train(sb_ctx* ctx, const float* X, size_t n_rows, size_t n_cols, const uint8_t* feature_types,
             float missing, const float* labels, const float* weights, const float* base_margin,
             const sb_train_params* p, int num_boost_round, sb_model** out) {
  SB_REQUIRE(ctx && X && labels && p && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(num_boost_round >= 0, SB_ERR_INVALID_ARG, "negative num_boost_round");
  SB_TRY(sb_train_params_validate(p));
  if (p->tree_method == SB_TREE_APPROX) {
    SB_REQUIRE(n_rows > 0 && n_cols > 0, SB_ERR_INVALID_ARG, "empty dataset: zero rows or columns");
    SB_CUDA(cudaSetDevice(ctx->device));
    *out = nullptr;
    sb::DBuf<float> dX;
    SB_TRY(dX.alloc(ctx, n_rows * n_cols));
    SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, ctx->stream));
    return sb::approx_train(ctx, dX.p, n_rows, n_cols, feature_types, missing, labels, weights, base_margin, p,
                            num_boost_round, out);
  }
  sb_ghist* g = nullptr;
  SB_TRY(sb_ghist_create(ctx, X, n_rows, n_cols, feature_types, missing, p->max_bin, &g));
  sb_booster* b = nullptr;
  int s = sb_booster_create(ctx, g, p, labels, weights, base_margin, &b);
  if (s == SB_OK) s = sb_booster_update(b, num_boost_round);
  if (s == SB_OK) s = sb_booster_model(b, out);
  sb_booster_destroy(b);
  sb_ghist_destroy(g);
  return s;
}

int sb_train_dart(sb_ctx* ctx, const float* X, size_t n_rows, size_t n_cols, const uint8_t* feature_types,
                  float missing, const float* labels, const float* weights, const float* base_margin,
                  const sb_train_params* p, double rate_drop, double skip_drop, int num_boost_round,
                  sb_model** out) {
  using namespace sb;
  SB_REQUIRE(ctx && X && labels && p && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(num_boost_round >= 0, SB_ERR_INVALID_ARG, "negative num_boost_round");
  SB_REQUIRE(rate_drop >= 0.0 && rate_drop <= 1.0, SB_ERR_INVALID_ARG,
             "invalid parameter rate_drop=%g: must be in [0, 1]", rate_drop);
  SB_REQUIRE(skip_drop >= 0.0 && skip_drop <= 1.0, SB_ERR_INVALID_ARG,
             "invalid parameter skip_drop=%g: must be in [0, 1]", skip_drop);
  SB_TRY(sb_train_params_validate(p));
  SB_REQUIRE(p->tree_method != SB_TREE_APPROX, SB_ERR_UNSUPPORTED, "booster=dart trains tree_method=hist only");
  SB_REQUIRE(n_rows > 0 && n_cols > 0, SB_ERR_INVALID_ARG, "empty dataset: zero rows or columns");
  *out = nullptr;
  SB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  // the rows stay on the device: every round predicts the ensemble on them
  DBuf<float> dX;
  SB_TRY(dX.alloc(ctx, n_rows * n_cols));
  SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, st));
  sb_ghist* g = nullptr;
  SB_TRY(sb_ghist_create_device(ctx, dX.p, n_rows, n_cols, feature_types, missing, p->max_bin, &g));
  std::unique_ptr<sb_ghist, int (*)(sb_ghist*)> own_g(g, sb_ghist_destroy);
  sb_booster* b = nullptr;
  SB_TRY(sb_booster_create(ctx, g, p, labels, weights, base_margin, &b));
  std::unique_ptr<sb_booster, int (*)(sb_booster*)> own_b(b, sb_booster_destroy);
  const int K = b->K;
  DBuf<float> dbm;
  if (base_margin) {
    SB_TRY(dbm.alloc(ctx, n_rows * K));
    SB_CUDA(cudaMemcpyAsync(dbm.p, base_margin, dbm.bytes(), cudaMemcpyHostToDevice, st));
  }
  std::vector<float> w;  // tree weights (model.rs:130-145)
  // one host ensemble for the whole loop: each round appends only the trees
  // the previous round grew (the device copy is rebuilt for the prediction)
  std::unique_ptr<sb_model, int (*)(sb_model*)> m(new sb_model, sb_model_destroy);
  m->ctx = ctx;
  SB_TRY(booster_export(b, m.get()));
  for (int rnd = 0; rnd < num_boost_round; ++rnd) {
    const int existing = (int)w.size();
    const std::vector<int> dropped = dart_dropout(p->seed, (uint64_t)rnd, existing, rate_drop, skip_drop);
    if (existing) {  // margins of the ensemble with the dropped trees at weight 0
      SB_TRY(booster_export_append(b, m.get()));
      m->weights = w;
      for (int t : dropped) m->weights[t] = 0.0f;
      m->dev_valid = false;
      SB_TRY(predict_margin_device(m.get(), dX.p, n_rows, n_cols, missing, dbm.p, 1, 0, b->d_margin.p));
      b->delta_pending = false;  // the booster grows the round's trees from these margins
    }
    SB_TRY(booster_run(b, 1));
    b->stats.rounds = b->rounds_done;
    const float kd = (float)dropped.size();
    const float wn = 1.0f / (kd + 1.0f), ws = kd / (kd + 1.0f);
    for (int c = 0; c < K; ++c) w.push_back(wn);
    for (int t : dropped) w[t] = w[t] * ws;
  }
  SB_TRY(booster_export_append(b, m.get()));
  m->weights = w;
  m->dev_valid = false;
  *out = m.release();
  return SB_OK;
}

}  // extern "C"
