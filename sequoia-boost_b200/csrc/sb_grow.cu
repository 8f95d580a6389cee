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
//   per level d: k_eval -> k_assign -> k_partition -> k_plan -> histograms
//   -> k_round_end.
// All frontier nodes of all K class trees are processed by each launch.
#include <algorithm>
#include <cstring>

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

struct Fill {
  unsigned int left, right, lsamp, rsamp;
};

struct BState {
  // shapes
  int K, F, FW, HB, total_bins, max_depth, maxn, maxw, cat_cap;
  size_t n, Fp;
  // binned data
  const uint16_t* bins;
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
  unsigned int* kept;       // sampled rows this round
  // gradients
  float* margin;            // [n][K]
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
  // sampling
  uint32_t* pool;           // [K][F]
  int* pool_len;            // [K]
  uint32_t* samp_scratch;   // [1024][F] when per-node sampling is on
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

__device__ __forceinline__ void atomic_max_f(unsigned int* a, float v) {
  atomicMax(a, __float_as_uint(fabsf(v)));  // non-negative floats order as integers
}

__device__ __forceinline__ float sigmoidf_ref(float x) {  // classification.rs:7-15
  if (x >= 0.0f) return __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-x)));
  float e = expf(x);
  return __fdiv_rn(e, __fadd_rn(1.0f, e));
}

// ---------------------------------------------------------------- K3
__global__ void k_gradient(BState S) {
  const unsigned long long round = *S.round + S.round_base;
  const uint64_t rk = sb_round_key(S.seed, round);
  unsigned int kept = 0;
  float mg[16], mh[16];
  const int K = S.K;
  for (int c = 0; c < 16; ++c) mg[c] = mh[c] = 0.0f;
  for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < S.n;
       r += (size_t)gridDim.x * blockDim.x) {
    if (!S.ext_gpair) {
      const float w0 = S.weights ? S.weights[r] : 1.0f;
      const float y = S.labels[r];
      if (K == 1) {
        const float m = S.margin[r];
        float g, h;
        if (S.objective == SB_OBJ_SQUARED_ERROR) {  // regression.rs:18-40
          float d = __fsub_rn(m, y);
          g = S.weights ? __fmul_rn(d, w0) : d;
          h = S.weights ? w0 : 1.0f;
        } else if (S.objective == SB_OBJ_PSEUDOHUBER) {  // regression.rs:51-85
          float d = __fsub_rn(m, y);
          float s = __fadd_rn(1.0f, __fmul_rn(d, d));
          float sq = __fsqrt_rn(s);
          g = __fmul_rn(__fdiv_rn(d, sq), w0);
          h = __fmul_rn(__fdiv_rn(1.0f, __fmul_rn(s, sq)), w0);
        } else {  // logistic, classification.rs:50-71
          float p = sigmoidf_ref(m);
          float w = w0;
          if (y == 1.0f) w = __fmul_rn(w, S.spw);
          g = __fmul_rn(__fsub_rn(p, y), w);
          h = __fmul_rn(fmaxf(__fmul_rn(p, __fsub_rn(1.0f, p)), 1e-16f), w);
        }
        S.gpair[r] = make_float2(g, h);
        mg[0] = fmaxf(mg[0], fabsf(g));
        mh[0] = fmaxf(mh[0], fabsf(h));
      } else {  // softmax, multiclass.rs:14-30, :64-91
        const float* mr = S.margin + r * K;
        float mx = -INFINITY;
        for (int c = 0; c < K; ++c)
          if (mr[c] > mx) mx = mr[c];
        float sum = 0.0f;
        for (int c = 0; c < K; ++c) sum = __fadd_rn(sum, expf(__fsub_rn(mr[c], mx)));
        const float inv = __fdiv_rn(1.0f, sum);
        const int label = (int)y;
        for (int c = 0; c < K; ++c) {
          float p = __fmul_rn(expf(__fsub_rn(mr[c], mx)), inv);
          float target = (c == label) ? 1.0f : 0.0f;
          float g = __fmul_rn(__fsub_rn(p, target), w0);
          float h = fmaxf(__fmul_rn(__fmul_rn(__fmul_rn(2.0f, p), __fsub_rn(1.0f, p)), w0), 1e-16f);
          S.gpair[(size_t)c * S.n + r] = make_float2(g, h);
          if (c < 16) {
            mg[c] = fmaxf(mg[c], fabsf(g));
            mh[c] = fmaxf(mh[c], fabsf(h));
          }
        }
      }
    } else {
      for (int c = 0; c < K && c < 16; ++c) {
        float2 v = S.gpair[(size_t)c * S.n + r];
        mg[c] = fmaxf(mg[c], fabsf(v.x));
        mh[c] = fmaxf(mh[c], fabsf(v.y));
      }
    }
    bool keep;
    if (S.ext_gpair) keep = !(S.rows0[r] & UNSAMPLED);  // the caller's subset
    else keep = S.subsample >= 1.0 || sb_u01(sb_row_draw(rk, r)) < S.subsample;
    if (!S.ext_gpair) S.rows0[r] = (uint32_t)r | (keep ? 0u : UNSAMPLED);
    kept += keep ? 1u : 0u;
  }
  for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xFFFFFFFFu, kept, o);
  if ((threadIdx.x & 31) == 0 && kept) atomicAdd(S.kept, kept);
  if (S.fixed) {
    for (int c = 0; c < K && c < 16; ++c) {
      float a = mg[c], b = mh[c];
      for (int o = 16; o > 0; o >>= 1) {
        a = fmaxf(a, __shfl_xor_sync(0xFFFFFFFFu, a, o));
        b = fmaxf(b, __shfl_xor_sync(0xFFFFFFFFu, b, o));
      }
      if ((threadIdx.x & 31) == 0) {
        atomic_max_f(&S.maxabs[2 * c], a);
        atomic_max_f(&S.maxabs[2 * c + 1], b);
      }
    }
  }
}

// Column subset of node `nid` (sampler.rs:52-70 with sb_sampling.h keys),
// intersected with the node's allowed set, as a bitmask.
__device__ void node_feature_mask(const BState& S, int k, int nid, uint64_t tkey, uint32_t* out,
                                  const uint32_t* allowed, bool allowed_all, uint32_t* scratch) {
  for (int w = 0; w < S.FW; ++w) out[w] = 0u;
  const uint32_t* pool = S.pool + (size_t)k * S.F;
  int len = S.pool_len[k];
  if (S.bylevel >= 1.0 && S.bynode >= 1.0) {
    for (int i = 0; i < len; ++i) out[pool[i] >> 5] |= 1u << (pool[i] & 31);
  } else {
    for (int i = 0; i < len; ++i) scratch[i] = pool[i];
    sb_splitmix gen{sb_node_key(tkey, (uint64_t)nid)};
    int l1 = sb_subsample(scratch, len, S.bylevel, &gen);
    int l2 = sb_subsample(scratch, l1, S.bynode, &gen);
    for (int i = 0; i < l2; ++i) out[scratch[i] >> 5] |= 1u << (scratch[i] & 31);
  }
  if (!allowed_all)
    for (int w = 0; w < S.FW; ++w) out[w] &= allowed[w];
}

// Per round: quantisation scales, the sampled-row fallback, the per-tree
// column pools and the root of every class tree.
__global__ void k_round_prep(BState S) {
  const unsigned long long round = *S.round + S.round_base;
  const int tid = threadIdx.x;
  if (tid == 0) *S.qerr = 0ull;
  if (tid == 0 && *S.kept == 0 && !S.ext_gpair) {  // train.rs:472-474
    uint64_t rk = sb_round_key(S.seed, round);
    S.rows0[sb_row_fallback(rk, S.n)] &= ~UNSAMPLED;
    *S.kept = 1;
  }
  for (int k = tid; k < S.K; k += blockDim.x) {
    if (S.fixed) {
      int sg = quant_shift(__uint_as_float(S.maxabs[2 * k]), S.bits);
      int sh = quant_shift(__uint_as_float(S.maxabs[2 * k + 1]), S.bits);
      S.shifts[2 * k] = sg;
      S.shifts[2 * k + 1] = sh;
      S.inv_scale[2 * k] = ldexp(1.0, -sg);
      S.inv_scale[2 * k + 1] = ldexp(1.0, -sh);
    }
    // colsample_bytree pool (train.rs:479-489)
    uint64_t tkey = sb_tree_key(S.seed, round, (uint64_t)(k + S.k_base));
    uint32_t* pool = S.pool + (size_t)k * S.F;
    for (int f = 0; f < S.F; ++f) pool[f] = (uint32_t)f;
    int len = S.F;
    if (S.bytree < 1.0) {
      sb_splitmix gen{tkey};
      len = sb_subsample(pool, S.F, S.bytree, &gen);
    }
    S.pool_len[k] = len;
    S.num_nodes[k] = 1;
    S.lvl_begin[k] = 0;
    S.lvl_count[k] = 1;
    S.prev_begin[k] = 0;
    S.cat_count[k] = 0;
    size_t r0 = NI(S, k, 0);
    S.seg[r0] = make_uint2(0u, (unsigned)S.n);
    S.nsamp[r0] = *S.kept;
    S.bounds[r0] = make_double2(-INFINITY, INFINITY);
    S.allowed_all[r0] = 1;
    S.built[r0] = 1;
    S.parent[r0] = -1;
    S.root_total[k] = make_longlong2(0, 0);
    node_feature_mask(S, k, 0, tkey, S.fmask + r0 * S.FW, nullptr, true,
                      S.samp_scratch ? S.samp_scratch + (size_t)tid * S.F : nullptr);
    HistItem it;
    it.rows = S.rows0;  // level 0 shares the root list of class 0
    it.begin = 0;
    it.end = (uint32_t)S.n;
    it.k = (uint32_t)k;
    it.root = 1;
    it.out = level_hist(S, 0, k, 0);
    it.total = &S.root_total[k];
    S.items[k] = it;
    S.prefix[k] = (uint64_t)k * S.n;
  }
  if (tid == 0) {
    S.prefix[S.K] = (uint64_t)S.K * S.n;
    *S.item_count = S.K;
  }
}

// FIXED: q = rint(x * 2^s), packed (q_g << 32) + q_h.
__global__ void k_quantize(BState S) {
  float eg = 0.0f, eh = 0.0f;
  const size_t total = (size_t)S.K * S.n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    int k = (int)(i / S.n);
    float2 v = S.gpair[i];
    int sg = S.shifts[2 * k], sh = S.shifts[2 * k + 1];
    float xg = ldexpf(v.x, sg), xh = ldexpf(v.y, sh);
    int qg = __float2int_rn(xg), qh = __float2int_rn(xh);
    S.gpk[i] = ((unsigned long long)(uint32_t)qg << 32) + (unsigned long long)(uint32_t)qh;
    eg = fmaxf(eg, fabsf(__fsub_rn(v.x, ldexpf((float)qg, -sg))));
    eh = fmaxf(eh, fabsf(__fsub_rn(v.y, ldexpf((float)qh, -sh))));
  }
  for (int o = 16; o > 0; o >>= 1) {
    eg = fmaxf(eg, __shfl_xor_sync(0xFFFFFFFFu, eg, o));
    eh = fmaxf(eh, __shfl_xor_sync(0xFFFFFFFFu, eh, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax((unsigned int*)&S.qerr[0], __float_as_uint(eg));
    atomicMax((unsigned int*)&S.qerr[1], __float_as_uint(eh));
  }
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
struct CatScratch {
  double g[MAX_CAT_BINS];
  double h[MAX_CAT_BINS];
  long long key[MAX_CAT_BINS];
  uint16_t ne[MAX_CAT_BINS];      // non-empty bins, ascending
  uint16_t order[MAX_CAT_BINS];   // sorted by ratio (stable)
};

// The result of a sequential replay of one feature.
struct Chosen {
  double gain;
  int cand;    // candidate index within the feature, -1 none
};

// Warp-parallel scan of one feature's candidates in the reference's order:
//   numeric  : bins ascending, direction A (missing right) before B
//   category : prefixes of the ratio-sorted non-empty bins
// MODE 0 returns the feature's max candidate gain (phase 1).
// MODE 1 replays `consider`'s rule `g > best + 1e-6` exactly from state
// b_in: a taken candidate must be a strict new prefix maximum P; any
// candidate with g > P + eps is certainly taken; so the outcome is the last
// certain record k*, followed by a short sequential resolution of the
// remaining (ambiguous) records after k*.
template <int MODE>
__device__ Chosen scan_feature(const BState& S, const char* H, int k, int f, const EvalNode& E,
                               double b_in, CatScratch* cs, double* s_gains, NodeSplit* out) {
  const int lane = threadIdx.x & 31;
  const int fs = (int)S.foff[f], nb = (int)S.foff[f + 1] - fs;
  const int dir = S.mono ? S.mono[f] : 0;
  Chosen res{b_in, -1};
  double fmax_g = -INFINITY;
  if (!S.is_cat[f]) {
    // missing statistics come from the feature's missing bin; present = sum
    double2 miss = hist_entry(S, H, S.total_bins + f, k);
    double pg = 0.0, ph = 0.0;
    for (int c0 = 0; c0 < nb; c0 += 32) {
      int i = c0 + lane;
      double2 v = i < nb ? hist_entry(S, H, fs + i, k) : make_double2(0.0, 0.0);
      pg += v.x;
      ph += v.y;
    }
    pg = warp_sum(pg);
    ph = warp_sum(ph);
    const bool has_missing = miss.y > 1e-6;
    for (int pass = 0; pass < (MODE == 0 ? 1 : 2); ++pass) {
      double cg = 0.0, ch = 0.0, P = b_in;
      // pass 0 (MODE 1): last certain record; pass 1: resolution
      __shared__ int s_kstar[EVAL_THREADS / 32];
      __shared__ double s_gstar[EVAL_THREADS / 32];
      const int w = threadIdx.x >> 5;
      if (pass == 0 && lane == 0) {
        s_kstar[w] = -1;
        s_gstar[w] = b_in;
      }
      __syncwarp();
      int kstar = pass == 1 ? s_kstar[w] : -1;
      double bstate = pass == 1 ? s_gstar[w] : b_in;
      int chosen = kstar;
      for (int c0 = 0; c0 < nb - 1; c0 += 32) {
        const int i = c0 + lane;
        double2 v = i < nb ? hist_entry(S, H, fs + i, k) : make_double2(0.0, 0.0);
        double sg = warp_incl_sum(v.x), shh = warp_incl_sum(v.y);
        double ag = cg + sg, ah = ch + shh;
        double tg = __shfl_sync(0xFFFFFFFFu, sg, 31), th = __shfl_sync(0xFFFFFFFFu, shh, 31);
        double gA = -INFINITY, gB = -INFINITY, wlA = 0, wrA = 0, wlB = 0, wrB = 0;
        if (i < nb - 1) {
          gA = cand_gain(S, E, dir, ag, ah, dsub(E.tg, ag), dsub(E.th, ah), &wlA, &wrA);
          if (has_missing)
            gB = cand_gain(S, E, dir, dadd(ag, miss.x), dadd(ah, miss.y), dsub(pg, ag), dsub(ph, ah),
                           &wlB, &wrB);
        }
        if (MODE == 0) {
          fmax_g = fmax(fmax_g, fmax(gA, gB));
        } else {
          double lm = fmax(gA, gB);
          double PA = warp_excl_max(lm, P);
          double PB = fmax(PA, gA);
          if (pass == 0) {
            int ci = -1;
            double cgain = 0;
            if (gB > PB + K_RT_EPS) { ci = 2 * i + 1; cgain = gB; }
            else if (gA > PA + K_RT_EPS) { ci = 2 * i; cgain = gA; }
            // the highest candidate index wins
            int best_ci = ci;
            for (int o = 16; o > 0; o >>= 1) best_ci = max(best_ci, __shfl_xor_sync(0xFFFFFFFFu, best_ci, o));
            if (best_ci >= 0 && ci == best_ci) {
              s_kstar[w] = ci;
              s_gstar[w] = cgain;
            }
            __syncwarp();
          } else {
            // records after k* in candidate order, resolved sequentially
            bool recA = (2 * i > kstar) && gA > PA;
            bool recB = (2 * i + 1 > kstar) && gB > PB;
            unsigned ma = __ballot_sync(0xFFFFFFFFu, recA), mb = __ballot_sync(0xFFFFFFFFu, recB);
            s_gains[lane] = gA;
            s_gains[32 + lane] = gB;
            __syncwarp();
            if (lane == 0 && (ma | mb)) {
              for (int L = 0; L < 32; ++L) {
                if ((ma >> L) & 1u) {
                  double gv = s_gains[L];
                  if (gv > bstate + K_RT_EPS) { bstate = gv; chosen = 2 * (c0 + L); }
                }
                if ((mb >> L) & 1u) {
                  double gv = s_gains[32 + L];
                  if (gv > bstate + K_RT_EPS) { bstate = gv; chosen = 2 * (c0 + L) + 1; }
                }
              }
            }
            bstate = __shfl_sync(0xFFFFFFFFu, bstate, 0);
            chosen = __shfl_sync(0xFFFFFFFFu, chosen, 0);
            __syncwarp();
            // the owner of the chosen candidate records its statistics
            if (out && chosen >= 0 && (chosen >> 1) == i) {
              const bool isB = chosen & 1;
              out->feature = f;
              out->bin = i;
              out->default_left = isB ? 1 : 0;
              out->is_cat = 0;
              out->ncat = 0;
              out->lg = isB ? dadd(ag, miss.x) : ag;
              out->lh = isB ? dadd(ah, miss.y) : ah;
              out->rg = isB ? dsub(pg, ag) : dsub(E.tg, ag);
              out->rh = isB ? dsub(ph, ah) : dsub(E.th, ah);
              out->wl = isB ? wlB : wlA;
              out->wr = isB ? wrB : wrA;
            }
            __syncwarp();
          }
          P = fmax(P, warp_max(lm));
        }
        cg += tg;
        ch += th;
      }
      if (MODE == 1 && pass == 1) {
        res.gain = bstate;
        res.cand = chosen;
      }
    }
    if (MODE == 0) res.gain = warp_max(fmax_g);  // every lane's candidates
    return res;
  }
  // ---- categorical (evaluate_categorical, hist.rs:607-653)
  const double lam = S.reg.lambda;
  int nne = 0;
  for (int c0 = 0; c0 < nb; c0 += 32) {
    int i = c0 + lane;
    double2 v = i < nb ? hist_entry(S, H, fs + i, k) : make_double2(0.0, -1.0);
    bool ne = i < nb && v.y > 0.0;
    unsigned m = __ballot_sync(0xFFFFFFFFu, ne);
    if (ne) {
      int pos = nne + __popc(m & ((1u << lane) - 1u));
      cs->ne[pos] = (uint16_t)i;
      cs->g[pos] = v.x;
      cs->h[pos] = v.y;
      cs->key[pos] = total_cmp_key(ddiv(v.x, dadd(v.y, lam)));
    }
    nne += __popc(m);
  }
  __syncwarp();
  if (nne < 2) {
    res.gain = MODE == 0 ? -INFINITY : b_in;
    return res;
  }
  for (int i = lane; i < nne; i += 32) {  // stable rank by key
    long long ki = cs->key[i];
    int r = 0;
    for (int j = 0; j < nne; ++j) {
      long long kj = cs->key[j];
      r += (kj < ki || (kj == ki && j < i)) ? 1 : 0;
    }
    cs->order[r] = (uint16_t)i;  // index into ne/g/h
  }
  __syncwarp();
  const int ncand = nne - 1;
  __shared__ int s_kstar_c[EVAL_THREADS / 32];
  __shared__ double s_gstar_c[EVAL_THREADS / 32];
  const int w = threadIdx.x >> 5;
  for (int pass = 0; pass < (MODE == 0 ? 1 : 2); ++pass) {
    double cg = 0.0, ch = 0.0, P = b_in;
    if (pass == 0 && lane == 0) {
      s_kstar_c[w] = -1;
      s_gstar_c[w] = b_in;
    }
    __syncwarp();
    int kstar = pass == 1 ? s_kstar_c[w] : -1;
    double bstate = pass == 1 ? s_gstar_c[w] : b_in;
    int chosen = kstar;
    for (int c0 = 0; c0 < ncand; c0 += 32) {
      const int pidx = c0 + lane;
      double vg = 0.0, vh = 0.0;
      if (pidx < nne) {
        int o = cs->order[pidx];
        vg = cs->g[o];
        vh = cs->h[o];
      }
      double lg = cg + warp_incl_sum(vg), lh = ch + warp_incl_sum(vh);
      double tg = __shfl_sync(0xFFFFFFFFu, lg - cg, 31), th = __shfl_sync(0xFFFFFFFFu, lh - ch, 31);
      double gv = -INFINITY, wl = 0, wr = 0;
      if (pidx < ncand) gv = cand_gain(S, E, dir, lg, lh, dsub(E.tg, lg), dsub(E.th, lh), &wl, &wr);
      if (MODE == 0) {
        fmax_g = fmax(fmax_g, gv);
      } else {
        double Pc = warp_excl_max(gv, P);
        if (pass == 0) {
          int ci = gv > Pc + K_RT_EPS ? pidx : -1;
          int best_ci = ci;
          for (int o = 16; o > 0; o >>= 1) best_ci = max(best_ci, __shfl_xor_sync(0xFFFFFFFFu, best_ci, o));
          if (best_ci >= 0 && ci == best_ci) {
            s_kstar_c[w] = ci;
            s_gstar_c[w] = gv;
          }
          __syncwarp();
        } else {
          bool rec = pidx > kstar && gv > Pc;
          unsigned m = __ballot_sync(0xFFFFFFFFu, rec);
          s_gains[lane] = gv;
          __syncwarp();
          if (lane == 0 && m) {
            for (int L = 0; L < 32; ++L)
              if ((m >> L) & 1u) {
                double x = s_gains[L];
                if (x > bstate + K_RT_EPS) { bstate = x; chosen = c0 + L; }
              }
          }
          bstate = __shfl_sync(0xFFFFFFFFu, bstate, 0);
          chosen = __shfl_sync(0xFFFFFFFFu, chosen, 0);
          __syncwarp();
          if (out && chosen == pidx) {
            out->feature = f;
            out->bin = 0;
            out->default_left = 0;
            out->is_cat = 1;
            out->ncat = pidx + 1;
            out->lg = lg;
            out->lh = lh;
            out->rg = dsub(E.tg, lg);
            out->rh = dsub(E.th, lh);
            out->wl = wl;
            out->wr = wr;
          }
          __syncwarp();
        }
        P = fmax(P, warp_max(gv));
      }
      cg += tg;
      ch += th;
    }
    if (MODE == 1 && pass == 1) {
      res.gain = bstate;
      res.cand = chosen;
      if (out && chosen >= 0 && chosen == res.cand) {
        // categories routed left, in sweep order (cats_left, hist.rs:630-636)
        for (int i = lane; i < MAX_CAT_BINS / 32; i += 32) out->cat_mask[i] = 0u;
        __syncwarp();
        for (int p = lane; p <= chosen; p += 32) {
          int b = cs->ne[cs->order[p]];
          out->cat_order[p] = (uint8_t)b;
          atomicOr(&out->cat_mask[b >> 5], 1u << (b & 31));
        }
        __syncwarp();
      }
    }
  }
  if (MODE == 0) res.gain = warp_max(fmax_g);
  return res;
}

// One CTA per frontier node: materialise a subtracted histogram if the node
// was not built, then find its best split with the reference's tie rule.
__global__ void __launch_bounds__(EVAL_THREADS) k_eval(BState S, int d) {
  extern __shared__ double ev_sm[];
  const int k = blockIdx.y, slot = blockIdx.x;
  if (slot >= S.lvl_count[k]) return;
  const int nid = S.lvl_begin[k] + slot;
  const size_t ni = NI(S, k, nid);
  char* H = level_hist(S, d, k, slot);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  double* s_M = ev_sm;                                    // [F]
  int* s_flist = reinterpret_cast<int*>(s_M + S.F);       // [F]
  double* s_gains = reinterpret_cast<double*>(s_flist + S.F + (S.F & 1));  // [64]
  CatScratch* s_cat = reinterpret_cast<CatScratch*>(s_gains + 64);        // [nwarps] if categorical
  __shared__ int s_nf;
  __shared__ EvalNode s_E;
  __shared__ NodeSplit s_best;

  if (d > 0 && !S.built[ni]) {  // sibling = parent - built child (K5)
    const int pslot = S.parent[ni] - S.prev_begin[k];
    const char* P = level_hist(S, d - 1, k, pslot);
    const char* B = level_hist(S, d, k, slot ^ 1);
    if (S.fixed) {
      const longlong2* p = reinterpret_cast<const longlong2*>(P);
      const longlong2* b = reinterpret_cast<const longlong2*>(B);
      longlong2* o = reinterpret_cast<longlong2*>(H);
      for (int i = tid; i < S.HB; i += blockDim.x) {
        longlong2 x = p[i], y = b[i];
        o[i] = make_longlong2(x.x - y.x, x.y - y.y);
      }
    } else {
      const double2* p = reinterpret_cast<const double2*>(P);
      const double2* b = reinterpret_cast<const double2*>(B);
      double2* o = reinterpret_cast<double2*>(H);
      for (int i = tid; i < S.HB; i += blockDim.x) {
        double2 x = p[i], y = b[i];
        o[i] = make_double2(dsub(x.x, y.x), dsub(x.y, y.y));
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (d == 0) {  // root statistics, summed by the root histogram launch
      double2 t;
      if (S.fixed) {
        longlong2 q = S.root_total[k];
        t = make_double2(dmul((double)q.x, S.inv_scale[2 * k]), dmul((double)q.y, S.inv_scale[2 * k + 1]));
      } else {
        t = reinterpret_cast<const double2*>(S.root_total)[k];
      }
      S.stats[ni] = t;
    }
    double2 st = S.stats[ni];
    double2 bd = S.bounds[ni];
    EvalNode E;
    E.tg = st.x;
    E.th = st.y;
    E.lo = bd.x;
    E.hi = bd.y;
    E.parent_gain = S.constrained
        ? gain_at_weight(st.x, st.y, S.reg, calc_weight_bounded(st.x, st.y, S.reg, bd.x, bd.y))
        : calc_gain(st.x, st.y, S.reg);
    s_E = E;
    s_best.loss_chg = 0.0;
    s_best.feature = -1;
    s_best.valid = 0;
    s_best.ncat = 0;
    s_best.is_cat = 0;
    s_best.default_left = 1;
    s_best.wl = s_best.wr = 0.0;
    s_best.lg = s_best.lh = s_best.rg = s_best.rh = 0.0;
    s_best.bin = 0;
  }
  // candidate features: sampled & allowed, with >= 2 bins, ascending
  if (warp == 0) {
    const uint32_t* fm = S.fmask + ni * S.FW;
    int cnt = 0;
    for (int w0 = 0; w0 < S.FW; w0 += 32) {
      int wi = w0 + lane;
      uint32_t word = wi < S.FW ? fm[wi] : 0u;
      // keep features with >= 2 bins
      for (int b = 0; b < 32 && word; ++b) {
        if ((word >> b) & 1u) {
          int f = wi * 32 + b;
          if (f >= S.F || S.foff[f + 1] - S.foff[f] < 2) word &= ~(1u << b);
        }
      }
      int pc = __popc(word);
      int incl = pc;
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      int pos = cnt + incl - pc;
      while (word) {
        int b = __ffs(word) - 1;
        word &= word - 1;
        s_flist[pos++] = wi * 32 + b;
      }
      cnt += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    if (lane == 0) s_nf = cnt;
  }
  __syncthreads();
  const EvalNode E = s_E;
  const int nf = s_nf;
  CatScratch* my_cs = S.cat_cap > 0 ? s_cat + warp : nullptr;
  // phase 1: every feature's max candidate gain
  for (int i = warp; i < nf; i += nwarps) {
    Chosen c = scan_feature<0>(S, H, k, s_flist[i], E, 0.0, my_cs, nullptr, nullptr);
    if (lane == 0) s_M[i] = c.gain;
  }
  __syncthreads();
  // phase 2: exact sequential replay over the features that can still win
  if (warp == 0) {
    double b = 0.0;
    for (int i = 0; i < nf; ++i) {
      if (!(s_M[i] > b + K_RT_EPS)) continue;
      Chosen c = scan_feature<1>(S, H, k, s_flist[i], E, b, my_cs, s_gains, &s_best);
      if (c.cand >= 0) {
        b = c.gain;
        if (lane == 0) s_best.loss_chg = b;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (tid == 0) {
    NodeSplit& o = S.split[ni];
    bool found = s_best.feature >= 0 && s_best.loss_chg > K_RT_EPS;
    bool valid = found && s_best.loss_chg > S.gamma && s_best.lh >= S.reg.mcw && s_best.rh >= S.reg.mcw;
    o.loss_chg = s_best.loss_chg;
    o.lg = s_best.lg;
    o.lh = s_best.lh;
    o.rg = s_best.rg;
    o.rh = s_best.rh;
    o.wl = s_best.wl;
    o.wr = s_best.wr;
    o.feature = s_best.feature;
    o.bin = s_best.bin;
    o.default_left = s_best.default_left;
    o.is_cat = s_best.is_cat;
    o.ncat = s_best.is_cat ? s_best.ncat : 0;
    o.valid = valid ? 1 : 0;
  }
  if (s_best.is_cat && s_best.feature >= 0) {
    NodeSplit& o = S.split[ni];
    for (int i = tid; i < MAX_CAT_BINS / 32; i += blockDim.x) o.cat_mask[i] = s_best.cat_mask[i];
    for (int i = tid; i < s_best.ncat; i += blockDim.x) o.cat_order[i] = s_best.cat_order[i];
  }
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
__global__ void __launch_bounds__(1024) k_assign(BState S, int d, int write_tiles) {
  __shared__ int sm_i[33];
  __shared__ int s_tile_carry;
  const unsigned long long round = *S.round;
  const int tid = threadIdx.x;
  if (tid == 0) s_tile_carry = 0;
  __syncthreads();
  const bool last = (d + 1 == S.max_depth);
  for (int k = 0; k < S.K; ++k) {
    const int begin = S.lvl_begin[k], cnt = S.lvl_count[k], nn0 = S.num_nodes[k];
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
        S.fill[ni] = Fill{0u, 0u, 0u, 0u};
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
          uint32_t* scratch = S.samp_scratch ? S.samp_scratch + (size_t)tid * S.F : nullptr;
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
      // partition tiles of this frontier node
      int tot_t;
      const int toff = s_tile_carry + block_scan_excl<int>(tiles, &tot_t, sm_i);
      if (write_tiles && act) {
        const uint2 sg = S.seg[ni];
        for (int q = 0; q < tiles && toff + q < S.ptile_cap; ++q) {
          unsigned b = sg.x + q * PART_TILE;
          unsigned e = min(sg.y, b + PART_TILE);
          S.ptiles[toff + q] = make_int4(k, nid, (int)b, (int)e);
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
      S.lvl_begin[k] = nn0;
      S.lvl_count[k] = 2 * carry_v;
      S.num_nodes[k] = nn0 + 2 * carry_v;
      S.cat_count[k] = carry_c;
    }
    __syncthreads();
  }
  if (tid == 0) *S.ptile_count = min(s_tile_carry, S.ptile_cap);
}

// K7 + K8: stable-count partition of every split node's rows into its two
// children (left rows fill from the segment start, right rows from its end),
// and the margin update (train.rs:326-328) for rows whose node is final.
__global__ void __launch_bounds__(256) k_partition(BState S, int d) {
  __shared__ unsigned int sm_u[33];
  __shared__ unsigned int s_base[2];
  const bool last = (d + 1 == S.max_depth);
  const int ntiles = *S.ptile_count;
  const uint32_t* rows_cur_all = (d & 1) ? S.rows1 : S.rows0;
  uint32_t* rows_nxt_all = (d & 1) ? S.rows0 : S.rows1;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tile = S.ptiles[t];
    const int k = tile.x, nid = tile.y;
    const size_t ni = NI(S, k, nid);
    const uint32_t* rows_cur = rows_cur_all + (d == 0 ? 0 : (size_t)k * S.n);
    uint32_t* rows_nxt = rows_nxt_all + (size_t)k * S.n;
    const NodeSplit& sp = S.split[ni];
    const int K = S.K;
    if (!sp.valid) {
      const float lv = S.leafval[ni];
      for (int p = tile.z + threadIdx.x; p < tile.w; p += blockDim.x) {
        uint32_t rv = rows_cur[p];
        uint32_t id = rv & ~UNSAMPLED;
        if (S.update_margin) S.margin[(size_t)id * K + k] += lv;
        if (S.row_leaf) S.row_leaf[id] = (rv & UNSAMPLED) ? -1 : nid;
      }
      continue;
    }
    const int f = sp.feature, sbin = sp.bin, dl = sp.default_left, isc = sp.is_cat;
    const int left_id = S.out_nodes[((size_t)(*S.round) * K + k) * S.maxn + nid].left;
    constexpr int PER = PART_TILE / 256;
    uint32_t rv[PER];
    bool gl[PER];
    unsigned nl = 0, nls = 0, nrs = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      int p = tile.z + q * 256 + threadIdx.x;
      rv[q] = UNSAMPLED;
      gl[q] = false;
      if (p < tile.w) {
        rv[q] = rows_cur[p];
        uint32_t id = rv[q] & ~UNSAMPLED;
        uint16_t b = S.bins[(size_t)id * S.Fp + f];
        bool go;
        if (b == MISSING_BIN) go = dl != 0;
        else if (isc) go = (sp.cat_mask[b >> 5] >> (b & 31)) & 1u;
        else go = (int)b <= sbin;
        gl[q] = go;
        if (last) {
          int child = go ? left_id : left_id + 1;
          size_t ci = NI(S, k, child);
          if (S.update_margin) S.margin[(size_t)id * K + k] += S.leafval[ci];
          if (S.row_leaf) S.row_leaf[id] = (rv[q] & UNSAMPLED) ? -1 : child;
        } else {
          nl += go ? 1u : 0u;
          bool smp = !(rv[q] & UNSAMPLED);
          nls += (go && smp) ? 1u : 0u;
          nrs += (!go && smp) ? 1u : 0u;
        }
      }
    }
    if (last) continue;
    const int nvalid = min(PART_TILE, tile.w - tile.z);
    unsigned totl;
    const unsigned loff = block_scan_excl<unsigned>(nl, &totl, sm_u);
    unsigned cnt_here = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) cnt_here += (tile.z + q * 256 + (int)threadIdx.x < tile.w) ? 1u : 0u;
    unsigned totall;
    const unsigned aoff = block_scan_excl<unsigned>(cnt_here, &totall, sm_u);
    unsigned ls = nls, rs = nrs;
    for (int o = 16; o > 0; o >>= 1) {
      ls += __shfl_xor_sync(0xFFFFFFFFu, ls, o);
      rs += __shfl_xor_sync(0xFFFFFFFFu, rs, o);
    }
    Fill* fl = &S.fill[ni];
    if ((threadIdx.x & 31) == 0) {
      if (ls) atomicAdd(&fl->lsamp, ls);
      if (rs) atomicAdd(&fl->rsamp, rs);
    }
    const unsigned totr = (unsigned)nvalid - totl;
    if (threadIdx.x == 0) {
      s_base[0] = atomicAdd(&fl->left, totl);
      s_base[1] = atomicAdd(&fl->right, totr);
    }
    __syncthreads();
    const uint2 sg = S.seg[ni];
    unsigned li = loff, ri = aoff - loff;  // right rows before mine = all before - left before
    const unsigned lbase = sg.x + s_base[0];
    const unsigned rbase = sg.y - s_base[1] - totr;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      int p = tile.z + q * 256 + threadIdx.x;
      if (p < tile.w) {
        if (gl[q]) rows_nxt[lbase + li++] = rv[q];
        else rows_nxt[rbase + ri++] = rv[q];
      }
    }
    __syncthreads();
  }
}

// After the partition: children segments and sampled counts, the smaller
// child to build (hist.rs:352-362: left when left_rows <= right_rows), and
// the histogram work list of level d + 1.
__global__ void __launch_bounds__(1024) k_plan(BState S, int d) {
  __shared__ int sm_i[33];
  __shared__ unsigned long long sm_u[33];
  __shared__ int s_items;
  __shared__ unsigned long long s_pos;
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_items = 0;
    s_pos = 0;
  }
  __syncthreads();
  const unsigned long long round = *S.round;
  const int dn = d + 1;
  for (int k = 0; k < S.K; ++k) {
    const int pbegin = S.prev_begin[k];
    const int pcount = S.lvl_begin[k] - pbegin;  // frontier of level d
    const int cbegin = S.lvl_begin[k];
    uint32_t* rows_nxt = ((dn & 1) ? S.rows1 : S.rows0) + (size_t)k * S.n;
    const sb_node* out = S.out_nodes + ((size_t)round * S.K + k) * S.maxn;
    for (int c0 = 0; c0 < pcount; c0 += blockDim.x) {
      const int slot = c0 + tid;
      int v = 0;
      unsigned long long len = 0;
      int bchild = -1;
      uint2 bseg = make_uint2(0, 0);
      if (slot < pcount) {
        const int nid = pbegin + slot;
        const size_t ni = NI(S, k, nid);
        if (S.split[ni].valid) {
          const Fill fl = S.fill[ni];
          const uint2 sg = S.seg[ni];
          const int l = out[nid].left, r = l + 1;
          const size_t li = NI(S, k, l), ri = NI(S, k, r);
          S.seg[li] = make_uint2(sg.x, sg.x + fl.left);
          S.seg[ri] = make_uint2(sg.x + fl.left, sg.y);
          S.nsamp[li] = fl.lsamp;
          S.nsamp[ri] = fl.rsamp;
          const bool build_left = fl.lsamp <= fl.rsamp;
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
        it.rows = rows_nxt;
        it.begin = bseg.x;
        it.end = bseg.y;
        it.k = (uint32_t)k;
        it.root = 0;
        it.out = level_hist(S, dn, k, bchild - cbegin);
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
  }
}

__global__ void k_round_end(BState S) {
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
    if (S.fixed)
      for (int i = 0; i < 2 * S.K; ++i) S.maxabs[i] = 0u;
  }
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
  sb::DBuf<float2> d_gpair;
  sb::DBuf<unsigned long long> d_gpk;
  sb::DBuf<unsigned int> d_maxabs;
  sb::DBuf<int> d_shifts;
  sb::DBuf<double> d_inv_scale;
  sb::DBuf<unsigned long long> d_qerr;
  sb::DBuf<char> d_hist0, d_hist1;
  sb::DBuf<longlong2> d_root_total;
  sb::DBuf<sb::HistItem> d_items;
  sb::DBuf<uint64_t> d_prefix;
  sb::DBuf<int> d_item_count;
  sb::DBuf<int4> d_ptiles;
  sb::DBuf<int> d_ptile_count;
  sb::DBuf<uint32_t> d_pool;
  sb::DBuf<int> d_pool_len;
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
  SB_REQUIRE(p->grow_policy == SB_GROW_DEPTHWISE, SB_ERR_UNSUPPORTED,
             "grow_policy=lossguide is not available on the GPU path yet");
  SB_REQUIRE(K >= 1 && K <= 16, SB_ERR_UNSUPPORTED, "at most 16 outputs per round on the GPU");
  b->D = p->max_depth;
  b->maxn = (1 << (b->D + 1)) - 1;
  b->maxw = 1 << (b->D - 1);
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
  SB_TRY(b->d_mono.alloc(ctx, F));
  SB_TRY(b->d_in_group.alloc(ctx, F));
  SB_TRY(b->d_iset.alloc(ctx, (size_t)F * FW));
  SB_CUDA(cudaMemcpyAsync(b->d_mono.p, mono_full.data(), F, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(b->d_in_group.p, in_group.data(), F, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(b->d_iset.p, iset.data(), iset.size() * 4, cudaMemcpyHostToDevice, st));
  SB_TRY(b->d_round.alloc(ctx, 1));
  SB_CUDA(cudaMemsetAsync(b->d_round.p, 0, 8, st));
  SB_TRY(b->d_stats.alloc(ctx, KN));
  SB_TRY(b->d_bounds.alloc(ctx, KN));
  SB_TRY(b->d_allowed.alloc(ctx, KN * FW));
  SB_TRY(b->d_fmask.alloc(ctx, KN * FW));
  SB_TRY(b->d_allowed_all.alloc(ctx, KN));
  SB_TRY(b->d_built.alloc(ctx, KN));
  SB_TRY(b->d_seg.alloc(ctx, KN));
  SB_TRY(b->d_nsamp.alloc(ctx, KN));
  SB_TRY(b->d_parent.alloc(ctx, KN));
  SB_TRY(b->d_split.alloc(ctx, KN));
  SB_CUDA(cudaMemsetAsync(b->d_split.p, 0, b->d_split.bytes(), st));
  SB_TRY(b->d_leafval.alloc(ctx, KN));
  SB_TRY(b->d_fill.alloc(ctx, KN));
  SB_TRY(b->d_lvl.alloc(ctx, 5 * K));
  SB_TRY(b->d_rows0.alloc(ctx, (size_t)K * b->n));
  SB_TRY(b->d_rows1.alloc(ctx, (size_t)K * b->n));
  SB_TRY(b->d_kept.alloc(ctx, 1));
  SB_CUDA(cudaMemsetAsync(b->d_kept.p, 0, 4, st));
  SB_TRY(b->d_margin.alloc(ctx, b->n * K));
  SB_TRY(b->d_gpair.alloc(ctx, (size_t)K * b->n));
  const bool fixed = p->hist_precision == SB_HIST_FIXED;
  if (fixed) SB_TRY(b->d_gpk.alloc(ctx, (size_t)K * b->n));
  SB_TRY(b->d_maxabs.alloc(ctx, 2 * K));
  SB_CUDA(cudaMemsetAsync(b->d_maxabs.p, 0, 8 * K, st));
  SB_TRY(b->d_shifts.alloc(ctx, 2 * K));
  SB_CUDA(cudaMemsetAsync(b->d_shifts.p, 0, 8 * K, st));
  SB_TRY(b->d_inv_scale.alloc(ctx, 2 * K));
  SB_TRY(b->d_qerr.alloc(ctx, 1));
  SB_CUDA(cudaMemsetAsync(b->d_qerr.p, 0, 8, st));
  const size_t hist_bytes = (size_t)K * b->maxw * HB * 16;
  SB_TRY(b->d_hist0.alloc(ctx, hist_bytes));
  SB_TRY(b->d_hist1.alloc(ctx, hist_bytes));
  SB_TRY(b->d_root_total.alloc(ctx, K));
  SB_TRY(b->d_items.alloc(ctx, (size_t)K * b->maxw + K));
  SB_TRY(b->d_prefix.alloc(ctx, (size_t)K * b->maxw + K + 1));
  SB_TRY(b->d_item_count.alloc(ctx, 1));
  const int ptile_cap = (int)((size_t)K * ((b->n + PART_TILE - 1) / PART_TILE + b->maxn + 1));
  SB_TRY(b->d_ptiles.alloc(ctx, ptile_cap));
  SB_TRY(b->d_ptile_count.alloc(ctx, 1));
  SB_TRY(b->d_pool.alloc(ctx, (size_t)K * F));
  SB_TRY(b->d_pool_len.alloc(ctx, K));
  if (p->colsample_bylevel < 1.0 || p->colsample_bynode < 1.0) SB_TRY(b->d_samp.alloc(ctx, (size_t)1024 * F));
  SB_TRY(b->d_tiles.alloc(ctx, g->tiles.size()));
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
  S.cat_cap = g->has_categorical ? (b->maxn / 2 + 1) * g->max_feature_bins : 0;
  S.n = b->n;
  S.Fp = g->Fp;
  S.bins = g->bins.p;
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
  S.rows0 = b->d_rows0.p;
  S.rows1 = b->d_rows1.p;
  S.kept = b->d_kept.p;
  S.margin = b->d_margin.p;
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
  S.samp_scratch = b->d_samp.p;
  S.row_leaf = nullptr;
  SB_TRY(booster_alloc_trees(b, K * 16));
  return SB_OK;
}

size_t eval_smem(const sb_booster* b) {
  size_t s = (size_t)b->S.F * 8 + (size_t)(b->S.F + 2) * 4 + 64 * 8 + 16;
  if (b->S.cat_cap) s += (EVAL_THREADS / 32) * sizeof(CatScratch);
  return s;
}

int booster_round(sb_booster* b) {
  sb_ctx* ctx = b->ctx;
  BState& S = b->S;
  cudaEvent_t r0 = nullptr, r1 = nullptr;
  if (b->timing) {
    if (!b->d_hist_rows.p) {
      SB_TRY(b->d_hist_rows.alloc(ctx, 1));
      SB_CUDA(cudaMemsetAsync(b->d_hist_rows.p, 0, 8, ctx->stream));
    }
    SB_CUDA(cudaEventCreate(&r0));
    SB_CUDA(cudaEventCreate(&r1));
    SB_CUDA(cudaEventRecord(r0, ctx->stream));
  }
  const unsigned gblocks = (unsigned)std::min<size_t>((b->n + 255) / 256, (size_t)ctx->num_sms * 16);
  SB_LAUNCH(ctx, k_gradient, gblocks, 256, 0, S);
  SB_LAUNCH(ctx, k_round_prep, 1, 32, 0, S);
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
  for (int d = 0; d < b->D; ++d) {
    dim3 eg((unsigned)std::min(1 << d, b->maxw), (unsigned)b->K);
    SB_LAUNCH(ctx, k_eval, eg, EVAL_THREADS, esm, S, d);
    SB_LAUNCH(ctx, k_assign, 1, 1024, 0, S, d, 1);
    unsigned pblocks = (unsigned)ctx->num_sms * 8;
    SB_LAUNCH(ctx, k_partition, pblocks, 256, 0, S, d);
    if (d + 1 < b->D) {
      SB_LAUNCH(ctx, k_plan, 1, 1024, 0, S, d);
      SB_TRY(hist(b->K * (1 << d)));
    }
  }
  SB_LAUNCH(ctx, k_round_end, 1, 32, 0, S);
  if (b->timing) {
    SB_CUDA(cudaEventRecord(r1, ctx->stream));
    b->ev.push_back(r0);
    b->ev.push_back(r1);
    b->ev_kind.push_back(1);
  }
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
  size_t esm = eval_smem(b);
  SB_CUDA(cudaFuncSetAttribute(k_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esm));
  return SB_OK;
}

int booster_export(const sb_booster* b, sb_model* m) {
  sb_ctx* ctx = b->ctx;
  const int ntrees = b->rounds_done * b->K;
  std::vector<int> nn(ntrees), nc(ntrees);
  std::vector<sb_node> nodes((size_t)ntrees * b->maxn);
  std::vector<uint32_t> cats(b->S.cat_cap ? (size_t)ntrees * b->S.cat_cap : 0);
  if (ntrees) {
    SB_CUDA(cudaMemcpyAsync(nn.data(), b->d_out_nnodes.p, ntrees * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(cudaMemcpyAsync(nc.data(), b->d_out_ncats.p, ntrees * 4, cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(cudaMemcpyAsync(nodes.data(), b->d_out_nodes.p, nodes.size() * sizeof(sb_node),
                            cudaMemcpyDeviceToHost, ctx->stream));
    if (!cats.empty())
      SB_CUDA(cudaMemcpyAsync(cats.data(), b->d_out_cats.p, cats.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  }
  SB_CUDA(cudaStreamSynchronize(ctx->stream));
  m->trees.resize(ntrees);
  m->weights.assign(ntrees, 1.0f);
  for (int t = 0; t < ntrees; ++t) {
    m->trees[t].nodes.assign(nodes.begin() + (size_t)t * b->maxn, nodes.begin() + (size_t)t * b->maxn + nn[t]);
    if (!cats.empty())
      m->trees[t].cats.assign(cats.begin() + (size_t)t * b->S.cat_cap,
                              cats.begin() + (size_t)t * b->S.cat_cap + nc[t]);
  }
  m->base_score = b->base_score;
  m->num_class = b->p.num_class;
  m->n_features = (int)b->g->F;
  m->objective = b->p.objective;
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

}  // namespace sb

extern "C" {

int sb_booster_create(sb_ctx* ctx, const sb_ghist* g, const sb_train_params* p, const float* labels,
                      const float* weights, const float* base_margin, sb_booster** out) {
  using namespace sb;
  SB_REQUIRE(ctx && g && p && labels && out, SB_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  SB_TRY(sb_train_params_validate(p));
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
  // base margin, train.rs:203-210 (host: the labels are on the host here)
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
  SB_CUDA(cudaMemcpyAsync(out, b->d_margin.p, b->d_margin.bytes(), cudaMemcpyDeviceToHost, b->ctx->stream));
  SB_CUDA(cudaStreamSynchronize(b->ctx->stream));
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
    delete b;
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

int sb_tree_build(sb_ctx* ctx, const sb_ghist* g, const sb_train_params* p, const sb_gradpair* gpair,
                  size_t n, const uint32_t* rows, size_t m, uint64_t round, uint32_t k,
                  int32_t* row_leaf, sb_model** out) {
  using namespace sb;
  SB_REQUIRE(ctx && g && p && gpair && out, SB_ERR_INVALID_ARG, "NULL argument");
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
  SB_CUDA(cudaMemcpyAsync(b.d_rows0.p, rl.data(), n * 4, cudaMemcpyHostToDevice, st));
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

}  // extern "C"
