// sb_internal.cuh — shared declarations of the sequoia-boost-b200 library.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "../../include/sb_gpu.h"
#include "../../include/sb_sampling.h"

namespace sb {

void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what, const char* file, int line);

}  // namespace sb

#define SB_CUDA(call)                                                      \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) return sb::cuda_status(e_, #call, __FILE__, __LINE__); \
  } while (0)

#define SB_TRY(expr)              \
  do {                            \
    int s_ = (expr);              \
    if (s_ != SB_OK) return s_;   \
  } while (0)

#define SB_REQUIRE(cond, code, ...)   \
  do {                                \
    if (!(cond)) {                    \
      sb::set_error(__VA_ARGS__);     \
      return (code);                  \
    }                                 \
  } while (0)

// Launch on the context stream, count it, and surface launch errors.
#define SB_LAUNCH(ctx, kern, grid, block, smem, ...)                        \
  do {                                                                      \
    kern<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);          \
    (ctx)->launches++;                                                      \
    SB_CUDA(cudaGetLastError());                                            \
  } while (0)

// The same on another stream of the context's device.
#define SB_LAUNCH_ON(ctx, st, kern, grid, block, smem, ...)                 \
  do {                                                                      \
    kern<<<(grid), (block), (smem), (st)>>>(__VA_ARGS__);                   \
    (ctx)->launches++;                                                      \
    SB_CUDA(cudaGetLastError());                                            \
  } while (0)

struct sb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  size_t smem_optin = 0;     // max dynamic shared memory per block
  size_t smem_per_sm = 0;
  std::atomic<uint64_t> launches{0};  // also counted by serving threads
};

namespace sb {

// Stream-ordered device allocation (pool-backed, cached across calls).
int dalloc(sb_ctx* ctx, void** p, size_t bytes);
// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`; never lowers it (another index, booster or model of the
// process may launch the same kernel with more).
int raise_smem_limit(const void* func, size_t bytes);
void dfree(sb_ctx* ctx, void* p);

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  sb_ctx* ctx = nullptr;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  int alloc(sb_ctx* c, size_t count) {
    release();
    ctx = c;
    n = count;
    if (count == 0) return SB_OK;
    return dalloc(c, (void**)&p, count * sizeof(T));
  }
  // alloc, then zero on the context stream (state that is read before every
  // path has written it then starts from zeros, not from the pool's leftovers)
  int alloc_zero(sb_ctx* c, size_t count) {
    int s = alloc(c, count);
    if (s != SB_OK || count == 0) return s;
    cudaError_t e = cudaMemsetAsync(p, 0, count * sizeof(T), c->stream);
    return e == cudaSuccess ? SB_OK : cuda_status(e, "cudaMemsetAsync", __FILE__, __LINE__);
  }
  void release() {
    if (p && ctx) dfree(ctx, p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// ----------------------------------------------------------------- data
constexpr uint16_t MISSING_BIN = 0xFFFF;
constexpr int MAX_CAT_BINS = 256;      // categorical features: <= 256 categories
constexpr uint32_t UNSAMPLED = 0x80000000u;  // row-list flag: not in the subset

// Layouts of the row-major bin codes that the histogram kernel reads.
//  TILED: row r holds feature f's code at position f (row stride Fp =
//         round_up(F, 8)); the code is the entry's index in its feature tile's
//         shared-memory partial, which holds the tile's bins in global order.
//         With u8 codes (every feature at most 255 bins) the code is the
//         feature's local bin, or its bin count when missing, and the partial
//         holds each feature's bins followed by its missing entry.
//  LANES: each tile gives each of the 32 lanes of a warp `slots` code
//         positions (row stride Fp = tiles * 32 * slots); lane l owns the
//         features placed in its slots, and the code is the entry's index e
//         in lane l's own column of the partial, stored at word e * 32 + l,
//         so the 32 lanes of a warp always add into 32 different banks.
enum { HIST_LAYOUT_TILED = 0, HIST_LAYOUT_LANES = 1 };

// A feature tile of the histogram: features [f0, f1), whose entries fit in the
// shared-memory partial of one CTA.
struct FeatureTile {
  int f0, f1;
  int bin0;       // foff[f0]
  int nbins;      // foff[f1] - foff[f0]
  int E;          // LANES: entries per lane (the partial has 32 * E words per plane)
  int ent_off;    // LANES, u8 TILED: offset of the tile's entry -> histogram-bin table
  int slot_off;   // LANES: position of the tile's first code in a row
  int reserved;
};

struct Ghist {  // sb_ghist
  sb_ctx* ctx = nullptr;
  size_t n = 0, F = 0, Fp = 0;   // Fp: row stride of the row-major codes, in codes
  size_t total_bins = 0;
  int max_bin = 0;
  float missing = NAN;
  int max_feature_bins = 0;
  int has_categorical = 0;
  int layout = HIST_LAYOUT_TILED;  // HIST_LAYOUT_*
  int slots = 0;                   // LANES: code positions per lane and tile
  int tiled_rl = 0;                // TILED: log2 of the rows one warp instruction covers
  // Bytes per row-major code: 1 (u8) when the layout is TILED and every
  // feature's bins and its missing entry fit a byte (at most 255 bins), else 2.
  int code_bytes = 2;
  // [n][Fp] bin codes of the histogram kernel: feature f of row r at
  // r * Fp + rpos[f], code = rbase[f] + local bin, or rmiss[f] for a missing
  // entry; unused positions hold 0xFFFF (0xFF). `bins` holds u16 codes,
  // `bins8` u8 codes (rbase 0, rmiss the feature's bin count); only the one
  // of `code_bytes` is allocated.
  DBuf<uint16_t> bins;
  DBuf<uint8_t> bins8;
  std::vector<int> h_rpos, h_rbase, h_rmiss;
  DBuf<int> rpos, rbase, rmiss;  // device copies of h_rpos, h_rbase, h_rmiss
  DBuf<int> ent_gbin;      // LANES: per tile, [E][32] histogram bin of each (entry, lane), -1 unused;
                           // u8 TILED: per tile, the histogram bin of each shared entry
  DBuf<int> slot_feat;     // LANES: [Fp] feature of each code position, -1 unused
  // [F][n] local bins, feature-major, MISSING_BIN for a missing entry (the
  // partition reads them): code = fbase[f] + local, fmiss[f] when missing
  DBuf<uint16_t> bins_col;
  DBuf<int> fbase;         // [F] 0
  DBuf<int> fmiss;         // [F] MISSING_BIN
  DBuf<uint32_t> foff;     // [F+1]
  DBuf<float> cuts;        // [total_bins]
  DBuf<uint8_t> is_cat;    // [F]
  std::vector<uint32_t> h_foff;
  std::vector<float> h_cuts;
  std::vector<uint8_t> h_is_cat;
  std::vector<FeatureTile> tiles;  // histogram feature tiles
  size_t hist_smem_bytes = 0;      // shared memory of the largest tile
};

// A binned matrix lives on the device of the context that built it; an entry
// point given a context of another device rejects it before any launch.
#define SB_SAME_DEVICE(ctx, g)                                                              \
  SB_REQUIRE((g)->ctx && (g)->ctx->device == (ctx)->device, SB_ERR_INVALID_ARG,            \
             "the binned matrix is on device %d, the context on device %d",                 \
             (g)->ctx ? (g)->ctx->device : -1, (ctx)->device)

int ghist_build(sb_ctx* ctx, const float* d_X, size_t n, size_t F, const uint8_t* h_ftypes,
                float missing, int max_bin, Ghist* g);
// The index's device cuts, histogram layout and bin codes from its host cuts
// (h_foff, h_cuts, h_is_cat; n, F, missing and max_bin set).
int ghist_bin(sb_ctx* ctx, const float* d_X, Ghist* g);

// tree_method=approx (sb_approx.cu): a matrix's columns sorted once, then
// hessian-weighted cuts (HistCuts::from_dmatrix_weighted) for any hessians.
struct ApproxState;
ApproxState* approx_state_new();
void approx_state_free(ApproxState* a);
int approx_prepare(sb_ctx* ctx, const float* d_X, size_t n, size_t F, const uint8_t* h_ftypes, float missing,
                   int max_bin, ApproxState* A);
// host cuts into g (h_foff, h_cuts, h_is_cat) for device hessians d_hess[n] >= 0
int approx_cuts(ApproxState* A, const float* d_hess, Ghist* g);

// ------------------------------------------------------------ histograms
// One node histogram to accumulate: rows[begin..end) of a row list.
struct HistItem {
  const uint32_t* rows;  // row list (the round's sampled rows)
  uint32_t begin, end;
  uint32_t k;            // class (gradient column)
  uint32_t root;         // 1: also accumulate the node total
  void* out;             // HB entries of 16 B (double2 or longlong2)
  void* total;           // double2* / longlong2* when root
};

struct HistLaunch {
  const Ghist* g;
  const void* gpair;     // FP32: float2 [K][n]; FIXED: uint64 packed [K][n]
  int fixed;
  int quant_bits;
  const HistItem* items; // device
  const uint64_t* prefix;  // device, exclusive prefix of item lengths, [count+1]
  const int* count;      // device: number of items
  int max_items;
  const FeatureTile* tiles;  // device
  int ntiles;
  unsigned long long* rows_done;  // device counter of sampled rows, or null
  const uint32_t* pool_mask;      // device [K][ceil(F/32)]: features to accumulate, or null
  size_t rows_bound = 0;          // most rows one launch accumulates (0: unknown, full grid)
  uint32_t min_units = 0;         // fewest (row, tile) units per active CTA (0: every CTA works)
};

// Zeroing of one job's node histograms in a batched launch.
struct ZeroJob {
  const HistItem* items;
  const int* count;
  size_t words;  // 64-bit words per node histogram
};

// Device tables of histogram launches over many jobs (sb_train_many): job j
// is described by Ls[j] (TILED layout; all FIXED or all FP32). Built once per
// batch by hist_jobs_prepare and kept alive while its launches run. A launch
// gives job j hist_grid[j] (zero_grid[j]) blocks, or none when the job builds
// nothing at that step: the caller's offset tables say which.
struct HistJobsPlan {
  DBuf<char> devs;     // the jobs' launch descriptions
  DBuf<ZeroJob> zero;  // [njobs]
  std::vector<unsigned> hist_grid, zero_grid;
  int njobs = 0;
  int fixed = 0;
  int rl = 0;  // rows per warp instruction (log2), the same for every job
  bool u8 = false;  // one-byte codes, the same for every job
  size_t smem = 0;
};
int hist_jobs_prepare(sb_ctx* ctx, const std::vector<HistLaunch>& Ls, HistJobsPlan* P);
// Zeroes the jobs' current node histograms and builds them: one launch each.
// d_xoff / d_zoff: [njobs + 1] block offsets of the two launches.
int launch_hist_jobs(sb_ctx* ctx, const HistJobsPlan& P, const unsigned* d_xoff, unsigned hist_blocks,
                     const unsigned* d_zoff, unsigned zero_blocks, int max_items);

// One layout of the histogram's bin codes (HIST_LAYOUT_*; LANES: positions
// per lane and tile, 1, 2 or 4).
struct HistChoice {
  int layout;
  int slots;
  int rl = -1;  // TILED: rows per warp instruction (log2); -1: by the feature count
};
int hist_prepare(sb_ctx* ctx, Ghist* g, HistChoice c);
int hist_default_choice(sb_ctx* ctx, Ghist* g, HistChoice* out);
std::vector<HistChoice> hist_candidates(sb_ctx* ctx, Ghist* g);
int hist_time(sb_ctx* ctx, const Ghist* g, float* ms);
int launch_hist(sb_ctx* ctx, const HistLaunch& L);
int launch_zero_items(sb_ctx* ctx, const Ghist* g, const HistItem* items, const int* count,
                      int max_items);
int hist_grid(sb_ctx* ctx, const Ghist* g, size_t rows_bound);
// Depthwise boosters that can share batched round launches (no lossguide,
// external gradients, timing, eval sets or row -> leaf output; TILED index).
bool booster_batchable(const sb_booster* b);
// `rounds` rounds of nb batchable boosters of one precision, on ctx's stream:
// one launch per kernel step over all of them, recorded once as a graph.
int boosters_train_batched(sb_ctx* ctx, sb_booster* const* bs, int nb, int rounds);
// rounds[j] rounds of each of nb boosters: the batchable ones in batches
// (one launch per kernel step for a batch) of similar-size jobs, up to nctx
// batches at once on the streams of ctxs; the others one round at a time in
// turn on their own streams. status[j] gets each job's result (entries not
// SB_OK on entry are skipped).
int boosters_train_many(sb_ctx* const* ctxs, int nctx, sb_booster* const* bs, const int* rounds, int nb,
                        int* status);

// ----------------------------------------------------------------- model
struct HostTree {
  std::vector<sb_node> nodes;
  std::vector<uint32_t> cats;
};

// One element of a root-to-leaf path for TreeSHAP: every split on the path
// that tests feature f, merged. A row follows the element when its value lies
// in [lo, hi), or when it is missing and every such split sends missing
// values the path's way. z = the product of the splits' cover fractions.
struct PathEl {
  int f;        // -1 for the path's first (bias) element
  int miss_ok;
  float lo, hi;
  double z, inv_z;
};

struct DevEnsemble {
  DBuf<int4> nodes;          // packed predict nodes
  DBuf<int> cat_end;         // per node: end of its category list
  DBuf<int64_t> tree_off;    // node offset per tree
  DBuf<uint32_t> cats;
  DBuf<float> weights;
  DBuf<double> tree_mean;
  // TreeSHAP: the root-to-leaf paths of every tree
  DBuf<PathEl> path_el;      // elements, path after path
  DBuf<int> path_off;        // [n_paths + 1] element offsets
  DBuf<float> path_leaf;     // [n_paths] leaf values
  DBuf<int> tree_path;       // [n_trees + 1] first path of each tree
  DBuf<int4> shap_chunk;     // {class, first path, end path, -} work units of TreeSHAP blocks
  int n_shap_chunks = 0;
  DBuf<int> path_fc;         // per element: its feature's index in its chunk's feature list (-1: bias)
  DBuf<int> chunk_fo;        // [n_shap_chunks + 1] offsets into chunk_f
  DBuf<int> chunk_f;         // the distinct features of each chunk's paths
  int shap_max_fc = 1;       // most distinct features in one chunk
  bool shap_valid = false;   // the TreeSHAP state above has been built (shap_prepare)
  bool shap_table = false;   // per-path contribution tables are in use
  DBuf<float> shap_tab;      // per path: [2^D][round_up(D, 4)] f32 contributions
  DBuf<long long> shap_tab_off;  // [n_paths] first float of each path's table
  DBuf<int4> tab_el;         // per element: {feature, lo, hi, (table-chunk feature index << 1) | miss_ok}
  DBuf<int4> tab_head;       // per path: {first element, elements, table offset low, high 32 bits}
  DBuf<int4> tab_chunk;      // {class, first tree, trees, -}: work units of the table kernel
  DBuf<int> tab_chunk_fo;    // [n_tab_chunks + 1] offsets into tab_chunk_f
  DBuf<int> tab_chunk_f;     // each table chunk's distinct features
  int n_tab_chunks = 0;
  int tab_max_fc = 1;
  int n_trees = 0;
  int max_depth = 0;
  int max_path_len = 0;      // elements, bias included
};

}  // namespace sb

struct sb_ghist : sb::Ghist {};

struct sb_model {
  sb_ctx* ctx = nullptr;
  std::vector<sb::HostTree> trees;
  std::vector<float> weights;
  float base_score = 0.0f;
  int num_class = 0;
  int n_features = 0;
  int objective = 0;
  int64_t best_iteration = -1;  // early stopping's pick (-1: none), model.rs:41
  bool dev_valid = false;
  sb::DevEnsemble dev;
};

namespace sb {

int n_outputs(int objective, int num_class);
int model_upload(sb_model* m);
int tree_depth(const HostTree& t);
double node_mean_value(const HostTree& t, int id);  // learner/shap.rs:288-302
// TreeSHAP (sb_shap.cu): the model's path data and tables, built once
int shap_prepare(sb_model* m);
// Margins of n device rows into d_out ([n][K]): base score, or the
// per-row base margins d_base_margin ([n][K] when bm_kind == 1, [n] when 2),
// plus the weighted leaf values of the first ntree_limit trees (0: all).
int predict_margin_device(sb_model* m, const float* d_X, size_t n, size_t F, float missing,
                          const float* d_base_margin, int bm_kind, size_t ntree_limit, float* d_out);
int predict_contribs_device(sb_model* m, const float* d_X, size_t n, size_t F, float missing, float* d_out);
int predict_interactions_device(sb_model* m, const float* d_X, size_t n, size_t F, float missing,
                                float* d_out);

// The trees a booster has grown so far, as they sit on the device: tree
// t = round * K + class at nodes[t * maxn ..], its categories at
// cats[t * cat_cap ..] (leaf values already scaled by eta).
struct BoosterTrees {
  sb_ctx* ctx;
  const sb_node* nodes;
  const uint32_t* cats;  // null when no tree can hold categorical splits
  int maxn, cat_cap, K, rounds_done;
  float base_score;      // margin space
  int objective, num_class;
  size_t n_features;
};

// An eval set attached to a booster (train_impl's `evals`, train.rs:243-246):
// its rows, labels, weights and incremental margin cache stay on the device.
struct EvalSet {
  DBuf<float> X, labels, weights, margin, preds;
  size_t n = 0;
  float missing = NAN;
  int rounds_in_margin = 0;  // rounds already added into `margin`
};

int booster_trees(const sb_booster* b, BoosterTrees* v);
std::vector<std::unique_ptr<EvalSet>>& booster_evals(sb_booster* b);

// ---------------------------------------------------- FP64 split math
// Written with explicit round-to-nearest intrinsics so that no FMA
// contraction changes a result bit: the fixed-point path reproduces the CPU
// oracle's gains exactly. Formulas: tree/gain.rs:78-126 and
// tree/constraints.rs:70-134.
struct RegP {
  double lambda, alpha, mds, mcw;
};

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ double threshold_l1(double g, double a) {
  if (g > a) return dsub(g, a);
  if (g < -a) return dadd(g, a);
  return 0.0;
}
__device__ __forceinline__ double clampd(double x, double lo, double hi) {
  if (x < lo) x = lo;
  if (x > hi) x = hi;
  return x;
}
__device__ __forceinline__ double calc_weight(double g, double h, const RegP& r) {
  if (h < r.mcw || h <= 0.0) return 0.0;
  double w = ddiv(-threshold_l1(g, r.alpha), dadd(h, r.lambda));
  if (r.mds > 0.0) w = clampd(w, -r.mds, r.mds);
  return w;
}
__device__ __forceinline__ double calc_gain(double g, double h, const RegP& r) {
  if (h < r.mcw || h <= 0.0) return 0.0;
  double t = threshold_l1(g, r.alpha);
  if (r.mds == 0.0) return ddiv(dmul(t, t), dadd(h, r.lambda));
  double w = calc_weight(g, h, r);
  return -dadd(dmul(dmul(2.0, t), w), dmul(dmul(dadd(h, r.lambda), w), w));
}
__device__ __forceinline__ double calc_weight_bounded(double g, double h, const RegP& r, double lo,
                                                      double hi) {
  if (h < r.mcw || h <= 0.0) return clampd(0.0, lo, hi);
  double w = ddiv(-threshold_l1(g, r.alpha), dadd(h, r.lambda));
  if (r.mds > 0.0) w = clampd(w, -r.mds, r.mds);
  return clampd(w, lo, hi);
}
__device__ __forceinline__ double gain_at_weight(double g, double h, const RegP& r, double w) {
  if (h < r.mcw || h <= 0.0) return 0.0;
  double t = threshold_l1(g, r.alpha);
  return -dadd(dmul(dmul(2.0, t), w), dmul(dmul(dadd(h, r.lambda), w), w));
}
__device__ __forceinline__ bool satisfies(int dir, double wl, double wr) {
  if (dir > 0) return wl <= wr;
  if (dir < 0) return wl >= wr;
  return true;
}
__device__ __forceinline__ long long total_cmp_key(double x) {
  long long b = __double_as_longlong(x);
  b ^= (long long)(((unsigned long long)(b >> 63)) >> 1);
  return b;
}

// Rust `f32 as u32`: saturating, NaN -> 0.
__host__ __device__ __forceinline__ uint32_t f32_as_u32(float v) {
  if (!(v > 0.0f)) return 0u;
  if (v >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)v;
}

// Objective::pred_transform over one row of K margins, in place: the
// logistic sigmoid (classification.rs:73-77) or the softmax
// (multiclass.rs:93-99), in f32 with explicit rounding; the identity for the
// regression objectives.
__device__ __forceinline__ void pred_transform_row(float* row, int K, int objective) {
  if (objective == SB_OBJ_LOGISTIC) {
    const float x = row[0];
    float p;
    if (x >= 0.0f) p = __fdiv_rn(1.0f, __fadd_rn(1.0f, expf(-x)));
    else {
      const float e = expf(x);
      p = __fdiv_rn(e, __fadd_rn(1.0f, e));
    }
    row[0] = p;
  } else if ((objective == SB_OBJ_SOFTMAX || objective == SB_OBJ_SOFTPROB) && K > 1) {
    float mx = -INFINITY;
    for (int c = 0; c < K; ++c)
      if (row[c] > mx) mx = row[c];
    float sum = 0.0f;
    for (int c = 0; c < K; ++c) {
      row[c] = expf(__fsub_rn(row[c], mx));
      sum = __fadd_rn(sum, row[c]);
    }
    const float inv = __fdiv_rn(1.0f, sum);
    for (int c = 0; c < K; ++c) row[c] = __fmul_rn(row[c], inv);
  }
}

// Power-of-two exponent of the fixed-point scale: q = rint(x * 2^s) keeps
// |q| <= 2^bits for |x| <= m.
__host__ __device__ __forceinline__ int quant_shift(float m, int bits) {
  if (!(m > 0.0f) || !(m < INFINITY)) return 0;
  int e = ilogbf(m);
  int s = (bits - 1) - e;
  if (s > 100) s = 100;
  if (s < -100) s = -100;
  return s;
}

// Rows a CTA may fold into its packed 32+32-bit partial before flushing.
__host__ __device__ __forceinline__ uint32_t fixed_rows_per_flush(int bits) {
  return (uint32_t)((0x7FFFFFFFull >> bits) - 1ull);
}

}  // namespace sb
