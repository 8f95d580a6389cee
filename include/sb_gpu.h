/*
 * sb_gpu.h — C ABI of sequoia-boost-b200: the B200 (sm_100a) backend for
 * sequoia-boost's `tree_method=hist` training and tree-ensemble prediction.
 *
 * Every entry point below stands in for one interface of the reference crate
 * (pgarrett-scripps/sequoia-boost, crates/sequoia-boost/src/…); each cites the
 * file:line it replaces. Plain pointers and sizes only: no CUDA or torch types
 * cross the boundary (device pointers are passed as `void*`/typed pointers
 * where an entry says "device").
 *
 * Conventions
 *  - Every function returns an `int` status: SB_OK (0) or one of SB_ERR_*;
 *    `sb_last_error()` gives a thread-local message for the last failure.
 *    Nothing exits, aborts or traps. (The reference's HistogramBackend is
 *    infallible and panics on misuse, tree/hist/mod.rs:31-45; its crate API
 *    returns Result<_, SequoiaError>, error.rs:6-76.)
 *  - Host buffers are borrowed for the duration of a call and never retained.
 *  - Device memory belongs to opaque handles (sb_ctx, sb_ghist, sb_booster,
 *    sb_model) and is released by the matching *_destroy.
 *  - One CUDA stream per sb_ctx; a context is not re-entrant (the caller
 *    serialises calls on it); distinct contexts are independent.
 *  - There is no CPU fallback: without a usable sm_100 device every compute
 *    entry returns SB_ERR_NO_DEVICE.
 */
#ifndef SB_GPU_H
#define SB_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
  SB_OK = 0,
  SB_ERR_INVALID_ARG = 1,  /* SequoiaError::InvalidParameter */
  SB_ERR_OOM = 2,          /* device allocation failed */
  SB_ERR_CUDA = 3,         /* any other CUDA runtime error */
  SB_ERR_TIMEOUT = 4,      /* a bounded device wait gave up */
  SB_ERR_UNSUPPORTED = 5,  /* valid for the reference, not built here */
  SB_ERR_NO_DEVICE = 6,    /* no CUDA device / wrong architecture */
  SB_ERR_DIMENSION = 7     /* SequoiaError::DimensionMismatch */
};

/* Thread-local text of the last error (never NULL). */
const char* sb_last_error(void);
/* Library version string. */
const char* sb_version(void);

/* ----------------------------------------------------------------- types */
/* GradPair{grad:f32, hess:f32} — objective/mod.rs:31-36 (8 bytes). */
typedef struct sb_gradpair { float grad; float hess; } sb_gradpair;
/* GradStats{grad:f64, hess:f64} — tree/gain.rs:18-23 (16 bytes). */
typedef struct sb_gradstats { double grad; double hess; } sb_gradstats;

/* Node — tree/regtree.rs:17-47. left/right are -1 for a leaf; for a
 * categorical node categories[cat_begin..cat_end) of the owning tree are the
 * category codes routed left. 40 bytes. */
typedef struct sb_node {
  int32_t left;
  int32_t right;
  uint32_t split_feature;
  float split_cond;
  float leaf_value;
  float sum_hess;
  float split_gain;
  uint8_t default_left;
  uint8_t is_categorical;
  uint16_t reserved;
  uint32_t cat_begin;
  uint32_t cat_end;
} sb_node;

enum { SB_FEAT_NUMERICAL = 0, SB_FEAT_CATEGORICAL = 1 }; /* data/meta.rs:8-14 */

enum { /* create_objective, objective/mod.rs:136-161 */
  SB_OBJ_SQUARED_ERROR = 0, /* reg:squarederror | reg:linear */
  SB_OBJ_PSEUDOHUBER = 1,   /* reg:pseudohubererror */
  SB_OBJ_LOGISTIC = 2,      /* binary:logistic | reg:logistic */
  SB_OBJ_SOFTMAX = 3,       /* multi:softmax */
  SB_OBJ_SOFTPROB = 4       /* multi:softprob */
};

enum { SB_GROW_DEPTHWISE = 0, SB_GROW_LOSSGUIDE = 1 }; /* config GrowPolicy */

enum { /* config TreeMethod (params.rs); Auto resolves to hist (train.rs:60-64) */
  SB_TREE_HIST = 0,   /* cuts and bins computed once */
  SB_TREE_APPROX = 1  /* hessian-weighted cuts recomputed every round and class
                         (train.rs:46-53); trains through sb_train only */
};

enum { /* histogram accumulation on the device */
  SB_HIST_FP32 = 0,  /* f32 shared-memory partials, f64 node histograms */
  SB_HIST_FIXED = 1  /* per-round power-of-two int quantised gradients,
                        exact int64 histograms (order independent) */
};

/* TrainingParams fields on the hist path — config/params.rs:76-151, defaults
 * :153-186. 8-byte fields first so the layout has no interior padding. */
typedef struct sb_train_params {
  uint64_t seed;              /* 0 */
  double base_score;          /* used when has_base_score != 0 */
  double eta;                 /* 0.3 */
  double gamma;               /* 0 */
  double min_child_weight;    /* 1 */
  double max_delta_step;      /* 0 */
  double subsample;           /* 1 */
  double colsample_bytree;    /* 1 */
  double colsample_bylevel;   /* 1 */
  double colsample_bynode;    /* 1 */
  double lambda;              /* 1 */
  double alpha;               /* 0 */
  double scale_pos_weight;    /* 1 */
  const int8_t* monotone;     /* n_monotone entries of -1/0/+1, or NULL */
  const uint32_t* interaction_offsets;  /* n_interaction_groups + 1 */
  const uint32_t* interaction_features; /* flattened groups */
  int32_t objective;          /* SB_OBJ_* */
  int32_t num_class;          /* 0 */
  int32_t has_base_score;     /* 0 = estimate from labels */
  int32_t max_depth;          /* 6 (0 = unlimited) */
  int32_t max_leaves;         /* 0 */
  int32_t grow_policy;        /* SB_GROW_* */
  int32_t max_bin;            /* 256 */
  int32_t hist_precision;     /* SB_HIST_*, default SB_HIST_FIXED (deterministic) */
  int32_t quantize_bits;      /* fixed-point magnitude bits, 0 = 16 */
  int32_t n_monotone;
  int32_t n_interaction_groups;
  int32_t tree_method;        /* SB_TREE_*, default SB_TREE_HIST */
} sb_train_params;

/* Fills `p` with the reference defaults (params.rs:153-186). */
void sb_train_params_default(sb_train_params* p);
/* TrainingParams::validate, params.rs:197-261, plus the limits of this
 * backend. SB_OK or SB_ERR_INVALID_ARG / SB_ERR_UNSUPPORTED. */
int sb_train_params_validate(const sb_train_params* p);

/* A read-only view of a tree ensemble (BoostedModel, learner/model.rs:34-54).
 * Tree t owns nodes[tree_node_offset[t] .. tree_node_offset[t+1]) and
 * categories[tree_cat_offset[t] .. tree_cat_offset[t+1]). */
typedef struct sb_model_view {
  const int64_t* tree_node_offset;  /* n_trees + 1 */
  const sb_node* nodes;
  const int64_t* tree_cat_offset;   /* n_trees + 1 */
  const uint32_t* categories;
  const float* tree_weights;        /* n_trees, or NULL for all 1.0 */
  int32_t n_trees;
  int32_t num_class;                /* 0/1 = single output */
  int32_t n_features;
  int32_t objective;                /* SB_OBJ_* for pred_transform */
  float base_score;                 /* margin space */
  int32_t reserved;
} sb_model_view;

/* --------------------------------------------------------------- context */
typedef struct sb_ctx sb_ctx;

/* Opens device `device` (must be sm_100) with its own stream. */
int sb_ctx_create(int device, sb_ctx** out);
int sb_ctx_destroy(sb_ctx* ctx);
int sb_ctx_synchronize(sb_ctx* ctx);
/* The context's cudaStream_t, for event timing by the caller. */
void* sb_ctx_stream(sb_ctx* ctx);
/* Number of kernels this context has launched so far. */
uint64_t sb_ctx_launch_count(const sb_ctx* ctx);

/* ------------------------------------------- binned matrix (cuts + ELLPACK)
 * Replaces HistCuts::from_dmatrix (data/quantile.rs:39-70, with
 * build_feature_cuts :203-245, build_categorical_cuts :187-200,
 * push_max_sentinel :319-323) and GHistIndex::from_dmatrix (data/ghist.rs:
 * :48-82, bin_of quantile.rs:166-181). `X` is a dense row-major f32 matrix;
 * an entry is missing when it is NaN (missing = NaN) or equal to `missing`
 * (data/dmatrix.rs:10-16). `feature_types` may be NULL (all numerical).
 * The device keeps local bins per feature as u16, 0xFFFF = missing. */
typedef struct sb_ghist sb_ghist;

int sb_ghist_create(sb_ctx* ctx, const float* X, size_t n_rows, size_t n_cols,
                    const uint8_t* feature_types, float missing, int max_bin,
                    sb_ghist** out);
/* Same from a device-resident matrix `d_X` (n_rows * n_cols floats). */
int sb_ghist_create_device(sb_ctx* ctx, const float* d_X, size_t n_rows, size_t n_cols,
                           const uint8_t* feature_types, float missing, int max_bin,
                           sb_ghist** out);
int sb_ghist_destroy(sb_ghist* g);
int sb_ghist_info(const sb_ghist* g, size_t* n_rows, size_t* n_cols, size_t* total_bins);
/* HistCuts accessors (quantile.rs:126-163): feature_offset[n_cols+1],
 * cut_values[total_bins], is_categorical[n_cols]. Any pointer may be NULL. */
int sb_ghist_cuts(const sb_ghist* g, uint32_t* feature_offset, float* cut_values,
                  uint8_t* is_categorical);
/* Local bin of every entry, row-major n_rows * n_cols, 0xFFFF = missing. The
 * reference's global bin is feature_offset[f] + local (ghist.rs:48-82). */
int sb_ghist_bins(const sb_ghist* g, uint16_t* local_bins);
/* The device ELLPACK the histogram kernel reads, in the manner of
 * GHistIndex::bins (ghist.rs:117), whose storage is tagged u16/u32: here
 * u8 or u16 row-major codes, n_rows rows of `row_stride` codes.
 * layout: 0 = TILED, 1 = LANES; code_bytes: 1 when the layout is TILED and
 * every feature has at most 255 bins (then feature f's code sits at position
 * f: its local bin, or its bin count when missing), else 2 (tile-relative
 * histogram entries); rows_per_instruction: rows one warp instruction of the
 * histogram kernel covers. Any pointer may be NULL. */
int sb_ghist_layout(const sb_ghist* g, int* layout, int* code_bytes, size_t* row_stride,
                    int* rows_per_instruction);
/* Copies the n_rows * row_stride codes (code_bytes each) to `codes` (host). */
int sb_ghist_codes(const sb_ghist* g, void* codes);

/* HistCuts::from_dmatrix_weighted (data/quantile.rs:81-122, with
 * build_feature_cuts_weighted :253-316) + GHistIndex::from_dmatrix: the cuts
 * and bins tree_method=approx uses in a round, numeric cuts placed at the
 * hessian-weighted quantiles of `hessians` (one per row, finite, >= 0; host). */
int sb_ghist_create_weighted(sb_ctx* ctx, const float* X, size_t n_rows, size_t n_cols,
                             const uint8_t* feature_types, float missing, int max_bin, const float* hessians,
                             sb_ghist** out);

/* -------------------------------------------- HistogramBackend (the seam)
 * trait HistogramBackend::build, tree/hist/mod.rs:31-45 / CpuBackend::build
 * :58-89: out[bin] = sum over rows r and r's bins of (grad_r, hess_r), f64,
 * overwritten, length total_bins. `precision` is SB_HIST_*; with
 * SB_HIST_FIXED the pairs are first quantised with the power-of-two scale of
 * this call's max |grad| / |hess| over the `n` pairs. */
int sb_hist_build(sb_ctx* ctx, const sb_ghist* g, const uint32_t* rows, size_t m,
                  const sb_gradpair* gpair, size_t n, int precision, int quantize_bits,
                  sb_gradstats* out, size_t total_bins);
/* HistogramBackend::subtract, hist/mod.rs:38-44 (and `subtracted` :25-28). */
int sb_hist_subtract(sb_ctx* ctx, const sb_gradstats* parent, const sb_gradstats* child,
                     sb_gradstats* out, size_t total_bins);

/* No counterpart in the reference. The FP32 form of sb_hist_build for callers
 * that cannot let a library allocate device memory, such as a process that
 * hands all free HBM to its own pool allocator at start-up, where any later
 * allocation by a library can fail at an arbitrary time. Inputs and output are
 * the caller's DEVICE buffers: d_rows[m] (row ids below n), d_gpair[n] and
 * d_out[total_bins] (overwritten), on the context's device.
 * Working memory is one static device array of SB_STATIC_SCRATCH_BYTES
 * (8 MiB). It is part of the library's device code, so every device on which
 * the library's kernels are loaded holds those 8 MiB until the process exits,
 * whether or not this entry point is ever called. The `g` index must have been
 * built on the context's device. The node histogram in it takes 16 bytes per bin plus one missing
 * bin per feature, so total_bins + n_cols must stay below about 524,000;
 * a larger index is rejected with SB_ERR_UNSUPPORTED.
 * The first call on a device looks up the array's address
 * (cudaGetSymbolAddress). The call copies small tables from host memory and
 * waits for its result, so it cannot be recorded into a CUDA graph: while the
 * context's stream is being captured it returns SB_ERR_UNSUPPORTED.
 * All calls on a device share the array, and the call clears the histogram
 * part itself: calls that overlap in time (from other threads, or other
 * contexts on the same device) race and must be serialised by the caller.
 * Returns after d_out is written. */
#define SB_STATIC_SCRATCH_BYTES (8u << 20)
int sb_hist_build_static(sb_ctx* ctx, const sb_ghist* g, const uint32_t* d_rows, size_t m,
                         const sb_gradpair* d_gpair, size_t n, sb_gradstats* d_out,
                         size_t total_bins);

/* ------------------------------------------------------------ objectives
 * Objective::gradient, objective/mod.rs:58-69, for the objectives of the hist
 * path: squared error and pseudo-Huber (objective/regression.rs:18-85),
 * logistic with scale_pos_weight (classification.rs:50-71) and softmax
 * (multiclass.rs:64-91). `preds` are margins [n_rows][K] (K = num_class for
 * the multiclass objectives, else 1), `labels` [n_rows], `weights` [n_rows] or
 * NULL; `out` receives GradPair [n_rows][K]. Host buffers. Computed by the
 * same device code as the boosting rounds' gradients. */
int sb_objective_gradient(sb_ctx* ctx, int objective, int num_class, double scale_pos_weight,
                          const float* preds, const float* labels, const float* weights, size_t n_rows,
                          sb_gradpair* out);

/* ---------------------------------------------------- tree / boosting loop */
typedef struct sb_model sb_model;
typedef struct sb_booster sb_booster;

/* HistTreeBuilder::build, tree/builder/hist.rs:139-202: one tree from the
 * binned matrix, `gpair[n]`, and the row subset `rows[m]` (ascending).
 * Column sampling is that of class `k` in round `round` (sb_sampling.h).
 * Leaves are NOT scaled by eta (the builder's contract). `row_leaf`, when not
 * NULL, receives for every row of the subset the node id it ends in (the
 * row-to-node assignment; -1 for rows outside the subset, length n). */
int sb_tree_build(sb_ctx* ctx, const sb_ghist* g, const sb_train_params* p,
                  const sb_gradpair* gpair, size_t n, const uint32_t* rows, size_t m,
                  uint64_t round, uint32_t k, int32_t* row_leaf, sb_model** out);

/* The device-resident boosting state of train_impl (learner/train.rs:183-383)
 * for the hist path: labels/weights/margins live on the device; each update
 * runs whole rounds (gradients, row sampling, one tree per output, margin
 * update) without host round trips. `base_margin` is NULL or n (or n*K)
 * floats (init_margin, train.rs:496-511). Host pointers. */
int sb_booster_create(sb_ctx* ctx, const sb_ghist* g, const sb_train_params* p,
                      const float* labels, const float* weights, const float* base_margin,
                      sb_booster** out);
/* Runs `n_rounds` boosting rounds (the unit of work of one training step). */
int sb_booster_update(sb_booster* b, int n_rounds);
/* Margins [n][K] (host). */
int sb_booster_margins(const sb_booster* b, float* out);
/* Gradient pairs of the last round, class-major [K][n] (host). */
int sb_booster_gradients(const sb_booster* b, sb_gradpair* out);
/* Replaces the booster's margins [n][K] (host buffer) before the next round,
 * which then takes its gradients from them; the last tree's leaf values are
 * not added on top. DART's rounds (train.rs:384-456) take their gradients
 * from the ensemble minus the dropped trees this way. */
int sb_booster_set_margins(sb_booster* b, const float* margins);
/* Rows sampled in round `round` (host, n bytes: 1 = in the subset). */
int sb_booster_row_mask(const sb_booster* b, uint64_t round, uint8_t* out);
/* Copies the trees grown so far into a new model handle. */
int sb_booster_model(const sb_booster* b, sb_model** out);
int sb_booster_destroy(sb_booster* b);

typedef struct sb_booster_stats {
  uint64_t rounds;             /* rounds completed */
  uint64_t hist_launches;      /* histogram-kernel launches (timed ones) */
  double hist_ms;              /* summed device time of those launches */
  double hist_bytes;           /* algorithmic bytes they processed */
  double round_ms;             /* summed device time of timed rounds */
  double quant_err_grad;       /* last round: max |g - deq(q(g))| */
  double quant_err_hess;       /* last round: max |h - deq(q(h))| */
  int32_t quant_shift_grad;    /* last round's power-of-two scale exponents */
  int32_t quant_shift_hess;
} sb_booster_stats;
/* No counterpart in the reference (an engine option). Rounds after the
 * second are recorded once as a CUDA graph and replayed with one launch each
 * (re-recorded when the booster's buffers change); 0 launches every kernel
 * separately. On by default. */
int sb_booster_set_graphs(sb_booster* b, int enable);
/* timing != 0 brackets every histogram launch with CUDA events (adds a
 * little overhead); stats accumulate until reset. */
int sb_booster_set_timing(sb_booster* b, int timing);
int sb_booster_stats_get(const sb_booster* b, sb_booster_stats* out);
int sb_booster_stats_reset(sb_booster* b);

/* train(params, dtrain, num_boost_round), learner/train.rs:107-113 (hist
 * branch): the whole job from host buffers — upload, cuts and binning,
 * `num_boost_round` rounds, model download. */
int sb_train(sb_ctx* ctx, const float* X, size_t n_rows, size_t n_cols,
             const uint8_t* feature_types, float missing, const float* labels,
             const float* weights, const float* base_margin, const sb_train_params* p,
             int num_boost_round, sb_model** out);

/* train() with booster = "dart" (learner/train.rs:384-456, model.rs:130-145):
 * before each round the margins of the ensemble minus that round's dropout
 * set (tree weights, dropped trees at 0) are predicted on the device and the
 * round's K trees grow from their gradients; the new trees get weight
 * 1 / (k + 1) and the k dropped trees are scaled by k / (k + 1), in f32. The
 * dropout set is skipped with probability skip_drop, else each tree drops
 * with probability rate_drop, at least one; its draws come from the
 * SplitMix64 stream of sb_dart_key (include/sb_sampling.h), not rand 0.8.
 * The returned model carries the tree weights. tree_method=hist only. */
int sb_train_dart(sb_ctx* ctx, const float* X, size_t n_rows, size_t n_cols,
                  const uint8_t* feature_types, float missing, const float* labels,
                  const float* weights, const float* base_margin, const sb_train_params* p,
                  double rate_drop, double skip_drop, int num_boost_round, sb_model** out);

/* One job of sb_train_many: the arguments of sb_train, plus its outputs. */
typedef struct sb_job {
  const float* X;               /* [n_rows][n_cols], host */
  size_t n_rows, n_cols;
  const uint8_t* feature_types; /* or NULL */
  float missing;
  const float* labels;
  const float* weights;         /* or NULL */
  const float* base_margin;     /* or NULL */
  const sb_train_params* params;
  int32_t num_boost_round;
  int32_t status;               /* out: SB_OK or the job's error */
  sb_model* out;                /* out: the trained model (destroy with sb_model_destroy) */
} sb_job;

/* No counterpart in the reference (it trains one job per call; cv() runs its
 * folds one after another). Trains independent jobs of any sizes together:
 * each gets its own binned matrix and device booster (set up by up to 8 host
 * threads), spread over n_streams streams (1..64). Depthwise jobs train in
 * batches of similar-size jobs of one precision (up to 8 batches at once, on
 * their own streams): each round of a batch is one launch per kernel step
 * for all its jobs. The others (lossguide, the LANES layout) are issued round
 * r of every job before round r + 1 of any. Each model
 * equals the one sb_train would give for its job. Returns the first failing
 * job's status. */
int sb_train_many(sb_ctx* ctx, sb_job* jobs, size_t n_jobs, int n_streams);

/* ------------------------------------------------------ model / predict */
/* Uploads a host ensemble (BoostedModel) to the device. */
int sb_model_create(sb_ctx* ctx, const sb_model_view* view, sb_model** out);
int sb_model_destroy(sb_model* m);
/* Sizes of the host export arrays. */
int sb_model_export_sizes(const sb_model* m, int32_t* n_trees, int64_t* n_nodes,
                          int64_t* n_categories);
/* Host export: tree_node_offset[n_trees+1], nodes[n_nodes],
 * tree_cat_offset[n_trees+1], categories[n_categories], tree_weights[n_trees].
 * Any pointer may be NULL. base_score / num_class / n_features / objective
 * via sb_model_info. */
int sb_model_export(const sb_model* m, int64_t* tree_node_offset, sb_node* nodes,
                    int64_t* tree_cat_offset, uint32_t* categories, float* tree_weights);
int sb_model_info(const sb_model* m, float* base_score, int32_t* num_class,
                  int32_t* n_features, int32_t* objective);

/* BoostedModel::predict_margin_limited, learner/model.rs:231-285: f32 sum in
 * tree order, tree t adds w_t * leaf to output t % K; `ntree_limit` 0 = all.
 * `base_margin` NULL or n / n*K floats. Host X [n][n_cols], out [n][K]. */
int sb_predict_margin(sb_model* m, const float* X, size_t n_rows, size_t n_cols,
                      float missing, const float* base_margin, size_t ntree_limit,
                      float* out);
/* BoostedModel::predict, model.rs:291-300 (margin then pred_transform). */
int sb_predict(sb_model* m, const float* X, size_t n_rows, size_t n_cols, float missing,
               const float* base_margin, float* out);
/* BoostedModel::predict_contribs, learner/shap.rs:321-367: out
 * [n][K][n_cols+1], bias last. */
int sb_predict_contribs(sb_model* m, const float* X, size_t n_rows, size_t n_cols,
                        float missing, float* out);
/* BoostedModel::predict_leaf, learner/model.rs:330-341: out [n][n_trees]
 * leaf node ids (RegTree::leaf_id_with, regtree.rs:213-242). */
int sb_predict_leaf(sb_model* m, const float* X, size_t n_rows, size_t n_cols, float missing,
                    uint32_t* out);
/* BoostedModel::predict_interactions, learner/shap.rs:395-509: out
 * [n][K][n_cols+1][n_cols+1]; [F][F] holds the sum of the trees' expected
 * values (no base score), the rest of the last row and column is 0. On a
 * B200: up to 239 features (an f32 matrix per row in shared memory). */
int sb_predict_interactions(sb_model* m, const float* X, size_t n_rows, size_t n_cols,
                            float missing, float* out);

/* ------------------------------------------------ eval sets (train.rs) */
/* train_with_eval's eval sets (learner/train.rs:121-140, 243-246, 319-379).
 * sb_booster_eval_add uploads an eval set (X [n][n_cols], labels, optional
 * weights, optional base_margin [n][K]) and starts its margin cache at
 * init_margin (train.rs:240-241). sb_booster_eval adds the rounds grown since
 * the last call into every cache (the same f32 sums as predict_margin) and
 * writes out[e * n_metrics + j], metric j of eval set e, computed on the
 * device after pred_transform (metric/mod.rs:37-262). Early stopping stays
 * with the caller; sb_model_set_best_iteration records its pick. */
enum {
  SB_METRIC_RMSE = 0,     /* Rmse, metric/mod.rs:37-60 */
  SB_METRIC_MAE = 1,      /* Mae, :62-85 */
  SB_METRIC_LOGLOSS = 2,  /* LogLoss, :87-113 */
  SB_METRIC_ERROR = 3,    /* ErrorRate, :115-142 */
  SB_METRIC_MLOGLOSS = 4, /* MLogLoss, :194-226 (multi-output models) */
  SB_METRIC_MERROR = 5    /* MError, :228-262 (multi-output models) */
};
#define SB_EVAL_MAX_METRICS 8
#define SB_EVAL_MAX_CLASSES 64
int sb_booster_eval_add(sb_booster* b, const float* X, size_t n_rows, size_t n_cols, float missing,
                        const float* labels, const float* weights, const float* base_margin,
                        int* eval_id);
int sb_booster_eval(sb_booster* b, int n_metrics, const int* metrics, double* out);
/* The margin cache of one eval set after the rounds grown so far: [n][K]. */
int sb_booster_eval_margins(sb_booster* b, int eval_id, float* out);
/* BoostedModel::set_best_iteration / best_iteration (model.rs:147-149,
 * 209-211); -1 = none. sb_predict then uses (best_iteration + 1) * K trees
 * (model.rs:213-219); sb_predict_margin's ntree_limit and the serving loop
 * are not affected. */
int sb_model_set_best_iteration(sb_model* m, int64_t best_iteration);
int sb_model_best_iteration(const sb_model* m, int64_t* best_iteration);

/* -------------------------------------------------------- serving loop */
/* No counterpart in the reference (it predicts one call at a time). A tree
 * ensemble kept resident in HBM answers margin requests (the output of
 * sb_predict_margin with ntree_limit 0 and no base_margin, [n][K]) and
 * TreeSHAP requests (the output of sb_predict_contribs, [n][K][n_cols+1])
 * from any number of threads, with continuous batching: requests queue in
 * three lanes (margin requests of at most 4096 rows, larger margin requests,
 * TreeSHAP requests); a dispatcher thread joins runs of queued requests of one
 * lane into device batches, admits a batch when its buffers fit in the free
 * part of the loop's memory budget, and keeps up to max(1, n_slots / 2) small
 * margin batches (highest stream priority), max(1, n_slots - n_slots / 2)
 * larger margin batches (middle priority) and max(1, n_slots / 2) TreeSHAP
 * batches (lowest priority) in flight, each on its own stream. Host buffers
 * may be pageable; page-locked X and out make the copies asynchronous. Set
 * CUDA_DEVICE_MAX_CONNECTIONS to at least 1.5 * n_slots + 2 (e.g. 32) in the
 * environment before the process's first CUDA call: with the default 8
 * hardware work queues, streams share queues and a margin batch can wait
 * behind a TreeSHAP kernel of another stream. */
typedef struct sb_server sb_server;
enum { SB_REQ_MARGIN = 0, SB_REQ_CONTRIBS = 1 };
typedef struct sb_server_stats {
  uint64_t submitted, completed, failed;
  uint64_t batches, rows;        /* device batches launched and their rows */
  uint64_t max_batch_requests;   /* most requests joined into one batch */
  uint64_t memory_waits;         /* times the queue head waited for memory */
  uint64_t mem_bytes, mem_peak;  /* budget and the most of it in use */
} sb_server_stats;
/* mem_bytes: device memory for request buffers (0 = half of what is free
 * now); n_slots: margin batches in flight over both margin lanes (1..64). The
 * model must outlive the loop. */
int sb_server_create(sb_ctx* ctx, sb_model* m, size_t mem_bytes, int n_slots, sb_server** out);
/* Queues a request; X [n_rows][n_cols] and out stay owned by the caller and
 * must stay valid until sb_server_wait returns for the ticket. */
int sb_server_submit(sb_server* s, int kind, const float* X, size_t n_rows, size_t n_cols,
                     float missing, float* out, uint64_t* ticket);
/* Blocks until the request is done (timeout_ms < 0: no limit); returns its
 * status (SB_ERR_OOM when it can never fit the budget, SB_ERR_TIMEOUT when
 * the wait ran out) and its submit-to-done latency. Each ticket is waited once. */
int sb_server_wait(sb_server* s, uint64_t ticket, int timeout_ms, double* latency_ms);
int sb_server_stats_get(sb_server* s, sb_server_stats* out);
/* Finishes every queued request, then stops the loop. */
int sb_server_destroy(sb_server* s);

#ifdef __cplusplus
}
#endif

#endif /* SB_GPU_H */
