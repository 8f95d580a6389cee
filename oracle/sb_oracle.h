/*
 * sb_oracle.h — TEST INFRASTRUCTURE ONLY. Not part of the product.
 *
 * C ABI of the CPU oracle: a C++ restatement of the reference's CPU
 * `tree_method=hist` path (pgarrett-scripps/sequoia-boost, crates/
 * sequoia-boost/src/…). Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference legs may load it, and only as the checker or the
 * timed CPU baseline — never as a compute path of the product.
 *
 * Parity status: the reference is Rust and cannot be compiled here (no Rust
 * toolchain in this image or on the GPU hosts), so the oracle could not be
 * diffed against the reference binary. It is pinned instead against every
 * known-answer test and invariant the reference's own unit tests hold for
 * this path (tests/golden/reference_kats.json, generated by
 * tests/golden/make_reference_kats.py from those tests). The reference's
 * random streams (rand 0.8 StdRng, not vendored) are unpinned: sampling
 * follows include/sb_sampling.h on both sides instead.
 */
#ifndef SB_ORACLE_H
#define SB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/sb_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_data orc_data;
typedef struct orc_model orc_model;

/* HistCuts::from_dmatrix + GHistIndex::from_dmatrix (dense X). NULL on error
 * (e.g. NaN values with a non-NaN missing sentinel, where the reference's
 * sort would panic). */
orc_data* orc_data_create(const float* X, size_t n, size_t F, const uint8_t* ftypes,
                          float missing, int max_bin);
/* HistCuts::from_dmatrix_weighted (data/quantile.rs:81-122, cuts of
 * tree_method=approx, weighted by one hessian per row) + GHistIndex. */
orc_data* orc_data_create_weighted(const float* X, size_t n, size_t F, const uint8_t* ftypes, float missing,
                                   int max_bin, const float* hessians);
void orc_data_destroy(orc_data* d);
size_t orc_data_total_bins(const orc_data* d);
int orc_data_is_dense(const orc_data* d);
void orc_data_cuts(const orc_data* d, uint32_t* off, float* vals, uint8_t* is_cat);
/* Global bin of every entry (n*F), UINT32_MAX for missing. */
void orc_data_dense_bins(const orc_data* d, uint32_t* out);
/* HistCuts::bin_of for one value. */
uint32_t orc_bin_of(const orc_data* d, size_t f, float v);

/* CpuBackend::build with `threads` workers (1 = sequential accumulate). */
void orc_hist_build(const orc_data* d, const uint32_t* rows, size_t m,
                    const sb_gradpair* gpair, sb_gradstats* out, int threads);

/* HistTreeBuilder::build: one tree (leaves not scaled by eta). */
orc_model* orc_tree_build(const orc_data* d, const sb_train_params* p,
                          const sb_gradpair* gpair, const uint32_t* rows, size_t m,
                          uint64_t round, uint32_t k, int threads);

/* train(): the hist branch of train_impl. `margins_out` (n*K) and
 * `metric_out` (per round train metric of the objective's default metric)
 * may be NULL. With p->hist_precision == SB_HIST_FIXED each class tree is
 * grown from the gradients rounded as the GPU's fixed-point form rounds them
 * (orc_quantize); with SB_HIST_FP32 from the plain f32 gradients. */
orc_model* orc_train(const orc_data* d, const float* X, const sb_train_params* p,
                     const float* labels, const float* weights, const float* base_margin,
                     int rounds, int threads, float* margins_out, double* metric_out);
/* dart_round (learner/train.rs:384-456): DART training with the dropout
 * draws of sb_dart_key's stream; tree weights via orc_model_export. */
orc_model* orc_train_dart(const orc_data* d, const float* X, const sb_train_params* p, double rate_drop,
                          double skip_drop, const float* labels, const float* weights, const float* base_margin,
                          int rounds, int threads, float* margins_out);

void orc_model_destroy(orc_model* m);
void orc_model_sizes(const orc_model* m, int32_t* n_trees, int64_t* n_nodes, int64_t* n_cats);
void orc_model_export(const orc_model* m, int64_t* node_off, sb_node* nodes, int64_t* cat_off,
                      uint32_t* cats, float* weights, float* base_score);
/* Per node: best gain minus the best gain of any other candidate (the
 * runner-up); +inf for leaves and nodes with a single candidate. */
void orc_model_node_gaps(const orc_model* m, double* out);

int orc_predict_margin(const sb_model_view* v, const float* X, size_t n, size_t F,
                       float missing, const float* base_margin, size_t ntree_limit, float* out);
int orc_predict_contribs(const sb_model_view* v, const float* X, size_t n, size_t F,
                         float missing, float* out);
/* predict_leaf (learner/model.rs:330-341): out [n][n_trees] leaf node ids. */
int orc_predict_leaf(const sb_model_view* v, const float* X, size_t n, size_t F, float missing,
                     uint32_t* out);
/* predict_interactions (learner/shap.rs:395-509): out [n][K][F+1][F+1]. */
int orc_predict_interactions(const sb_model_view* v, const float* X, size_t n, size_t F,
                             float missing, float* out);
/* Objective::gradient over margins [n][K] -> out [n][K]. */
void orc_gradient(int objective, int num_class, double scale_pos_weight, const float* preds,
                  const float* labels, const float* weights, size_t n, sb_gradpair* out);
/* Objective::pred_transform in place over [n][K]. */
void orc_pred_transform(int objective, int num_class, float* preds, size_t n);
/* Metrics: 0 rmse, 1 logloss, 2 mlogloss (preds already transformed). */
double orc_metric(int kind, const float* preds, const float* labels, const float* weights,
                  size_t n, int num_class);
/* The base margin train_impl starts from (train.rs:203-210). */
float orc_base_margin(const sb_train_params* p, const float* labels, const float* weights,
                      size_t n);
/* Fixed-point rounding of the GPU path: q = rint(x * 2^s), out = q * 2^-s,
 * with s = (bits-1) - floor(log2(max |x|)) per component. */
void orc_quantize(const sb_gradpair* in, size_t n, int bits, sb_gradpair* out, int* shift_g,
                  int* shift_h);
/* Column subset of node `nid` of class `k` in round `round` (make_sampler +
 * ColumnSampler::sample over sb_sampling.h keys). Returns its length. */
int orc_sample_features(size_t F, const sb_train_params* p, uint64_t round, uint32_t k,
                        uint64_t nid, uint32_t* out);
/* Bernoulli row subset of a round (sample_rows). Returns its length. */
size_t orc_sample_rows(size_t n, const sb_train_params* p, uint64_t round, uint32_t* out);
/* TrainingParams::validate. 0 = ok. */
int orc_validate(const sb_train_params* p);

#ifdef __cplusplus
}
#endif

#endif
