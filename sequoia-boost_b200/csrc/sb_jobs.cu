// sb_jobs.cu — sb_train_many: many independent training jobs (k-fold splits,
// parameter sweeps) of uneven sizes trained together on one GPU.
//
// Each job gets its own binned matrix and device booster (train(), learner/
// train.rs:107-113, per job), set up by a few host threads at once, jobs
// spread round-robin over a pool of streams. Depthwise jobs of one precision
// and one row grouping then train in batches: every round of a batch is one
// launch per kernel step for all its jobs (their grids laid end to end, each
// block running its job's state), recorded once as a CUDA graph and
// replayed. Jobs are sorted by size into up to 8 batches of similar jobs that
// run at once on their own streams. The jobs that cannot share launches
// (lossguide, eval sets, the LANES layout) are issued round r of every job
// before round r + 1 of any over the pool.
#include <algorithm>
#include <thread>
#include <vector>

#include "sb_internal.cuh"

extern "C" {

int sb_train_many(sb_ctx* ctx, sb_job* jobs, size_t n_jobs, int n_streams) {
  using namespace sb;
  SB_REQUIRE(ctx && (jobs || n_jobs == 0), SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_streams >= 1 && n_streams <= 64, SB_ERR_INVALID_ARG, "n_streams must be in [1, 64]");
  for (size_t j = 0; j < n_jobs; ++j) {
    jobs[j].out = nullptr;
    jobs[j].status = SB_OK;
    SB_REQUIRE(jobs[j].X && jobs[j].labels && jobs[j].params, SB_ERR_INVALID_ARG, "job %zu: NULL argument", j);
    SB_REQUIRE(jobs[j].num_boost_round >= 0, SB_ERR_INVALID_ARG, "job %zu: negative num_boost_round", j);
  }
  SB_CUDA(cudaSetDevice(ctx->device));
  const int S = (int)std::min<size_t>((size_t)n_streams, std::max<size_t>(n_jobs, 1));
  std::vector<sb_ctx*> sctx(S, nullptr);
  std::vector<sb_ghist*> gh(n_jobs, nullptr);
  std::vector<sb_booster*> bo(n_jobs, nullptr);
  int rc = SB_OK;
  for (int s = 0; s < S && rc == SB_OK; ++s) rc = sb_ctx_create(ctx->device, &sctx[s]);
  // set-up: bin each job's matrix and create its booster on its stream.
  // Binning waits for its cuts on the host, so host threads set up jobs in
  // parallel: thread t takes the streams s with s % T == t (a stream's jobs
  // stay on one thread).
  if (rc == SB_OK) {
    const int T = std::max(1, std::min(S, (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency()))));
    auto setup = [&](int t) {
      cudaSetDevice(ctx->device);
      for (size_t j = 0; j < n_jobs; ++j) {
        if ((int)(j % S) % T != t) continue;
        sb_job& jb = jobs[j];
        sb_ctx* c = sctx[j % S];
        int s = sb_train_params_validate(jb.params);
        if (s == SB_OK)
          s = sb_ghist_create(c, jb.X, jb.n_rows, jb.n_cols, jb.feature_types, jb.missing, jb.params->max_bin,
                              &gh[j]);
        if (s == SB_OK) s = sb_booster_create(c, gh[j], jb.params, jb.labels, jb.weights, jb.base_margin, &bo[j]);
        jb.status = s;
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(setup, t);
    setup(0);
    for (std::thread& th : pool) th.join();
  }
  // rounds: the jobs that can share launches run as one batch (one launch
  // per kernel step for all of them), the others interleaved over the pool
  if (rc == SB_OK && n_jobs > 0) {
    std::vector<int> rounds(n_jobs), status(n_jobs);
    for (size_t j = 0; j < n_jobs; ++j) {
      rounds[j] = jobs[j].num_boost_round;
      status[j] = jobs[j].status;
    }
    boosters_train_many(sctx.data(), std::min(S, 8), bo.data(), rounds.data(), (int)n_jobs, status.data());
    for (size_t j = 0; j < n_jobs; ++j) jobs[j].status = status[j];
  }
  // models
  for (size_t j = 0; j < n_jobs && rc == SB_OK; ++j)
    if (jobs[j].status == SB_OK) {
      jobs[j].status = sb_booster_model(bo[j], &jobs[j].out);
      if (jobs[j].out) jobs[j].out->ctx = ctx;  // the job streams end here; the model lives on
    }
  for (size_t j = 0; j < n_jobs; ++j) {
    sb_booster_destroy(bo[j]);
    sb_ghist_destroy(gh[j]);
  }
  for (sb_ctx* c : sctx)
    if (c) sb_ctx_destroy(c);
  if (rc != SB_OK) return rc;
  for (size_t j = 0; j < n_jobs; ++j)
    if (jobs[j].status != SB_OK) {
      set_error("job %zu failed with status %d", j, jobs[j].status);
      return jobs[j].status;
    }
  return SB_OK;
}

}  // extern "C"
