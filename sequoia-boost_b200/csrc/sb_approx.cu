// sb_approx.cu — tree_method=approx: hessian-weighted cuts recomputed every
// round, then the hist builder on the re-binned matrix.
//
// Replaces HistCuts::from_dmatrix_weighted with build_feature_cuts_weighted
// (data/quantile.rs:81-122, :253-316) and the Prepared::Approx branch of the
// round loop (learner/train.rs:46-53), for which the reference sorts every
// column again in every round.
//
// Here each column is sorted once (a stable radix sort of (feature, value)
// keys, so equal values keep row order, as the reference's stable sort does).
// A round then takes, per column whose cuts depend on the weights (numeric
// with more distinct values than max_bin), the class tree's hessians in value
// order:
//   pass 1  one thread per column adds the weights in value order in f64,
//           exactly the reference's sequential `cum += w as f64`, and keeps
//           the running sum at every CHUNK-th element (the total is its last);
//   pass 2  one thread per (column, chunk) resumes from that running sum and
//           marks the elements where the count of crossed boundaries
//           #{b <= max_bin : b * step <= cum + 1e-12} grows: the reference
//           pushes that element's value there (step = total / max_bin).
// The host drops repeated values among the marked ones (`v > last_pushed`)
// and adds the sentinel next_up(max). Columns whose cuts do not depend on the
// weights (categorical, or at most max_bin distinct values) keep the cuts of
// the first round. All f64 arithmetic uses explicit round-to-nearest
// operations so that no contraction changes a comparison.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "sb_internal.cuh"

namespace sb {
namespace {

constexpr int APPROX_CHUNK = 2048;  // elements per pass-2 thread

__device__ __forceinline__ bool missing_value(float v, float missing, bool miss_nan) {
  return miss_nan ? isnan(v) : (v == missing);
}

// Order-preserving u32 of a non-NaN float, with -0.0 and +0.0 equal (the
// reference compares values with partial_cmp, where they are equal).
__device__ __forceinline__ uint32_t sortable(float v) {
  if (v == 0.0f) v = 0.0f;
  const uint32_t u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Keys (feature << 32 | sortable value) of every entry, in row-major order;
// missing entries sort last (feature F).
__global__ void k_approx_keys(const float* __restrict__ X, size_t n, int F, float missing,
                              unsigned long long* __restrict__ keys, uint32_t* __restrict__ rows,
                              unsigned int* __restrict__ nan_seen) {
  const bool miss_nan = isnan(missing);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * (size_t)F;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / F;
    const int f = (int)(i - r * F);
    const float v = X[i];
    const bool mis = missing_value(v, missing, miss_nan);
    if (!mis && isnan(v)) *nan_seen = 1u;
    keys[i] = mis ? ((unsigned long long)F << 32) : (((unsigned long long)f << 32) | sortable(v));
    rows[i] = (uint32_t)r;
  }
}

// Column starts (first sorted position of each feature), the sorted values,
// and each column's distinct-value count.
__global__ void k_approx_columns(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ rows,
                                 const float* __restrict__ X, size_t total, int F,
                                 unsigned long long* __restrict__ coff, float* __restrict__ sval,
                                 unsigned int* __restrict__ distinct) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(keys[i] >> 32);
    const int fp = i == 0 ? -1 : (int)(keys[i - 1] >> 32);
    for (int g = fp + 1; g <= f && g <= F; ++g) coff[g] = i;  // features fp+1..f start here
    if (i + 1 == total)
      for (int g = f + 1; g <= F; ++g) coff[g] = total;
    if (f >= F) continue;
    const float v = X[(size_t)rows[i] * F + f];
    sval[i] = v;
    const bool first = fp != f || (uint32_t)keys[i - 1] != (uint32_t)keys[i];
    if (first) atomicAdd(&distinct[f], 1u);
  }
}

// Pass 1: the sequential f64 sum of each weighted column's hessians in value
// order, recorded before every chunk and at the end.
__global__ void k_approx_pass1(const int* __restrict__ wfeat, int nw, const unsigned long long* __restrict__ coff,
                               const uint32_t* __restrict__ srow, const float* __restrict__ hess,
                               const unsigned long long* __restrict__ ck_off, double* __restrict__ ck) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nw) return;
  const int f = wfeat[j];
  const size_t b = coff[f], e = coff[f + 1];
  double* out = ck + ck_off[j];
  double cum = 0.0;
  size_t c = 0;
  for (size_t i0 = b; i0 < e; i0 += APPROX_CHUNK) {
    out[c++] = cum;
    const size_t i1 = i0 + APPROX_CHUNK < e ? i0 + APPROX_CHUNK : e;
    size_t i = i0;
    for (; i + 8 <= i1; i += 8) {  // the gathers do not depend on the sum: issue them together
      float w[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) w[u] = __ldg(hess + srow[i + u]);
#pragma unroll
      for (int u = 0; u < 8; ++u) cum = __dadd_rn(cum, (double)w[u]);
    }
    for (; i < i1; ++i) cum = __dadd_rn(cum, (double)__ldg(hess + srow[i]));
  }
  out[c] = cum;  // the total
}

// #{b in [1, max_bin] : fl(b * step) <= y}; fl(b * step) does not decrease with b.
__device__ __forceinline__ int crossed(double y, double step, int max_bin) {
  int lo = 0, hi = max_bin;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__dmul_rn((double)mid, step) <= y) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Pass 2: per (weighted column, chunk), the elements at which the count of
// crossed boundaries grows (hessians are >= 0, so the running sum and the
// count never decrease). Events go to the column's list (at most max_bin).
__global__ void k_approx_pass2(const int* __restrict__ wfeat, int nw, const unsigned long long* __restrict__ coff,
                               const uint32_t* __restrict__ srow, const float* __restrict__ hess,
                               const unsigned long long* __restrict__ ck_off, const double* __restrict__ ck,
                               const unsigned long long* __restrict__ chunk_first, unsigned long long n_chunks,
                               const float* __restrict__ sval, int max_bin, unsigned int* __restrict__ ev_count,
                               uint32_t* __restrict__ ev_pos, float* __restrict__ ev_val) {
  for (unsigned long long q = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; q < n_chunks;
       q += (unsigned long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nw;  // the column: last j with chunk_first[j] <= q
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (chunk_first[mid] <= q) lo = mid; else hi = mid;
    }
    const int j = lo, f = wfeat[j];
    const unsigned long long c = q - chunk_first[j];
    const size_t b = coff[f], e = coff[f + 1];
    const size_t n_ch = (e - b + APPROX_CHUNK - 1) / APPROX_CHUNK;
    const double total = ck[ck_off[j] + n_ch];
    if (!(total > 0.0)) continue;  // the unweighted positions are taken instead
    const double step = __ddiv_rn(total, (double)max_bin);
    double cum = ck[ck_off[j] + c];
    int prev = crossed(__dadd_rn(cum, 1e-12), step, max_bin);
    const size_t i0 = b + (size_t)c * APPROX_CHUNK;
    const size_t i1 = i0 + APPROX_CHUNK < e ? i0 + APPROX_CHUNK : e;
    for (size_t i = i0; i < i1 && prev < max_bin; ++i) {
      cum = __dadd_rn(cum, (double)__ldg(hess + srow[i]));
      const int now = crossed(__dadd_rn(cum, 1e-12), step, max_bin);
      if (now > prev) {
        const unsigned int slot = atomicAdd(&ev_count[j], 1u);
        if (slot < (unsigned int)max_bin) {
          ev_pos[(size_t)j * max_bin + slot] = (uint32_t)(i - b);
          ev_val[(size_t)j * max_bin + slot] = sval[i];
        }
        prev = now;
      }
    }
  }
}

}  // namespace

// The sorted columns of one matrix, kept across rounds.
struct ApproxState {
  sb_ctx* ctx = nullptr;
  size_t n = 0, F = 0;
  int max_bin = 0;
  float missing = NAN;
  std::vector<uint8_t> is_cat;
  DBuf<uint32_t> srow;                 // rows of present entries, sorted by (feature, value)
  DBuf<float> sval;                    // their values
  std::vector<unsigned long long> coff;  // [F + 1] column starts
  DBuf<unsigned long long> d_coff;
  std::vector<int> wfeat;              // columns whose cuts depend on the weights
  DBuf<int> d_wfeat;
  std::vector<std::vector<float>> fixed_cuts;  // the others' cuts, per column
  std::vector<float> max_val;          // last sorted value per column
  DBuf<unsigned long long> ck_off, chunk_first;
  unsigned long long n_chunks = 0, ck_total = 0;
  DBuf<double> ck;
  std::vector<unsigned long long> h_ck_off;  // per weighted column: its first checkpoint
  DBuf<unsigned int> ev_count;
  DBuf<uint32_t> ev_pos;
  DBuf<float> ev_val;
};

namespace {

void push_sentinel(std::vector<float>& out, float max_val) {  // push_max_sentinel, quantile.rs:319-323
  if (out.back() <= max_val) out.push_back(std::nextafterf(max_val, INFINITY));
}

}  // namespace

ApproxState* approx_state_new() { return new ApproxState; }
void approx_state_free(ApproxState* a) { delete a; }

int approx_prepare(sb_ctx* ctx, const float* d_X, size_t n, size_t F, const uint8_t* h_ftypes, float missing,
                   int max_bin, ApproxState* A) {
  SB_REQUIRE(n > 0 && F > 0, SB_ERR_INVALID_ARG, "empty dataset: zero rows or columns");
  SB_REQUIRE(max_bin >= 2 && max_bin <= 1024, SB_ERR_UNSUPPORTED, "max_bin must be in [2, 1024] on the GPU, got %d",
             max_bin);
  SB_REQUIRE(F < 4096 && n < (size_t)UNSAMPLED, SB_ERR_UNSUPPORTED, "at most 4095 features and 2^31-1 rows");
  A->ctx = ctx;
  A->n = n;
  A->F = F;
  A->max_bin = max_bin;
  A->missing = missing;
  A->is_cat.assign(F, 0);
  if (h_ftypes)
    for (size_t f = 0; f < F; ++f) A->is_cat[f] = h_ftypes[f] == SB_FEAT_CATEGORICAL ? 1 : 0;
  cudaStream_t st = ctx->stream;
  const size_t N = n * F;
  DBuf<unsigned long long> keys, keys2;
  DBuf<uint32_t> rows, rows2;
  DBuf<unsigned int> distinct, nan_seen;
  SB_TRY(nan_seen.alloc_zero(ctx, 1));
  SB_TRY(keys.alloc(ctx, N));
  SB_TRY(keys2.alloc(ctx, N));
  SB_TRY(rows.alloc(ctx, N));
  SB_TRY(rows2.alloc(ctx, N));
  const unsigned blocks = (unsigned)std::min<size_t>((N + 255) / 256, (size_t)ctx->num_sms * 32);
  SB_LAUNCH(ctx, k_approx_keys, blocks, 256, 0, d_X, n, (int)F, missing, keys.p, rows.p, nan_seen.p);
  unsigned int h_nan = 0;
  SB_CUDA(cudaMemcpyAsync(&h_nan, nan_seen.p, 4, cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  SB_REQUIRE(h_nan == 0, SB_ERR_INVALID_ARG,
             "the matrix holds NaN while the missing sentinel is %g (the reference's sort panics on NaN here)",
             (double)missing);
  int end_bit = 32;
  while ((1ull << (end_bit - 32)) <= F) ++end_bit;  // the feature field holds 0..F
  size_t temp_bytes = 0;
  SB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys.p, keys2.p, rows.p, rows2.p, N, 0, end_bit, st));
  DBuf<unsigned char> temp;
  SB_TRY(temp.alloc(ctx, std::max<size_t>(temp_bytes, 1)));
  SB_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, keys.p, keys2.p, rows.p, rows2.p, N, 0, end_bit, st));
  ctx->launches++;
  SB_TRY(A->d_coff.alloc(ctx, F + 1));
  SB_TRY(A->sval.alloc(ctx, N));
  SB_TRY(distinct.alloc_zero(ctx, F));
  SB_LAUNCH(ctx, k_approx_columns, blocks, 256, 0, keys2.p, rows2.p, d_X, N, (int)F, A->d_coff.p, A->sval.p,
            distinct.p);
  A->coff.assign(F + 1, 0);
  std::vector<unsigned int> h_distinct(F);
  SB_CUDA(cudaMemcpyAsync(A->coff.data(), A->d_coff.p, (F + 1) * 8, cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaMemcpyAsync(h_distinct.data(), distinct.p, F * 4, cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  // keep the sorted rows (the present part of rows2)
  const size_t present = A->coff[F];
  SB_TRY(A->srow.alloc(ctx, std::max<size_t>(present, 1)));
  if (present)
    SB_CUDA(cudaMemcpyAsync(A->srow.p, rows2.p, present * 4, cudaMemcpyDeviceToDevice, st));
  std::vector<float> hv(present);
  if (present) SB_CUDA(cudaMemcpyAsync(hv.data(), A->sval.p, present * 4, cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  // columns with weight-independent cuts get them now (build_categorical_cuts
  // :187-200, or every distinct value, :270-279); the others are weighted
  A->fixed_cuts.assign(F, {});
  A->max_val.assign(F, 0.0f);
  A->wfeat.clear();
  for (size_t f = 0; f < F; ++f) {
    const size_t b = A->coff[f], e = A->coff[f + 1];
    std::vector<float>& out = A->fixed_cuts[f];
    if (b == e) {  // no present value: one degenerate bin
      out.push_back(0.0f);
      continue;
    }
    A->max_val[f] = hv[e - 1];
    if (A->is_cat[f] || h_distinct[f] <= (unsigned)max_bin) {
      out.push_back(hv[b]);
      for (size_t i = b + 1; i < e; ++i)
        if (hv[i - 1] != hv[i]) out.push_back(hv[i]);
      if (!A->is_cat[f]) push_sentinel(out, hv[e - 1]);
      if (A->is_cat[f])
        SB_REQUIRE(out.size() <= (size_t)MAX_CAT_BINS, SB_ERR_UNSUPPORTED,
                   "categorical feature %zu has more than %d categories", f, MAX_CAT_BINS);
      continue;
    }
    A->wfeat.push_back((int)f);
  }
  // per weighted column: its chunks and checkpoint slots
  const size_t nw = A->wfeat.size();
  std::vector<unsigned long long> cko(nw), chf(nw);
  A->n_chunks = 0;
  A->ck_total = 0;
  A->h_ck_off.assign(nw, 0);
  for (size_t j = 0; j < nw; ++j) {
    const int f = A->wfeat[j];
    const unsigned long long len = A->coff[f + 1] - A->coff[f];
    const unsigned long long nc = (len + APPROX_CHUNK - 1) / APPROX_CHUNK;
    cko[j] = A->ck_total;
    A->h_ck_off[j] = A->ck_total;
    A->ck_total += nc + 1;
    chf[j] = A->n_chunks;
    A->n_chunks += nc;
  }
  if (nw) {
    SB_TRY(A->d_wfeat.alloc(ctx, nw));
    SB_TRY(A->ck_off.alloc(ctx, nw));
    SB_TRY(A->chunk_first.alloc(ctx, nw));
    SB_TRY(A->ck.alloc(ctx, A->ck_total));
    SB_TRY(A->ev_count.alloc(ctx, nw));
    SB_TRY(A->ev_pos.alloc(ctx, nw * (size_t)max_bin));
    SB_TRY(A->ev_val.alloc(ctx, nw * (size_t)max_bin));
    SB_CUDA(cudaMemcpyAsync(A->d_wfeat.p, A->wfeat.data(), nw * 4, cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemcpyAsync(A->ck_off.p, cko.data(), nw * 8, cudaMemcpyHostToDevice, st));
    SB_CUDA(cudaMemcpyAsync(A->chunk_first.p, chf.data(), nw * 8, cudaMemcpyHostToDevice, st));
  }
  SB_CUDA(cudaStreamSynchronize(st));
  return SB_OK;
}

// HistCuts::from_dmatrix_weighted for the hessians d_hess (device, one per
// row, >= 0): host cuts into g (h_foff, h_cuts, h_is_cat).
int approx_cuts(ApproxState* A, const float* d_hess, Ghist* g) {
  sb_ctx* ctx = A->ctx;
  cudaStream_t st = ctx->stream;
  const size_t F = A->F, nw = A->wfeat.size();
  const int max_bin = A->max_bin;
  std::vector<double> ck(A->ck_total);
  std::vector<unsigned int> cnt(nw);
  std::vector<uint32_t> pos(nw * (size_t)max_bin);
  std::vector<float> val(nw * (size_t)max_bin);
  if (nw) {
    SB_LAUNCH(ctx, k_approx_pass1, (unsigned)((nw + 63) / 64), 64, 0, A->d_wfeat.p, (int)nw, A->d_coff.p,
              A->srow.p, d_hess, A->ck_off.p, A->ck.p);
    SB_CUDA(cudaMemsetAsync(A->ev_count.p, 0, nw * 4, st));
    const unsigned blocks = (unsigned)std::min<unsigned long long>((A->n_chunks + 127) / 128,
                                                                   (unsigned long long)ctx->num_sms * 16);
    SB_LAUNCH(ctx, k_approx_pass2, std::max(blocks, 1u), 128, 0, A->d_wfeat.p, (int)nw, A->d_coff.p, A->srow.p,
              d_hess, A->ck_off.p, A->ck.p, A->chunk_first.p, A->n_chunks, A->sval.p, max_bin, A->ev_count.p,
              A->ev_pos.p, A->ev_val.p);
    SB_CUDA(cudaMemcpyAsync(ck.data(), A->ck.p, ck.size() * 8, cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(cnt.data(), A->ev_count.p, nw * 4, cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(pos.data(), A->ev_pos.p, pos.size() * 4, cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(val.data(), A->ev_val.p, val.size() * 4, cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
  }
  g->h_foff.assign(F + 1, 0);
  g->h_cuts.clear();
  g->h_is_cat = A->is_cat;
  size_t j = 0;
  for (size_t f = 0; f < F; ++f) {
    if (j < nw && A->wfeat[j] == (int)f) {
      const size_t b = A->coff[f], len = A->coff[f + 1] - b;
      const size_t nc = (len + APPROX_CHUNK - 1) / APPROX_CHUNK;
      const double total = ck[A->h_ck_off[j] + nc];
      std::vector<float> vals;
      if (total > 0.0) {  // the marked elements in value order
        SB_REQUIRE(cnt[j] <= (unsigned)max_bin, SB_ERR_CUDA, "internal: %u cut events on feature %zu", cnt[j], f);
        std::vector<std::pair<uint32_t, float>> ev(cnt[j]);
        for (unsigned t = 0; t < cnt[j]; ++t) ev[t] = {pos[j * max_bin + t], val[j * max_bin + t]};
        std::sort(ev.begin(), ev.end(),
                  [](const std::pair<uint32_t, float>& x, const std::pair<uint32_t, float>& y) { return x.first < y.first; });
        for (const auto& e : ev) vals.push_back(e.second);
      } else {  // all weights zero: the unweighted positions (quantile.rs:298-311)
        std::vector<float> col(len);
        SB_CUDA(cudaMemcpyAsync(col.data(), A->sval.p + b, len * 4, cudaMemcpyDeviceToHost, st));
        SB_CUDA(cudaStreamSynchronize(st));
        for (int bb = 1; bb <= max_bin; ++bb) {
          const double q = (double)bb / (double)max_bin;
          const size_t c = (size_t)std::ceil(q * (double)len);
          vals.push_back(col[std::min(std::max(c, (size_t)1) - 1, len - 1)]);
        }
      }
      std::vector<float> out;
      float last = -INFINITY;
      for (float v : vals)  // `if v > last_pushed`, quantile.rs:290-293
        if (v > last) {
          out.push_back(v);
          last = v;
        }
      SB_REQUIRE(!out.empty(), SB_ERR_CUDA, "internal: no weighted cut on feature %zu", f);
      push_sentinel(out, A->max_val[f]);
      g->h_cuts.insert(g->h_cuts.end(), out.begin(), out.end());
      ++j;
    } else {
      const std::vector<float>& c = A->fixed_cuts[f];
      g->h_cuts.insert(g->h_cuts.end(), c.begin(), c.end());
    }
    g->h_foff[f + 1] = (uint32_t)g->h_cuts.size();
  }
  return SB_OK;
}

}  // namespace sb

extern "C" {

int sb_ghist_create_weighted(sb_ctx* ctx, const float* X, size_t n_rows, size_t n_cols,
                             const uint8_t* feature_types, float missing, int max_bin, const float* hessians,
                             sb_ghist** out) {
  using namespace sb;
  SB_REQUIRE(ctx && X && hessians && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_rows > 0 && n_cols > 0, SB_ERR_INVALID_ARG, "empty dataset: zero rows or columns");
  for (size_t i = 0; i < n_rows; ++i)
    SB_REQUIRE(hessians[i] >= 0.0f && std::isfinite(hessians[i]), SB_ERR_INVALID_ARG,
               "hessian %zu (%g) is not a finite value >= 0", i, (double)hessians[i]);
  *out = nullptr;
  SB_CUDA(cudaSetDevice(ctx->device));
  DBuf<float> dX, dh;
  SB_TRY(dX.alloc(ctx, n_rows * n_cols));
  SB_TRY(dh.alloc(ctx, n_rows));
  SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  SB_CUDA(cudaMemcpyAsync(dh.p, hessians, dh.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  ApproxState A;
  SB_TRY(approx_prepare(ctx, dX.p, n_rows, n_cols, feature_types, missing, max_bin, &A));
  std::unique_ptr<sb_ghist> g(new sb_ghist);
  g->ctx = ctx;
  g->n = n_rows;
  g->F = n_cols;
  g->max_bin = max_bin;
  g->missing = missing;
  SB_TRY(approx_cuts(&A, dh.p, g.get()));
  SB_TRY(ghist_bin(ctx, dX.p, g.get()));
  *out = g.release();
  return SB_OK;
}

}  // extern "C"
