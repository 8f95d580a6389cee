// sb_bin.cu — quantile cuts (K1) and ELLPACK binning (K2) on the device.
//
// Replaces HistCuts::from_dmatrix (data/quantile.rs:39-70) with
// build_feature_cuts (:203-245), build_categorical_cuts (:187-200),
// push_max_sentinel (:319-323), and GHistIndex::from_dmatrix
// (data/ghist.rs:48-82) with bin_of (quantile.rs:166-181).
//
// The reference sorts every column and reads order statistics at ranks
// idx_b = min(max(ceil(b/max_bin*n),1)-1, n-1). Here the same order statistics
// are found without sorting: values map to order-preserving 32-bit keys and a
// three-level radix select (11 + 11 + 10 key bits) counts, per feature, only
// the key ranges that contain a wanted rank (or, while a feature may still
// have <= max_bin distinct values, every non-empty range). Three streaming
// passes over X give exact values, identical to the sorted-array reads.
#include <cstring>

#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

#include "sb_internal.cuh"

namespace sb {
namespace {

constexpr int MODE_ENUM = 0;   // may have <= max_bin distinct values: refine all
constexpr int MODE_QUANT = 1;  // > max_bin distinct: refine wanted ranks only
constexpr int MODE_DONE = 2;   // no present values: single cut 0.0

struct FPlan {
  unsigned long long n;  // present values
  int mode;
  int nslots;            // slots refined at the next level
  int err;               // 1: NaN with non-NaN sentinel, 2: too many categories
  int pad;
};

__device__ __forceinline__ bool is_missing_d(float v, float missing, bool miss_nan) {
  return miss_nan ? isnan(v) : (v == missing);
}

// Order-preserving key; -0.0 and +0.0 share the key of +0.0 (partial_cmp
// equality).
__device__ __forceinline__ uint32_t f2key(float v) {
  if (v == 0.0f) v = 0.0f;
  uint32_t u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key2f(uint32_t k) {
  uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  return __uint_as_float(u);
}

constexpr int TILE_F = 32;
constexpr int TILE_R = 128;
constexpr int COUNT_THREADS = 256;

// Levels 2 and 3 of the radix select: one streaming pass over a (TILE_R rows
// x TILE_F features) tile staged in shared memory; each warp walks one
// feature's column so equal cells of consecutive rows aggregate before the
// atomic. Only values in the ranges the previous level refined are counted.
template <int LEVEL>
__global__ void __launch_bounds__(COUNT_THREADS) k_cuts_count(const float* __restrict__ X, size_t n, int F,
                                                    float missing, int S,
                                                    unsigned int* __restrict__ cnt2,
                                                    unsigned int* __restrict__ cnt3,
                                                    const short* __restrict__ map2,
                                                    const short* __restrict__ map3,
                                                    FPlan* __restrict__ plan) {
  __shared__ float tile[TILE_R][TILE_F + 1];
  const bool miss_nan = isnan(missing);
  size_t r0 = (size_t)blockIdx.x * TILE_R;
  int f0 = blockIdx.y * TILE_F;
  int nf = min(TILE_F, F - f0);
  int nr = (int)min((size_t)TILE_R, n - r0);
  {  // every load of the thread's tile cells in flight together
    constexpr int PER = TILE_R * TILE_F / COUNT_THREADS;
    float v[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int i = threadIdx.x + u * COUNT_THREADS;
      const int rr = i / TILE_F, ff = i % TILE_F;
      v[u] = (rr < nr && ff < nf) ? __ldg(X + (r0 + rr) * (size_t)F + f0 + ff) : NAN;
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int i = threadIdx.x + u * COUNT_THREADS;
      tile[i / TILE_F][i % TILE_F] = v[u];
    }
  }
  __syncthreads();
  static_assert(LEVEL == 2 || LEVEL == 3, "level 1 counts in k_cuts_count1");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int STEPS = TILE_R / 32;
  for (int ff = warp; ff < nf; ff += COUNT_THREADS / 32) {
    const int f = f0 + ff;
    if (plan[f].mode == MODE_DONE) continue;
    // the counter of each of the lane's rows: the lookups of the steps are
    // independent, so they are all issued before the first atomic
    unsigned int* addr[STEPS];
#pragma unroll
    for (int q = 0; q < STEPS; ++q) {
      const int rr = q * 32 + lane;
      addr[q] = nullptr;
      if (rr < nr) {
        const float v = tile[rr][ff];
        bool miss = is_missing_d(v, missing, miss_nan);
        if (!miss && !miss_nan && isnan(v)) {
          plan[f].err = 1;
          miss = true;
        }
        if (!miss) {
          const uint32_t key = f2key(v);
          const int s2 = map2[(size_t)f * 2048 + (key >> 21)];
          if (s2 >= 0) {
            const uint32_t d2 = (key >> 10) & 0x7FFu;
            if (LEVEL == 2) {
              addr[q] = cnt2 + ((size_t)f * S + s2) * 2048 + d2;
            } else {
              const int s3 = map3[((size_t)f * S + s2) * 2048 + d2];
              if (s3 >= 0) addr[q] = cnt3 + ((size_t)f * S + s3) * 1024 + (key & 0x3FFu);
            }
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < STEPS; ++q) {
      const unsigned active = __ballot_sync(0xFFFFFFFFu, addr[q] != nullptr);
      if (addr[q]) {
        const unsigned peers = __match_any_sync(active, (unsigned long long)addr[q]);
        if (lane == __ffs(peers) - 1) atomicAdd(addr[q], (unsigned)__popc(peers));
      }
    }
  }
}

// Level 1 of the radix select with shared-memory counters: a block takes
// C1_FEATS consecutive features over a range of rows (4 lanes per row, one
// feature each, so a warp reads 8 rows' 16-byte segments) and counts the top
// 11 key bits of their present values in shared memory, then adds its
// non-zero counters into cnt1. The counts are integers, so they equal those
// of counting value by value in any order; values that would otherwise meet
// in the few hot global counters of a feature's dense key range add in
// shared memory.
constexpr int C1_FEATS = 4;
__global__ void __launch_bounds__(256) k_cuts_count1(const float* __restrict__ X, size_t n, int F, float missing,
                                                     size_t rows_per_block, unsigned int* __restrict__ cnt1,
                                                     FPlan* __restrict__ plan) {
  __shared__ unsigned int s_c[C1_FEATS * 2048];
  const bool miss_nan = isnan(missing);
  const int f0 = blockIdx.y * C1_FEATS;
  const int nf = min(C1_FEATS, F - f0);
  const size_t r0 = (size_t)blockIdx.x * rows_per_block;
  const size_t r1 = min(n, r0 + rows_per_block);
  for (int i = threadIdx.x; i < C1_FEATS * 2048; i += blockDim.x) s_c[i] = 0u;
  __syncthreads();
  const int j = threadIdx.x % C1_FEATS;
  const bool on = j < nf;
  const size_t step = blockDim.x / C1_FEATS;
  bool bad = false;  // NaN while the missing sentinel is not NaN
  auto count = [&](float v) {
    bool miss = is_missing_d(v, missing, miss_nan);
    if (!miss && !miss_nan && isnan(v)) {
      bad = true;
      miss = true;
    }
    if (!miss) atomicAdd(&s_c[j * 2048 + (f2key(v) >> 21)], 1u);
  };
  size_t r = r0 + threadIdx.x / C1_FEATS;
  if (on) {
    for (; r + 3 * step < r1; r += 4 * step) {
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = __ldg(X + (r + u * step) * (size_t)F + f0 + j);
#pragma unroll
      for (int u = 0; u < 4; ++u) count(v[u]);
    }
    for (; r < r1; r += step) count(__ldg(X + r * (size_t)F + f0 + j));
  }
  if (bad) plan[f0 + j].err = 1;
  __syncthreads();
  for (int i = threadIdx.x; i < nf * 2048; i += blockDim.x) {
    const unsigned c = s_c[i];
    if (c) atomicAdd(&cnt1[(size_t)(f0 + i / 2048) * 2048 + (i % 2048)], c);
  }
}

// Block-wide exclusive scan of one value per thread (1024 threads).
template <typename T>
__device__ T block_excl_scan(T v, T* total, T* sm /* >= 33 */) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
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
  T res = sm[warp] + (x - v);
  if (total) *total = sm[32];
  __syncthreads();
  return res;
}

// Planning step of level LEVEL for feature blockIdx.x (1024 threads).
// Reads the level's counts over the refined slots, decides enum/quantile,
// and writes the next level's slots and lookup map (or the final cuts).
template <int LEVEL>
__global__ void __launch_bounds__(1024) k_cuts_plan(
    int F, int S, int max_bin, const uint8_t* __restrict__ is_cat,
    const unsigned int* __restrict__ cnt1, const unsigned int* __restrict__ cnt2,
    const unsigned int* __restrict__ cnt3, short* __restrict__ map2, short* __restrict__ map3,
    uint32_t* __restrict__ slot_prefix,   // [2][F][S] (cur, next) by level parity
    unsigned long long* __restrict__ slot_base,  // [2][F][S]
    unsigned long long* __restrict__ trank,      // [F][S]
    float* __restrict__ cut_tmp, int* __restrict__ ncut, FPlan* __restrict__ plan) {
  constexpr int D = (LEVEL == 3) ? 1024 : 2048;
  constexpr int CPT = D / 1024;  // cells per thread
  __shared__ unsigned long long sm_u64[33];
  __shared__ unsigned long long s_trank[1100];
  __shared__ int s_carry;
  __shared__ int s_mode;
  __shared__ unsigned long long s_E;
  __shared__ float s_vals[1100];
  int f = blockIdx.x;
  const int tid = threadIdx.x;
  FPlan& P = plan[f];
  const int cur = (LEVEL + 1) & 1, nxt = LEVEL & 1;  // parity buffers
  uint32_t* pre_cur = slot_prefix + ((size_t)cur * F + f) * S;
  unsigned long long* base_cur = slot_base + ((size_t)cur * F + f) * S;
  uint32_t* pre_nxt = slot_prefix + ((size_t)nxt * F + f) * S;
  unsigned long long* base_nxt = slot_base + ((size_t)nxt * F + f) * S;
  const bool cat = is_cat && is_cat[f];

  if (LEVEL == 1) {
    // total present count
    unsigned long long c = 0;
    for (int d = tid; d < 2048; d += 1024) c += cnt1[(size_t)f * 2048 + d];
    unsigned long long tot;
    block_excl_scan<unsigned long long>(c, &tot, sm_u64);
    if (tid == 0) {
      P.n = tot;
      P.mode = tot == 0 ? MODE_DONE : MODE_ENUM;
      pre_cur[0] = 0;
      base_cur[0] = 0;
      P.nslots = 1;
    }
    __syncthreads();
  }
  if (P.mode == MODE_DONE) {
    if (LEVEL == 3 || P.n == 0) {
      if (tid == 0) {
        ncut[f] = 1;
        cut_tmp[(size_t)f * (S + 1)] = 0.0f;
      }
    }
    return;
  }
  const int nslots = P.nslots;
  auto cell_cnt = [&](int s, int d) -> unsigned long long {
    if (LEVEL == 1) return cnt1[(size_t)f * 2048 + d];
    if (LEVEL == 2) return cnt2[((size_t)f * S + s) * 2048 + d];
    return cnt3[((size_t)f * S + s) * 1024 + d];
  };

  // Pass A: number of non-empty cells.
  unsigned long long E = 0;
  for (int s = 0; s < nslots; ++s)
    for (int i = 0; i < CPT; ++i) E += cell_cnt(s, tid * CPT + i) ? 1 : 0;
  unsigned long long Etot;
  block_excl_scan<unsigned long long>(E, &Etot, sm_u64);
  if (tid == 0) {
    int mode = P.mode;
    if (mode == MODE_ENUM) {
      if (cat) {
        if (Etot > (unsigned long long)MAX_CAT_BINS) P.err = 2;
      } else if (Etot > (unsigned long long)max_bin) {
        mode = MODE_QUANT;
      }
    }
    s_mode = mode;
    s_E = Etot;
    s_carry = 0;
  }
  __syncthreads();
  const int mode = s_mode;
  if (P.err == 2) {
    if (tid == 0) P.mode = MODE_DONE;
    return;
  }
  const unsigned long long n = P.n;
  const int T = max_bin + 1;  // ranks b = 1..max_bin, then n-1
  if (mode == MODE_QUANT) {
    if (P.mode == MODE_ENUM) {
      for (int j = tid; j < T; j += 1024) {
        unsigned long long r;
        if (j < max_bin) {
          double q = (double)(j + 1) / (double)max_bin;
          unsigned long long c = (unsigned long long)ceil(q * (double)n);
          if (c < 1) c = 1;
          r = c - 1;
          if (r > n - 1) r = n - 1;
        } else {
          r = n - 1;
        }
        trank[(size_t)f * S + j] = r;
      }
      __syncthreads();
    }
    for (int j = tid; j < T; j += 1024) s_trank[j] = trank[(size_t)f * S + j];
    __syncthreads();
  }

  // Pass B: slot by slot, scan the cells in key order.
  for (int s = 0; s < nslots; ++s) {
    unsigned long long c[CPT];
    unsigned long long mine = 0;
    for (int i = 0; i < CPT; ++i) {
      c[i] = cell_cnt(s, tid * CPT + i);
      mine += c[i];
    }
    unsigned long long slot_total;
    unsigned long long rank0 = base_cur[s] + block_excl_scan<unsigned long long>(mine, &slot_total, sm_u64);
    uint32_t prefix = pre_cur[s];
    // which cells become next-level slots (or final values)
    int take[CPT];
    int ntake = 0;
    unsigned long long rlo = rank0;
    for (int i = 0; i < CPT; ++i) {
      take[i] = 0;
      if (c[i]) {
        if (mode == MODE_ENUM) {
          take[i] = 1;
        } else {
          // any wanted rank in [rlo, rlo + c)?
          int lo = 0, hi = T;
          while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (s_trank[mid] < rlo) lo = mid + 1; else hi = mid;
          }
          take[i] = (lo < T && s_trank[lo] < rlo + c[i]) ? 1 : 0;
        }
      }
      ntake += take[i];
      rlo += c[i];
    }
    unsigned long long ntot;
    int idx = s_carry + (int)block_excl_scan<unsigned long long>((unsigned long long)ntake, &ntot, sm_u64);
    rlo = rank0;
    for (int i = 0; i < CPT; ++i) {
      int d = tid * CPT + i;
      if (take[i]) {
        if (idx < S + 64) {
          if (LEVEL < 3) {
            uint32_t np = (LEVEL == 1) ? (uint32_t)d : ((prefix << 11) | (uint32_t)d);
            if (idx < S) {
              pre_nxt[idx] = np;
              base_nxt[idx] = rlo;
              if (LEVEL == 1) map2[(size_t)f * 2048 + d] = (short)idx;
              else map3[((size_t)f * S + s) * 2048 + d] = (short)idx;
            }
          } else {
            uint32_t key = (prefix << 10) | (uint32_t)d;
            float v = key2f(key);
            if (mode == MODE_ENUM) {
              if (idx < 1100) s_vals[idx] = v;
            } else {
              // every wanted rank inside this cell takes the cell's value
              int lo = 0, hi = T;
              while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (s_trank[mid] < rlo) lo = mid + 1; else hi = mid;
              }
              for (int j = lo; j < T && s_trank[j] < rlo + c[i]; ++j) s_vals[j] = v;
            }
          }
        }
        idx++;
      }
      rlo += c[i];
    }
    __syncthreads();
    if (tid == 0) s_carry += (int)ntot;
    __syncthreads();
  }
  if (LEVEL < 3) {
    if (tid == 0) {
      P.mode = mode;
      P.nslots = s_carry > S ? S : s_carry;
      if (s_carry > S) P.err = 3;  // cannot happen: slots are bounded by max_bin + 1
    }
    return;
  }
  // Final cut list (quantile.rs:203-245 / :187-200), one thread.
  if (tid == 0) {
    float* out = cut_tmp + (size_t)f * (S + 1);
    int m = 0;
    if (mode == MODE_ENUM) {
      int E3 = s_carry;
      for (int i = 0; i < E3; ++i) out[m++] = s_vals[i];
      if (!cat) {
        float mx = s_vals[E3 - 1];
        if (out[m - 1] <= mx) out[m++] = nextafterf(mx, INFINITY);
      }
    } else {
      float last = -INFINITY;
      for (int j = 0; j < max_bin; ++j) {
        float v = s_vals[j];
        if (v > last) {
          out[m++] = v;
          last = v;
        }
      }
      float mx = s_vals[max_bin];
      if (out[m - 1] <= mx) out[m++] = nextafterf(mx, INFINITY);
    }
    ncut[f] = m;
    P.mode = MODE_DONE;
  }
}

// K2: local bin of every entry; categorical exact match (unseen -> 0). The
// histogram codes go to row r at position rpos[f] (rbase[f] + local bin, or
// rmiss[f] when missing); the feature-major copy holds the local bin itself,
// MISSING_BIN when missing.
// The local bin of value v of a feature whose `len` cuts start at `cuts`:
// bin_of (quantile.rs:166-181), the categorical form an exact match,
// MISSING_BIN for a missing value.
__device__ __forceinline__ uint16_t local_bin(float v, bool miss, const float* cuts, uint32_t len, bool cat) {
  if (miss) return MISSING_BIN;
  if (cat) {
    uint32_t lo = 0, hi = len, found = 0;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      const float c = cuts[mid];
      if (c < v) lo = mid + 1;
      else if (c > v) hi = mid;
      else { found = mid; break; }
    }
    return (uint16_t)found;
  }
  uint32_t lo = 0, hi = len;  // partition_point(c <= v)
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (cuts[mid] <= v) lo = mid + 1; else hi = mid;
  }
  return (uint16_t)(lo < len - 1 ? lo : len - 1);
}

// A block bins BIN_TILES tiles of BIN_TR rows x BIN_TF features. It first
// copies its features' cuts into shared memory (when they fit in
// `sh_cut_cap` floats; else it searches them in global memory), so the
// binary searches read shared memory. Per tile it reads the rows' values in
// row order, writes the row-major codes row by row, and writes the
// feature-major local bins column by column from a shared-memory copy of
// the tile, so both layouts are stored with coalesced writes.
constexpr int BIN_TR = 64, BIN_TF = 32, BIN_TILES = 16, BIN_THREADS = 256;
template <typename Code>
__global__ void __launch_bounds__(BIN_THREADS) k_bin(const float* __restrict__ X, size_t n, int F, size_t Fp,
                                             float missing, const uint32_t* __restrict__ foff,
                                             const float* __restrict__ cuts,
                                             const uint8_t* __restrict__ is_cat,
                                             const int* __restrict__ rpos,
                                             const int* __restrict__ rbase,
                                             const int* __restrict__ rmiss,
                                             Code* __restrict__ bins,
                                             uint16_t* __restrict__ bins_col, int sh_cut_cap) {
  extern __shared__ float s_cut[];
  __shared__ uint16_t tl[BIN_TF][BIN_TR + 2];  // local bins [feature][row]
  __shared__ uint32_t s_off[BIN_TF + 1];
  __shared__ int s_pos[BIN_TF], s_base[BIN_TF], s_miss[BIN_TF];
  __shared__ uint8_t s_cat[BIN_TF];
  const bool miss_nan = isnan(missing);
  const int f0 = blockIdx.y * BIN_TF;
  const int nf = min(BIN_TF, F - f0);
  const uint32_t c0 = foff[f0], ncut = foff[f0 + nf] - c0;
  const bool sh = ncut <= (uint32_t)sh_cut_cap;
  for (int i = threadIdx.x; i <= nf; i += blockDim.x) s_off[i] = foff[f0 + i] - c0;
  for (int i = threadIdx.x; i < nf; i += blockDim.x) {
    s_pos[i] = rpos[f0 + i];
    s_base[i] = rbase[f0 + i];
    s_miss[i] = rmiss[f0 + i];
    s_cat[i] = is_cat[f0 + i];
  }
  if (sh)
    for (uint32_t i = threadIdx.x; i < ncut; i += blockDim.x) s_cut[i] = cuts[c0 + i];
  __syncthreads();
  const float* cb = sh ? s_cut : cuts + c0;
  for (int t = 0; t < BIN_TILES; ++t) {
    const size_t r0 = ((size_t)blockIdx.x * BIN_TILES + t) * BIN_TR;
    if (r0 >= n) break;
    const int nr = (int)min((size_t)BIN_TR, n - r0);
    // all of a thread's values of the tile are loaded before the searches,
    // so its loads are in flight together
    constexpr int PER = BIN_TR * BIN_TF / BIN_THREADS;
    float v[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int i = threadIdx.x + u * BIN_THREADS;
      const int rr = i / BIN_TF, ff = i % BIN_TF;
      v[u] = (rr < nr && ff < nf) ? __ldg(X + (r0 + rr) * (size_t)F + f0 + ff) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int i = threadIdx.x + u * BIN_THREADS;
      const int rr = i / BIN_TF, ff = i % BIN_TF;
      if (rr < nr && ff < nf) {
        const size_t r = r0 + rr;
        const uint32_t s0 = s_off[ff];
        const uint16_t local =
            local_bin(v[u], is_missing_d(v[u], missing, miss_nan), cb + s0, s_off[ff + 1] - s0, s_cat[ff] != 0);
        tl[ff][rr] = local;
        bins[r * Fp + s_pos[ff]] = local == MISSING_BIN ? (Code)s_miss[ff] : (Code)(s_base[ff] + (int)local);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < BIN_TR * BIN_TF; i += blockDim.x) {
      const int ff = i / BIN_TR, rr = i % BIN_TR;
      if (rr < nr && ff < nf) bins_col[(size_t)(f0 + ff) * n + r0 + rr] = tl[ff][rr];
    }
    __syncthreads();
  }
}

}  // namespace

namespace {

// Indexes with fewer rows take the default layout without timing.
constexpr size_t TUNE_MIN_ROWS = 200000;

// Shape bucket of the autotuner: device, features, most bins of a feature,
// log2 of the rows, categorical features present.
struct TuneKey {
  int device, F, max_bins, log2_rows, categorical;
  bool operator<(const TuneKey& o) const {
    return std::tie(device, F, max_bins, log2_rows, categorical) <
           std::tie(o.device, o.F, o.max_bins, o.log2_rows, o.categorical);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, HistChoice> g_tuned;

}  // namespace

int bin_codes(sb_ctx* ctx, const float* d_X, Ghist* g);

int ghist_build(sb_ctx* ctx, const float* d_X, size_t n, size_t F, const uint8_t* h_ftypes,
                float missing, int max_bin, Ghist* g) {
  SB_REQUIRE(n > 0 && F > 0, SB_ERR_INVALID_ARG, "empty dataset: zero rows or columns");
  SB_REQUIRE(max_bin >= 2 && max_bin <= 1024, SB_ERR_UNSUPPORTED,
             "max_bin must be in [2, 1024] on the GPU, got %d", max_bin);
  SB_REQUIRE(n < (size_t)UNSAMPLED, SB_ERR_UNSUPPORTED, "at most 2^31-1 rows");
  SB_REQUIRE(F <= 4096, SB_ERR_UNSUPPORTED, "at most 4096 features");
  g->ctx = ctx;
  g->n = n;
  g->F = F;
  g->Fp = (F + 7) / 8 * 8;
  g->max_bin = max_bin;
  g->missing = missing;
  cudaStream_t st = ctx->stream;

  std::vector<uint8_t> hcat(F, 0);
  bool any_cat = false;
  if (h_ftypes)
    for (size_t f = 0; f < F; ++f) {
      hcat[f] = h_ftypes[f] == SB_FEAT_CATEGORICAL ? 1 : 0;
      any_cat |= hcat[f] != 0;
    }
  // slots per feature and level: <= max_bin + 1 wanted ranks, or <= max_bin
  // distinct values, or <= MAX_CAT_BINS categories
  const int S = std::max(max_bin + 1, any_cat ? MAX_CAT_BINS + 1 : 0);
  SB_TRY(g->is_cat.alloc(ctx, F));
  SB_CUDA(cudaMemcpyAsync(g->is_cat.p, hcat.data(), F, cudaMemcpyHostToDevice, st));

  DBuf<unsigned int> cnt1, cnt2, cnt3;
  DBuf<short> map2, map3;
  DBuf<uint32_t> slot_prefix;
  DBuf<unsigned long long> slot_base, trank;
  DBuf<float> cut_tmp;
  DBuf<int> ncut;
  DBuf<FPlan> plan;
  SB_TRY(cnt1.alloc(ctx, F * 2048));
  SB_TRY(cnt2.alloc(ctx, F * (size_t)S * 2048));
  SB_TRY(cnt3.alloc(ctx, F * (size_t)S * 1024));
  SB_TRY(map2.alloc(ctx, F * 2048));
  SB_TRY(map3.alloc(ctx, F * (size_t)S * 2048));
  SB_TRY(slot_prefix.alloc(ctx, 2 * F * (size_t)S));
  SB_TRY(slot_base.alloc(ctx, 2 * F * (size_t)S));
  SB_TRY(trank.alloc(ctx, F * (size_t)S));
  SB_TRY(cut_tmp.alloc(ctx, F * (size_t)(S + 1)));
  SB_TRY(ncut.alloc(ctx, F));
  SB_TRY(plan.alloc(ctx, F));
  SB_CUDA(cudaMemsetAsync(cnt1.p, 0, cnt1.bytes(), st));
  SB_CUDA(cudaMemsetAsync(cnt2.p, 0, cnt2.bytes(), st));
  SB_CUDA(cudaMemsetAsync(cnt3.p, 0, cnt3.bytes(), st));
  SB_CUDA(cudaMemsetAsync(map2.p, 0xFF, map2.bytes(), st));
  SB_CUDA(cudaMemsetAsync(map3.p, 0xFF, map3.bytes(), st));
  SB_CUDA(cudaMemsetAsync(plan.p, 0, plan.bytes(), st));

  dim3 cgrid((unsigned)((n + TILE_R - 1) / TILE_R), (unsigned)((F + TILE_F - 1) / TILE_F));
  SB_REQUIRE(cgrid.x <= 0x7FFFFFFFu, SB_ERR_UNSUPPORTED, "too many rows");
  {  // level 1: shared counters; about 8 blocks per SM over all feature groups
    const size_t groups = (F + C1_FEATS - 1) / C1_FEATS;
    size_t nrb = std::max<size_t>(1, ((size_t)8 * ctx->num_sms + groups - 1) / groups);
    nrb = std::min(nrb, (n + 1023) / 1024);
    const size_t rpb = (n + nrb - 1) / nrb;
    nrb = (n + rpb - 1) / rpb;
    SB_LAUNCH(ctx, k_cuts_count1, dim3((unsigned)nrb, (unsigned)groups), 256, 0, d_X, n, (int)F, missing, rpb,
              cnt1.p, plan.p);
  }
  SB_LAUNCH(ctx, k_cuts_plan<1>, (unsigned)F, 1024, 0, (int)F, S, max_bin, g->is_cat.p, cnt1.p,
            cnt2.p, cnt3.p, map2.p, map3.p, slot_prefix.p, slot_base.p, trank.p, cut_tmp.p, ncut.p,
            plan.p);
  SB_LAUNCH(ctx, k_cuts_count<2>, cgrid, COUNT_THREADS, 0, d_X, n, (int)F, missing, S, cnt2.p, cnt3.p,
            map2.p, map3.p, plan.p);
  SB_LAUNCH(ctx, k_cuts_plan<2>, (unsigned)F, 1024, 0, (int)F, S, max_bin, g->is_cat.p, cnt1.p,
            cnt2.p, cnt3.p, map2.p, map3.p, slot_prefix.p, slot_base.p, trank.p, cut_tmp.p, ncut.p,
            plan.p);
  SB_LAUNCH(ctx, k_cuts_count<3>, cgrid, COUNT_THREADS, 0, d_X, n, (int)F, missing, S, cnt2.p, cnt3.p,
            map2.p, map3.p, plan.p);
  SB_LAUNCH(ctx, k_cuts_plan<3>, (unsigned)F, 1024, 0, (int)F, S, max_bin, g->is_cat.p, cnt1.p,
            cnt2.p, cnt3.p, map2.p, map3.p, slot_prefix.p, slot_base.p, trank.p, cut_tmp.p, ncut.p,
            plan.p);

  std::vector<int> h_ncut(F);
  std::vector<float> h_tmp(F * (size_t)(S + 1));
  std::vector<FPlan> h_plan(F);
  SB_CUDA(cudaMemcpyAsync(h_ncut.data(), ncut.p, F * sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaMemcpyAsync(h_tmp.data(), cut_tmp.p, cut_tmp.bytes(), cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaMemcpyAsync(h_plan.data(), plan.p, plan.bytes(), cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  for (size_t f = 0; f < F; ++f) {
    SB_REQUIRE(h_plan[f].err != 1, SB_ERR_INVALID_ARG,
               "feature %zu holds NaN while the missing sentinel is %g (the reference's sort "
               "panics on NaN here)", f, (double)missing);
    SB_REQUIRE(h_plan[f].err != 2, SB_ERR_UNSUPPORTED,
               "categorical feature %zu has more than %d categories", f, MAX_CAT_BINS);
    SB_REQUIRE(h_plan[f].err == 0, SB_ERR_CUDA, "internal cut planning error on feature %zu", f);
  }
  g->h_foff.assign(F + 1, 0);
  g->h_cuts.clear();
  g->h_is_cat = hcat;
  g->max_feature_bins = 0;
  g->has_categorical = 0;
  for (size_t f = 0; f < F; ++f) {
    int m = h_ncut[f];
    SB_REQUIRE(m >= 1 && m <= S + 1, SB_ERR_CUDA, "internal cut count error on feature %zu", f);
    g->h_cuts.insert(g->h_cuts.end(), h_tmp.begin() + f * (S + 1), h_tmp.begin() + f * (S + 1) + m);
    g->h_foff[f + 1] = (uint32_t)g->h_cuts.size();
    g->max_feature_bins = std::max(g->max_feature_bins, m);
    if (hcat[f]) g->has_categorical = 1;
  }
  return ghist_bin(ctx, d_X, g);
}

// The rest of the index from the host cuts (h_foff, h_cuts, h_is_cat): device
// copies of the cuts, the histogram layout and the bin codes of every entry.
int ghist_bin(sb_ctx* ctx, const float* d_X, Ghist* g) {
  const size_t n = g->n, F = g->F;
  cudaStream_t st = ctx->stream;
  g->total_bins = g->h_cuts.size();
  g->max_feature_bins = 0;
  g->has_categorical = 0;
  for (size_t f = 0; f < F; ++f) {
    g->max_feature_bins = std::max(g->max_feature_bins, (int)(g->h_foff[f + 1] - g->h_foff[f]));
    if (g->h_is_cat[f]) g->has_categorical = 1;
  }
  if (!g->is_cat.p) {
    SB_TRY(g->is_cat.alloc(ctx, F));
    SB_CUDA(cudaMemcpyAsync(g->is_cat.p, g->h_is_cat.data(), F, cudaMemcpyHostToDevice, st));
  }
  SB_TRY(g->foff.alloc(ctx, F + 1));
  SB_TRY(g->cuts.alloc(ctx, g->total_bins));
  SB_CUDA(cudaMemcpyAsync(g->foff.p, g->h_foff.data(), (F + 1) * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(g->cuts.p, g->h_cuts.data(), g->total_bins * 4, cudaMemcpyHostToDevice, st));

  // the histogram layout fixes the row codes: the default choice, or the
  // fastest candidate for this shape (timed once per shape and device)
  HistChoice choice;
  SB_TRY(hist_default_choice(ctx, g, &choice));
  const char* at = std::getenv("SB_HIST_AUTOTUNE");
  const bool tune = !std::getenv("SB_HIST_LAYOUT") && !std::getenv("SB_HIST_ROWS") &&
                    !(at && std::strcmp(at, "0") == 0) && n >= TUNE_MIN_ROWS;
  const std::vector<HistChoice> cands = tune ? hist_candidates(ctx, g) : std::vector<HistChoice>();
  if (tune && cands.size() > 1) {
    int lg = 0;
    while ((size_t(2) << lg) <= n) ++lg;
    const TuneKey key{ctx->device, (int)F, g->max_feature_bins, lg, g->has_categorical};
    bool cached = false;
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      auto it = g_tuned.find(key);
      if (it != g_tuned.end()) {
        choice = it->second;
        cached = true;
      }
    }
    if (!cached) {
      float best_t = 1e30f;
      HistChoice best = choice, last{-1, -1};
      for (const HistChoice& c : cands) {
        SB_TRY(hist_prepare(ctx, g, c));
        SB_TRY(bin_codes(ctx, d_X, g));
        float t = 0.0f;
        SB_TRY(hist_time(ctx, g, &t));
        last = c;
        if (t < best_t) {
          best_t = t;
          best = c;
        }
      }
      {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tuned[key] = best;
      }
      if (best.layout == last.layout && best.slots == last.slots && best.rl == last.rl) return SB_OK;  // built already
      choice = best;
    }
  }
  SB_TRY(hist_prepare(ctx, g, choice));
  return bin_codes(ctx, d_X, g);
}

// The bin codes of every entry for the planned layout (and the feature-major
// local bins).
int bin_codes(sb_ctx* ctx, const float* d_X, Ghist* g) {
  const size_t n = g->n, F = g->F;
  const float missing = g->missing;
  cudaStream_t st = ctx->stream;
  // feature-major codes are the local bins themselves
  const std::vector<int> zeros(F, 0), miss(F, (int)MISSING_BIN);
  SB_TRY(g->fbase.alloc(ctx, F));
  SB_TRY(g->fmiss.alloc(ctx, F));
  SB_CUDA(cudaMemcpyAsync(g->fbase.p, zeros.data(), F * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(g->fmiss.p, miss.data(), F * 4, cudaMemcpyHostToDevice, st));
  DBuf<int>& rpos = g->rpos;
  DBuf<int>& rbase = g->rbase;
  DBuf<int>& rmiss = g->rmiss;
  SB_TRY(rpos.alloc(ctx, F));
  SB_TRY(rbase.alloc(ctx, F));
  SB_TRY(rmiss.alloc(ctx, F));
  SB_CUDA(cudaMemcpyAsync(rpos.p, g->h_rpos.data(), F * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(rbase.p, g->h_rbase.data(), F * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(rmiss.p, g->h_rmiss.data(), F * 4, cudaMemcpyHostToDevice, st));
  SB_TRY(g->bins_col.alloc(ctx, n * F));
  const size_t rows_per_block = (size_t)BIN_TR * BIN_TILES;
  const dim3 bgrid((unsigned)((n + rows_per_block - 1) / rows_per_block), (unsigned)((F + BIN_TF - 1) / BIN_TF));
  // the blocks' cuts go to shared memory up to the default 48 KB per block
  // (less the static tile arrays); wider groups search them in global memory
  const int sh_cap = (int)((48 * 1024 - 6 * 1024) / sizeof(float));
  size_t sh_cuts = 0;
  for (size_t f0 = 0; f0 < F; f0 += BIN_TF) {
    const size_t c = g->h_foff[std::min(F, f0 + BIN_TF)] - g->h_foff[f0];
    if (c <= (size_t)sh_cap) sh_cuts = std::max(sh_cuts, c);
  }
  const size_t bsm = sh_cuts * sizeof(float);
  if (g->code_bytes == 1) {  // u8 codes: the u16 matrix is not kept
    g->bins.release();
    SB_TRY(g->bins8.alloc(ctx, n * g->Fp));
    SB_CUDA(cudaMemsetAsync(g->bins8.p, 0xFF, g->bins8.bytes(), st));  // unused positions: 0xFF
    SB_LAUNCH(ctx, k_bin<uint8_t>, bgrid, BIN_THREADS, bsm, d_X, n, (int)F, g->Fp, missing, g->foff.p, g->cuts.p,
              g->is_cat.p, rpos.p, rbase.p, rmiss.p, g->bins8.p, g->bins_col.p, (int)sh_cuts);
  } else {
    g->bins8.release();
    SB_TRY(g->bins.alloc(ctx, n * g->Fp));
    SB_CUDA(cudaMemsetAsync(g->bins.p, 0xFF, g->bins.bytes(), st));  // unused positions: 0xFFFF
    SB_LAUNCH(ctx, k_bin<uint16_t>, bgrid, BIN_THREADS, bsm, d_X, n, (int)F, g->Fp, missing, g->foff.p, g->cuts.p,
              g->is_cat.p, rpos.p, rbase.p, rmiss.p, g->bins.p, g->bins_col.p, (int)sh_cuts);
  }
  SB_CUDA(cudaStreamSynchronize(st));  // the host vectors are released on return
  return SB_OK;
}

}  // namespace sb

extern "C" {

int sb_ghist_create_device(sb_ctx* ctx, const float* d_X, size_t n_rows, size_t n_cols,
                           const uint8_t* feature_types, float missing, int max_bin, sb_ghist** out) {
  SB_REQUIRE(ctx && d_X && out, SB_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  SB_CUDA(cudaSetDevice(ctx->device));
  sb_ghist* g = new sb_ghist;
  int s = sb::ghist_build(ctx, d_X, n_rows, n_cols, feature_types, missing, max_bin, g);
  if (s != SB_OK) {
    delete g;
    return s;
  }
  *out = g;
  return SB_OK;
}

int sb_ghist_create(sb_ctx* ctx, const float* X, size_t n_rows, size_t n_cols,
                    const uint8_t* feature_types, float missing, int max_bin, sb_ghist** out) {
  SB_REQUIRE(ctx && X && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_REQUIRE(n_rows > 0 && n_cols > 0, SB_ERR_INVALID_ARG, "empty dataset: zero rows or columns");
  *out = nullptr;
  SB_CUDA(cudaSetDevice(ctx->device));
  sb::DBuf<float> dX;
  SB_TRY(dX.alloc(ctx, n_rows * n_cols));
  SB_CUDA(cudaMemcpyAsync(dX.p, X, dX.bytes(), cudaMemcpyHostToDevice, ctx->stream));
  return sb_ghist_create_device(ctx, dX.p, n_rows, n_cols, feature_types, missing, max_bin, out);
}

int sb_ghist_destroy(sb_ghist* g) {
  if (g) {
    cudaSetDevice(g->ctx->device);
    delete g;
  }
  return SB_OK;
}

int sb_ghist_info(const sb_ghist* g, size_t* n_rows, size_t* n_cols, size_t* total_bins) {
  SB_REQUIRE(g != nullptr, SB_ERR_INVALID_ARG, "ghist is NULL");
  if (n_rows) *n_rows = g->n;
  if (n_cols) *n_cols = g->F;
  if (total_bins) *total_bins = g->total_bins;
  return SB_OK;
}

int sb_ghist_cuts(const sb_ghist* g, uint32_t* feature_offset, float* cut_values, uint8_t* is_cat) {
  SB_REQUIRE(g != nullptr, SB_ERR_INVALID_ARG, "ghist is NULL");
  if (feature_offset) std::memcpy(feature_offset, g->h_foff.data(), (g->F + 1) * 4);
  if (cut_values) std::memcpy(cut_values, g->h_cuts.data(), g->total_bins * 4);
  if (is_cat) std::memcpy(is_cat, g->h_is_cat.data(), g->F);
  return SB_OK;
}

int sb_ghist_bins(const sb_ghist* g, uint16_t* local_bins) {
  SB_REQUIRE(g && local_bins, SB_ERR_INVALID_ARG, "NULL argument");
  SB_CUDA(cudaSetDevice(g->ctx->device));
  std::vector<uint16_t> col(g->n * g->F);  // feature-major local bins
  SB_CUDA(cudaMemcpyAsync(col.data(), g->bins_col.p, col.size() * 2, cudaMemcpyDeviceToHost, g->ctx->stream));
  SB_CUDA(cudaStreamSynchronize(g->ctx->stream));
  for (size_t f = 0; f < g->F; ++f)
    for (size_t r = 0; r < g->n; ++r) local_bins[r * g->F + f] = col[f * g->n + r];
  return SB_OK;
}

int sb_ghist_layout(const sb_ghist* g, int* layout, int* code_bytes, size_t* row_stride,
                    int* rows_per_instruction) {
  SB_REQUIRE(g != nullptr, SB_ERR_INVALID_ARG, "ghist is NULL");
  if (layout) *layout = g->layout;
  if (code_bytes) *code_bytes = g->code_bytes;
  if (row_stride) *row_stride = g->Fp;
  if (rows_per_instruction) *rows_per_instruction = g->layout == sb::HIST_LAYOUT_TILED ? 1 << g->tiled_rl : 1;
  return SB_OK;
}

int sb_ghist_codes(const sb_ghist* g, void* codes) {
  SB_REQUIRE(g && codes, SB_ERR_INVALID_ARG, "NULL argument");
  SB_CUDA(cudaSetDevice(g->ctx->device));
  const void* src = g->code_bytes == 1 ? (const void*)g->bins8.p : (const void*)g->bins.p;
  SB_CUDA(cudaMemcpyAsync(codes, src, g->n * g->Fp * (size_t)g->code_bytes, cudaMemcpyDeviceToHost,
                          g->ctx->stream));
  SB_CUDA(cudaStreamSynchronize(g->ctx->stream));
  return SB_OK;
}

}  // extern "C"
