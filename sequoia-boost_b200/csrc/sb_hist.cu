// sb_hist.cu — gradient histogram construction (K4) and subtraction (K5).
//
// Replaces CpuBackend::build / accumulate (tree/hist/mod.rs:58-119) and
// `subtracted` / HistogramBackend::subtract (:25-28, :38-44).
//
// Design: a persistent grid (one CTA of 1024 threads per SM) splits the
// concatenated rows of every node to build (all frontier nodes of all class
// trees in one launch) evenly over CTAs (fewer CTAs for a launch known to
// hold few rows). A CTA keeps one node's histogram for one feature tile in
// shared memory, walks its rows in small batches per warp (the low lanes load
// the row ids ahead and the gradient pairs, shuffles hand them to the warp;
// TILED keeps two batches in flight), adds every code of a row into the
// shared partial, and flushes the non-zero entries to the node's HBM
// histogram with global atomics when it moves to the next piece.
//   codes  TILED layout: lane l reads features 4l..4l+3 of the tile (one
//          8-byte load per row) and a code is the entry's index in the tile's
//          partial, where a feature's bins are contiguous. LANES layout: each
//          tile gives lane l `S` (1, 2 or 4) code positions of the row, packed
//          with features so that every lane's entries fit its own column, and
//          entry e of lane l sits at word e * 32 + l: the 32 lanes of a warp
//          always add into 32 different banks.
//   sums   FP32 form: f32 shared atomics, f64 node histograms. FIXED form:
//          gradients rounded to |q| <= 2^bits with a per-round power-of-two
//          scale; one int32 and one uint32 shared atomic per entry, exact
//          because a CTA flushes at least every fixed_rows_per_flush(bits)
//          rows; int64 node histograms (order independent).
// Each feature also owns one extra "missing" bin (index total_bins + f), so a
// node's missing-value statistics are summed directly instead of being
// recovered as total - present.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "sb_internal.cuh"

namespace sb {
namespace {

constexpr int HIST_THREADS = 1024;
constexpr int MAX_TILE_FEATURES = 128;  // 4 features per lane
constexpr int ROWS_PER_WARP = 8;        // LANES: rows per warp batch
constexpr int TILED_ROWS = 4;           // TILED: rows per warp batch (two batches in flight)

struct HistDev {
  const uint16_t* bins;  // u16 codes, or null with u8 codes in bins8
  const uint8_t* bins8;
  const uint32_t* foff;
  size_t Fp;             // row stride of bins (u16)
  const int* ent_gbin;   // LANES: (entry, lane) -> histogram bin, per tile; u8 TILED: entry -> bin
  const int* slot_feat;  // LANES: feature of each code position of a row
  size_t n;              // gradient column stride
  int total_bins;
  const void* gpair;
  const HistItem* items;
  const uint64_t* prefix;
  const int* count;
  const FeatureTile* tiles;
  int ntiles;
  uint32_t flush_rows;   // FIXED: max rows per shared partial
  unsigned long long* rows_done;  // sampled rows accumulated (or null)
  const uint32_t* pool_mask;      // [K][FW] features to accumulate (or null: all)
  int FW;
  int rl;                         // TILED: log2 of the rows one warp instruction covers
  uint32_t min_units;             // fewest (row, tile) units per active CTA (0: all CTAs)
};

__device__ __forceinline__ int find_item(const uint64_t* prefix, int count, uint64_t pos) {
  int lo = 0, hi = count;  // last i with prefix[i] <= pos
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (prefix[mid] <= pos) lo = mid; else hi = mid;
  }
  return lo;
}

// One addition into each plane of the shared partial, at the 32-bit shared
// address `a` (g plane) and `a + hoff` (h plane), with `red` (no value
// returned). FIXED: int32 g and uint32 h; FP32: f32 bits.
template <bool FIXED>
__device__ __forceinline__ void add_pair(unsigned a, unsigned hoff, uint32_t vg, uint32_t vh) {
  if (FIXED) {
    asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(a), "r"(vg));
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a + hoff), "r"(vh));
  } else {
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a), "f"(__uint_as_float(vg)));
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a + hoff), "f"(__uint_as_float(vh)));
  }
}

// The shared partial is two planes of nent 32-bit words, g then h (FIXED:
// int32 / uint32 integers; FP32: floats), so a warp's atomics spread over all
// 32 banks. Every entry costs one add into each plane.
// RL >= 0: the rows per warp instruction (as log2) fixed at compile time;
// RL < 0: read from the launch description.
// U8: one-byte codes, the feature's local bin (its bin count when missing);
// a feature's bins and its missing entry are contiguous in the partial, so an
// entry's address is the feature's first entry plus the code, and the flush
// maps entries to histogram bins through the tile's table (ent_gbin).
template <bool U8> struct CodeWord { using T = uint2; };     // 4 u16 codes
template <> struct CodeWord<true> { using T = uint32_t; };   // 4 u8 codes

template <bool FIXED, int RL, bool U8>
__device__ __forceinline__ void hist_tiled_body(const HistDev& a, unsigned bx, unsigned gdx) {
  using CW = typename CodeWord<U8>::T;
  extern __shared__ unsigned long long sh_u64[];
  unsigned* sh_g = reinterpret_cast<unsigned*>(sh_u64);
  __shared__ double s_tot_d[2];
  __shared__ unsigned long long s_tot_u[2];

  const int count = *a.count;
  if (count <= 0) return;
  const uint64_t W = a.prefix[count];
  if (W == 0) return;
  const uint64_t U = W * (uint64_t)a.ntiles;
  // with a.min_units set (batched jobs, whose launches overlap), a launch
  // holding few rows uses fewer CTAs of at least that many (row, tile) units,
  // so that zeroing and flushing a shared partial is paid for by enough rows;
  // the other CTAs return. A lone launch spreads its rows over every CTA.
  const uint64_t mu = a.min_units ? a.min_units : 1;
  const uint64_t act = min((uint64_t)gdx, max((uint64_t)1, (U + mu - 1) / mu));
  if (bx >= act) return;
  const uint64_t lo = U * bx / act, hi = U * (bx + 1) / act;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;

  uint64_t u = lo;
  while (u < hi) {
    const int t = (int)(u / W);
    const uint64_t pos = u - (uint64_t)t * W;
    const int it = find_item(a.prefix, count, pos);
    const HistItem item = a.items[it];
    const uint64_t item_lo = a.prefix[it], item_hi = a.prefix[it + 1];
    uint64_t piece_hi_u = (uint64_t)t * W + item_hi;
    if (piece_hi_u > hi) piece_hi_u = hi;
    uint64_t n_pos = piece_hi_u - u;
    if (FIXED && n_pos > a.flush_rows) n_pos = a.flush_rows;
    const uint32_t pbeg = item.begin + (uint32_t)(pos - item_lo);
    const uint32_t pend = pbeg + (uint32_t)n_pos;
    const FeatureTile tile = a.tiles[t];
    const int nf = tile.f1 - tile.f0;
    const int nent = tile.nbins + nf;
    unsigned* sh_h = sh_g + nent;
    const unsigned sh_base = (unsigned)__cvta_generic_to_shared(sh_g), hoff = 4u * (unsigned)nent;
    const bool want_total = item.root && t == 0;

    // A warp instruction covers 2^rl rows: lane `lane` works on row slot
    // lane >> (5 - rl) of it and owns the 4 consecutive features
    // f0 + 4 * grp .. +3 of the tile, grp = its lane within the row's group
    // (only features of the tree's column pool are added); one 8-byte load
    // per row fetches their 4 bins. Tiles start at multiples of 4, hold at
    // most 4 * 32 >> rl features, and rows are padded to a multiple of 8
    // bins, so the load is aligned and stays inside the row.
    const int rl = RL >= 0 ? RL : a.rl;
    const int grp = lane & ((32 >> rl) - 1), rsub = lane >> (5 - rl);
    const int fl0 = 4 * grp;
    const bool lane_on = fl0 < nf;
    bool fon[4];
    unsigned eb[4];  // U8: shared address of each owned feature's first entry
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int fl = fl0 + j;
      const int f = tile.f0 + fl;
      bool on = fl < nf;
      eb[j] = sh_base;
      if (U8 && on) eb[j] = sh_base + 4u * (a.foff[f] - (unsigned)tile.bin0 + (unsigned)fl);
      if (on && a.pool_mask && !((a.pool_mask[(size_t)item.k * a.FW + (f >> 5)] >> (f & 31)) & 1u)) on = false;
      fon[j] = on;
    }
    for (int i = threadIdx.x; i < 2 * nent; i += blockDim.x) sh_g[i] = 0u;
    if (threadIdx.x < 2) {
      s_tot_d[threadIdx.x] = 0.0;
      s_tot_u[threadIdx.x] = 0ull;
    }
    __syncthreads();

    // Rows go through a warp in batches of TILED_ROWS << rl, double-buffered:
    // the codes and gradient pairs of the next batch are loaded before the
    // adds of the current one, so the gather is in flight while the shared
    // atomics issue. Lane i < the batch size holds row i of a batch (its id,
    // loaded two batches ahead, and its gradient pair); the other lanes get
    // them by shuffles. Step q of a batch covers its rows (q << rl) + slot,
    // and every lane loads its 4 codes of its row.
    double tg = 0.0, th = 0.0;
    long long tqg = 0;
    unsigned long long tqh = 0;
    unsigned int nsampled = 0;
    const size_t gcol = (size_t)item.k * a.n;
    const uint16_t* bins_tile = U8 ? nullptr : a.bins + tile.f0 + fl0;
    const uint8_t* bins8_tile = U8 ? a.bins8 + tile.f0 + fl0 : nullptr;
    constexpr int R = TILED_ROWS;
    const uint32_t B = (uint32_t)R << rl;  // rows per batch (<= 32)
    const uint32_t stride = (uint32_t)nwarps * B;
    // the gradient pair of the batch at p (lanes < its rows), counted into the totals
    auto load_grad = [&](uint32_t rid, uint32_t nr, uint32_t& g, uint32_t& h) {
      g = 0u;
      h = 0u;
      if (lane < (int)nr) {
        if (FIXED) {
          const unsigned long long pk = reinterpret_cast<const unsigned long long*>(a.gpair)[gcol + rid];
          g = (uint32_t)(pk >> 32);
          h = (uint32_t)(pk & 0xFFFFFFFFull);
        } else {
          const float2 v = reinterpret_cast<const float2*>(a.gpair)[gcol + rid];
          g = __float_as_uint(v.x);
          h = __float_as_uint(v.y);
        }
        nsampled++;
        if (want_total) {
          if (FIXED) {
            tqg += (int)g;
            tqh += h;
          } else {
            tg += (double)__uint_as_float(g);
            th += (double)__uint_as_float(h);
          }
        }
      }
    };
    // the codes of the batch's rows (the lists hold sampled rows only)
    auto load_codes = [&](uint32_t rid, uint32_t nr, CW (&bv)[R]) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const uint32_t src = ((uint32_t)q << rl) + (uint32_t)rsub;
        const uint32_t id = __shfl_sync(0xFFFFFFFFu, rid, src);
        if constexpr (U8)
          bv[q] = (src < nr && lane_on) ? __ldg(reinterpret_cast<const uint32_t*>(bins8_tile + (size_t)id * a.Fp)) : 0u;
        else
          bv[q] = (src < nr && lane_on) ? __ldg(reinterpret_cast<const uint2*>(bins_tile + (size_t)id * a.Fp))
                                        : make_uint2(0u, 0u);
      }
    };
    uint32_t p = pbeg + warp * B;
    uint32_t rid_c = ((uint32_t)lane < B && p + lane < pend) ? item.rows[p + lane] : 0u;
    uint32_t nrow_c = p < pend ? min(pend - p, B) : 0u;
    uint32_t g_c, h_c;
    CW bv_c[R];
    load_grad(rid_c, nrow_c, g_c, h_c);
    load_codes(rid_c, nrow_c, bv_c);
    uint32_t rid_n = ((uint32_t)lane < B && p + stride + lane < pend) ? item.rows[p + stride + lane] : 0u;
    for (; p < pend; p += stride) {
      const uint32_t pn = p + stride;
      const uint32_t nrow_n = pn < pend ? min(pend - pn, B) : 0u;
      uint32_t g_n, h_n;
      CW bv_n[R];
      load_grad(rid_n, nrow_n, g_n, h_n);
      load_codes(rid_n, nrow_n, bv_n);
      const uint32_t rid_nn =
          ((uint32_t)lane < B && pn + stride + lane < pend) ? item.rows[pn + stride + lane] : 0u;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const uint32_t src = ((uint32_t)q << rl) + (uint32_t)rsub;
        const uint32_t vg = __shfl_sync(0xFFFFFFFFu, g_c, src);
        const uint32_t vh = __shfl_sync(0xFFFFFFFFu, h_c, src);
        if (((uint32_t)q << rl) >= nrow_c) break;  // no row of this step in any lane
        const bool row_on = src < nrow_c;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          unsigned addr;
          if constexpr (U8) {
            addr = eb[j] + 4u * ((bv_c[q] >> (8 * j)) & 0xFFu);  // the feature's entry of the local bin
          } else {
            const uint32_t w = j < 2 ? bv_c[q].x : bv_c[q].y;
            addr = sh_base + 4u * ((j & 1) ? (w >> 16) : (w & 0xFFFFu));  // the tile-relative code
          }
          if (fon[j] && row_on) add_pair<FIXED>(addr, hoff, vg, vh);
        }
      }
      g_c = g_n;
      h_c = h_n;
      nrow_c = nrow_n;
      rid_n = rid_nn;
#pragma unroll
      for (int q = 0; q < R; ++q) bv_c[q] = bv_n[q];
    }
    if (a.rows_done && t == 0 && nsampled) atomicAdd(a.rows_done, (unsigned long long)nsampled);
    if (want_total && (uint32_t)lane < B) {  // every lane that held rows of a batch
      if (FIXED) {
        atomicAdd(&s_tot_u[0], (unsigned long long)tqg);
        atomicAdd(&s_tot_u[1], tqh);
      } else {
        atomicAdd(&s_tot_d[0], tg);
        atomicAdd(&s_tot_d[1], th);
      }
    }
    __syncthreads();
    // flush the partial into the node's HBM histogram
    for (int i = threadIdx.x; i < nent; i += blockDim.x) {
      const int gi = U8 ? a.ent_gbin[tile.ent_off + i]
                        : (i < tile.nbins ? tile.bin0 + i : a.total_bins + tile.f0 + (i - tile.nbins));
      if (FIXED) {
        const long long gq = (long long)(int)sh_g[i];
        const unsigned long long hq = sh_h[i];
        unsigned long long* o = reinterpret_cast<unsigned long long*>(item.out) + 2 * (size_t)gi;
        if (gq) atomicAdd(o, (unsigned long long)gq);
        if (hq) atomicAdd(o + 1, hq);
      } else {
        const float g = __uint_as_float(sh_g[i]), h = __uint_as_float(sh_h[i]);
        double* o = reinterpret_cast<double*>(item.out) + 2 * (size_t)gi;
        if (g != 0.0f) atomicAdd(o, (double)g);
        if (h != 0.0f) atomicAdd(o + 1, (double)h);
      }
    }
    if (want_total && threadIdx.x == 0) {
      if (FIXED) {
        unsigned long long* o = reinterpret_cast<unsigned long long*>(item.total);
        atomicAdd(o, s_tot_u[0]);
        atomicAdd(o + 1, s_tot_u[1]);
      } else {
        double* o = reinterpret_cast<double*>(item.total);
        atomicAdd(o, s_tot_d[0]);
        atomicAdd(o + 1, s_tot_d[1]);
      }
    }
    __syncthreads();
    u += n_pos;
  }
}

template <bool FIXED, int RL, bool U8>
__global__ void __launch_bounds__(HIST_THREADS, 1) k_hist(HistDev a) {
  hist_tiled_body<FIXED, RL, U8>(a, blockIdx.x, gridDim.x);
}

// Many indexes' histogram launches as one (sb_train_many): the x-blocks are
// every job's own persistent grid laid end to end; block x belongs to job j
// when xoff[j] <= x < xoff[j + 1], and runs job j's launch description.
struct HistJobs {
  const HistDev* devs;   // [njobs]
  const unsigned* xoff;  // [njobs + 1]
  int njobs;
};

__device__ __forceinline__ int hist_job_of(const unsigned* xoff, int njobs, unsigned x) {
  int lo = 0, hi = njobs;  // the last job whose first block is <= x
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (xoff[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

template <bool FIXED, int RL, bool U8>
__global__ void __launch_bounds__(HIST_THREADS, 1) k_hist_jobs(HistJobs H) {
  const int j = hist_job_of(H.xoff, H.njobs, blockIdx.x);
  hist_tiled_body<FIXED, RL, U8>(H.devs[j], blockIdx.x - H.xoff[j], H.xoff[j + 1] - H.xoff[j]);
}

template <bool FIXED, bool U8>
const void* tiled_jobs_pick(int rl) {
  switch (rl) {
    case 1: return (const void*)k_hist_jobs<FIXED, 1, U8>;
    case 2: return (const void*)k_hist_jobs<FIXED, 2, U8>;
    case 3: return (const void*)k_hist_jobs<FIXED, 3, U8>;
    default: return (const void*)k_hist_jobs<FIXED, 0, U8>;
  }
}

template <bool FIXED, bool U8>
const void* tiled_pick(int rl) {
  switch (rl) {
    case 1: return (const void*)k_hist<FIXED, 1, U8>;
    case 2: return (const void*)k_hist<FIXED, 2, U8>;
    case 3: return (const void*)k_hist<FIXED, 3, U8>;
    default: return (const void*)k_hist<FIXED, 0, U8>;
  }
}

// The batched TILED kernel for a precision, rows per warp instruction (log2)
// and code width.
const void* tiled_jobs_kernel(bool fixed, int rl, bool u8) {
  if (u8) return fixed ? tiled_jobs_pick<true, true>(rl) : tiled_jobs_pick<false, true>(rl);
  return fixed ? tiled_jobs_pick<true, false>(rl) : tiled_jobs_pick<false, false>(rl);
}

// The TILED kernel for a precision, rows per warp instruction (log2) and
// code width.
const void* tiled_kernel(bool fixed, int rl, bool u8) {
  if (u8) return fixed ? tiled_pick<true, true>(rl) : tiled_pick<false, true>(rl);
  return fixed ? tiled_pick<true, false>(rl) : tiled_pick<false, false>(rl);
}

// LANES layout (see sb_internal.cuh): lane l of every warp owns the features
// in its `S` code positions of the tile, and entry e of lane l lives at word
// e * 32 + l of each plane, so every shared atomic instruction of a warp hits
// 32 different banks. A row costs one S x u16 load per lane and 2 * S shared
// atomic instructions per warp; the partial is flushed through the tile's
// (entry, lane) -> histogram-bin table.
template <int S> struct Codes;
template <> struct Codes<1> {
  using T = unsigned short;
  __device__ static T none() { return 0xFFFFu; }
  __device__ static int get(T v, int) { return (int)v; }
};
template <> struct Codes<2> {
  using T = unsigned int;
  __device__ static T none() { return 0xFFFFFFFFu; }
  __device__ static int get(T v, int s) { return (int)((v >> (16 * s)) & 0xFFFFu); }
};
template <> struct Codes<4> {
  using T = uint2;
  __device__ static T none() { return make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu); }
  __device__ static int get(T v, int s) {
    const unsigned w = s < 2 ? v.x : v.y;
    return (int)((w >> (16 * (s & 1))) & 0xFFFFu);
  }
};

template <bool FIXED, int S>
__global__ void __launch_bounds__(HIST_THREADS, 1) k_hist_lanes(HistDev a) {
  using C = Codes<S>;
  using CT = typename C::T;
  extern __shared__ unsigned long long sh_u64[];
  unsigned* sh_g = reinterpret_cast<unsigned*>(sh_u64);
  __shared__ double s_tot_d[2];
  __shared__ unsigned long long s_tot_u[2];

  const int count = *a.count;
  if (count <= 0) return;
  const uint64_t W = a.prefix[count];
  if (W == 0) return;
  const uint64_t U = W * (uint64_t)a.ntiles;
  const uint64_t lo = U * blockIdx.x / gridDim.x, hi = U * (blockIdx.x + 1) / gridDim.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;

  uint64_t u = lo;
  while (u < hi) {
    const int t = (int)(u / W);
    const uint64_t pos = u - (uint64_t)t * W;
    const int it = find_item(a.prefix, count, pos);
    const HistItem item = a.items[it];
    const uint64_t item_lo = a.prefix[it], item_hi = a.prefix[it + 1];
    uint64_t piece_hi_u = (uint64_t)t * W + item_hi;
    if (piece_hi_u > hi) piece_hi_u = hi;
    uint64_t n_pos = piece_hi_u - u;
    if (FIXED && n_pos > a.flush_rows) n_pos = a.flush_rows;
    const uint32_t pbeg = item.begin + (uint32_t)(pos - item_lo);
    const uint32_t pend = pbeg + (uint32_t)n_pos;
    const FeatureTile tile = a.tiles[t];
    const int words = 32 * tile.E;  // per plane
    unsigned* sh_h = sh_g + words;
    const unsigned sh_base = (unsigned)__cvta_generic_to_shared(sh_g), hoff = 4u * (unsigned)words;
    const bool want_total = item.root && t == 0;

    // the features of this lane's code positions that the tree's column pool
    // keeps (unused positions are off)
    const int slot0 = tile.slot_off + lane * S;
    bool fon[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int f = a.slot_feat[slot0 + s];
      bool on = f >= 0;
      if (on && a.pool_mask && !((a.pool_mask[(size_t)item.k * a.FW + (f >> 5)] >> (f & 31)) & 1u)) on = false;
      fon[s] = on;
    }
    for (int i = threadIdx.x; i < 2 * words; i += blockDim.x) sh_g[i] = 0u;
    if (threadIdx.x < 2) {
      s_tot_d[threadIdx.x] = 0.0;
      s_tot_u[threadIdx.x] = 0ull;
    }
    __syncthreads();

    double tg = 0.0, th = 0.0;
    long long tqg = 0;
    unsigned long long tqh = 0;
    unsigned int nsampled = 0;
    const size_t gcol = (size_t)item.k * a.n;
    const uint16_t* bins_lane = a.bins + slot0;
    const uint32_t stride = (uint32_t)nwarps * ROWS_PER_WARP;
    uint32_t p = pbeg + warp * ROWS_PER_WARP;
    uint32_t next_rid = 0u;
    if (lane < ROWS_PER_WARP && p + lane < pend) next_rid = item.rows[p + lane];
    for (; p < pend; p += stride) {
      const uint32_t my_rid = next_rid;
      const uint32_t pn = p + stride + lane;
      next_rid = (lane < ROWS_PER_WARP && pn < pend) ? item.rows[pn] : 0u;
      const uint32_t nrow = min(pend - p, (uint32_t)ROWS_PER_WARP);
      uint32_t my_g = 0u, my_h = 0u;  // FIXED ints or FP32 float bits
      if (lane < (int)nrow) {
        if (FIXED) {
          const unsigned long long pk = reinterpret_cast<const unsigned long long*>(a.gpair)[gcol + my_rid];
          my_g = (uint32_t)(pk >> 32);
          my_h = (uint32_t)(pk & 0xFFFFFFFFull);
        } else {
          const float2 v = reinterpret_cast<const float2*>(a.gpair)[gcol + my_rid];
          my_g = __float_as_uint(v.x);
          my_h = __float_as_uint(v.y);
        }
        nsampled++;
        if (want_total) {
          if (FIXED) {
            tqg += (int)my_g;
            tqh += my_h;
          } else {
            tg += (double)__uint_as_float(my_g);
            th += (double)__uint_as_float(my_h);
          }
        }
      }
      CT cv[ROWS_PER_WARP];
#pragma unroll
      for (int q = 0; q < ROWS_PER_WARP; ++q) {
        const uint32_t id = __shfl_sync(0xFFFFFFFFu, my_rid, q);
        cv[q] = (uint32_t)q < nrow ? __ldg(reinterpret_cast<const CT*>(bins_lane + (size_t)id * a.Fp)) : C::none();
      }
#pragma unroll
      for (int q = 0; q < ROWS_PER_WARP; ++q) {
        const uint32_t vg = __shfl_sync(0xFFFFFFFFu, my_g, q);
        const uint32_t vh = __shfl_sync(0xFFFFFFFFu, my_h, q);
        if ((uint32_t)q >= nrow) break;
#pragma unroll
        for (int s = 0; s < S; ++s)
          if (fon[s]) add_pair<FIXED>(sh_base + 4u * (unsigned)(C::get(cv[q], s) * 32 + lane), hoff, vg, vh);
      }
    }
    if (a.rows_done && t == 0 && nsampled) atomicAdd(a.rows_done, (unsigned long long)nsampled);
    if (want_total && lane < ROWS_PER_WARP) {
      if (FIXED) {
        atomicAdd(&s_tot_u[0], (unsigned long long)tqg);
        atomicAdd(&s_tot_u[1], tqh);
      } else {
        atomicAdd(&s_tot_d[0], tg);
        atomicAdd(&s_tot_d[1], th);
      }
    }
    __syncthreads();
    // flush the partial into the node's HBM histogram
    const int* eg = a.ent_gbin + tile.ent_off;
    for (int i = threadIdx.x; i < words; i += blockDim.x) {
      const int gi = eg[i];
      if (gi < 0) continue;
      if (FIXED) {
        const long long gq = (long long)(int)sh_g[i];
        const unsigned long long hq = sh_h[i];
        unsigned long long* o = reinterpret_cast<unsigned long long*>(item.out) + 2 * (size_t)gi;
        if (gq) atomicAdd(o, (unsigned long long)gq);
        if (hq) atomicAdd(o + 1, hq);
      } else {
        const float g = __uint_as_float(sh_g[i]), h = __uint_as_float(sh_h[i]);
        double* o = reinterpret_cast<double*>(item.out) + 2 * (size_t)gi;
        if (g != 0.0f) atomicAdd(o, (double)g);
        if (h != 0.0f) atomicAdd(o + 1, (double)h);
      }
    }
    if (want_total && threadIdx.x == 0) {
      if (FIXED) {
        unsigned long long* o = reinterpret_cast<unsigned long long*>(item.total);
        atomicAdd(o, s_tot_u[0]);
        atomicAdd(o + 1, s_tot_u[1]);
      } else {
        double* o = reinterpret_cast<double*>(item.total);
        atomicAdd(o, s_tot_d[0]);
        atomicAdd(o + 1, s_tot_d[1]);
      }
    }
    __syncthreads();
    u += n_pos;
  }
}

__global__ void k_zero_items(const HistItem* __restrict__ items, const int* __restrict__ count,
                             size_t words) {
  int it = blockIdx.y;
  if (it >= *count) return;
  unsigned long long* o = reinterpret_cast<unsigned long long*>(items[it].out);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < words;
       i += (size_t)gridDim.x * blockDim.x)
    o[i] = 0ull;
  if (items[it].root && blockIdx.x == 0 && threadIdx.x < 2)
    reinterpret_cast<unsigned long long*>(items[it].total)[threadIdx.x] = 0ull;
}

// k_zero_items for many jobs: job j's blocks are xoff[j] .. xoff[j + 1] - 1.
__global__ void k_zero_items_jobs(const ZeroJob* __restrict__ zj, const unsigned* __restrict__ xoff, int njobs) {
  const int j = hist_job_of(xoff, njobs, blockIdx.x);
  const unsigned bx = blockIdx.x - xoff[j], gdx = xoff[j + 1] - xoff[j];
  const ZeroJob z = zj[j];
  const int it = blockIdx.y;
  if (it >= *z.count) return;
  unsigned long long* o = reinterpret_cast<unsigned long long*>(z.items[it].out);
  for (size_t i = (size_t)bx * blockDim.x + threadIdx.x; i < z.words; i += (size_t)gdx * blockDim.x) o[i] = 0ull;
  if (z.items[it].root && bx == 0 && threadIdx.x < 2)
    reinterpret_cast<unsigned long long*>(z.items[it].total)[threadIdx.x] = 0ull;
}

__global__ void k_subtract(const double2* __restrict__ p, const double2* __restrict__ c,
                           double2* __restrict__ o, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    double2 a = p[i], b = c[i];
    o[i] = make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
  }
}

__global__ void k_fixed_to_f64(const longlong2* __restrict__ in, double2* __restrict__ out, size_t n,
                               double sg, double sh) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    longlong2 v = in[i];
    out[i] = make_double2(__dmul_rn((double)v.x, sg), __dmul_rn((double)v.y, sh));
  }
}

}  // namespace

namespace {

// TILED layout: contiguous feature ranges whose bins and missing entries fit
// the shared-memory budget, at most 128 features (4 per lane), starting at
// multiples of 4 features.
// Rows per warp instruction of the TILED kernel (as log2): a narrow matrix
// leaves most of a warp's lanes without features when one row takes the
// whole warp (4 features per lane), so up to 8 rows share an instruction:
// at most 128 >> rl features per tile. SB_HIST_ROWS (1, 2, 4, 8) forces it.
static int tiled_rows_log(size_t F) {
  if (const char* e = std::getenv("SB_HIST_ROWS")) {
    const int v = std::atoi(e);
    if (v == 1) return 0;
    if (v == 2) return 1;
    if (v == 4) return 2;
    if (v == 8) return 3;
  }
  return F <= 16 ? 3 : F <= 32 ? 2 : F <= 64 ? 1 : 0;
}

int plan_tiled(Ghist* g, size_t budget, int rl) {
  g->tiles.clear();
  const size_t F = g->F;
  g->tiled_rl = rl >= 0 ? rl : tiled_rows_log(F);
  const size_t max_tile = (size_t)MAX_TILE_FEATURES >> g->tiled_rl;
  size_t f0 = 0, maxb = 0;
  while (f0 < F) {
    size_t f1 = f0;
    while (f1 < F && f1 - f0 < max_tile) {
      size_t bins = g->h_foff[f1 + 1] - g->h_foff[f0];
      if ((bins + (f1 + 1 - f0)) * 8 > budget) break;
      f1++;
    }
    SB_REQUIRE(f1 > f0, SB_ERR_UNSUPPORTED, "feature %zu has too many bins for shared memory", f0);
    if (f1 < F && f1 - f0 >= 4) f1 -= (f1 - f0) % 4;  // next tile starts on a multiple of 4
    SB_REQUIRE(f1 == F || (f1 - f0) % 4 == 0, SB_ERR_UNSUPPORTED,
               "features %zu.. need more shared memory than one CTA has", f0);
    FeatureTile t{};
    t.f0 = (int)f0;
    t.f1 = (int)f1;
    t.bin0 = (int)g->h_foff[f0];
    t.nbins = (int)(g->h_foff[f1] - g->h_foff[f0]);
    maxb = std::max(maxb, (size_t)(t.nbins + (t.f1 - t.f0)) * 8);
    SB_REQUIRE(t.nbins + (t.f1 - t.f0) < 0xFFFF, SB_ERR_UNSUPPORTED, "histogram tile too large");
    g->tiles.push_back(t);
    f0 = f1;
  }
  g->layout = HIST_LAYOUT_TILED;
  g->slots = 0;
  g->Fp = (F + 7) / 8 * 8;
  // one-byte codes when every feature's local bins and its missing code fit
  // (SB_HIST_CODES=2 keeps two bytes)
  size_t max_nb = 0;
  for (size_t f = 0; f < F; ++f) max_nb = std::max<size_t>(max_nb, g->h_foff[f + 1] - g->h_foff[f]);
  const char* cb = std::getenv("SB_HIST_CODES");
  g->code_bytes = (max_nb <= 255 && !(cb && std::atoi(cb) == 2)) ? 1 : 2;
  g->h_rpos.assign(F, 0);
  g->h_rbase.assign(F, 0);
  g->h_rmiss.assign(F, 0);
  int ent_off = 0;
  for (FeatureTile& t : g->tiles) {
    t.ent_off = ent_off;
    ent_off += t.nbins + (t.f1 - t.f0);
    for (int f = t.f0; f < t.f1; ++f) {
      g->h_rpos[f] = f;
      if (g->code_bytes == 1) {  // the local bin; the bin count when missing
        g->h_rbase[f] = 0;
        g->h_rmiss[f] = (int)(g->h_foff[f + 1] - g->h_foff[f]);
      } else {  // the entry in the tile's partial: bins, then one missing entry per feature
        g->h_rbase[f] = (int)g->h_foff[f] - t.bin0;
        g->h_rmiss[f] = t.nbins + (f - t.f0);
      }
    }
  }
  g->hist_smem_bytes = maxb;
  return SB_OK;
}

// u8 TILED: the histogram bin of every shared entry, per tile: feature fl of
// the tile owns entries foff[f] - bin0 + fl .. + its bin count (the last one
// its missing entry, bin total_bins + f).
std::vector<int> tiled_u8_entries(const Ghist* g) {
  std::vector<int> eg;
  for (const FeatureTile& t : g->tiles) {
    eg.resize((size_t)t.ent_off + t.nbins + (t.f1 - t.f0), -1);
    for (int f = t.f0; f < t.f1; ++f) {
      const int nb = (int)(g->h_foff[f + 1] - g->h_foff[f]);
      const size_t e0 = (size_t)t.ent_off + (g->h_foff[f] - t.bin0) + (f - t.f0);
      for (int b = 0; b < nb; ++b) eg[e0 + b] = (int)g->h_foff[f] + b;
      eg[e0 + nb] = (int)(g->total_bins + f);
    }
  }
  return eg;
}

// One feature's place in the LANES layout.
struct LanePlace {
  int lane, slot, eb;  // lane, code position within the lane, first entry
};

// Longest-processing-time packing of features [f0, f1) into 32 lanes of
// `slots` positions with at most `emax` entries (bins + the missing entry)
// per lane. Returns the largest lane load, or -1 when the features do not fit.
int pack_lanes(const Ghist* g, size_t f0, size_t f1, int slots, int emax, std::vector<LanePlace>* out) {
  const size_t m = f1 - f0;
  if (m > (size_t)32 * slots) return -1;
  std::vector<int> order(m);
  for (size_t i = 0; i < m; ++i) order[i] = (int)(f0 + i);
  auto ent = [&](int f) { return (int)(g->h_foff[f + 1] - g->h_foff[f]) + 1; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ent(a) > ent(b); });
  int load[32] = {0}, used[32] = {0};
  out->assign(m, LanePlace{0, 0, 0});
  int emx = 1;
  for (int f : order) {
    int best = -1;
    for (int l = 0; l < 32; ++l)
      if (used[l] < slots && (best < 0 || load[l] < load[best])) best = l;
    if (best < 0 || load[best] + ent(f) > emax) return -1;
    (*out)[f - f0] = LanePlace{best, used[best]++, load[best]};
    load[best] += ent(f);
    emx = std::max(emx, load[best]);
  }
  return emx;
}

// LANES layout: tiles grow feature by feature while their features still pack
// into the 32 lanes.
int plan_lanes(Ghist* g, size_t budget, int slots, std::vector<std::vector<LanePlace>>* places) {
  const size_t F = g->F;
  const int emax = (int)std::min<size_t>(budget / (2 * 32 * 4), 0xFFFE);
  std::vector<FeatureTile> tiles;
  places->clear();
  size_t f0 = 0;
  int ent_off = 0;
  std::vector<LanePlace> cur, best;
  while (f0 < F) {
    size_t f1 = f0;
    int E = -1;
    while (f1 < F) {
      int e = pack_lanes(g, f0, f1 + 1, slots, emax, &cur);
      if (e < 0) break;
      E = e;
      best = cur;
      f1++;
    }
    if (f1 == f0) return SB_ERR_UNSUPPORTED;  // one feature's bins exceed a lane
    FeatureTile t{};
    t.f0 = (int)f0;
    t.f1 = (int)f1;
    t.bin0 = (int)g->h_foff[f0];
    t.nbins = (int)(g->h_foff[f1] - g->h_foff[f0]);
    t.E = E;
    t.ent_off = ent_off;
    t.slot_off = (int)tiles.size() * 32 * slots;
    ent_off += 32 * E;
    tiles.push_back(t);
    places->push_back(best);
    f0 = f1;
  }
  g->tiles = tiles;
  return SB_OK;
}

size_t lanes_smem(const Ghist* g) {
  size_t m = 0;
  for (const FeatureTile& t : g->tiles) m = std::max(m, (size_t)t.E * 32 * 4 * 2);
  return m;
}

}  // namespace

namespace {

size_t smem_budget(const sb_ctx* ctx) {
  return ctx->smem_optin > 8192 ? ctx->smem_optin - 4096 : ctx->smem_optin;
}

}  // namespace

// Plans the histogram's bin-code layout and feature tiles for one choice
// (HIST_LAYOUT_TILED, or HIST_LAYOUT_LANES with 1, 2 or 4 code positions per
// lane and tile). SB_ERR_UNSUPPORTED when a feature's entries do not fit one
// lane's column.
int hist_prepare(sb_ctx* ctx, Ghist* g, HistChoice c) {
  const size_t budget = smem_budget(ctx);
  const size_t F = g->F;
  if (c.layout == HIST_LAYOUT_TILED) {
    SB_TRY(plan_tiled(g, budget, c.rl));
    if (g->code_bytes == 1) {
      const std::vector<int> eg = tiled_u8_entries(g);
      SB_TRY(g->ent_gbin.alloc(ctx, eg.size()));
      SB_CUDA(cudaMemcpyAsync(g->ent_gbin.p, eg.data(), eg.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
      SB_CUDA(cudaStreamSynchronize(ctx->stream));  // the pageable copy must finish before eg goes away
    }
  } else {
    const int slots = c.slots;
    SB_REQUIRE(slots == 1 || slots == 2 || slots == 4, SB_ERR_INVALID_ARG, "internal: %d slots", slots);
    std::vector<std::vector<LanePlace>> places;
    SB_REQUIRE(plan_lanes(g, budget, slots, &places) == SB_OK, SB_ERR_UNSUPPORTED,
               "a feature has too many bins for the lane layout");
    g->layout = HIST_LAYOUT_LANES;
    g->slots = slots;
    g->code_bytes = 2;
    g->Fp = g->tiles.size() * 32 * slots;
    g->h_rpos.assign(F, 0);
    g->h_rbase.assign(F, 0);
    g->h_rmiss.assign(F, 0);
    size_t ent_total = 0;
    for (const FeatureTile& t : g->tiles) ent_total += (size_t)32 * t.E;
    std::vector<int> eg(ent_total, -1), sf(g->Fp, -1);
    for (size_t ti = 0; ti < g->tiles.size(); ++ti) {
      const FeatureTile& t = g->tiles[ti];
      for (int f = t.f0; f < t.f1; ++f) {
        const LanePlace& pl = places[ti][f - t.f0];
        const int nb = (int)(g->h_foff[f + 1] - g->h_foff[f]);
        g->h_rpos[f] = t.slot_off + pl.lane * slots + pl.slot;
        g->h_rbase[f] = pl.eb;
        g->h_rmiss[f] = pl.eb + nb;
        sf[g->h_rpos[f]] = f;
        for (int b = 0; b < nb; ++b) eg[t.ent_off + (size_t)(pl.eb + b) * 32 + pl.lane] = (int)g->h_foff[f] + b;
        eg[t.ent_off + (size_t)(pl.eb + nb) * 32 + pl.lane] = (int)(g->total_bins + f);
      }
    }
    SB_TRY(g->ent_gbin.alloc(ctx, eg.size()));
    SB_TRY(g->slot_feat.alloc(ctx, sf.size()));
    SB_CUDA(cudaMemcpyAsync(g->ent_gbin.p, eg.data(), eg.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    SB_CUDA(cudaMemcpyAsync(g->slot_feat.p, sf.data(), sf.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    // the pageable copies above must finish before the vectors go away
    SB_CUDA(cudaStreamSynchronize(ctx->stream));
    g->hist_smem_bytes = lanes_smem(g);
  }
  for (int fixed = 0; fixed < 2; ++fixed)
    for (int rl = 0; rl < 4; ++rl)
      for (int u8 = 0; u8 < 2; ++u8) SB_TRY(raise_smem_limit(tiled_kernel(fixed != 0, rl, u8 != 0), g->hist_smem_bytes));
  SB_TRY(raise_smem_limit((const void*)k_hist_lanes<false, 1>, g->hist_smem_bytes));
  SB_TRY(raise_smem_limit((const void*)k_hist_lanes<true, 1>, g->hist_smem_bytes));
  SB_TRY(raise_smem_limit((const void*)k_hist_lanes<false, 2>, g->hist_smem_bytes));
  SB_TRY(raise_smem_limit((const void*)k_hist_lanes<true, 2>, g->hist_smem_bytes));
  SB_TRY(raise_smem_limit((const void*)k_hist_lanes<false, 4>, g->hist_smem_bytes));
  SB_TRY(raise_smem_limit((const void*)k_hist_lanes<true, 4>, g->hist_smem_bytes));
  return SB_OK;
}

// The layout an index takes without timing: TILED, or what SB_HIST_LAYOUT
// ("tiled" or "lanes") in the environment forces. On the 10M x 100 binary
// workload TILED measured 0.41 ms per histogram launch against 0.48 ms for
// LANES with 4 positions per lane, so LANES is only chosen by timing.
int hist_default_choice(sb_ctx* ctx, Ghist* g, HistChoice* out) {
  const size_t F = g->F;
  const char* force = std::getenv("SB_HIST_LAYOUT");
  const bool force_lanes = force && std::strcmp(force, "lanes") == 0;
  *out = HistChoice{HIST_LAYOUT_TILED, 0};
  if (!force_lanes) return SB_OK;
  const int slots = F <= 32 ? 1 : (F <= 64 ? 2 : 4);
  std::vector<std::vector<LanePlace>> places;
  const std::vector<FeatureTile> keep = g->tiles;
  const bool ok = plan_lanes(g, smem_budget(ctx), slots, &places) == SB_OK;
  g->tiles = keep;
  SB_REQUIRE(ok, SB_ERR_UNSUPPORTED, "SB_HIST_LAYOUT=lanes: a feature has too many bins");
  *out = HistChoice{HIST_LAYOUT_LANES, slots};
  return SB_OK;
}

// The choices the autotuner times: TILED, and for up to 64 features (where
// one row per warp instruction keeps at most 16 of a warp's lanes busy)
// TILED with 2, 4 or 8 rows per instruction and LANES with 1 and 2 positions
// per lane where the features pack. Wider matrices take TILED: on
// the 10M x 100 workload a whole round measured TILED faster at every level
// (ncu: LANES cut the shared-atomic wavefronts by 2.4x but waited longer on
// its 23 % longer rows), while a single timed launch ranked LANES first.
std::vector<HistChoice> hist_candidates(sb_ctx* ctx, Ghist* g) {
  std::vector<HistChoice> out{HistChoice{HIST_LAYOUT_TILED, 0, 0}};
  if (g->F > 64) return out;
  // TILED with 2, 4, 8 rows per warp instruction while a tile still holds
  // every feature (128 >> rl features)
  for (int rl = 1; rl <= 3 && (size_t)(MAX_TILE_FEATURES >> rl) >= g->F; ++rl)
    out.push_back(HistChoice{HIST_LAYOUT_TILED, 0, rl});
  const std::vector<FeatureTile> keep = g->tiles;
  for (int slots : {1, 2}) {
    std::vector<std::vector<LanePlace>> places;
    if (plan_lanes(g, smem_budget(ctx), slots, &places) == SB_OK) out.push_back(HistChoice{HIST_LAYOUT_LANES, slots});
  }
  g->tiles = keep;
  return out;
}

namespace {

const void* hist_kernel(const Ghist* g, bool fixed) {
  if (g->layout == HIST_LAYOUT_LANES) {
    switch (g->slots) {
      case 1: return fixed ? (const void*)k_hist_lanes<true, 1> : (const void*)k_hist_lanes<false, 1>;
      case 2: return fixed ? (const void*)k_hist_lanes<true, 2> : (const void*)k_hist_lanes<false, 2>;
      default: return fixed ? (const void*)k_hist_lanes<true, 4> : (const void*)k_hist_lanes<false, 4>;
    }
  }
  return tiled_kernel(fixed, g->tiled_rl, g->code_bytes == 1);
}

}  // namespace

// The persistent grid: every resident CTA, or for a launch known to hold
// few rows one CTA per HIST_MIN_ROWS_PER_CTA (row, tile) units, so that a
// small job's launch zeroes and flushes few shared partials and leaves SMs
// to the launches of other streams.
constexpr size_t HIST_MIN_ROWS_PER_CTA = 4096;
int hist_grid(sb_ctx* ctx, const Ghist* g, size_t rows_bound) {
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hist_kernel(g, true), HIST_THREADS,
                                                g->hist_smem_bytes);
  if (per_sm < 1) per_sm = 1;
  const size_t full = (size_t)ctx->num_sms * per_sm;
  if (rows_bound == 0) return (int)full;
  const size_t want = (rows_bound * g->tiles.size() + HIST_MIN_ROWS_PER_CTA - 1) / HIST_MIN_ROWS_PER_CTA;
  return (int)std::max<size_t>(1, std::min(full, want));
}

// The kernel's description of one launch.
static HistDev hist_dev(const HistLaunch& L) {
  HistDev a;
  a.bins = L.g->code_bytes == 1 ? nullptr : L.g->bins.p;
  a.bins8 = L.g->code_bytes == 1 ? L.g->bins8.p : nullptr;
  a.foff = L.g->foff.p;
  a.Fp = L.g->Fp;
  a.ent_gbin = L.g->ent_gbin.p;
  a.slot_feat = L.g->slot_feat.p;
  a.n = L.g->n;
  a.total_bins = (int)L.g->total_bins;
  a.gpair = L.gpair;
  a.items = L.items;
  a.prefix = L.prefix;
  a.count = L.count;
  a.tiles = L.tiles;
  a.ntiles = L.ntiles;
  a.flush_rows = fixed_rows_per_flush(L.quant_bits);
  a.rows_done = L.rows_done;
  a.pool_mask = L.pool_mask;
  a.FW = (int)((L.g->F + 31) / 32);
  a.rl = L.g->tiled_rl;
  a.min_units = L.min_units;
  return a;
}

int launch_hist(sb_ctx* ctx, const HistLaunch& L) {
  const HistDev a = hist_dev(L);
  const int grid = hist_grid(ctx, L.g, L.rows_bound);
  const size_t sm = L.g->hist_smem_bytes;
  void (*kern)(HistDev) = reinterpret_cast<void (*)(HistDev)>(
      const_cast<void*>(tiled_kernel(L.fixed, L.g->tiled_rl, L.g->code_bytes == 1)));
  if (L.g->layout == HIST_LAYOUT_LANES) {
    switch (L.g->slots) {
      case 1: kern = L.fixed ? k_hist_lanes<true, 1> : k_hist_lanes<false, 1>; break;
      case 2: kern = L.fixed ? k_hist_lanes<true, 2> : k_hist_lanes<false, 2>; break;
      default: kern = L.fixed ? k_hist_lanes<true, 4> : k_hist_lanes<false, 4>;
    }
  }
  SB_LAUNCH(ctx, kern, grid, HIST_THREADS, sm, a);
  return SB_OK;
}

int launch_zero_items(sb_ctx* ctx, const Ghist* g, const HistItem* items, const int* count,
                      int max_items) {
  if (max_items <= 0) return SB_OK;
  size_t words = (g->total_bins + g->F) * 2;
  dim3 grid((unsigned)std::min<size_t>((words + 255) / 256, 64), (unsigned)max_items);
  SB_LAUNCH(ctx, k_zero_items, grid, 256, 0, items, count, words);
  return SB_OK;
}

int hist_jobs_prepare(sb_ctx* ctx, const std::vector<HistLaunch>& Ls, HistJobsPlan* P) {
  const int nj = (int)Ls.size();
  SB_REQUIRE(nj > 0, SB_ERR_INVALID_ARG, "internal: no jobs");
  std::vector<HistDev> devs(nj);
  std::vector<ZeroJob> zero(nj);
  P->fixed = Ls[0].fixed;
  P->smem = 0;
  P->hist_grid.assign(nj, 0);
  P->zero_grid.assign(nj, 0);
  for (int j = 0; j < nj; ++j) {
    const HistLaunch& L = Ls[j];
    SB_REQUIRE(L.g->layout == HIST_LAYOUT_TILED && L.fixed == P->fixed && L.g->tiled_rl == Ls[0].g->tiled_rl &&
                   L.g->code_bytes == Ls[0].g->code_bytes,
               SB_ERR_INVALID_ARG,
               "internal: batched histograms need the TILED layout, one precision, one row grouping and one "
               "code width");
    devs[j] = hist_dev(L);
    const size_t words = (L.g->total_bins + L.g->F) * 2;
    zero[j] = ZeroJob{L.items, L.count, words};
    P->hist_grid[j] = (unsigned)hist_grid(ctx, L.g, L.rows_bound);
    P->zero_grid[j] = (unsigned)std::min<size_t>((words + 255) / 256, 64);
    P->smem = std::max(P->smem, L.g->hist_smem_bytes);
  }
  P->njobs = nj;
  cudaStream_t st = ctx->stream;
  SB_TRY(P->devs.alloc(ctx, nj * sizeof(HistDev)));
  SB_TRY(P->zero.alloc(ctx, nj));
  SB_CUDA(cudaMemcpyAsync(P->devs.p, devs.data(), nj * sizeof(HistDev), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(P->zero.p, zero.data(), nj * sizeof(ZeroJob), cudaMemcpyHostToDevice, st));
  P->rl = Ls[0].g->tiled_rl;
  P->u8 = Ls[0].g->code_bytes == 1;
  SB_TRY(raise_smem_limit(tiled_jobs_kernel(P->fixed != 0, P->rl, P->u8), P->smem));
  SB_CUDA(cudaStreamSynchronize(st));  // the host tables are released on return
  return SB_OK;
}

int launch_hist_jobs(sb_ctx* ctx, const HistJobsPlan& P, const unsigned* d_xoff, unsigned hist_blocks,
                     const unsigned* d_zoff, unsigned zero_blocks, int max_items) {
  if (max_items <= 0 || hist_blocks == 0) return SB_OK;
  SB_LAUNCH(ctx, k_zero_items_jobs, dim3(zero_blocks, (unsigned)max_items), 256, 0, P.zero.p, d_zoff, P.njobs);
  HistJobs H;
  H.devs = reinterpret_cast<const HistDev*>(P.devs.p);
  H.xoff = d_xoff;
  H.njobs = P.njobs;
  void (*kern)(HistJobs) =
      reinterpret_cast<void (*)(HistJobs)>(const_cast<void*>(tiled_jobs_kernel(P.fixed != 0, P.rl, P.u8)));
  SB_LAUNCH(ctx, kern, hist_blocks, HIST_THREADS, P.smem, H);
  return SB_OK;
}

// Device time of fixed-point histogram launches over min(n, 2^20) rows
// spread over the whole matrix (one row drawn from each of m equal strides,
// ascending): the gathers of a round's deeper levels, on codes mostly
// outside L2. Best of two after a warm-up launch: the autotuner's measure.
int hist_time(sb_ctx* ctx, const Ghist* g, float* ms) {
  const size_t m = std::min<size_t>(g->n, (size_t)1 << 20);
  const size_t HB = g->total_bins + g->F;
  cudaStream_t st = ctx->stream;
  DBuf<uint32_t> rows;
  DBuf<unsigned long long> gp;
  DBuf<longlong2> out;
  DBuf<HistItem> item;
  DBuf<uint64_t> prefix;
  DBuf<int> count;
  DBuf<FeatureTile> tiles;
  SB_TRY(rows.alloc(ctx, m));
  SB_TRY(gp.alloc_zero(ctx, g->n));
  SB_TRY(out.alloc(ctx, HB));
  SB_TRY(item.alloc(ctx, 1));
  SB_TRY(prefix.alloc(ctx, 2));
  SB_TRY(count.alloc(ctx, 1));
  SB_TRY(tiles.alloc(ctx, g->tiles.size()));
  std::vector<uint32_t> h_rows(m);
  const size_t stride = g->n / m;
  for (size_t i = 0; i < m; ++i) h_rows[i] = (uint32_t)(i * stride + sb_mix64(i) % stride);
  HistItem it{};
  it.rows = rows.p;
  it.begin = 0;
  it.end = (uint32_t)m;
  it.out = out.p;
  const uint64_t h_prefix[2] = {0, (uint64_t)m};
  const int one = 1;
  SB_CUDA(cudaMemcpyAsync(rows.p, h_rows.data(), m * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(item.p, &it, sizeof(it), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(prefix.p, h_prefix, sizeof(h_prefix), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(count.p, &one, sizeof(one), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(tiles.p, g->tiles.data(), g->tiles.size() * sizeof(FeatureTile), cudaMemcpyHostToDevice,
                          st));
  HistLaunch L;
  L.g = g;
  L.gpair = gp.p;
  L.fixed = 1;
  L.quant_bits = 16;
  L.items = item.p;
  L.prefix = prefix.p;
  L.count = count.p;
  L.max_items = 1;
  L.tiles = tiles.p;
  L.ntiles = (int)g->tiles.size();
  L.rows_done = nullptr;
  L.pool_mask = nullptr;
  cudaEvent_t e0, e1;
  SB_CUDA(cudaEventCreate(&e0));
  SB_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int rc = SB_OK;
  for (int rep = 0; rep < 3 && rc == SB_OK; ++rep) {
    cudaMemsetAsync(out.p, 0, out.bytes(), st);
    cudaEventRecord(e0, st);
    rc = launch_hist(ctx, L);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = SB_ERR_CUDA;
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    if (rep > 0) best = std::min(best, t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = best;
  return rc;
}

// per-node seam helpers (defined in sb_grow.cu)
int quantize_pairs(sb_ctx* ctx, const float2* d_gp, size_t n, int bits, unsigned long long* d_packed,
                   int* h_shift_g, int* h_shift_h);

}  // namespace sb

extern "C" {

int sb_hist_build(sb_ctx* ctx, const sb_ghist* g, const uint32_t* rows, size_t m,
                  const sb_gradpair* gpair, size_t n, int precision, int quantize_bits,
                  sb_gradstats* out, size_t total_bins) {
  using namespace sb;
  SB_REQUIRE(ctx && g && gpair && out, SB_ERR_INVALID_ARG, "NULL argument");
  SB_SAME_DEVICE(ctx, g);
  SB_REQUIRE(m == 0 || rows, SB_ERR_INVALID_ARG, "rows is NULL");
  SB_REQUIRE(total_bins == g->total_bins, SB_ERR_DIMENSION,
             "dimension mismatch: out length expected %zu, got %zu", g->total_bins, total_bins);
  SB_REQUIRE(n == g->n, SB_ERR_DIMENSION, "dimension mismatch: gpair length expected %zu, got %zu",
             g->n, n);
  SB_REQUIRE(precision == SB_HIST_FP32 || precision == SB_HIST_FIXED, SB_ERR_INVALID_ARG,
             "unknown precision %d", precision);
  int bits = quantize_bits ? quantize_bits : 16;
  SB_REQUIRE(bits >= 8 && bits <= 23, SB_ERR_INVALID_ARG, "quantize_bits must be in [8, 23]");
  for (size_t i = 0; i < m; ++i)
    SB_REQUIRE(rows[i] < n, SB_ERR_INVALID_ARG, "row %u out of range", rows[i]);
  SB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t HB = g->total_bins + g->F;
  DBuf<uint32_t> d_rows;
  DBuf<float2> d_gp;
  DBuf<unsigned long long> d_packed;
  DBuf<double2> d_hist, d_out;
  DBuf<HistItem> d_item;
  DBuf<uint64_t> d_prefix;
  DBuf<int> d_count;
  DBuf<FeatureTile> d_tiles;
  SB_TRY(d_rows.alloc(ctx, std::max<size_t>(m, 1)));
  SB_TRY(d_gp.alloc(ctx, n));
  SB_TRY(d_hist.alloc(ctx, HB));
  SB_TRY(d_out.alloc(ctx, HB));
  SB_TRY(d_item.alloc(ctx, 1));
  SB_TRY(d_prefix.alloc(ctx, 2));
  SB_TRY(d_count.alloc(ctx, 1));
  SB_TRY(d_tiles.alloc(ctx, g->tiles.size()));
  if (m) SB_CUDA(cudaMemcpyAsync(d_rows.p, rows, m * 4, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_gp.p, gpair, n * 8, cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_tiles.p, g->tiles.data(), g->tiles.size() * sizeof(FeatureTile),
                          cudaMemcpyHostToDevice, st));
  int sg = 0, shh = 0;
  const void* gsrc = d_gp.p;
  if (precision == SB_HIST_FIXED) {
    SB_TRY(d_packed.alloc(ctx, n));
    SB_TRY(quantize_pairs(ctx, d_gp.p, n, bits, d_packed.p, &sg, &shh));
    gsrc = d_packed.p;
  }
  HistItem it;
  it.rows = d_rows.p;
  it.begin = 0;
  it.end = (uint32_t)m;
  it.k = 0;
  it.root = 0;
  it.out = d_hist.p;
  it.total = nullptr;
  uint64_t prefix[2] = {0, (uint64_t)m};
  int one = 1;
  SB_CUDA(cudaMemcpyAsync(d_item.p, &it, sizeof(it), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_prefix.p, prefix, sizeof(prefix), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(d_count.p, &one, sizeof(int), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemsetAsync(d_hist.p, 0, d_hist.bytes(), st));
  HistLaunch L;
  L.g = g;
  L.gpair = gsrc;
  L.fixed = precision == SB_HIST_FIXED;
  L.quant_bits = bits;
  L.items = d_item.p;
  L.prefix = d_prefix.p;
  L.count = d_count.p;
  L.max_items = 1;
  L.tiles = d_tiles.p;
  L.ntiles = (int)g->tiles.size();
  L.rows_done = nullptr;
  L.pool_mask = nullptr;
  if (m) SB_TRY(launch_hist(ctx, L));
  const double2* res = d_hist.p;
  if (L.fixed) {
    SB_LAUNCH(ctx, k_fixed_to_f64, 256, 256, 0, reinterpret_cast<const longlong2*>(d_hist.p), d_out.p,
              HB, std::ldexp(1.0, -sg), std::ldexp(1.0, -shh));
    res = d_out.p;
  }
  SB_CUDA(cudaMemcpyAsync(out, res, total_bins * sizeof(double2), cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  return SB_OK;
}

int sb_hist_subtract(sb_ctx* ctx, const sb_gradstats* parent, const sb_gradstats* child,
                     sb_gradstats* out, size_t total_bins) {
  using namespace sb;
  SB_REQUIRE(ctx && parent && child && out, SB_ERR_INVALID_ARG, "NULL argument");
  if (total_bins == 0) return SB_OK;
  SB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  DBuf<double2> p, c, o;
  SB_TRY(p.alloc(ctx, total_bins));
  SB_TRY(c.alloc(ctx, total_bins));
  SB_TRY(o.alloc(ctx, total_bins));
  SB_CUDA(cudaMemcpyAsync(p.p, parent, p.bytes(), cudaMemcpyHostToDevice, st));
  SB_CUDA(cudaMemcpyAsync(c.p, child, c.bytes(), cudaMemcpyHostToDevice, st));
  unsigned blocks = (unsigned)std::min<size_t>((total_bins + 255) / 256, (size_t)ctx->num_sms * 8);
  SB_LAUNCH(ctx, k_subtract, blocks, 256, 0, p.p, c.p, o.p, total_bins);
  SB_CUDA(cudaMemcpyAsync(out, o.p, o.bytes(), cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  return SB_OK;
}

}  // extern "C"
