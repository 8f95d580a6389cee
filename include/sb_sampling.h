/*
 * sb_sampling.h — the row / column sampling streams of sequoia-boost-b200.
 *
 * The reference draws its Bernoulli row subsample (crates/sequoia-boost/src/
 * learner/train.rs:304-306, :465-476), its per-tree column pool (train.rs:
 * :479-489, :516-534) and its per-node column subsets (tree/sampler.rs:52-70)
 * from `rand 0.8` StdRng. That crate is not vendored and has no lock file, so
 * its stream cannot be reproduced; only the sampling *algorithms* are kept:
 *
 *   rows   : keep row r with probability `subsample`; at least one row.
 *   pool   : k = clamp(round(ratio * F), 1, F); shuffle; truncate; sort.
 *   node   : subsample(subsample(pool, bylevel), bynode), drawn per node.
 *
 * The random numbers come from counter-based SplitMix64 keys, so a row's or a
 * node's draw does not depend on the order in which the GPU visits it. The
 * CUDA kernels and the CPU oracle both include this header, which makes their
 * samples identical on the same seed.
 */
#ifndef SB_SAMPLING_H
#define SB_SAMPLING_H

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define SB_HD __host__ __device__ __forceinline__
#else
#define SB_HD static inline
#endif

/* SplitMix64 finaliser (Steele, Lea, Flood 2014). */
SB_HD uint64_t sb_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* Uniform double in [0, 1) from the top 53 bits. */
SB_HD double sb_u01(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

/* Key of boosting round `round` (shared by the round's class trees). */
SB_HD uint64_t sb_round_key(uint64_t seed, uint64_t round) {
  return sb_mix64(seed ^ sb_mix64(round + 0x5EED0001ULL));
}

/* Bernoulli draw of row `row` in a round: kept iff sb_u01(...) < subsample. */
SB_HD uint64_t sb_row_draw(uint64_t round_key, uint64_t row) {
  return sb_mix64(round_key + row * 0xD1B54A32D192ED03ULL);
}

/* Row taken when the Bernoulli draw kept none (train.rs:472-474). */
SB_HD uint64_t sb_row_fallback(uint64_t round_key, uint64_t n_rows) {
  return sb_mix64(round_key ^ 0xFA11BAC4ULL) % n_rows;
}

/* Key of the class-`k` tree of a round: seeds its colsample_bytree pool. */
SB_HD uint64_t sb_tree_key(uint64_t seed, uint64_t round, uint64_t k) {
  return sb_mix64(seed ^ sb_mix64((round << 20) + k) ^ 0x706F6F6CULL);
}

/* Key of node `nid` of a tree: seeds its bylevel/bynode subset. */
SB_HD uint64_t sb_node_key(uint64_t tree_key, uint64_t nid) {
  return sb_mix64(tree_key ^ sb_mix64(nid + 0x6E6F6465ULL));
}

/* Key of a DART round's dropout draws (train.rs:397-425): a sequential
 * stream seeded with it draws skip (u01 < skip_drop), then one u01 per
 * existing tree (dropped if < rate_drop), then, when none was dropped, the
 * one tree to drop (bounded draw). The host side of the DART loop uses it. */
SB_HD uint64_t sb_dart_key(uint64_t seed, uint64_t round) {
  return sb_mix64(seed ^ sb_mix64(round + 0x0DA27ULL) ^ 0x64617274ULL);
}

/* Sequential SplitMix64 stream. */
typedef struct sb_splitmix { uint64_t s; } sb_splitmix;

SB_HD uint64_t sb_splitmix_next(sb_splitmix* g) {
  uint64_t z = (g->s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* Uniform integer in [0, n) by a 64x64->128 multiply (Lemire, no rejection). */
SB_HD uint64_t sb_splitmix_bounded(sb_splitmix* g, uint64_t n) {
  uint64_t x = sb_splitmix_next(g);
#if defined(__CUDA_ARCH__)
  return __umul64hi(x, n);
#else
  return (uint64_t)(((unsigned __int128)x * n) >> 64);
#endif
}

/*
 * Fisher-Yates shuffle from the back (as SliceRandom::shuffle) followed by a
 * truncation to k = clamp(round(ratio*len), 1, len); returns k. The first k
 * entries are the sample, in shuffled order. ratio >= 1 or len <= 1 keeps
 * the pool and draws nothing.
 */
SB_HD int sb_shuffle_truncate(uint32_t* idx, int len, double ratio, sb_splitmix* g) {
  if (ratio >= 1.0 || len <= 1) return len;
  /* f64::round and C round() both round half away from zero. */
  long long k = (long long)round(ratio * (double)len);
  if (k < 1) k = 1;
  if (k > len) k = len;
  for (int i = len - 1; i >= 1; --i) {
    int j = (int)sb_splitmix_bounded(g, (uint64_t)(i + 1));
    uint32_t t = idx[i]; idx[i] = idx[j]; idx[j] = t;
  }
  return (int)k;
}

/*
 * subsample(pool, ratio): in place on `idx[0..len)`; returns the new length.
 * Same steps as tree/sampler.rs:60-70 and train.rs:479-489: shuffle, truncate,
 * sort ascending.
 */
SB_HD int sb_subsample(uint32_t* idx, int len, double ratio, sb_splitmix* g) {
  if (ratio >= 1.0 || len <= 1) return len;
  int k = sb_shuffle_truncate(idx, len, ratio, g);
  for (int i = 1; i < k; ++i) { /* insertion sort (pools are small) */
    uint32_t v = idx[i];
    int j = i - 1;
    while (j >= 0 && idx[j] > v) { idx[j + 1] = idx[j]; --j; }
    idx[j + 1] = v;
  }
  return k;
}

#endif /* SB_SAMPLING_H */
