/*
 * Seeded synthetic-input generators for list ranking and tree rooting.
 *
 * These are the benchmark inputs (the role KaGen plays for the reference's
 * bench/input/generation.cpp:64-96): random successor lists, locality-biased
 * lists, random recursive forests and caterpillar forests.  Every generator is
 * a pure function of (seed, index), written in plain C so that the CUDA
 * generator kernels and the CPU oracle compute bit-identical arrays.
 *
 *  - ks_mix64          : the SplitMix64 finaliser (Vigna, public domain
 *                        algorithm) used as a counter-based hash.
 *  - ks_perm_*         : a keyed 4-round balanced Feistel network over
 *                        [0, 2^bits) with cycle walking down to [0, n) --
 *                        a seeded pseudo-random permutation computable per
 *                        index in O(1) on host and device alike.
 */
#ifndef KASCADE_B200_GEN_COMMON_H
#define KASCADE_B200_GEN_COMMON_H

#include <stdint.h>

#if defined(__CUDACC__)
#define KS_HD __host__ __device__ __forceinline__
#else
#define KS_HD static inline
#endif

KS_HD uint64_t ks_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* Hash of (seed, stream, index): independent streams per generator role. */
KS_HD uint64_t ks_hash3(uint64_t seed, uint64_t stream, uint64_t idx) {
  return ks_mix64(ks_mix64(seed ^ (stream * 0xD1B54A32D192ED03ull)) + idx);
}

/* Uniform integer in [0, bound) from a 64-bit hash (multiply-shift). */
KS_HD uint64_t ks_bounded(uint64_t h, uint64_t bound) {
  /* (h >> 32) * bound >> 32 is exact for bound < 2^32 */
  return ((h >> 32) * bound) >> 32;
}

typedef struct {
  uint64_t n;
  uint64_t half_mask;
  uint32_t half_bits;
  uint32_t pad;
  uint64_t keys[4];
} ks_perm;

KS_HD ks_perm ks_perm_make(uint64_t n, uint64_t seed) {
  ks_perm p;
  uint32_t bits = 0;
  while (bits < 64 && (1ull << bits) < n) bits++;
  if (bits < 2) bits = 2;
  if (bits & 1u) bits++;
  p.n = n;
  p.half_bits = bits / 2;
  p.half_mask = (p.half_bits >= 64) ? ~0ull : ((1ull << p.half_bits) - 1ull);
  p.pad = 0;
  for (int i = 0; i < 4; ++i) p.keys[i] = ks_hash3(seed, 0x5045524Dull + (uint64_t)i, 0);
  return p;
}

KS_HD uint64_t ks_perm_encrypt(const ks_perm* p, uint64_t x) {
  uint64_t l = x >> p->half_bits;
  uint64_t r = x & p->half_mask;
  for (int i = 0; i < 4; ++i) {
    uint64_t nl = r;
    uint64_t nr = l ^ (ks_mix64(r ^ p->keys[i]) & p->half_mask);
    l = nl;
    r = nr;
  }
  return (l << p->half_bits) | r;
}

/* The permutation of [0, n): cycle walking keeps every value below n. */
KS_HD uint64_t ks_perm_apply(const ks_perm* p, uint64_t x) {
  uint64_t y = ks_perm_encrypt(p, x);
  while (y >= p->n) y = ks_perm_encrypt(p, y);
  return y;
}

/* ---------------------------------------------------------------------------
 * Lists.  The list visits elements in "order position" k = 0..n-1; the
 * element at position k has the element at position k+1 as successor and the
 * element at position n-1 (the tail) is the root (succ == self).
 * ------------------------------------------------------------------------ */

#define KS_LAYOUT_RANDOM 0u /* order = a random permutation of [0, n)          */
#define KS_LAYOUT_RUNS 1u   /* order = runs of KS_RUN consecutive indices,
                               runs visited in random order                     */
#define KS_LAYOUT_IDENTITY 2u /* order = 0, 1, ..., n-1 (a sequential path)     */
#define KS_RUN 64u

/* Element at order position k. `perm` must be made with n (RANDOM) or with
 * n / KS_RUN runs (RUNS). */
KS_HD uint64_t ks_list_elem(const ks_perm* perm, uint32_t layout, uint64_t n, uint64_t k) {
  if (layout == KS_LAYOUT_RANDOM) return ks_perm_apply(perm, k);
  if (layout == KS_LAYOUT_RUNS) {
    uint64_t full = (n / KS_RUN) * KS_RUN;
    if (k >= full) return k; /* a trailing partial run keeps its place at the end */
    return ks_perm_apply(perm, k / KS_RUN) * KS_RUN + (k % KS_RUN);
  }
  return k;
}

KS_HD ks_perm ks_list_perm(uint64_t n, uint64_t seed, uint32_t layout) {
  uint64_t m = (layout == KS_LAYOUT_RUNS) ? (n / KS_RUN) : n;
  if (m == 0) m = 1;
  return ks_perm_make(m, ks_hash3(seed, 0x4C495354ull, layout));
}

/* Weight of element i: uniform integer in [0, 2^wbits). */
KS_HD uint32_t ks_weight(uint64_t seed, uint64_t i, uint32_t wbits) {
  uint64_t h = ks_hash3(seed, 0x57454947ull, i);
  if (wbits >= 32) return (uint32_t)(h >> 32);
  return (uint32_t)(h >> (64 - wbits));
}

/* ---------------------------------------------------------------------------
 * Forests, given as parent arrays (a root is its own parent).  Vertices are
 * generated in "local" ids and relabelled by a random permutation of [0, n).
 * ------------------------------------------------------------------------ */

/* Block [start, end) of block b when n is split into `blocks` near-equal parts
 * (the last block takes the remainder). */
KS_HD void ks_block_range(uint64_t n, uint64_t blocks, uint64_t b, uint64_t* start, uint64_t* end) {
  uint64_t sz = n / blocks;
  *start = b * sz;
  *end = (b + 1 == blocks) ? n : (b + 1) * sz;
}

/* Random recursive trees: in each block, local vertex i > start picks its
 * parent uniformly in [start, i); `start` is the tree root. Returns the local
 * parent of local vertex v. */
KS_HD uint64_t ks_rrt_parent_local(uint64_t n, uint64_t trees, uint64_t seed, uint64_t v) {
  uint64_t sz = n / trees;
  uint64_t b = (sz == 0) ? 0 : v / sz;
  if (b >= trees) b = trees - 1;
  uint64_t s, e;
  ks_block_range(n, trees, b, &s, &e);
  if (v == s) return v;
  return s + ks_bounded(ks_hash3(seed, 0x52525450ull, v), v - s);
}

/* Caterpillars: each block is one caterpillar whose first `spine` local
 * vertices form a path (local id start is the root, start+i hangs below
 * start+i-1); every other vertex is a leaf attached to a uniformly random
 * spine vertex. */
KS_HD uint64_t ks_cat_parent_local(uint64_t n, uint64_t cats, uint64_t spine, uint64_t seed, uint64_t v) {
  uint64_t sz = n / cats;
  uint64_t b = (sz == 0) ? 0 : v / sz;
  if (b >= cats) b = cats - 1;
  uint64_t s, e;
  ks_block_range(n, cats, b, &s, &e);
  uint64_t len = e - s;
  uint64_t sp = spine < len ? spine : len;
  uint64_t i = v - s;
  if (i == 0) return v;
  if (i < sp) return v - 1;
  return s + ks_bounded(ks_hash3(seed, 0x43415450ull, v), sp);
}

#define KS_FOREST_RRT 0u
#define KS_FOREST_CATERPILLAR 1u

KS_HD ks_perm ks_forest_perm(uint64_t n, uint64_t seed) {
  return ks_perm_make(n ? n : 1, ks_hash3(seed, 0x52454C42ull, 0));
}

/* Relabelled forest: returns (label(v), label(parent_local(v))) for local v. */
KS_HD void ks_forest_edge(const ks_perm* perm, uint32_t kind, uint64_t n, uint64_t blocks,
                          uint64_t spine, uint64_t seed, uint64_t v, uint64_t* at,
                          uint64_t* parent) {
  uint64_t pl = (kind == KS_FOREST_RRT) ? ks_rrt_parent_local(n, blocks, seed, v)
                                        : ks_cat_parent_local(n, blocks, spine, seed, v);
  *at = ks_perm_apply(perm, v);
  *parent = ks_perm_apply(perm, pl);
}

#endif /* KASCADE_B200_GEN_COMMON_H */
