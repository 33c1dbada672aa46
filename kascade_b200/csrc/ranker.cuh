// Internal interface of the ruling-set list ranker.
//
// Pipeline for a list of n elements held as 16 B records (Rec):
//   prepare   : counter-hash ruler sampling + ruler ids       (level 0 from the
//               caller's arrays, deeper levels in place)
//   chase     : every ruler walks its successors until the next ruler,
//               stamping (ruler id, distance) into each record it passes and
//               writing the ruler's sub-list record for the next level
//   recurse   : the sub-list of rulers is ranked the same way, down to a
//               one-CTA shared-memory base case (or pointer doubling when a
//               level does not shrink)
//   propagate : one coalesced pass: rank = rank(ruler) - distance, root =
//               root(ruler); elements ahead of their list's first ruler walk
//               forward to the first stamped element
#pragma once

#include "common.cuh"
#include "ctx.cuh"

namespace ks {

struct Params {
  uint32_t spacing0 = 48;      // mean elements per ruler, level 0
  uint32_t spacing_deep = 24;  // mean elements per ruler, deeper levels
  uint32_t max_levels = 6;
  uint32_t base_max = 8192;    // one-CTA base case bound
  uint32_t chains = 2;         // chains in flight per thread (1, 2 or 4)
  uint32_t block = 256;
  uint32_t seed = 0x6b617363u;
  uint32_t algorithm = KASCADE_ALGO_SPARSE_RULING_SET;
  uint32_t level0_log_min = 1u << 25;  // level 0 uses the write-free path from this size on
  uint32_t max_chain = 0;              // write-free chase hop cap (0: 64 x spacing0 + 1024)
};

Params make_params(const kascade_ctx& ctx, const kascade_opts* opts, uint64_t n);

// Mean ruler spacing for an instance of n elements (the size-class table).
uint32_t spacing_for(const kascade_ctx& ctx, uint64_t n);

// Where results of level 0 go ------------------------------------------------
// A sink receives, for element x, its rank, its root (level-0 index) and
// whether x itself is a root.

// Level-0 output description for the write-free (log) pipeline.
struct LogTarget {
  uint64_t* root;
  uint64_t* rank;
  uint32_t limit;        // elements [0, limit) produce output
  int keep_roots;        // leave roots' entries untouched
  int heads_are_rulers;  // every list head is a ruler: no element is left unreached
  // a batch of instances in one index space: roots are reported relative to
  // their instance (seg_off: nseg instance offsets, hint[k]: the instance
  // holding element k * 4096); null for a single instance
  const uint64_t* seg_off = nullptr;
  const uint32_t* hint = nullptr;
  uint32_t nseg = 0;
  // bit x set: element x's rank output is one more than its rank in the list
  // (a tree rooting's leaves, whose down and up edge share one element)
  const uint32_t* plus_one = nullptr;
  // heads_are_rulers: how many elements at or above limit a valid input logs
  // (device memory; null: every element from limit to n)
  const uint32_t* beyond_want = nullptr;
};

// Plain arrays. keep_roots: leave root entries untouched (the reference's
// in-place contract); otherwise roots get (x, 0).
struct SinkPlain {
  static constexpr bool kWriteFree = true;
  uint64_t* root;
  uint64_t* rank;
  int keep_roots;
  // elements [0, limit(n)) produce output
  uint32_t limit(uint32_t n) const { return n; }
  LogTarget log_target(uint32_t n) const { return LogTarget{root, rank, n, keep_roots, 0}; }
  __device__ __forceinline__ void put(uint32_t x, uint64_t rk, uint32_t rt, bool is_root) const {
    if (is_root) {
      if (!keep_roots) {
        __stcs(root + x, (unsigned long long)x);
        __stcs(rank + x, 0ull);
      }
      return;
    }
    __stcs(root + x, (unsigned long long)rt);
    __stcs(rank + x, (unsigned long long)rk);
  }
};

// Euler tour: elements 0..nv-1 are the vertices' up edges (roots: the tour's
// terminal element), so only those produce output.
// leaf_bits (optional): bit v set for a leaf whose down and up edge are one
// element of weight 0, whose rank is then one less than the leaf's depth.
struct SinkTour {
  static constexpr bool kWriteFree = true;
  uint64_t* root;
  uint64_t* depth;
  uint32_t nv;
  int keep_roots;
  const uint32_t* leaf_bits = nullptr;
  // the tour's down-edge count in device memory when the records are sized
  // for a bound (2 nv) rather than the tour's length
  const uint32_t* downs_dev = nullptr;
  uint32_t limit(uint32_t n) const { return n < nv ? n : nv; }
  // the tour build makes every tour head a ruler
  LogTarget log_target(uint32_t n) const {
    LogTarget t{root, depth, limit(n), keep_roots, 1};
    t.plus_one = leaf_bits;
    t.beyond_want = downs_dev;
    return t;
  }
  __device__ __forceinline__ void put(uint32_t x, uint64_t rk, uint32_t rt, bool is_root) const {
    if (x >= nv) return;
    if (is_root) {
      if (!keep_roots) {
        __stcs(root + x, (unsigned long long)x);
        __stcs(depth + x, 0ull);
      }
      return;
    }
    if (leaf_bits) rk += (__ldg(leaf_bits + (x >> 5)) >> (x & 31)) & 1u;
    __stcs(root + x, (unsigned long long)rt);
    __stcs(depth + x, (unsigned long long)rk);
  }
};

// A batch of independent instances concatenated into one index space:
// roots are reported relative to their instance.  seg_off holds the nseg
// instance offsets (non-decreasing), hint[k] the instance containing element
// k * 4096.  Elements at or beyond `total` (tour down edges) give no output.
// plus_one (optional): bit x set for a forest leaf whose down and up edge are
// one element, whose rank is then one less than the leaf's depth.
struct SinkBatch {
  static constexpr bool kWriteFree = true;
  uint64_t* root;
  uint64_t* rank;
  uint32_t total;
  const uint64_t* seg_off;
  const uint32_t* hint;
  uint32_t nseg;
  const uint32_t* plus_one = nullptr;
  uint32_t limit(uint32_t n) const { return n < total ? n : total; }
  LogTarget log_target(uint32_t n) const {
    LogTarget t{root, rank, limit(n), 0, 0, seg_off, hint, nseg};
    t.plus_one = plus_one;
    return t;
  }
  __device__ __forceinline__ uint64_t base_of(uint32_t x) const {
    uint32_t j = __ldg(hint + (x >> 12));
    while (j + 1 < nseg && __ldg(seg_off + j + 1) <= x) ++j;
    return __ldg(seg_off + j);
  }
  __device__ __forceinline__ void put(uint32_t x, uint64_t rk, uint32_t rt, bool is_root) const {
    if (x >= total) return;
    const uint64_t b = base_of(x);
    if (is_root) {
      __stcs(root + x, (unsigned long long)(x - b));
      __stcs(rank + x, 0ull);
      return;
    }
    if (plus_one) rk += (__ldg(plus_one + (x >> 5)) >> (x & 31)) & 1u;
    __stcs(root + x, (unsigned long long)(rt - b));
    __stcs(rank + x, (unsigned long long)rk);
  }
};

// Deeper levels write Out records.
struct SinkOut {
  static constexpr bool kWriteFree = false;
  Out* out;
  uint32_t limit(uint32_t n) const { return n; }
  __device__ __forceinline__ void put(uint32_t x, uint64_t rk, uint32_t rt, bool is_root) const {
    st_out(out + x, is_root ? 0ull : rk, rt);
  }
};

// Weight readers for building level-0 records.
enum class WKind { Unit, U32, I64 };

// Build level-0 records from (succ, weights), sample rulers and number them.
// ruler_elem must hold n entries; *r_out receives the ruler count.
kascade_status prepare_arrays(kascade_ctx& ctx, const uint64_t* succ, WKind wk, const void* w,
                              uint32_t n, Rec* rec, uint32_t* ruler_elem, uint32_t* r_out,
                              const Params& p, cudaStream_t s, uint32_t** r_dev = nullptr);

// Rank level-0 records that carry ruler tags (r0 rulers, listed in
// ruler_elem0) and deliver the results to the sink.
template <class Sink>
kascade_status rank_records(kascade_ctx& ctx, Rec* rec, uint32_t n, uint32_t r0,
                            uint32_t* ruler_elem0, const Sink& sink, const Params& p,
                            cudaStream_t s);

// Rank a deeper level (records written by the chase of the level above, tags
// unassigned); results go to out[0..n).  elem0 maps this level's elements to
// level-0 indices.
kascade_status rank_sublist(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* elem0, Out* out,
                            int level, const Params& p, cudaStream_t s);

// The recursion without host waits (see ranker.cu): r0_dev holds the level-0
// ruler count, cap1 bounds it.  Errors, including a level that outgrows its
// capacity (KASCADE_ERR_TIMEOUT: rerun on the host-driven path), land in the
// device status word.
template <class Sink>
kascade_status rank_records_dev(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* r0_dev, uint32_t cap1,
                                uint32_t* ruler_elem0, const Sink& sink, const Params& p, cudaStream_t s);
uint32_t dev_cap_next(uint32_t cap, uint32_t spacing);
constexpr int MAX_DEV_LEVELS = 8;
// Levels 1.. of that recursion: rec1 / out1 hold cap1 elements, cnt (device,
// MAX_DEV_LEVELS + 2 words) holds level 1's size in cnt[1] once the level-0
// chase has run; pred1 (optional, cap1 bits): level-1 elements a level-0
// chain ended at (the others head their lists and become rulers); fills out1
// and cnt[2..L], *levels = L.
kascade_status rank_deep_dev(kascade_ctx& ctx, Rec* rec1, Out* out1, uint32_t cap1, uint32_t* cnt,
                             const uint32_t* elem0_1, const uint32_t* pred1, const Params& p, cudaStream_t s,
                             int* levels);
// *copy = *cnt, and KASCADE_ERR_TIMEOUT in the status word when it exceeds cap.
// lv[0] = base + *add: level 0's size in the device-driven level array when
// only the device knows it (a tour's length), reported in place of the call's n.
kascade_status launch_set_level0(kascade_ctx& ctx, uint32_t* lv, uint32_t base, const uint32_t* add,
                                 cudaStream_t s);
kascade_status launch_check_count(kascade_ctx& ctx, const uint32_t* cnt, uint32_t cap, uint32_t* copy,
                                  cudaStream_t s);
// Level sizes cnt[1..L] travel back with the call's status read.
kascade_status report_dev_levels(kascade_ctx& ctx, const uint32_t* cnt, int L, uint32_t n, cudaStream_t s);

kascade_status compute_stats(kascade_ctx& ctx, const uint64_t* root, const int64_t* rank, uint64_t n, int level,
                             kascade_stats* out, kascade_tree_stats* per_tree, uint64_t per_tree_cap,
                             uint64_t* per_tree_count, cudaStream_t s);

// Write-free level 0: read-only chase that logs (element, ruler, distance),
// recursion on the ruler sub-list, then two radix passes over the log by
// element and a dense placement into the outputs.  With r0_dev the ruler
// count stays on the device (r0 is then its capacity) and so does the
// recursion: no host wait; a chain past the hop cap or a level past its
// capacity reports KASCADE_ERR_TIMEOUT in the status word (rerun on the
// host-driven path).  Without it, a chain past the hop cap returns
// KASCADE_ERR_TIMEOUT directly (level 0 again on the stamping path).
kascade_status rank_level0_log(kascade_ctx& ctx, const Rec* rec, uint32_t n, uint32_t r0,
                               const uint32_t* ruler_elem0, const LogTarget& t, const Params& p,
                               cudaStream_t s, const uint32_t* r0_dev = nullptr);


// Pointer doubling on level-0 records (tags ignored).
template <class Sink>
kascade_status pointer_double_records(kascade_ctx& ctx, const Rec* rec, uint32_t n,
                                      const uint32_t* elem0, const Sink& sink,
                                      cudaStream_t s);

// Validation: *ok = 1 if no element has two predecessors.
kascade_status check_is_list(kascade_ctx& ctx, const uint64_t* succ, uint64_t n, int* ok,
                             cudaStream_t s);

}  // namespace ks
