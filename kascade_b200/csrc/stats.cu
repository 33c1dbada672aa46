// Device-side result statistics: the bench's compute_stats
// (bench/detail/stats.cpp:110-143 basic, 24-108 per tree) over root and rank
// arrays already in HBM.
//
//   pass 1  per element: warp-level aggregation of (size, rank sum, max rank)
//           by root (match_any), then one set of global atomics per distinct
//           root of a warp into arrays indexed by root; grid-wide count of
//           roots (root[i] == i), rank sum and max rank
//   pass 2  per root: the extensive figures (trees, non-trivial trees, size
//           and rank sums, max size) and a root-ordered list of the
//           non-trivial trees (stream compaction by one exclusive scan)
//
// Semantics kept from the reference, quirks included: a tree's max_rank
// starts at 0 (TreeStats, bench/detail/stats.hpp:23-27, updated with
// std::max at stats.cpp:38), so a tree whose ranks are all negative reports
// 0; the basic average divides the rank sum taken as an unsigned 64-bit value
// (stats.cpp:124-137 fold into std::size_t) by n.
#include <algorithm>
#include <climits>
#include <cstring>

#include "ranker.cuh"
#include "sort.cuh"

namespace ks {
namespace {

constexpr unsigned FULL = 0xffffffffu;

struct __align__(16) StatAcc {
  unsigned long long num_roots;
  unsigned long long rank_sum;  // int64 sum, two's complement
  long long max_rank;
  unsigned long long trees;
  unsigned long long nontrivial;
  unsigned long long nt_size_sum;
  unsigned long long nt_rank_sum;
  unsigned long long max_size;
};

__global__ void __launch_bounds__(256) k_stats_elems(const uint64_t* __restrict__ root, const int64_t* __restrict__ rank,
                                                     uint64_t n, int per_tree, unsigned long long* __restrict__ tsize,
                                                     unsigned long long* __restrict__ tsum,
                                                     long long* __restrict__ tmax, StatAcc* acc, DevStatus* st) {
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long roots = 0, sum = 0;
  long long mx = LLONG_MIN;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    const uint64_t i = base + threadIdx.x;
    const bool valid = i < n;
    unsigned long long r = 0;
    long long k = 0;
    if (valid) {
      r = __ldcs(reinterpret_cast<const unsigned long long*>(root) + i);
      k = __ldcs(reinterpret_cast<const long long*>(rank) + i);
      if (r >= n) {
        set_error(st, KASCADE_ERR_OUT_OF_RANGE, i);
        r = i;
      }
      roots += (r == i);
      sum += (unsigned long long)k;
      mx = max(mx, k);
    }
    if (per_tree) {
      // lanes with the same root combine; the lowest such lane updates HBM
      const unsigned long long key = valid ? r : ~0ull;
      const uint32_t peers = __match_any_sync(FULL, key);
      unsigned long long c = valid ? 1ull : 0ull, s = (unsigned long long)k;
      long long m = valid ? k : LLONG_MIN;
      // reduce over the peer set: every peer reads every peer's values
      uint32_t pm = peers;
      unsigned long long cs = 0, ss = 0;
      long long ms = LLONG_MIN;
      while (pm) {
        const int src = __ffs(pm) - 1;
        pm &= pm - 1;
        cs += __shfl_sync(peers, c, src);
        ss += __shfl_sync(peers, s, src);
        ms = max(ms, (long long)__shfl_sync(peers, m, src));
      }
      if (valid && lane == (uint32_t)(__ffs(peers) - 1)) {
        atomicAdd(tsize + r, cs);
        atomicAdd(tsum + r, ss);
        atomicMax(tmax + r, ms);
      }
    }
  }
  // grid-wide basic figures: one atomic per warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    roots += __shfl_down_sync(FULL, roots, o);
    sum += __shfl_down_sync(FULL, sum, o);
    mx = max(mx, (long long)__shfl_down_sync(FULL, mx, o));
  }
  if (lane == 0) {
    atomicAdd(&acc->num_roots, roots);
    atomicAdd(&acc->rank_sum, sum);
    atomicMax(&acc->max_rank, mx);
  }
}

__global__ void __launch_bounds__(256) k_stats_fill(unsigned long long* __restrict__ tsize,
                                                    unsigned long long* __restrict__ tsum,
                                                    long long* __restrict__ tmax, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    tsize[i] = 0;
    tsum[i] = 0;
    tmax[i] = 0;  // TreeStats::max_rank = 0
  }
}

// Per root: the extensive figures and a flag per non-trivial tree.
__global__ void __launch_bounds__(256) k_stats_trees(const unsigned long long* __restrict__ tsize,
                                                     const unsigned long long* __restrict__ tsum, uint64_t n,
                                                     uint32_t* __restrict__ nt_flag, StatAcc* acc) {
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long trees = 0, nt = 0, ntsz = 0, ntsum = 0, mxs = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long sz = tsize[i];
    uint32_t f = 0;
    if (sz) {
      trees++;
      mxs = max(mxs, sz);
      if (sz > 1) {
        nt++;
        ntsz += sz;
        ntsum += tsum[i];
        f = 1;
      }
    }
    if (nt_flag) nt_flag[i] = f;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    trees += __shfl_down_sync(FULL, trees, o);
    nt += __shfl_down_sync(FULL, nt, o);
    ntsz += __shfl_down_sync(FULL, ntsz, o);
    ntsum += __shfl_down_sync(FULL, ntsum, o);
    mxs = max(mxs, (unsigned long long)__shfl_down_sync(FULL, mxs, o));
  }
  if (lane == 0) {
    atomicAdd(&acc->trees, trees);
    atomicAdd(&acc->nontrivial, nt);
    atomicAdd(&acc->nt_size_sum, ntsz);
    atomicAdd(&acc->nt_rank_sum, ntsum);
    atomicMax(&acc->max_size, mxs);
  }
}

__global__ void __launch_bounds__(256) k_stats_list(const unsigned long long* __restrict__ tsize,
                                                    const unsigned long long* __restrict__ tsum,
                                                    const long long* __restrict__ tmax, uint64_t n,
                                                    const uint32_t* __restrict__ nt_flag,
                                                    const uint32_t* __restrict__ pos, kascade_tree_stats* out,
                                                    uint64_t cap) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (!nt_flag[i]) continue;
    const uint64_t p = pos[i];
    if (p < cap) out[p] = kascade_tree_stats{i, tsize[i], tmax[i], (int64_t)tsum[i]};
  }
}

double safe_div(double a, double b) { return b == 0.0 ? 0.0 : a / b; }

}  // namespace

kascade_status compute_stats(kascade_ctx& ctx, const uint64_t* root, const int64_t* rank, uint64_t n, int level,
                             kascade_stats* out, kascade_tree_stats* per_tree, uint64_t per_tree_cap,
                             uint64_t* per_tree_count, cudaStream_t s) {
  const bool extensive = level >= KASCADE_STATS_REDUCED_EXTENSIVE;
  StatAcc* acc = alloc<StatAcc>(ctx, 1);
  if (!acc) return KASCADE_ERR_OOM;
  StatAcc init{};
  init.max_rank = LLONG_MIN;
  KS_CUDA(cudaMemcpyAsync(acc, &init, sizeof(StatAcc), cudaMemcpyHostToDevice, s));
  unsigned long long *tsize = nullptr, *tsum = nullptr;
  long long* tmax = nullptr;
  if (extensive) {
    tsize = alloc<unsigned long long>(ctx, n);
    tsum = alloc<unsigned long long>(ctx, n);
    tmax = alloc<long long>(ctx, n);
    if (!tsize || !tsum || !tmax) return KASCADE_ERR_OOM;
    k_stats_fill<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(tsize, tsum, tmax, n);
    KS_CHECK_LAUNCH();
  }
  {
    ProfScope ps(ctx, "stats", s);
    k_stats_elems<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(root, rank, n, extensive ? 1 : 0, tsize, tsum, tmax, acc,
                                                           ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  const bool want_list = level >= KASCADE_STATS_EXTENSIVE && per_tree;
  uint32_t* flag = nullptr;
  uint32_t* pos = nullptr;
  if (extensive) {
    if (want_list) {
      flag = alloc<uint32_t>(ctx, n);
      pos = alloc<uint32_t>(ctx, n);
      if (!flag || !pos) return KASCADE_ERR_OOM;
    }
    k_stats_trees<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(tsize, tsum, n, flag, acc);
    KS_CHECK_LAUNCH();
    if (want_list) {
      KS_TRY(exclusive_scan_u32(ctx, flag, pos, n, nullptr, s));
      k_stats_list<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(tsize, tsum, tmax, n, flag, pos, per_tree,
                                                            per_tree_cap);
      KS_CHECK_LAUNCH();
    }
  }
  StatAcc h{};
  KS_CUDA(cudaMemcpyAsync(&h, acc, sizeof(StatAcc), cudaMemcpyDeviceToHost, s));
  KS_CUDA(cudaStreamSynchronize(s));
  std::memset(out, 0, sizeof(*out));
  out->num_trees = h.num_roots;
  out->max_rank = n ? h.max_rank : 0;
  // the reference folds the int64 ranks into a std::size_t sum and divides
  // that unsigned value (stats.cpp:124-137)
  out->avg_rank = safe_div((double)h.rank_sum, (double)n);
  if (extensive) {
    out->ext_num_trees = h.trees;
    out->num_nontrivial_trees = h.nontrivial;
    out->nontrivial_size_sum = h.nt_size_sum;
    out->nontrivial_rank_sum = (int64_t)h.nt_rank_sum;
    out->max_size = h.max_size;
    const uint64_t trivial = h.trees - h.nontrivial;
    out->avg_size = safe_div((double)(h.nt_size_sum + trivial), (double)h.trees);
    out->nontrivial_avg_size = safe_div((double)h.nt_size_sum, (double)h.nontrivial);
    out->nontrivial_avg_rank = safe_div((double)(long long)h.nt_rank_sum, (double)h.nt_size_sum);
  }
  if (per_tree_count) *per_tree_count = want_list ? h.nontrivial : 0;
  return KASCADE_OK;
}

}  // namespace ks
