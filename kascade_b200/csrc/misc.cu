// Small kernels behind the C ABI: seeded input generators, the initial
// ranking state, and pack / unpack of an active sub-list.
#include <algorithm>

#include "ctx.cuh"
#include "gen_common.h"

namespace ks {

namespace {

__global__ void __launch_bounds__(256) k_gen_list(uint64_t n, ks_perm perm, uint32_t layout, uint64_t* __restrict__ succ) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t e = ks_list_elem(&perm, layout, n, k);
    succ[e] = (k + 1 < n) ? ks_list_elem(&perm, layout, n, k + 1) : e;
  }
}

__global__ void __launch_bounds__(256) k_gen_weights(uint64_t n, uint64_t seed, uint32_t wbits, uint32_t* __restrict__ w) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    w[i] = ks_weight(seed, i, wbits);
}

__global__ void __launch_bounds__(256) k_gen_forest(uint64_t n, ks_perm perm, uint32_t kind, uint64_t blocks,
                                                    uint64_t spine, uint64_t seed, uint64_t* __restrict__ parent) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t at, par;
    ks_forest_edge(&perm, kind, n, blocks, spine, seed, v, &at, &par);
    parent[at] = par;
  }
}

// list_ranking.cpp:60-80
__global__ void __launch_bounds__(256) k_initial_state(const uint64_t* __restrict__ succ, uint64_t n,
                                                       uint64_t* __restrict__ root, int64_t* __restrict__ rank) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = succ[i];
    root[i] = s;
    rank[i] = (s == i) ? 0 : 1;
  }
}

__global__ void __launch_bounds__(256) k_fill_u64(uint64_t* __restrict__ a, uint64_t n, uint64_t v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) a[i] = v;
}

__global__ void __launch_bounds__(256) k_pack_index(const uint64_t* __restrict__ active, uint64_t k, uint64_t n,
                                                    uint64_t* __restrict__ to_packed, DevStatus* st) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < k; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a = active[j];
    if (a >= n || (j > 0 && active[j - 1] >= a)) {
      set_error(st, KASCADE_ERR_INVALID_ARG, j);
      continue;
    }
    to_packed[a] = j;
  }
}

// pack.hpp:23-80 on one rank
__global__ void __launch_bounds__(256) k_pack(const uint64_t* __restrict__ succ, const int64_t* __restrict__ rank,
                                              uint64_t n, const uint64_t* __restrict__ active, uint64_t k,
                                              const uint64_t* __restrict__ to_packed, uint64_t* __restrict__ succ_packed,
                                              int64_t* __restrict__ rank_packed, DevStatus* st) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < k; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a = active[j];
    if (a >= n) continue;
    const uint64_t s = succ[a];
    const uint64_t ps = (s < n) ? to_packed[s] : ~0ull;
    if (ps == ~0ull) {
      set_error(st, KASCADE_ERR_INVALID_ARG, j);
      continue;
    }
    succ_packed[j] = ps;
    rank_packed[j] = rank[a];
  }
}

// pack.hpp:81-175 (the unpack closure) on one rank
__global__ void __launch_bounds__(256) k_unpack(const uint64_t* __restrict__ succ_packed,
                                                const int64_t* __restrict__ rank_packed,
                                                const uint64_t* __restrict__ active, uint64_t k, uint64_t n,
                                                uint64_t* __restrict__ succ, int64_t* __restrict__ rank, DevStatus* st) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < k; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a = active[j], sp = succ_packed[j];
    if (a >= n || sp >= k) {
      set_error(st, KASCADE_ERR_INVALID_ARG, j);
      continue;
    }
    succ[a] = active[sp];
    rank[a] = rank_packed[j];
  }
}

}  // namespace

kascade_status gen_list(uint64_t n, uint64_t seed, uint32_t layout, uint64_t* succ, cudaStream_t s) {
  if (n == 0) return KASCADE_OK;
  ks_perm p = ks_list_perm(n, seed, layout);
  k_gen_list<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16), 256, 0, s>>>(n, p, layout, succ);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status gen_weights(uint64_t n, uint64_t seed, uint32_t wbits, uint32_t* w, cudaStream_t s) {
  if (n == 0) return KASCADE_OK;
  k_gen_weights<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16), 256, 0, s>>>(n, seed, wbits, w);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status gen_forest(uint64_t n, uint64_t seed, uint32_t kind, uint64_t blocks, uint64_t spine, uint64_t* parent,
                          cudaStream_t s) {
  if (n == 0) return KASCADE_OK;
  ks_perm p = ks_forest_perm(n, seed);
  k_gen_forest<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16), 256, 0, s>>>(n, p, kind, blocks, spine,
                                                                                          seed, parent);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status initial_state(kascade_ctx& ctx, const uint64_t* succ, uint64_t n, uint64_t* root, int64_t* rank,
                             cudaStream_t s) {
  if (n == 0) return KASCADE_OK;
  k_initial_state<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(succ, n, root, rank);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status pack_impl(kascade_ctx& ctx, const uint64_t* succ, const int64_t* rank, uint64_t n,
                         const uint64_t* active, uint64_t k, uint64_t* succ_packed, int64_t* rank_packed,
                         cudaStream_t s) {
  if (k == 0) return KASCADE_OK;
  uint64_t* to_packed = alloc<uint64_t>(ctx, n);
  if (!to_packed) return KASCADE_ERR_OOM;
  k_fill_u64<<<grid_for(ctx, n, 256, 8), 256, 0, s>>>(to_packed, n, ~0ull);
  KS_CHECK_LAUNCH();
  k_pack_index<<<grid_for(ctx, k, 256, 8), 256, 0, s>>>(active, k, n, to_packed, ctx.d_status);
  KS_CHECK_LAUNCH();
  k_pack<<<grid_for(ctx, k, 256, 8), 256, 0, s>>>(succ, rank, n, active, k, to_packed, succ_packed, rank_packed,
                                                  ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status unpack_impl(kascade_ctx& ctx, const uint64_t* succ_packed, const int64_t* rank_packed,
                           const uint64_t* active, uint64_t k, uint64_t* succ, int64_t* rank, uint64_t n,
                           cudaStream_t s) {
  if (k == 0) return KASCADE_OK;
  k_unpack<<<grid_for(ctx, k, 256, 8), 256, 0, s>>>(succ_packed, rank_packed, active, k, n, succ, rank, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

}  // namespace ks
