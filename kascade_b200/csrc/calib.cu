// Random-access calibration: the rate at which this GPU serves random 16 B
// record accesses in an array far larger than L2.  It measures the ceiling
// the ruler chase runs against (the hop of a chase is one dependent random
// 16 B load, optionally followed by a 16 B write to the same record).
//   mode 0: independent random reads
//   mode 1: independent random read + write back of the same record
//   mode 2: dependent chains (each read gives the next address), reads only
//   mode 3: dependent chains, read + write back
// and, for wider records (16 B of each read; the next address in its first
// 16 B), dependent chains:
//   mode 4: 32 B records, the whole 32 B written back
//   mode 5: 64 B records, the whole 64 B written back
//   mode 6: 64 B records, 16 B written back
//   mode 7: 32 B records, reads only
#include "ctx.cuh"
#include "gen_common.h"

namespace ks {
namespace {

__global__ void __launch_bounds__(256) k_cal_init(uint4* __restrict__ a, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = make_uint4((uint32_t)(ks_mix64(i) % n), 1u, 2u, 3u);
}

__global__ void __launch_bounds__(256) k_cal_independent(uint4* __restrict__ a, uint64_t n, uint64_t m, int write,
                                                         unsigned long long* sink) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t acc = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += 4 * stride) {
    uint64_t idx[4];
    uint4 v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) idx[j] = ks_mix64(i + j * stride + 0x9E37ull) % n;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (i + j * stride < m) v[j] = __ldcg(a + idx[j]);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (i + j * stride >= m) continue;
      acc += v[j].y;
      if (write) {
        v[j].w += 1;
        __stcg(a + idx[j], v[j]);
      }
    }
  }
  if (acc == 0x123456789ull) *sink = acc;
}

__global__ void __launch_bounds__(256) k_cal_chains(uint4* __restrict__ a, uint64_t n, uint64_t hops, int write,
                                                    unsigned long long* sink) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t x0 = (uint32_t)(ks_mix64(t) % n), x1 = (uint32_t)(ks_mix64(t + 0x5151ull) % n);
  uint64_t acc = 0;
  for (uint64_t h = 0; h < hops; ++h) {
    uint4 v0 = __ldcg(a + x0), v1 = __ldcg(a + x1);
    if (write) {
      v0.w = (uint32_t)h;
      v1.w = (uint32_t)h;
      __stcg(a + x0, v0);
      __stcg(a + x1, v1);
    }
    acc += v0.y + v1.y;
    x0 = v0.x;
    x1 = v1.x;
  }
  if (acc == 0x123456789ull) *sink = acc;
}

template <int W>
__global__ void __launch_bounds__(256) k_cal_init_wide(uint4* __restrict__ a, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    a[i * W] = make_uint4((uint32_t)(ks_mix64(i) % n), 1u, 2u, 3u);
#pragma unroll
    for (int k = 1; k < W; ++k) a[i * W + k] = make_uint4(0u, 0u, 0u, 0u);
  }
}

// W uint4 per record; write_all: rewrite the whole record, else its first 16 B
template <int W>
__global__ void __launch_bounds__(256) k_cal_chains_wide(uint4* __restrict__ a, uint64_t n, uint64_t hops, int write,
                                                         int write_all, unsigned long long* sink) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t x0 = (uint32_t)(ks_mix64(t) % n), x1 = (uint32_t)(ks_mix64(t + 0x5151ull) % n);
  uint64_t acc = 0;
  for (uint64_t h = 0; h < hops; ++h) {
    uint4 v0 = __ldcg(a + (uint64_t)x0 * W), v1 = __ldcg(a + (uint64_t)x1 * W);
    if (write) {
      v0.w = (uint32_t)h;
      v1.w = (uint32_t)h;
      __stcg(a + (uint64_t)x0 * W, v0);
      __stcg(a + (uint64_t)x1 * W, v1);
      if (write_all) {
#pragma unroll
        for (int k = 1; k < W; ++k) {
          __stcg(a + (uint64_t)x0 * W + k, make_uint4((uint32_t)h, 0u, 0u, 0u));
          __stcg(a + (uint64_t)x1 * W + k, make_uint4((uint32_t)h, 0u, 0u, 0u));
        }
      }
    }
    acc += v0.y + v1.y;
    x0 = v0.x;
    x1 = v1.x;
  }
  if (acc == 0x123456789ull) *sink = acc;
}

}  // namespace
}  // namespace ks

using namespace ks;

extern "C" KASCADE_API kascade_status kascade_calibrate_random_access(kascade_ctx* c, uint64_t n_records, uint32_t mode,
                                                                      uint32_t blocks_per_sm, double* gaccess_per_s) {
  if (!c || !gaccess_per_s || mode > 7 || n_records < 1024 || n_records > (1ull << 32)) return KASCADE_ERR_INVALID_ARG;
  KS_CUDA(cudaSetDevice(c->device));
  KS_TRY(arena_begin_call(*c, nullptr));
  const int W = (mode == 4 || mode == 7) ? 2 : (mode == 5 || mode == 6) ? 4 : 1;
  uint4* a = alloc<uint4>(*c, n_records * W);
  unsigned long long* sink = alloc<unsigned long long>(*c, 1);
  if (!a || !sink) return KASCADE_ERR_OOM;
  const unsigned bps = blocks_per_sm ? blocks_per_sm : 8;
  const unsigned grid = (unsigned)(c->sm_count * bps);
  if (W == 1)
    k_cal_init<<<c->sm_count * 8, 256>>>(a, n_records);
  else if (W == 2)
    k_cal_init_wide<2><<<c->sm_count * 8, 256>>>(a, n_records);
  else
    k_cal_init_wide<4><<<c->sm_count * 8, 256>>>(a, n_records);
  KS_CHECK_LAUNCH();
  cudaEvent_t e0, e1;
  KS_CUDA(cudaEventCreate(&e0));
  KS_CUDA(cudaEventCreate(&e1));
  double accesses = 0;
  const uint64_t m = n_records;
  const uint64_t threads = (uint64_t)grid * 256;
  const uint64_t hops = (m / (threads * 2)) ? m / (threads * 2) : 1;
  for (int rep = 0; rep < 4; ++rep) {
    if (rep == 1) cudaEventRecord(e0);
    if (mode < 2)
      k_cal_independent<<<grid, 256>>>(a, n_records, m, mode == 1, sink);
    else if (mode < 4)
      k_cal_chains<<<grid, 256>>>(a, n_records, hops, mode == 3, sink);
    else if (W == 2)
      k_cal_chains_wide<2><<<grid, 256>>>(a, n_records, hops, mode == 4, 1, sink);
    else
      k_cal_chains_wide<4><<<grid, 256>>>(a, n_records, hops, 1, mode == 5, sink);
  }
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  KS_CHECK_LAUNCH();
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  accesses = (mode < 2) ? (double)m : (double)threads * 2.0 * (double)hops;
  *gaccess_per_s = accesses * 3.0 / (ms / 1000.0) / 1e9;
  return KASCADE_OK;
}
