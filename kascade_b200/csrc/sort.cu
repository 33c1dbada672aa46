// Exclusive scan (reduce-then-scan) and LSD radix sort with digits of up to
// 8 bits, the key's bits spread evenly over the passes.
//
// Radix sort, per pass over 2048-key tiles:
//   hist    : per-tile digit counts, stored digit-major (count[d][tile])
//   scan    : one exclusive scan over all counts gives every (digit, tile)
//             its global output offset
//   scatter : each tile ranks its keys stably inside the tile (warp
//             ballots per digit bit + per-warp digit counters), stages the tile sorted
//             by digit in shared memory, and writes runs of equal digits
//             contiguously to their global offsets
// It is the counting-sort role of make_graph (lib/kascade/successor_utils.cpp:
// 236-260) done as a deterministic device sort.
#include <algorithm>

#include "sort.cuh"

namespace ks {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

constexpr int RADIX_BITS = 8;
constexpr int RADIX = 1 << RADIX_BITS;
constexpr int SORT_THREADS = 256;
constexpr int SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;  // 2048
constexpr int SORT_WARPS = SORT_THREADS / 32;
constexpr int WARP_ITEMS = SORT_TILE / SORT_WARPS;  // 512 consecutive keys per warp

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const uint32_t* __restrict__ in, uint64_t count,
                                                              uint32_t* __restrict__ sums) {
  __shared__ uint32_t sm[33];
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
  uint32_t acc = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    uint64_t x = base + (uint64_t)i * SCAN_THREADS + threadIdx.x;
    if (x < count) acc += in[x];
  }
  uint32_t total;
  block_exclusive_scan(acc, sm, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Scans its tile (blocked: thread t owns items t*ITEMS..) and adds offs[block].
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                            uint64_t count, const uint32_t* __restrict__ offs,
                                                            uint32_t* __restrict__ total_out) {
  __shared__ uint32_t sm[33];
  __shared__ uint32_t tile[SCAN_TILE];
  uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    uint64_t x = base + (uint64_t)i * SCAN_THREADS + threadIdx.x;
    tile[i * SCAN_THREADS + threadIdx.x] = (x < count) ? in[x] : 0u;
  }
  __syncthreads();
  uint32_t v[SCAN_ITEMS];
  uint32_t acc = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    v[i] = tile[threadIdx.x * SCAN_ITEMS + i];
    acc += v[i];
  }
  uint32_t total;
  uint32_t pre = block_exclusive_scan(acc, sm, &total);
  uint32_t off = (offs ? offs[blockIdx.x] : 0u) + pre;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    tile[threadIdx.x * SCAN_ITEMS + i] = off;
    off += v[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    uint64_t x = base + (uint64_t)i * SCAN_THREADS + threadIdx.x;
    if (x < count) out[x] = tile[i * SCAN_THREADS + threadIdx.x];
  }
  if (total_out && threadIdx.x == SCAN_THREADS - 1 && blockIdx.x == gridDim.x - 1) *total_out = off;
}

template <bool FROM_PARENT>
__device__ __forceinline__ void load_pair(const SortSource& src, const uint32_t* keys, const uint32_t* vals,
                                          uint32_t n, uint32_t i, uint32_t& k, uint32_t& v, DevStatus* st) {
  if (FROM_PARENT) {
    unsigned long long p = __ldcs(reinterpret_cast<const unsigned long long*>(src.parent) + i);
    if (p >= n) {
      set_error(st, KASCADE_ERR_OUT_OF_RANGE, i);
      p = i;
    }
    k = (uint32_t)p;
    v = i;
  } else {
    k = keys[i];
    v = vals ? vals[i] : i;
  }
}

template <bool FROM_PARENT>
__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist(SortSource src, const uint32_t* __restrict__ keys,
                                                            uint32_t n, int shift, uint32_t dmask, uint32_t num_tiles,
                                                            uint32_t* __restrict__ hist, DevStatus* st) {
  __shared__ uint32_t cnt[RADIX];
  for (uint32_t tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    cnt[threadIdx.x] = 0;
    __syncthreads();
    uint64_t base = (uint64_t)tile * SORT_TILE;
    uint32_t kv[SORT_ITEMS];
#pragma unroll
    for (int i = 0; i < SORT_ITEMS; ++i) {  // loads first, all in flight together
      uint64_t x = base + (uint64_t)i * SORT_THREADS + threadIdx.x;
      kv[i] = 0xFFFFFFFFu;
      if (x < n) {
        if (FROM_PARENT) {
          unsigned long long p = __ldg(reinterpret_cast<const unsigned long long*>(src.parent) + x);
          kv[i] = (p >= n) ? (uint32_t)x : (uint32_t)p;
        } else {
          kv[i] = keys[x];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < SORT_ITEMS; ++i) {
      uint64_t x = base + (uint64_t)i * SORT_THREADS + threadIdx.x;
      if (x < n) atomicAdd(&cnt[(kv[i] >> shift) & dmask], 1u);
    }
    __syncthreads();
    hist[(uint64_t)threadIdx.x * num_tiles + tile] = cnt[threadIdx.x];
    __syncthreads();
  }
}

template <bool FROM_PARENT>
__global__ void __launch_bounds__(SORT_THREADS) k_sort_scatter(SortSource src, const uint32_t* __restrict__ keys,
                                                               const uint32_t* __restrict__ vals, uint32_t n, int shift,
                                                               int bits,
                                                               uint32_t num_tiles, const uint32_t* __restrict__ offs,
                                                               uint32_t* __restrict__ keys_out,
                                                               uint32_t* __restrict__ vals_out, DevStatus* st) {
  __shared__ uint32_t wcnt[SORT_WARPS][RADIX];  // per-warp digit counts -> exclusive offsets
  __shared__ uint32_t dstart[RADIX];            // tile-local start of each digit run
  __shared__ uint32_t gofs[RADIX];              // global start of each digit run
  __shared__ uint32_t sk[SORT_TILE];
  __shared__ uint32_t sv[SORT_TILE];
  __shared__ uint32_t sm[33];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  for (uint32_t tile = blockIdx.x; tile < num_tiles; tile += gridDim.x) {
    for (int d = threadIdx.x; d < RADIX * SORT_WARPS; d += SORT_THREADS) (&wcnt[0][0])[d] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)tile * SORT_TILE + (uint64_t)warp * WARP_ITEMS;
    uint32_t kk[SORT_ITEMS], vv[SORT_ITEMS], rk[SORT_ITEMS];
    // all of the tile's loads first (independent, in flight together), then
    // the ranking, which waits on each key in turn
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; ++j) {
      const uint64_t x = base + (uint64_t)j * 32 + lane;
      kk[j] = 0xFFFFFFFFu;
      vv[j] = 0;
      if (x < n) load_pair<FROM_PARENT>(src, keys, vals, n, (uint32_t)x, kk[j], vv[j], st);
    }
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; ++j) {
      const uint64_t x = base + (uint64_t)j * 32 + lane;
      const bool valid = x < n;
      const uint32_t k = kk[j], v = vv[j];
      const uint32_t d = valid ? ((k >> shift) & ((1u << bits) - 1u)) : 0xFFFFu;
      // lanes with the same digit (and validity): one ballot per digit bit,
      // measured faster than a warp match instruction here (sort scatter
      // 2.46 -> 2.22 ms on a 2^26-vertex forest)
      uint32_t peers = __ballot_sync(FULL, valid);
      if (!valid) peers = ~peers;
#pragma unroll
      for (int b = 0; b < RADIX_BITS; ++b) {
        if (b >= bits) break;  // warp-uniform
        const bool bit = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(FULL, bit);
        peers &= bit ? bal : ~bal;
      }
      const uint32_t before = __popc(peers & lt);
      uint32_t cur = 0;
      if (valid) cur = wcnt[warp][d];
      __syncwarp();
      if (valid && before == 0) wcnt[warp][d] = cur + __popc(peers);
      __syncwarp();
      kk[j] = k;
      vv[j] = v;
      rk[j] = cur + before;  // rank among this warp's keys of digit d
    }
    __syncthreads();
    // per digit: exclusive prefix over warps, tile total
    {
      const uint32_t d = threadIdx.x;  // SORT_THREADS == RADIX
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < SORT_WARPS; ++w) {
        uint32_t c = wcnt[w][d];
        wcnt[w][d] = run;
        run += c;
      }
      uint32_t total;
      uint32_t start = block_exclusive_scan(run, sm, &total);
      dstart[d] = start;
      gofs[d] = offs[(uint64_t)d * num_tiles + tile];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; ++j) {
      const uint64_t x = base + (uint64_t)j * 32 + lane;
      if (x < n) {
        const uint32_t d = (kk[j] >> shift) & ((1u << bits) - 1u);
        const uint32_t pos = dstart[d] + wcnt[warp][d] + rk[j];
        sk[pos] = kk[j];
        sv[pos] = vv[j];
      }
    }
    __syncthreads();
    const uint64_t tile_base = (uint64_t)tile * SORT_TILE;
    const uint32_t tile_n = (uint32_t)(((uint64_t)SORT_TILE < n - tile_base) ? (uint64_t)SORT_TILE : (n - tile_base));
    for (uint32_t i = threadIdx.x; i < tile_n; i += SORT_THREADS) {
      const uint32_t k = sk[i];
      const uint32_t d = (k >> shift) & ((1u << bits) - 1u);
      const uint32_t g = gofs[d] + (i - dstart[d]);
      keys_out[g] = k;
      vals_out[g] = sv[i];
    }
    __syncthreads();
  }
}

}  // namespace

kascade_status exclusive_scan_u32(kascade_ctx& ctx, const uint32_t* in, uint32_t* out, uint64_t count,
                                  uint32_t* total, cudaStream_t s) {
  if (count == 0) {
    if (total) KS_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), s));
    return KASCADE_OK;
  }
  uint64_t blocks = (count + SCAN_TILE - 1) / SCAN_TILE;
  if (blocks == 1) {
    k_scan_down<<<1, SCAN_THREADS, 0, s>>>(in, out, count, nullptr, total);
    KS_CHECK_LAUNCH();
    return KASCADE_OK;
  }
  uint32_t* sums = alloc<uint32_t>(ctx, blocks);
  if (!sums) return KASCADE_ERR_OOM;
  k_scan_reduce<<<(unsigned)blocks, SCAN_THREADS, 0, s>>>(in, count, sums);
  KS_CHECK_LAUNCH();
  KS_TRY(exclusive_scan_u32(ctx, sums, sums, blocks, nullptr, s));
  k_scan_down<<<(unsigned)blocks, SCAN_THREADS, 0, s>>>(in, out, count, sums, total);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status radix_sort_pairs(kascade_ctx& ctx, const SortSource& src, uint32_t n, int key_bits, uint32_t** keys_out,
                                uint32_t** vals_out, cudaStream_t s) {
  if (key_bits < 1) key_bits = 1;
  const uint32_t num_tiles = (uint32_t)(((uint64_t)n + SORT_TILE - 1) / SORT_TILE);
  uint32_t* kb[2] = {alloc<uint32_t>(ctx, n ? n : 1), alloc<uint32_t>(ctx, n ? n : 1)};
  uint32_t* vb[2] = {alloc<uint32_t>(ctx, n ? n : 1), alloc<uint32_t>(ctx, n ? n : 1)};
  uint32_t* hist = alloc<uint32_t>(ctx, (uint64_t)RADIX * (num_tiles ? num_tiles : 1));
  if (!kb[0] || !kb[1] || !vb[0] || !vb[1] || !hist) return KASCADE_ERR_OOM;
  if (n == 0) {
    *keys_out = kb[0];
    *vals_out = vb[0];
    return KASCADE_OK;
  }
  const unsigned grid = (unsigned)std::min<uint64_t>(num_tiles, (uint64_t)ctx.usable_sms() * 8);
  const unsigned grid_scatter = (unsigned)std::min<uint64_t>(num_tiles, (uint64_t)ctx.usable_sms() * 4);
  int cur = 0;
  // passes of at most RADIX_BITS bits, the key's bits spread evenly over them
  // (26 bits: 7 + 7 + 6 + 6 rather than 8 + 8 + 8 + 2): fewer ballots per key
  // and longer runs per digit
  const int passes = (key_bits + RADIX_BITS - 1) / RADIX_BITS;
  int shift = 0;
  for (int p = 0; p < passes; ++p) {
    const int bits = key_bits / passes + (p < key_bits % passes ? 1 : 0);
    const uint32_t dmask = (1u << bits) - 1u;
    const bool first = (p == 0) && src.parent != nullptr;
    const uint32_t* kin = (p == 0) ? src.keys : kb[cur];
    const uint32_t* vin = (p == 0) ? src.vals : vb[cur];
    const int dst = (p == 0) ? 0 : cur ^ 1;
    {
      ProfScope ps(ctx, "sort_hist", s);
      if (first)
        k_sort_hist<true><<<grid, SORT_THREADS, 0, s>>>(src, kin, n, shift, dmask, num_tiles, hist, ctx.d_status);
      else
        k_sort_hist<false><<<grid, SORT_THREADS, 0, s>>>(src, kin, n, shift, dmask, num_tiles, hist, ctx.d_status);
      KS_CHECK_LAUNCH();
    }
    {
      ProfScope ps(ctx, "sort_scan", s);
      KS_TRY(exclusive_scan_u32(ctx, hist, hist, (uint64_t)RADIX * num_tiles, nullptr, s));
    }
    {
      ProfScope ps(ctx, "sort_scatter", s);
      if (first)
        k_sort_scatter<true><<<grid_scatter, SORT_THREADS, 0, s>>>(src, kin, vin, n, shift, bits, num_tiles, hist,
                                                                    kb[dst], vb[dst], ctx.d_status);
      else
        k_sort_scatter<false><<<grid_scatter, SORT_THREADS, 0, s>>>(src, kin, vin, n, shift, bits, num_tiles, hist,
                                                                     kb[dst], vb[dst], ctx.d_status);
      KS_CHECK_LAUNCH();
    }
    cur = dst;
    shift += bits;
  }
  *keys_out = kb[cur];
  *vals_out = vb[cur];
  return KASCADE_OK;
}

}  // namespace ks
