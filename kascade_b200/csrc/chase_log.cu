// Write-free level 0 of the ruling-set ranker.
//
// On B200 a random 16 B read costs a 128 B DRAM fetch, and writing a record
// back after reading it roughly halves the random-access rate (random read:
// ~45 G/s, read + write back: ~17-22 G/s; see `bench.py --calibrate`).  This
// path therefore never writes at a random address:
//
//   chase     read-only walk of every chain; each visited element appends
//             (element, ruler id, distance from ruler) to a log made of
//             1024-entry chunks that each warp takes from a global counter,
//             so the log is written with coalesced 16 B stores
//   recurse   the ruler sub-list (written by the chase in dense id space) is
//             ranked by the deeper levels
//   resolve   one pass over the log: rank = rank(ruler) - distance,
//             root = root(ruler), then partition by element into windows of
//             2^21 elements (one global atomic per window and log chunk)
//   scatter   windows are processed in order, so the outputs of about one
//             window (32 MB) are live in L2 at a time and reach DRAM as full
//             sectors; a byte flag marks every written element
//   heads     elements ahead of their list's first ruler were never visited:
//             they are found by their clear flag and walk forward to the first
//             flagged element (tours make their heads rulers and skip this)
//
// Reference counterparts: the chase of sparse_ruling_set.cpp:147-273 (whose
// per-element writes are the reference's messages), ruler_propagation.hpp:
// 148-256 (pull) and post_invert.hpp:195-264 (unreached fix-up).
#include <algorithm>

#include "ranker.cuh"

namespace ks {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t LOG_CHUNK = 1024;  // entries per warp-owned log chunk
constexpr uint32_t WIN_SHIFT = 19;    // 2^19 elements per output window (8.5 MB of outputs)
constexpr uint32_t WIN = 1u << WIN_SHIFT;
constexpr uint32_t MAX_BUCKETS = 8192;  // windows for 2^32 elements
constexpr uint32_t CURSOR_STRIDE = 8;   // one 32 B sector per window cursor (spreads the atomics)
constexpr uint32_t FLAG_ONLY = 0xFFFFFFFFu;
constexpr uint32_t SCATTER_ITEM = 1024;

struct __align__(16) LogEnt {
  uint32_t x;
  uint32_t id;
  uint64_t off;
};
struct __align__(16) OutEnt {
  uint32_t x;
  uint32_t root;  // FLAG_ONLY: mark reached, leave the outputs untouched
  uint64_t rank;
};

__device__ __forceinline__ void st_log(LogEnt* p, uint32_t x, uint32_t id, uint64_t off) {
  __stcs(reinterpret_cast<uint4*>(p), make_uint4(x, id, (uint32_t)off, (uint32_t)(off >> 32)));
}

// Warp-cooperative append of one entry per emitting lane.  pos/end describe
// the warp's current log chunk and are warp-uniform.
__device__ __forceinline__ void log_append(bool emit, uint32_t x, uint32_t id, uint64_t off, uint32_t& pos,
                                           uint32_t& end, LogEnt* __restrict__ log, uint32_t* __restrict__ chunk_fill,
                                           uint32_t* __restrict__ chunk_cursor, uint32_t nchunks, uint32_t lane,
                                           uint32_t lt, DevStatus* st) {
  uint32_t m = __ballot_sync(FULL, emit);
  while (m != 0u) {
    if (pos == end) {
      uint32_t ch = 0;
      if (lane == 0) ch = atomicAdd(chunk_cursor, 1u);
      ch = __shfl_sync(FULL, ch, 0);
      if (ch >= nchunks) {
        // more entries than elements: the input is not a forest of lists
        if (lane == 0) set_error(st, KASCADE_ERR_NOT_A_LIST, ch);
        return;
      }
      pos = ch * LOG_CHUNK;
      end = pos + LOG_CHUNK;
    }
    const uint32_t take = min((uint32_t)__popc(m), end - pos);
    const uint32_t my = __popc(m & lt);
    const bool mine = emit && my < take;
    if (mine) st_log(log + pos + my, x, id, off);
    const uint32_t served = __ballot_sync(FULL, mine);
    m &= ~served;
    emit = emit && !mine;
    pos += take;
    if (pos == end && lane == 0) chunk_fill[(pos - 1) / LOG_CHUNK] = LOG_CHUNK;
  }
}

template <int C>
__global__ void __launch_bounds__(512) k_chase_log(const Rec* __restrict__ rec, uint32_t n,
                                                   const uint32_t* __restrict__ ruler_elem, uint32_t r,
                                                   Rec* __restrict__ rec_next, uint32_t* __restrict__ work,
                                                   LogEnt* __restrict__ log, uint32_t* __restrict__ chunk_fill,
                                                   uint32_t* __restrict__ chunk_cursor, uint32_t nchunks,
                                                   uint32_t max_hops, DevStatus* st) {
  constexpr uint32_t BATCH = 32u * C;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt = lanemask_lt();
  uint32_t cid[C], cx[C], hops[C];
  uint64_t acc[C];
  uint32_t act = 0;
  uint32_t q_base = 0, q_left = 0;
  bool drained = false;
  uint32_t lpos = 0, lend = 0;  // warp-uniform log chunk
#pragma unroll
  for (int c = 0; c < C; ++c) {
    cid[c] = cx[c] = hops[c] = 0;
    acc[c] = 0;
  }
  while (true) {
    if (!drained) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        bool need = !(act & (1u << c));
        uint32_t m = __ballot_sync(FULL, need);
        while (m != 0u && !drained) {
          if (q_left == 0u) {
            uint32_t b = 0;
            if (lane == 0) b = atomicAdd(work, BATCH);
            b = __shfl_sync(FULL, b, 0);
            if (b >= r) {
              drained = true;
              break;
            }
            q_base = b;
            q_left = min(BATCH, r - b);
          }
          const uint32_t take = min((uint32_t)__popc(m), q_left);
          const uint32_t my_rank = __popc(m & lt);
          const bool mine = need && my_rank < take;
          uint32_t x0 = 0, id = 0;
          if (mine) {
            id = q_base + my_rank;
            x0 = __ldg(ruler_elem + id);
            const Rec r0 = ld_rec_cg(rec + x0);
            if (r0.b == x0) {
              Rec o;
              o.a = 0;
              o.b = id;
              o.c = TAG_UNREACHED;
              st_rec_cg(rec_next + id, o);
            } else {
              cid[c] = id;
              cx[c] = r0.b;
              acc[c] = r0.a;
              hops[c] = 0;
              act |= 1u << c;
            }
          }
          // every ruler (root rulers included) logs itself at distance 0
          log_append(mine, x0, id, 0ull, lpos, lend, log, chunk_fill, chunk_cursor, nchunks, lane, lt, st);
          const uint32_t served = __ballot_sync(FULL, mine);
          m &= ~served;
          need = need && !mine;
          q_base += take;
          q_left -= take;
        }
      }
    }
    if (!__any_sync(FULL, act != 0u)) {
      if (drained) break;
      continue;
    }
    Rec rr[C];
#pragma unroll
    for (int c = 0; c < C; ++c)
      if (act & (1u << c)) rr[c] = ld_rec_cg(rec + cx[c]);
#pragma unroll
    for (int c = 0; c < C; ++c) {
      bool emit = false;
      const uint32_t x = cx[c];
      const uint64_t d = acc[c];
      if (act & (1u << c)) {
        if (tag_ruler(rr[c].c)) {
          Rec o;
          o.a = acc[c];
          o.b = tag_id(rr[c].c);
          o.c = TAG_UNREACHED;
          st_rec_cg(rec_next + cid[c], o);
          act &= ~(1u << c);
        } else {
          emit = true;
          acc[c] += rr[c].a;
          cx[c] = rr[c].b;
          // Ruler gaps are geometric: a chain longer than max_hops (64x the
          // mean spacing, probability ~e^-64) is treated as a sign of an
          // invalid input (a ruler-free cycle behind a ruler); the chain
          // stops and the host reruns level 0 on the stamping path, which
          // tells the two cases apart exactly.
          if (++hops[c] > max_hops) {
            atomicOr(&st->counter[0], 1ull);
            Rec o;  // keep the next level's records in range (the level is redone anyway)
            o.a = 0;
            o.b = cid[c];
            o.c = TAG_UNREACHED;
            st_rec_cg(rec_next + cid[c], o);
            act &= ~(1u << c);
          }
        }
      }
      log_append(emit, x, cid[c], d, lpos, lend, log, chunk_fill, chunk_cursor, nchunks, lane, lt, st);
    }
  }
  if (lane == 0 && lend != 0 && lpos != lend) chunk_fill[(lend - 1) / LOG_CHUNK] = LOG_CHUNK - (lend - lpos);
}

// resolve + partition: one log chunk per block iteration.
__global__ void __launch_bounds__(256) k_resolve_partition(const LogEnt* __restrict__ log,
                                                           const uint32_t* __restrict__ chunk_fill, uint32_t nchunks,
                                                           const Out* __restrict__ out1, uint32_t limit,
                                                           int keep_roots, uint32_t nb, OutEnt* __restrict__ part,
                                                           uint32_t* __restrict__ bcursor,
                                                           unsigned long long* __restrict__ logged, DevStatus* st) {
  constexpr int PER = LOG_CHUNK / 256;
  extern __shared__ uint32_t dyn[];
  uint32_t* bcnt = dyn;        // nb entries
  uint32_t* bbase = dyn + nb;  // nb entries
  unsigned long long block_logged = 0;
  for (uint32_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const uint32_t fill = chunk_fill[ch];
    if (fill == 0) continue;  // uniform over the block
    block_logged += fill;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) bcnt[b] = 0;
    __syncthreads();
    OutEnt e[PER];
    uint32_t bk[PER], loc[PER];
    bool v[PER];
    LogEnt le[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const uint32_t j = threadIdx.x + i * 256;
      v[i] = j < fill;
      if (v[i]) {
        uint4 raw = __ldcs(reinterpret_cast<const uint4*>(log + (uint64_t)ch * LOG_CHUNK + j));
        le[i].x = raw.x;
        le[i].id = raw.y;
        le[i].off = (uint64_t)raw.z | ((uint64_t)raw.w << 32);
      }
    }
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      if (v[i] && le[i].x >= limit) v[i] = false;  // e.g. tour down edges: no output
      if (!v[i]) continue;
      const Out o = ld_out(out1 + le[i].id);
      e[i].x = le[i].x;
      e[i].rank = o.rank - le[i].off;
      e[i].root = (keep_roots && o.root == le[i].x) ? FLAG_ONLY : o.root;
      bk[i] = le[i].x >> WIN_SHIFT;
      loc[i] = atomicAdd(&bcnt[bk[i]], 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x)
      if (bcnt[b]) bbase[b] = atomicAdd(bcursor + (uint64_t)b * CURSOR_STRIDE, bcnt[b]);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      if (!v[i]) continue;
      const uint32_t pos = bbase[bk[i]] + loc[i];
      if (pos >= WIN) {
        set_error(st, KASCADE_ERR_NOT_A_LIST, e[i].x);  // an element logged twice
        continue;
      }
      OutEnt* dst = part + (uint64_t)bk[i] * WIN + pos;
      *reinterpret_cast<uint4*>(dst) = make_uint4(e[i].x, e[i].root, (uint32_t)e[i].rank, (uint32_t)(e[i].rank >> 32));
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && block_logged) atomicAdd(logged, block_logged);
}

// Windowed scatter: work items are handed out in window order.
__global__ void __launch_bounds__(256) k_scatter(const OutEnt* __restrict__ part, const uint32_t* __restrict__ bcursor,
                                                 uint32_t nb, uint32_t* __restrict__ work, uint64_t* __restrict__ root_out,
                                                 uint64_t* __restrict__ rank_out, uint8_t* __restrict__ flags) {
  __shared__ uint32_t item;
  constexpr uint32_t IPB = WIN / SCATTER_ITEM;
  const uint32_t total = nb * IPB;
  while (true) {
    if (threadIdx.x == 0) item = atomicAdd(work, 1u);
    __syncthreads();
    const uint32_t it = item;
    __syncthreads();
    if (it >= total) break;
    const uint32_t b = it / IPB, k = it % IPB;
    const uint32_t cnt = min(bcursor[(uint64_t)b * CURSOR_STRIDE], WIN);  // beyond WIN only on invalid input
    const uint32_t beg = k * SCATTER_ITEM;
    if (beg >= cnt) continue;
    const uint32_t stop = min(beg + SCATTER_ITEM, cnt);
    const OutEnt* src = part + (uint64_t)b * WIN;
    for (uint32_t j = beg + threadIdx.x; j < stop; j += 256) {
      const uint4 raw = __ldcs(reinterpret_cast<const uint4*>(src + j));
      const uint32_t x = raw.x;
      if (raw.y != FLAG_ONLY) {
        root_out[x] = raw.y;
        rank_out[x] = (uint64_t)raw.z | ((uint64_t)raw.w << 32);
      }
      if (flags) flags[x] = 1;
    }
  }
}

// Elements never visited (ahead of their list's first ruler).
__global__ void __launch_bounds__(256) k_find_unreached(const uint8_t* __restrict__ flags, uint32_t n,
                                                        uint32_t* __restrict__ ulist, uint32_t* __restrict__ ucount,
                                                        uint32_t ucap, DevStatus* st) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t groups = ((uint64_t)n + 15) / 16;
  for (uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x; g0 < groups; g0 += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t g = g0 + threadIdx.x;
    uint32_t zero_mask = 0;
    if (g < groups) {
      uint4 v = __ldcs(reinterpret_cast<const uint4*>(flags) + g);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const uint32_t byte = (w[k >> 2] >> (8 * (k & 3))) & 0xFFu;
        if (byte == 0 && g * 16 + k < n) zero_mask |= 1u << k;
      }
    }
    uint32_t cnt = __popc(zero_mask);
    // warp-level exclusive scan of counts, one atomic per warp
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(FULL, incl, o);
      if (lane >= (uint32_t)o) incl += y;
    }
    const uint32_t wtotal = __shfl_sync(FULL, incl, 31);
    uint32_t base = 0;
    if (lane == 31 && wtotal) base = atomicAdd(ucount, wtotal);
    base = __shfl_sync(FULL, base, 31);
    uint32_t pos = base + incl - cnt;
    while (zero_mask) {
      const int k = __ffs(zero_mask) - 1;
      zero_mask &= zero_mask - 1;
      if (pos < ucap)
        ulist[pos] = (uint32_t)(g * 16 + k);
      else
        set_error(st, KASCADE_ERR_TOO_LARGE, pos);
      pos++;
    }
  }
}

__global__ void __launch_bounds__(256) k_walk_unreached(const Rec* __restrict__ rec, const uint8_t* __restrict__ flags,
                                                        const uint32_t* __restrict__ ulist,
                                                        const uint32_t* __restrict__ ucount, uint32_t ucap, uint32_t n,
                                                        uint64_t* __restrict__ root_out, uint64_t* __restrict__ rank_out,
                                                        DevStatus* st) {
  const uint32_t cnt = min(*ucount, ucap);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const uint32_t u = ulist[i];
    uint64_t acc = 0;
    uint32_t y = u, mark = u, power = 1, lam = 0, hops = 0;
    bool ok = true;
    while (true) {
      const Rec r = ld_rec_cg(rec + y);
      acc += r.a;
      y = r.b;
      if (flags[y]) break;
      if (y == mark || ++hops > n) {
        set_error(st, KASCADE_ERR_CYCLE, u);
        ok = false;
        break;
      }
      if (++lam == power) {
        mark = y;
        power <<= 1;
        lam = 0;
      }
    }
    if (!ok) continue;
    const Rec ry = ld_rec_cg(rec + y);
    uint64_t base_rank;
    uint64_t base_root;
    if (ry.b == y) {  // a root: rank 0 whatever its output slot holds
      base_rank = 0;
      base_root = y;
    } else {
      base_rank = rank_out[y];
      base_root = root_out[y];
    }
    root_out[u] = base_root;
    rank_out[u] = acc + base_rank;
  }
}

int g_chase_occ[5][3] = {{-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}};

template <int C>
kascade_status launch_chase_log_c(kascade_ctx& ctx, const Rec* rec, uint32_t n, const uint32_t* ruler_elem, uint32_t r,
                                  Rec* rec_next, uint32_t* work, LogEnt* log, uint32_t* chunk_fill,
                                  uint32_t* chunk_cursor, uint32_t nchunks, uint32_t max_hops, unsigned grid,
                                  uint32_t block, cudaStream_t s) {
  ProfScope ps(ctx, "chase", s);
  k_chase_log<C><<<grid, block, 0, s>>>(rec, n, ruler_elem, r, rec_next, work, log, chunk_fill, chunk_cursor, nchunks,
                                      max_hops, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

template <int C>
unsigned chase_grid(const kascade_ctx& ctx, uint32_t r, uint32_t block) {
  const int bi = block == 128 ? 0 : block == 512 ? 2 : 1;
  if (g_chase_occ[C][bi] < 0) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_chase_log<C>, (int)block, 0) != cudaSuccess) {
      cudaGetLastError();
      nb = 1;
    }
    g_chase_occ[C][bi] = nb < 1 ? 1 : nb;
  }
  unsigned grid = (unsigned)(ctx.usable_sms() * g_chase_occ[C][bi]);
  const uint64_t warps_per_block = block / 32;
  const uint64_t need = ((uint64_t)r + 32ull * C - 1) / (32ull * C);
  const uint64_t need_blocks = (need + warps_per_block - 1) / warps_per_block;
  if (need_blocks < grid) grid = (unsigned)(need_blocks ? need_blocks : 1);
  return grid;
}

}  // namespace

kascade_status rank_level0_log(kascade_ctx& ctx, const Rec* rec, uint32_t n, uint32_t r0, const uint32_t* ruler_elem0,
                               const LogTarget& t, const Params& p, cudaStream_t s) {
  const int C = (p.chains == 1 || p.chains == 4) ? (int)p.chains : 2;
  const uint32_t block = p.block;
  const unsigned grid = C == 1   ? chase_grid<1>(ctx, r0, block)
                        : C == 4 ? chase_grid<4>(ctx, r0, block)
                                 : chase_grid<2>(ctx, r0, block);
  const uint64_t warps = (uint64_t)grid * (block / 32);
  const uint32_t nchunks = (uint32_t)(((uint64_t)n + LOG_CHUNK - 1) / LOG_CHUNK + warps + 1);
  LogEnt* log = alloc<LogEnt>(ctx, (uint64_t)nchunks * LOG_CHUNK);
  uint32_t* chunk_fill = alloc<uint32_t>(ctx, nchunks);
  uint32_t* counters = alloc<uint32_t>(ctx, 8);  // chunk cursor, chase work, scatter work, unreached count
  unsigned long long* logged = alloc<unsigned long long>(ctx, 1);
  Rec* rec1 = alloc<Rec>(ctx, r0);
  Out* out1 = alloc<Out>(ctx, r0);
  if (!log || !chunk_fill || !counters || !logged || !rec1 || !out1) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(chunk_fill, 0, sizeof(uint32_t) * nchunks, s));
  KS_CUDA(cudaMemsetAsync(counters, 0, sizeof(uint32_t) * 8, s));
  KS_CUDA(cudaMemsetAsync(logged, 0, sizeof(unsigned long long), s));
  uint32_t* chunk_cursor = counters + 0;
  uint32_t* chase_work = counters + 1;
  uint32_t* scatter_work = counters + 2;
  uint32_t* ucount = counters + 3;
  const uint64_t cap = p.max_chain ? p.max_chain : 64ull * p.spacing0 + 1024;
  const uint32_t max_hops = cap < n ? (uint32_t)cap : n;
  switch (C) {
    case 1:
      KS_TRY(launch_chase_log_c<1>(ctx, rec, n, ruler_elem0, r0, rec1, chase_work, log, chunk_fill, chunk_cursor,
                                   nchunks, max_hops, grid, block, s));
      break;
    case 4:
      KS_TRY(launch_chase_log_c<4>(ctx, rec, n, ruler_elem0, r0, rec1, chase_work, log, chunk_fill, chunk_cursor,
                                   nchunks, max_hops, grid, block, s));
      break;
    default:
      KS_TRY(launch_chase_log_c<2>(ctx, rec, n, ruler_elem0, r0, rec1, chase_work, log, chunk_fill, chunk_cursor,
                                   nchunks, max_hops, grid, block, s));
  }
  {
    // a chain hit the hop cap: let the caller rerun level 0 on the stamping path
    uint32_t over = 0;
    KS_TRY(read_u32(ctx, reinterpret_cast<const uint32_t*>(&ctx.d_status->counter[0]), &over, s));
    if (over) return KASCADE_ERR_TIMEOUT;
  }
  // level-1 elements are level-0 rulers: their level-0 index is ruler_elem0
  KS_TRY(rank_sublist(ctx, rec1, r0, ruler_elem0, out1, 1, p, s));

  const uint32_t limit = t.limit < n ? t.limit : n;
  const uint32_t nb = (uint32_t)(((uint64_t)limit + WIN - 1) / WIN);
  OutEnt* part = alloc<OutEnt>(ctx, (uint64_t)(nb ? nb : 1) * WIN);
  uint32_t* bcursor = alloc<uint32_t>(ctx, (uint64_t)(nb ? nb : 1) * CURSOR_STRIDE);
  if (!part || !bcursor) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(bcursor, 0, sizeof(uint32_t) * (nb ? nb : 1) * CURSOR_STRIDE, s));
  {
    ProfScope ps(ctx, "resolve", s);
    const unsigned g = (unsigned)std::min<uint64_t>(nchunks, (uint64_t)ctx.usable_sms() * 8);
    const size_t smem = 2 * sizeof(uint32_t) * (nb ? nb : 1);
    if (smem > 48 * 1024) {
      static bool raised = false;
      if (!raised) {
        KS_CUDA(cudaFuncSetAttribute(k_resolve_partition, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(2 * sizeof(uint32_t) * MAX_BUCKETS)));
        raised = true;
      }
    }
    k_resolve_partition<<<g, 256, smem, s>>>(log, chunk_fill, nchunks, out1, limit, t.keep_roots, nb, part, bcursor,
                                             logged, ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  uint32_t lg[2] = {0, 0};
  KS_TRY(read_u32(ctx, reinterpret_cast<const uint32_t*>(logged), &lg[0], s));
  KS_TRY(read_u32(ctx, reinterpret_cast<const uint32_t*>(logged) + 1, &lg[1], s));
  const uint64_t total_logged = (uint64_t)lg[0] | ((uint64_t)lg[1] << 32);
  if (total_logged > n) return KASCADE_ERR_NOT_A_LIST;
  const bool need_heads = total_logged < n;
  if (need_heads && t.heads_are_rulers) return KASCADE_ERR_CYCLE;  // a tour element no ruler reaches
  uint8_t* flags = nullptr;
  if (need_heads) {
    flags = alloc<uint8_t>(ctx, (uint64_t)n + 16);
    if (!flags) return KASCADE_ERR_OOM;
    KS_CUDA(cudaMemsetAsync(flags, 0, (size_t)n + 16, s));
  }
  {
    ProfScope ps(ctx, "scatter", s);
    k_scatter<<<ctx.usable_sms() * 8, 256, 0, s>>>(part, bcursor, nb, scatter_work, t.root, t.rank, flags);
    KS_CHECK_LAUNCH();
  }
  if (need_heads) {
    // the log is dead after resolve: reuse it for the list of unreached elements
    uint32_t* ulist = reinterpret_cast<uint32_t*>(log);
    const uint32_t ucap = n;
    ProfScope ps(ctx, "heads", s);
    const uint64_t groups = ((uint64_t)n + 15) / 16;
    k_find_unreached<<<grid_for(ctx, groups, 256, 8), 256, 0, s>>>(flags, n, ulist, ucount, ucap, ctx.d_status);
    KS_CHECK_LAUNCH();
    k_walk_unreached<<<ctx.usable_sms() * 4, 256, 0, s>>>(rec, flags, ulist, ucount, ucap, n, t.root, t.rank,
                                                      ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  return KASCADE_OK;
}

}  // namespace ks
