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
//   resolve   first radix pass over the log by element window (2^20
//             elements), resolving each entry on the way: rank = rank(ruler)
//             - distance, root = root(ruler).  Tiles of 2 K entries are
//             sorted by window in shared memory and written as one run per
//             window; the ruler lookups mostly hit L1 (a log chunk holds the
//             entries of a few hundred chains)
//   partition second radix pass: each window into 128 sub-windows of 2^13
//   place     one sub-window at a time: outputs assembled in shared memory
//             and written densely, so no output store is random
//   heads     elements ahead of their list's first ruler were never visited:
//             the place step finds them (no entry in their slot), presets
//             their root output to a NOT_REACHED sentinel and lists them;
//             each walks forward to the first element with outputs (tours
//             make their heads rulers and report an unreached element as a
//             ruler-free cycle)
//
// Calls that must leave roots' outputs untouched (the in-place contract) use
// the stamping level 0 instead: the sentinel presets would overwrite them.
//
// Reference counterparts: the chase of sparse_ruling_set.cpp:147-273 (whose
// per-element writes are the reference's messages), ruler_propagation.hpp:
// 148-256 (pull) and post_invert.hpp:195-264 (unreached fix-up).
#include <algorithm>
#include <atomic>

#include "ranker.cuh"

namespace ks {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t LOG_CHUNK = 1024;  // entries per warp-owned log chunk
constexpr uint32_t WIN_SHIFT = 20;    // 2^20 elements per window (first partition pass)
constexpr uint32_t WIN = 1u << WIN_SHIFT;
constexpr uint32_t SUB_SHIFT = 13;  // 2^13 elements per sub-window (second pass; resolved in shared memory)
constexpr uint32_t SUB = 1u << SUB_SHIFT;
constexpr uint32_t SUBS = WIN / SUB;    // sub-windows per window
constexpr uint32_t MAX_BUCKETS = 4096;  // windows for 2^32 elements
constexpr uint32_t CURSOR_STRIDE = 8;   // one 32 B sector per cursor (spreads the atomics)
constexpr uint32_t PT_THREADS = 256;    // partition: threads per block
// entries per thread (a tile is PT_THREADS x ITEMS entries) and resident
// blocks per SM of the two partition passes: 2048-entry tiles, 4 blocks per
// SM (more tiles in flight per SM than 4096-entry tiles at 2 blocks)
constexpr uint32_t P1_ITEMS = 8, P1_BLOCKS = 4;
constexpr uint32_t P2_ITEMS = 8, P2_BLOCKS = 4;
constexpr uint32_t FIN_THREADS = 512;  // place: threads per block (one sub-window per iteration; 2 blocks per SM)
constexpr uint32_t FIN_GROUP = 8;      // place: entries a thread has in flight
constexpr uint32_t NO_ROOT = 0xFFFFFFFFu;          // shared-memory root slot not written
constexpr unsigned long long NOT_REACHED = ~0ull;  // root output of an element no chain reached

struct __align__(16) LogEnt {
  uint32_t x;
  uint32_t id;
  uint64_t off;
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
                                                   const uint32_t* __restrict__ r_dev,
                                                   Rec* __restrict__ rec_next, uint32_t* __restrict__ work,
                                                   LogEnt* __restrict__ log, uint32_t* __restrict__ chunk_fill,
                                                   uint32_t* __restrict__ chunk_cursor, uint32_t nchunks,
                                                   uint32_t max_hops, uint32_t* __restrict__ has_pred,
                                                   DevStatus* st) {
  constexpr uint32_t BATCH = 32u * C;
  // has_pred holds one bit per ruler of the capacity; a count past the
  // capacity (reported by the caller's count check, and the level redone)
  // leaves tags beyond it, whose bits are not recorded
  const uint32_t pred_cap = r;
  if (r_dev) r = min(r, *r_dev);  // the ruler count on the device, r its capacity
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
          // back at its own ruler: a rootless cycle holding one ruler
          if (tag_id(rr[c].c) == cid[c])
            set_error(st, KASCADE_ERR_CYCLE, cid[c]);
          else if (has_pred && tag_id(rr[c].c) < pred_cap)  // that ruler has a predecessor in the ruler sub-list
            atomicOr(has_pred + (tag_id(rr[c].c) >> 5), 1u << (tag_id(rr[c].c) & 31));
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

// Exclusive prefix sum of v[0, m) in place (shared memory, m <= MAX_BUCKETS);
// returns the total to every thread.  Called by all threads of the block.
__device__ uint32_t block_exclusive_scan(uint32_t* v, uint32_t m) {
  __shared__ uint32_t warp_sum[PT_THREADS / 32];
  const uint32_t per = (m + PT_THREADS - 1) / PT_THREADS;
  const uint32_t lo = min(threadIdx.x * per, m), hi = min(lo + per, m);
  uint32_t sum = 0;
  for (uint32_t i = lo; i < hi; ++i) sum += v[i];
  const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  uint32_t inc = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(FULL, inc, d);
    if (lane >= (uint32_t)d) inc += t;
  }
  if (lane == 31) warp_sum[wid] = inc;
  __syncthreads();
  uint32_t before = 0, total = 0;
  for (uint32_t k = 0; k < PT_THREADS / 32; ++k) {
    if (k < wid) before += warp_sum[k];
    total += warp_sum[k];
  }
  uint32_t run = before + inc - sum;
  for (uint32_t i = lo; i < hi; ++i) {
    const uint32_t c = v[i];
    v[i] = run;
    run += c;
  }
  __syncthreads();
  return total;
}

// Radix partition of 16 B entries by element index.  A block loads a
// tile of PT_TILE entries into registers, counts them per bucket in shared
// memory, takes one global cursor step per bucket the tile touches, sorts
// the tile by bucket in shared memory and writes each bucket's run with
// consecutive threads: every global store is part of a contiguous run, so
// L2 sees whole lines instead of one 16 B piece per store.
//   FROM_LOG (first pass): tiles of PT_TILE_CHUNKS log chunks, buckets are
//     windows of WIN elements.  Each log entry (element, ruler id, distance)
//     is resolved on the way: rank = rank(ruler) - distance, root =
//     root(ruler), from the rulers' results of the recursion.  A log chunk
//     holds the entries of a few hundred chains, so most of these lookups
//     hit L1.  Entries of elements at or above `limit` (tour down edges: no
//     output) are only counted, in `beyond`
//   otherwise (second pass): tiles inside one window's region, buckets are
//     its SUBS sub-windows
// More entries than a bucket holds means some element was logged twice.
//   used (first pass, optional): the chunks the chase took (its chunk
//     cursor); the chunks after them are empty and are skipped
template <bool FROM_LOG, uint32_t ITEMS, uint32_t BLOCKS>
__global__ void __launch_bounds__(PT_THREADS, BLOCKS) k_partition(const LogEnt* __restrict__ src,
                                                             const uint32_t* __restrict__ src_info, uint32_t nchunks,
                                                             const Out* __restrict__ out1, uint32_t limit,
                                                             uint32_t nb, LogEnt* __restrict__ dst,
                                                             uint32_t* __restrict__ dcursor,
                                                             uint32_t* __restrict__ beyond,
                                                             const uint32_t* __restrict__ used, DevStatus* st) {
  constexpr uint32_t PT_TILE = PT_THREADS * ITEMS;
  constexpr uint32_t PT_TILE_CHUNKS = PT_TILE / LOG_CHUNK;
  static_assert(PT_TILE % LOG_CHUNK == 0 && WIN % PT_TILE == 0, "tiles hold whole log chunks");
  extern __shared__ __align__(16) unsigned char smraw[];
  uint4* stage = reinterpret_cast<uint4*>(smraw);
  const uint32_t nbk = FROM_LOG ? nb : SUBS;
  uint32_t* cnt = reinterpret_cast<uint32_t*>(stage + PT_TILE);  // counts, then the tile's offsets
  uint32_t* gbase = cnt + nbk;                                   // the tile's start in each bucket
  __shared__ uint32_t fills[PT_TILE_CHUNKS];
  __shared__ uint32_t nbeyond;
  if (FROM_LOG && used) nchunks = min(nchunks, __ldcg(used));
  const uint32_t ntiles =
      FROM_LOG ? (nchunks + PT_TILE_CHUNKS - 1) / PT_TILE_CHUNKS : nb * (WIN / PT_TILE);
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    uint32_t w = 0, valid_end = 0;  // second pass: window and its entry count
    uint64_t src0;                  // index of the tile's first entry
    if (FROM_LOG) {
      src0 = (uint64_t)t * PT_TILE;
    } else {
      w = t / (WIN / PT_TILE);
      const uint32_t k0 = (t % (WIN / PT_TILE)) * PT_TILE;
      const uint32_t c = min(__ldcg(src_info + (uint64_t)w * CURSOR_STRIDE), WIN);
      if (k0 >= c) continue;  // block-uniform
      valid_end = c - k0;
      src0 = (uint64_t)w * WIN + k0;
    }
    for (uint32_t b = threadIdx.x; b < nbk; b += PT_THREADS) cnt[b] = 0;
    if (FROM_LOG && threadIdx.x < PT_TILE_CHUNKS) {
      // a flat source (no fill table) holds `limit` entries in full chunks
      const uint32_t c = t * PT_TILE_CHUNKS + threadIdx.x;
      fills[threadIdx.x] = c >= nchunks ? 0u : src_info ? __ldcg(src_info + c) : min(LOG_CHUNK, limit - c * LOG_CHUNK);
    }
    if (threadIdx.x == 0) nbeyond = 0;
    __syncthreads();
    uint4 v[ITEMS];
    uint32_t pos[ITEMS];
    uint32_t mine_beyond = 0;
#pragma unroll
    for (uint32_t k = 0; k < ITEMS; ++k) {
      const uint32_t e = k * PT_THREADS + threadIdx.x;
      const bool valid = FROM_LOG ? (e % LOG_CHUNK) < fills[e / LOG_CHUNK] : e < valid_end;
      v[k] = valid ? __ldcs(reinterpret_cast<const uint4*>(src + src0 + e)) : make_uint4(NO_ROOT, 0, 0, 0);
    }
    if (FROM_LOG && out1) {
      const uint64_t pol = l2_keep_policy();
#pragma unroll
      for (uint32_t k = 0; k < ITEMS; ++k) {
        if (v[k].x >= limit) continue;
        const Out o = ld_out_nc_keep(out1 + v[k].y, pol);
        const uint64_t rank = o.rank - ((uint64_t)v[k].z | ((uint64_t)v[k].w << 32));
        v[k] = make_uint4(v[k].x, o.root, (uint32_t)rank, (uint32_t)(rank >> 32));
      }
    }
#pragma unroll
    for (uint32_t k = 0; k < ITEMS; ++k) {
      pos[k] = NO_ROOT;
      const uint32_t x = v[k].x;
      if (x < limit) {
        const uint32_t b = FROM_LOG ? x >> WIN_SHIFT : (x >> SUB_SHIFT) & (SUBS - 1);
        pos[k] = atomicAdd(&cnt[b], 1u);
      } else if (FROM_LOG && x != NO_ROOT) {
        ++mine_beyond;
      }
    }
    if (FROM_LOG && mine_beyond) atomicAdd(&nbeyond, mine_beyond);
    __syncthreads();
    // one cursor step per bucket the tile touches.  In the second pass (one
    // bucket per thread) the step's result stays in a register until the
    // sorted tile is in place, so its round trip overlaps the scan and the
    // sort (1.60 -> 1.58 ms at 2^28; the first pass measured slower so)
    const bool one_per_thread = !FROM_LOG && nbk <= PT_THREADS;
    uint32_t g_mine = 0;
    for (uint32_t b = threadIdx.x; b < nbk; b += PT_THREADS) {
      const uint32_t c = cnt[b];
      const uint64_t ci = FROM_LOG ? (uint64_t)b * CURSOR_STRIDE : ((uint64_t)w * SUBS + b) * CURSOR_STRIDE;
      const uint32_t g = c ? atomicAdd(dcursor + ci, c) : 0u;
      if (one_per_thread)
        g_mine = g;
      else
        gbase[b] = g;
    }
    if (FROM_LOG && threadIdx.x == 0 && nbeyond) atomicAdd(beyond, nbeyond);
    const uint32_t total = block_exclusive_scan(cnt, nbk);  // cnt now holds the tile's offsets
#pragma unroll
    for (uint32_t k = 0; k < ITEMS; ++k) {
      if (pos[k] == NO_ROOT) continue;
      const uint32_t x = v[k].x;
      const uint32_t b = FROM_LOG ? x >> WIN_SHIFT : (x >> SUB_SHIFT) & (SUBS - 1);
      stage[cnt[b] + pos[k]] = v[k];
    }
    if (one_per_thread && threadIdx.x < nbk) gbase[threadIdx.x] = g_mine;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < total; i += PT_THREADS) {
      const uint4 e = stage[i];
      const uint32_t b = FROM_LOG ? e.x >> WIN_SHIFT : (e.x >> SUB_SHIFT) & (SUBS - 1);
      const uint32_t p = gbase[b] + (i - cnt[b]);
      const uint32_t cap = FROM_LOG ? WIN : SUB;
      if (p >= cap) {
        set_error(st, KASCADE_ERR_NOT_A_LIST, e.x);  // an element logged twice
        continue;
      }
      const uint64_t d = FROM_LOG ? (uint64_t)b * WIN + p : (uint64_t)w * WIN + (uint64_t)b * SUB + p;
      __stcg(reinterpret_cast<uint4*>(dst + d), e);
    }
    __syncthreads();
  }
}

// Place: one sub-window (SUB elements) per block iteration.  Its entries
// (element, root, rank) are read in order and placed in shared memory by
// element, then the sub-window's outputs are written densely.  Elements
// without an entry were reached by no chain: their root output becomes
// NOT_REACHED and they join the unreached list (or, when every list head is
// a ruler, they lie on a ruler-free cycle).  A batch's roots are written
// relative to their instance.
__global__ void __launch_bounds__(FIN_THREADS, 2) k_place(const LogEnt* __restrict__ part2,
                                                            const uint32_t* __restrict__ cursor2, uint32_t nb,
                                                            uint32_t limit, uint32_t n,
                                                            const uint32_t* __restrict__ beyond, int heads_are_rulers,
                                                            uint64_t* __restrict__ root_out,
                                                            uint64_t* __restrict__ rank_out,
                                                            uint32_t* __restrict__ ulist,
                                                            uint32_t* __restrict__ ucount, uint32_t ucap,
                                                            const uint64_t* __restrict__ seg_off,
                                                            const uint32_t* __restrict__ hint, uint32_t nseg,
                                                            const uint32_t* __restrict__ plus_one,
                                                            const uint32_t* __restrict__ beyond_want, DevStatus* st) {
  extern __shared__ __align__(16) unsigned char smraw[];
  unsigned long long* rank_s = reinterpret_cast<unsigned long long*>(smraw);  // SUB entries
  uint32_t* root_s = reinterpret_cast<uint32_t*>(rank_s + SUB);               // SUB entries
  __shared__ uint32_t plus_s[SUB / 32];                                       // the sub-window's plus_one words
  const uint32_t lane = threadIdx.x & 31u;
  if (blockIdx.x == 0 && threadIdx.x == 0 && heads_are_rulers) {
    const uint32_t want = beyond_want ? *beyond_want : n - limit;
    if (*beyond > want) set_error(st, KASCADE_ERR_NOT_A_LIST, *beyond);
    if (*beyond < want) set_error(st, KASCADE_ERR_CYCLE, *beyond);
  }
  const uint32_t items = nb * SUBS;
  for (uint32_t it = blockIdx.x; it < items; it += gridDim.x) {
    const uint32_t lo = it * SUB;  // == window * WIN + sub-window * SUB
    if (lo >= limit) continue;     // block-uniform
    const uint32_t len = min(SUB, limit - lo);
    const uint32_t cnt = min(__ldcg(cursor2 + (uint64_t)it * CURSOR_STRIDE), SUB);
    for (uint32_t i = threadIdx.x; i < SUB; i += FIN_THREADS) root_s[i] = NO_ROOT;
    // lo is a multiple of SUB: the sub-window's bits are whole words
    if (plus_one)
      for (uint32_t i = threadIdx.x; i < (len + 31) / 32; i += FIN_THREADS) plus_s[i] = __ldg(plus_one + (lo >> 5) + i);
    __syncthreads();
    const LogEnt* src = part2 + (uint64_t)it * SUB;
    for (uint32_t g = 0; g < SUB / FIN_THREADS; g += FIN_GROUP) {
      uint4 e[FIN_GROUP];
#pragma unroll
      for (uint32_t j = 0; j < FIN_GROUP; ++j) {
        const uint32_t i = (g + j) * FIN_THREADS + threadIdx.x;
        e[j] = i < cnt ? __ldcs(reinterpret_cast<const uint4*>(src + i)) : make_uint4(NO_ROOT, 0, 0, 0);
      }
#pragma unroll
      for (uint32_t j = 0; j < FIN_GROUP; ++j) {
        if (e[j].x == NO_ROOT) continue;
        const uint32_t xl = e[j].x - lo;
        if (xl >= len) {  // not this sub-window's: the partition passes wrote nothing like it
          set_error(st, KASCADE_ERR_NOT_A_LIST, e[j].x);
          continue;
        }
        if (atomicExch(&root_s[xl], e[j].y) != NO_ROOT) set_error(st, KASCADE_ERR_NOT_A_LIST, e[j].x);
        rank_s[xl] = (uint64_t)e[j].z | ((uint64_t)e[j].w << 32);
      }
    }
    __syncthreads();
    // a batch: the instance holding this thread's first element, its offset
    // and the next instance's; a thread's elements only move forward
    uint32_t jseg = 0;
    unsigned long long cur_off = 0, next_off = ~0ull;
    if (seg_off) {
      const uint32_t x0 = lo + threadIdx.x;
      jseg = __ldg(hint + (x0 >> 12));
      while (jseg + 1 < nseg && __ldg(seg_off + jseg + 1) <= x0) ++jseg;
      cur_off = __ldg(seg_off + jseg);
      next_off = jseg + 1 < nseg ? __ldg(seg_off + jseg + 1) : ~0ull;
    }
    for (uint32_t i0 = 0; i0 < len; i0 += FIN_THREADS) {
      const uint32_t i = i0 + threadIdx.x;
      bool un = false;
      if (i < len) {
        const uint32_t r = root_s[i];
        un = r == NO_ROOT;
        if (seg_off) {
          while (lo + i >= next_off) {
            ++jseg;
            cur_off = next_off;
            next_off = jseg + 1 < nseg ? __ldg(seg_off + jseg + 1) : ~0ull;
          }
        }
        const unsigned long long ibase = un ? 0ull : cur_off;
        __stcs(reinterpret_cast<unsigned long long*>(root_out) + lo + i,
               un ? NOT_REACHED : (unsigned long long)r - ibase);
        const unsigned long long add = plus_one ? (plus_s[i >> 5] >> (i & 31)) & 1u : 0u;
        __stcs(reinterpret_cast<unsigned long long*>(rank_out) + lo + i, un ? 0ull : rank_s[i] + add);
      }
      const uint32_t m = __ballot_sync(FULL, un);
      if (m == 0u) continue;
      if (heads_are_rulers) {
        if (un) set_error(st, KASCADE_ERR_CYCLE, lo + i);
        continue;
      }
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(ucount, (uint32_t)__popc(m));
      base = __shfl_sync(FULL, base, 0);
      if (un) {
        const uint32_t p = base + __popc(m & lanemask_lt());
        if (p < ucap)
          ulist[p] = lo + i;
        else
          set_error(st, KASCADE_ERR_TOO_LARGE, p);
      }
    }
    __syncthreads();
  }
}

// Each unreached element walks forward to the first element with outputs:
// one the place step wrote (root output not NOT_REACHED) or one another
// walker finished.  Walkers write the rank, fence, then the root, and readers
// load the root, fence, then the rank, so a root seen set comes with its
// rank.  Elements at or above `limit` (a batch's tour down edges) have no
// outputs and are walked through.  Roots already relative to their instance
// stay so: a walker and the element it stops at share an instance.
__global__ void __launch_bounds__(256) k_walk_unreached(const Rec* __restrict__ rec, const uint32_t* __restrict__ ulist,
                                                        const uint32_t* __restrict__ ucount, uint32_t ucap, uint32_t n,
                                                        uint32_t limit, uint64_t* root_out, uint64_t* rank_out,
                                                        DevStatus* st) {
  const uint32_t cnt = min(*ucount, ucap);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const uint32_t u = ulist[i];
    uint64_t acc = 0;
    uint32_t y = u, mark = u, power = 1, lam = 0, hops = 0;
    unsigned long long base_root = NOT_REACHED;
    bool ok = true;
    while (true) {
      const Rec r = ld_rec_cg(rec + y);
      acc += r.a;
      y = r.b;
      if (y >= n) {  // not reachable for a validated input; keeps every load in range
        set_error(st, KASCADE_ERR_OUT_OF_RANGE, u);
        ok = false;
        break;
      }
      if (y < limit) {
        base_root = __ldcg(reinterpret_cast<const unsigned long long*>(root_out) + y);
        if (base_root != NOT_REACHED) break;
      }
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
    __threadfence();
    const unsigned long long base_rank = __ldcg(reinterpret_cast<const unsigned long long*>(rank_out) + y);
    rank_out[u] = acc + base_rank;
    __threadfence();
    root_out[u] = base_root;
  }
}

// A chain that hit the hop cap, as a status: the device-driven call then
// reruns on the host-driven path, whose level 0 tells the cases apart.
__global__ void k_hop_cap_status(DevStatus* st) {
  if (st->counter[0]) set_error(st, KASCADE_ERR_TIMEOUT, st->counter[0]);
}

constexpr uint32_t TILE1 = PT_THREADS * P1_ITEMS, TILE2 = PT_THREADS * P2_ITEMS;
auto k_part1 = k_partition<true, P1_ITEMS, P1_BLOCKS>;
auto k_part2 = k_partition<false, P2_ITEMS, P2_BLOCKS>;

// Kernel attributes are per device: the shared-memory limits are raised once
// on each.
kascade_status raise_smem_limits() {
  static std::atomic<uint64_t> raised{0};
  int dev = 0;
  KS_CUDA(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (raised.load() & bit) return KASCADE_OK;
  KS_CUDA(cudaFuncSetAttribute(k_part1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(TILE1 * sizeof(LogEnt) + 2 * sizeof(uint32_t) * MAX_BUCKETS)));
  KS_CUDA(cudaFuncSetAttribute(k_part2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(TILE2 * sizeof(LogEnt) + 2 * sizeof(uint32_t) * SUBS)));
  KS_CUDA(cudaFuncSetAttribute(k_place, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(SUB * (sizeof(unsigned long long) + sizeof(uint32_t)))));
  raised.fetch_or(bit);
  return KASCADE_OK;
}

int g_chase_occ[5][3] = {{-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}};

template <int C>
kascade_status launch_chase_log_c(kascade_ctx& ctx, const Rec* rec, uint32_t n, const uint32_t* ruler_elem, uint32_t r,
                                  const uint32_t* r_dev, Rec* rec_next, uint32_t* work, LogEnt* log,
                                  uint32_t* chunk_fill, uint32_t* chunk_cursor, uint32_t nchunks, uint32_t max_hops,
                                  uint32_t* has_pred, unsigned grid, uint32_t block, cudaStream_t s) {
  ProfScope ps(ctx, "chase", s);
  k_chase_log<C><<<grid, block, 0, s>>>(rec, n, ruler_elem, r, r_dev, rec_next, work, log, chunk_fill, chunk_cursor,
                                      nchunks, max_hops, has_pred, ctx.d_status);
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
                               const LogTarget& t, const Params& p, cudaStream_t s, const uint32_t* r0_dev) {
  if (r0_dev) ctx.last_levels.assign(1, n);  // the deeper sizes come back with the status
  const int C = (p.chains == 1 || p.chains == 4) ? (int)p.chains : 2;
  const uint32_t block = p.block;
  const unsigned grid = C == 1   ? chase_grid<1>(ctx, r0, block)
                        : C == 4 ? chase_grid<4>(ctx, r0, block)
                                 : chase_grid<2>(ctx, r0, block);
  const uint64_t warps = (uint64_t)grid * (block / 32);
  const uint32_t nchunks = (uint32_t)(((uint64_t)n + LOG_CHUNK - 1) / LOG_CHUNK + warps + 1);
  LogEnt* log = alloc<LogEnt>(ctx, (uint64_t)nchunks * LOG_CHUNK);
  uint32_t* chunk_fill = alloc<uint32_t>(ctx, nchunks);
  uint32_t* counters = alloc<uint32_t>(ctx, 8);  // chunk cursor, chase work, unreached count, beyond
  Rec* rec1 = alloc<Rec>(ctx, r0);
  Out* out1 = alloc<Out>(ctx, r0);
  uint32_t* lv = r0_dev ? alloc<uint32_t>(ctx, MAX_DEV_LEVELS + 2) : nullptr;  // level sizes (device)
  // device-driven levels: the rulers a chain ended at (level-1 list heads are the others)
  const uint64_t pwords = ((uint64_t)r0 + 31) / 32;
  uint32_t* pred1 = r0_dev ? alloc<uint32_t>(ctx, pwords) : nullptr;
  if (!log || !chunk_fill || !counters || !rec1 || !out1 || (r0_dev && (!lv || !pred1))) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(chunk_fill, 0, sizeof(uint32_t) * nchunks, s));
  KS_CUDA(cudaMemsetAsync(counters, 0, sizeof(uint32_t) * 8, s));
  if (r0_dev) {
    KS_CUDA(cudaMemsetAsync(lv, 0, sizeof(uint32_t) * (MAX_DEV_LEVELS + 2), s));
    KS_CUDA(cudaMemsetAsync(pred1, 0, sizeof(uint32_t) * pwords, s));
    // a tour sized for a bound: its length is the output slots plus the down edges
    if (t.beyond_want) KS_TRY(launch_set_level0(ctx, lv, t.limit, t.beyond_want, s));
    KS_TRY(launch_check_count(ctx, r0_dev, r0, lv + 1, s));
  }
  const uint32_t* r_dev = r0_dev ? lv + 1 : nullptr;
  uint32_t* chunk_cursor = counters + 0;
  uint32_t* chase_work = counters + 1;
  uint32_t* ucount = counters + 2;
  uint32_t* beyond = counters + 3;
  const uint64_t cap = p.max_chain ? p.max_chain : 64ull * p.spacing0 + 1024;
  const uint32_t max_hops = cap < n ? (uint32_t)cap : n;
  switch (C) {
    case 1:
      KS_TRY(launch_chase_log_c<1>(ctx, rec, n, ruler_elem0, r0, r_dev, rec1, chase_work, log, chunk_fill,
                                   chunk_cursor, nchunks, max_hops, pred1, grid, block, s));
      break;
    case 4:
      KS_TRY(launch_chase_log_c<4>(ctx, rec, n, ruler_elem0, r0, r_dev, rec1, chase_work, log, chunk_fill,
                                   chunk_cursor, nchunks, max_hops, pred1, grid, block, s));
      break;
    default:
      KS_TRY(launch_chase_log_c<2>(ctx, rec, n, ruler_elem0, r0, r_dev, rec1, chase_work, log, chunk_fill,
                                   chunk_cursor, nchunks, max_hops, pred1, grid, block, s));
  }
  // level-1 elements are level-0 rulers: their level-0 index is ruler_elem0
  int levels = 0;
  if (r0_dev) {
    k_hop_cap_status<<<1, 1, 0, s>>>(ctx.d_status);
    KS_CHECK_LAUNCH();
    KS_TRY(rank_deep_dev(ctx, rec1, out1, r0, lv, ruler_elem0, pred1, p, s, &levels));
  } else {
    // a chain hit the hop cap: let the caller rerun level 0 on the stamping path
    uint32_t over = 0;
    KS_TRY(read_u32(ctx, reinterpret_cast<const uint32_t*>(&ctx.d_status->counter[0]), &over, s));
    if (over) return KASCADE_ERR_TIMEOUT;
    KS_TRY(rank_sublist(ctx, rec1, r0, ruler_elem0, out1, 1, p, s));
  }

  const uint32_t limit = t.limit < n ? t.limit : n;
  const uint32_t nb = (uint32_t)(((uint64_t)limit + WIN - 1) / WIN);
  const uint32_t nb1 = nb ? nb : 1;
  // first pass: log -> windows (part); second pass: windows -> sub-windows,
  // into the log's memory when it is large enough (the log is dead by then)
  const uint64_t part2_need = (((uint64_t)limit + SUB - 1) / SUB) * SUB;
  LogEnt* part = alloc<LogEnt>(ctx, (uint64_t)nb1 * WIN);
  LogEnt* part2 = (uint64_t)nchunks * LOG_CHUNK >= part2_need ? log : alloc<LogEnt>(ctx, part2_need ? part2_need : 1);
  uint32_t* cursor = alloc<uint32_t>(ctx, (uint64_t)nb1 * (SUBS + 1) * CURSOR_STRIDE);
  if (!part || !part2 || !cursor) return KASCADE_ERR_OOM;
  uint32_t* cursor1 = cursor;
  uint32_t* cursor2 = cursor + (uint64_t)nb1 * CURSOR_STRIDE;
  KS_CUDA(cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * nb1 * (SUBS + 1) * CURSOR_STRIDE, s));
  const size_t smem1 = TILE1 * sizeof(LogEnt) + 2 * sizeof(uint32_t) * nb1;
  const size_t smem2 = TILE2 * sizeof(LogEnt) + 2 * sizeof(uint32_t) * SUBS;
  auto k1 = k_part1;
  auto k2 = k_part2;
  KS_TRY(raise_smem_limits());
  {
    ProfScope ps(ctx, "resolve", s);
    const uint32_t tiles1 = (nchunks + TILE1 / LOG_CHUNK - 1) / (TILE1 / LOG_CHUNK);
    k1<<<(unsigned)std::min<uint64_t>(tiles1, (uint64_t)ctx.usable_sms() * P1_BLOCKS), PT_THREADS, smem1, s>>>(
        log, chunk_fill, nchunks, out1, limit, nb, part, cursor1, beyond, chunk_cursor, ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  const uint32_t tiles2 = nb * (WIN / TILE2);
  if (tiles2) {
    ProfScope ps(ctx, "partition", s);
    k2<<<(unsigned)std::min<uint64_t>(tiles2, (uint64_t)ctx.usable_sms() * P2_BLOCKS), PT_THREADS, smem2, s>>>(
        part, cursor1, 0, nullptr, limit, nb, part2, cursor2, beyond, nullptr, ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  // the first pass's output is dead after the second: it holds the unreached list
  uint32_t* ulist = reinterpret_cast<uint32_t*>(part);
  const uint32_t ucap = limit;
  {
    ProfScope ps(ctx, "place", s);
    const uint32_t items = nb * SUBS;
    const size_t smem = SUB * (sizeof(unsigned long long) + sizeof(uint32_t));
    k_place<<<(unsigned)std::max<uint64_t>(1, std::min<uint64_t>(items, (uint64_t)ctx.usable_sms() * 2)),
                FIN_THREADS, smem, s>>>(part2, cursor2, nb, limit, n, beyond, t.heads_are_rulers, t.root, t.rank,
                                        ulist, ucount, ucap, t.seg_off, t.hint, t.nseg, t.plus_one, t.beyond_want,
                                        ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  if (!t.heads_are_rulers) {
    ProfScope ps(ctx, "heads", s);
    k_walk_unreached<<<ctx.usable_sms() * 4, 256, 0, s>>>(rec, ulist, ucount, ucap, n, limit, t.root, t.rank,
                                                      ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  if (r0_dev) return report_dev_levels(ctx, lv, levels, n, s);
  return KASCADE_OK;
}

}  // namespace ks
