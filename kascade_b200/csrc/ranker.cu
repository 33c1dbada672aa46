// Ruling-set list ranker and pointer doubling for one B200.
//
// Reference counterparts (niklas-uhl/kascade):
//   ruler sampling      lib/kascade/sparse_ruling_set_detail/ruler_selection.hpp:18-115,
//                       sparse_ruling_set.cpp:106-136 (shuffled candidates) -> here a
//                       counter hash of the index, plus every root
//   ruler chasing       sparse_ruling_set.cpp:147-273 (init / work_on_item) and
//                       ruler_chasing_engine.hpp:57-101 (sync rounds) -> one
//                       persistent kernel, every hop a dependent 16 B load
//   unreached fix-up    post_invert.hpp:195-264 -> elements ahead of their list's
//                       first ruler walk forward during propagation
//   pack / recursion    pack.hpp:23-79, sparse_ruling_set.cpp:291-310, 376-392
//                       -> the chase writes the ruler sub-list directly in
//                       dense ruler-id space
//   propagation (pull)  ruler_propagation.hpp:148-256 -> one coalesced pass
//   pointer doubling    pointer_doubling_generic.hpp:43-60, 171-212, 418-438,
//                       609-700 -> double-buffered jump kernel
#include <cstddef>
#include <cstdio>

#include "ranker.cuh"
#include "tma.cuh"

namespace ks {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int PREP_ITEMS = 8;
constexpr int PROP_ITEMS = 8;
constexpr int BASE_THREADS = 1024;
constexpr int BASE_PER_THREAD = 8;  // base_max <= BASE_THREADS * BASE_PER_THREAD

// Weight sources; T is the narrowest type that holds one weight (fewer live
// registers in the prepare kernel).
struct WUnit {
  using T = uint32_t;
  __device__ __forceinline__ T operator()(uint64_t) const { return 1u; }
};
struct WU32 {
  using T = uint32_t;
  const uint32_t* p;
  __device__ __forceinline__ T operator()(uint64_t x) const { return __ldcs(p + x); }
};
struct WI64 {
  using T = uint64_t;
  const int64_t* p;
  __device__ __forceinline__ T operator()(uint64_t x) const {
    return (uint64_t)__ldcs(reinterpret_cast<const long long*>(p) + x);
  }
};

inline uint32_t thresh_for(uint32_t spacing) {
  if (spacing <= 1) return 0xFFFFFFFFu;
  double t = 4294967296.0 / (double)spacing;
  return t >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)t;
}
inline uint32_t salt_for(uint32_t seed, int level) { return mix32(seed + 0x9E3779B9u * (uint32_t)(level + 1)); }

// ---------------------------------------------------------------------------
// prepare: build records, sample rulers (every root is a ruler), number them.
// One atomicAdd per 2048-element tile hands out dense ruler ids.
// ---------------------------------------------------------------------------
template <class W>
__global__ void __launch_bounds__(256, 4) k_prepare_arrays(const uint64_t* __restrict__ succ, W w, uint32_t n,
                                                        uint64_t start, Rec* __restrict__ rec,
                                                        uint32_t* __restrict__ ruler_elem,
                                                        uint32_t* __restrict__ counter, uint32_t salt,
                                                        uint32_t thresh, DevStatus* st) {
  __shared__ uint32_t sm[33];
  __shared__ uint32_t sbase;
  const uint64_t tile_sz = (uint64_t)blockDim.x * PREP_ITEMS;
  for (uint64_t tile = start + (uint64_t)blockIdx.x * tile_sz; tile < n; tile += (uint64_t)gridDim.x * tile_sz) {
    uint32_t sv[PREP_ITEMS];
    typename W::T wv[PREP_ITEMS];
    uint32_t rl = 0, cnt = 0;
#pragma unroll
    for (int i = 0; i < PREP_ITEMS; ++i) {
      uint64_t x = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      sv[i] = 0;
      wv[i] = 0;
      if (x < n) {
        unsigned long long s = __ldcs(reinterpret_cast<const unsigned long long*>(succ) + x);
        if (s >= n) {
          set_error(st, KASCADE_ERR_OUT_OF_RANGE, x);
          s = x;
        }
        sv[i] = (uint32_t)s;
        wv[i] = w(x);
        if (s == x || sampled((uint32_t)x, salt, thresh)) {
          rl |= 1u << i;
          cnt++;
        }
      }
    }
    uint32_t total;
    uint32_t pre = block_exclusive_scan(cnt, sm, &total);
    if (threadIdx.x == 0) {
      uint32_t b = total ? atomicAdd(counter, total) : 0u;
      if ((uint64_t)b + total > MAX_RULERS) set_error(st, KASCADE_ERR_TOO_LARGE, b);
      sbase = b;
    }
    __syncthreads();
    uint32_t id = sbase + pre;
#pragma unroll
    for (int i = 0; i < PREP_ITEMS; ++i) {
      uint64_t x = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      if (x < n) {
        Rec r;
        r.a = wv[i];
        r.b = sv[i];
        r.c = TAG_UNREACHED;
        if (rl & (1u << i)) {
          if (id < MAX_RULERS) {
            r.c = TAG_RULER | id;
            ruler_elem[id] = (uint32_t)x;
          }
          id++;
        }
        rec[x] = r;
      }
    }
    __syncthreads();
  }
}

// The same work for 16 B-aligned inputs, with the input tiles moved by bulk
// (TMA) copies: a persistent block keeps PT_STAGES tiles of succ (and
// weights) in flight into shared memory while it numbers the rulers of an
// earlier tile and writes its records, so the loads no longer wait behind the
// block scan and the ruler-id atomic.  Full tiles only; the caller hands the
// tail to k_prepare_arrays.
constexpr int PT_TILE = 2048;
constexpr int PT_STAGES = 4;
constexpr int PT_ITEMS = PT_TILE / 256;

template <bool W32>
__global__ void __launch_bounds__(256) k_prepare_tma(const uint64_t* __restrict__ succ, const uint32_t* __restrict__ w,
                                                     uint32_t n, uint32_t ntiles, Rec* __restrict__ rec,
                                                     uint32_t* __restrict__ ruler_elem,
                                                     uint32_t* __restrict__ counter, uint32_t salt, uint32_t thresh,
                                                     DevStatus* st) {
  constexpr uint32_t SB = PT_TILE * 8, WB = W32 ? PT_TILE * 4 : 0, STAGE = SB + WB;
  extern __shared__ __align__(128) unsigned char dyn[];
  __shared__ __align__(8) uint64_t bar[PT_STAGES];
  __shared__ uint32_t sm[33];
  __shared__ uint32_t sbase;
  const uint32_t tid = threadIdx.x;
  if (tid == 0) {
    for (int i = 0; i < PT_STAGES; ++i) mbar_init(&bar[i], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // the k-th tile of this block goes to stage k % PT_STAGES
  auto issue = [&](uint32_t k) {
    const uint32_t t = blockIdx.x + k * gridDim.x;
    if (t >= ntiles) return;
    unsigned char* dst = dyn + (k % PT_STAGES) * STAGE;
    uint64_t* b = &bar[k % PT_STAGES];
    mbar_expect_tx(b, STAGE);
    bulk_g2s(dst, succ + (uint64_t)t * PT_TILE, SB, b);
    if (W32) bulk_g2s(dst + SB, w + (uint64_t)t * PT_TILE, WB, b);
  };
  if (tid == 0)
    for (uint32_t k = 0; k < PT_STAGES; ++k) issue(k);
  for (uint32_t k = 0;; ++k) {
    const uint32_t t = blockIdx.x + k * gridDim.x;
    if (t >= ntiles) break;
    const uint32_t sg = k % PT_STAGES;
    const bool ok = mbar_wait_bounded(&bar[sg], (k / PT_STAGES) & 1u);
    if (__syncthreads_or(!ok)) {
      // a copy never completed: report it and let the copies in flight land
      // before the block's shared memory goes away
      if (tid == 0) {
        set_error(st, KASCADE_ERR_TIMEOUT, t);
        for (uint32_t j = k; j < k + PT_STAGES; ++j)
          if (blockIdx.x + j * gridDim.x < ntiles) mbar_wait_bounded(&bar[j % PT_STAGES], (j / PT_STAGES) & 1u);
      }
      __syncthreads();
      return;
    }
    const uint64_t* ss = reinterpret_cast<const uint64_t*>(dyn + sg * STAGE);
    const uint32_t* ws = reinterpret_cast<const uint32_t*>(dyn + sg * STAGE + SB);
    const uint64_t base = (uint64_t)t * PT_TILE;
    uint32_t sv[PT_ITEMS], wv[PT_ITEMS];
    uint32_t rl = 0, cnt = 0;
#pragma unroll
    for (int i = 0; i < PT_ITEMS; ++i) {
      const uint32_t j = i * 256 + tid;
      const uint32_t x = (uint32_t)(base + j);
      unsigned long long sx = ss[j];
      if (sx >= n) {
        set_error(st, KASCADE_ERR_OUT_OF_RANGE, x);
        sx = x;
      }
      sv[i] = (uint32_t)sx;
      wv[i] = W32 ? ws[j] : 1u;
      if (sx == x || sampled(x, salt, thresh)) {
        rl |= 1u << i;
        cnt++;
      }
    }
    __syncthreads();  // the stage is read: refill it with this block's tile k + PT_STAGES
    if (tid == 0) {
      fence_proxy_async();
      issue(k + PT_STAGES);
    }
    uint32_t total;
    const uint32_t pre = block_exclusive_scan(cnt, sm, &total);
    if (tid == 0) {
      const uint32_t b = total ? atomicAdd(counter, total) : 0u;
      if ((uint64_t)b + total > MAX_RULERS) set_error(st, KASCADE_ERR_TOO_LARGE, b);
      sbase = b;
    }
    __syncthreads();
    uint32_t id = sbase + pre;
#pragma unroll
    for (int i = 0; i < PT_ITEMS; ++i) {
      const uint32_t x = (uint32_t)(base + i * 256 + tid);
      Rec r;
      r.a = wv[i];
      r.b = sv[i];
      r.c = TAG_UNREACHED;
      if (rl & (1u << i)) {
        if (id < MAX_RULERS) {
          r.c = TAG_RULER | id;
          ruler_elem[id] = x;
        }
        id++;
      }
      st_rec_cs(rec + x, r);
    }
    __syncthreads();
  }
}

// Deeper levels: the chase of the level above wrote the records (tag
// unreached); sample rulers in place and record each ruler's level-0 index.
// n_dev (device-driven recursion): the level's size is read from device
// memory, n is then its capacity; rulers beyond cap_next are reported as an
// overflow (KASCADE_ERR_TIMEOUT, the caller reruns on the host-driven path).
// has_pred (optional): bit x set when a chain of the level above ended at x;
// an element without it heads its list at this level and becomes a ruler, so
// no element of this level is left for propagation to walk to its first
// ruler (a batch's level holds one list per instance, and the longest of
// those walks would set the propagation's duration).
__global__ void __launch_bounds__(256) k_prepare_level(Rec* __restrict__ rec, uint32_t n,
                                                       const uint32_t* __restrict__ n_dev, uint32_t cap_next,
                                                       const uint32_t* __restrict__ elem0,
                                                       uint32_t* __restrict__ ruler_elem,
                                                       uint32_t* __restrict__ elem0_next,
                                                       uint32_t* __restrict__ counter, uint32_t salt,
                                                       uint32_t thresh, const uint32_t* __restrict__ has_pred,
                                                       DevStatus* st) {
  __shared__ uint32_t sm[33];
  __shared__ uint32_t sbase;
  if (n_dev) n = min(*n_dev, n);
  const uint64_t tile_sz = (uint64_t)blockDim.x * PREP_ITEMS;
  for (uint64_t tile = (uint64_t)blockIdx.x * tile_sz; tile < n; tile += (uint64_t)gridDim.x * tile_sz) {
    Rec rv[PREP_ITEMS];
    uint32_t rl = 0, cnt = 0;
#pragma unroll
    for (int i = 0; i < PREP_ITEMS; ++i) {
      uint64_t x = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      if (x < n) {
        rv[i] = rec[x];
        if (rv[i].b >= n) {  // never for records the level above wrote; kept as a guard
          set_error(st, KASCADE_ERR_OUT_OF_RANGE, x);
          rv[i].b = (uint32_t)x;
        }
        const bool head = has_pred && !((__ldg(has_pred + (x >> 5)) >> (x & 31)) & 1u);
        if (rv[i].b == (uint32_t)x || head || sampled((uint32_t)x, salt, thresh)) {
          rl |= 1u << i;
          cnt++;
        }
      }
    }
    uint32_t total;
    uint32_t pre = block_exclusive_scan(cnt, sm, &total);
    if (threadIdx.x == 0) sbase = total ? atomicAdd(counter, total) : 0u;
    __syncthreads();
    uint32_t id = sbase + pre;
#pragma unroll
    for (int i = 0; i < PREP_ITEMS; ++i) {
      uint64_t x = tile + (uint64_t)i * blockDim.x + threadIdx.x;
      if (x < n) {
        Rec r = rv[i];
        r.c = TAG_UNREACHED;
        if (rl & (1u << i)) {
          if (id < cap_next) {
            r.c = TAG_RULER | id;
            ruler_elem[id] = (uint32_t)x;
            elem0_next[id] = elem0 ? elem0[x] : (uint32_t)x;
          } else {
            set_error(st, KASCADE_ERR_TIMEOUT, id);  // more rulers than the next level holds
          }
          id++;
        }
        rec[x] = r;
      }
    }
    __syncthreads();
  }
}

// A chain that ends on an error still leaves its ruler a valid next-level
// record (a self loop), so that later levels only ever see in-range indices.
__device__ __forceinline__ void end_chain_on_error(Rec* rec_next, uint32_t id) {
  Rec o;
  o.a = 0;
  o.b = id;
  o.c = TAG_UNREACHED;
  st_rec_cg(rec_next + id, o);
}

// ---------------------------------------------------------------------------
// chase: persistent, C chains in flight per thread, rulers handed out to each
// warp in batches of 32*C from one global counter.  A hop reads the 16 B
// record of the next element; an unreached element is stamped with
// (distance from ruler, ruler id) in the same record.  A chain ends at the
// next ruler (or root) and writes its ruler's sub-list record:
// (weight = distance to that ruler, successor = that ruler's id).
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(512) k_chase(Rec* __restrict__ rec, uint32_t n, const uint32_t* __restrict__ n_dev,
                                               const uint32_t* __restrict__ ruler_elem, uint32_t r,
                                               const uint32_t* __restrict__ r_dev, Rec* __restrict__ rec_next,
                                               uint32_t* __restrict__ work, uint32_t* __restrict__ has_pred,
                                               DevStatus* st) {
  // device-driven recursion: sizes from device memory, n and r capacities
  // (has_pred holds one bit per ruler of the capacity; a count past it is
  // reported by the caller's count check and the level redone)
  const uint32_t pred_cap = r;
  if (n_dev) n = min(*n_dev, n);
  if (r_dev) r = min(*r_dev, r);
  constexpr uint32_t BATCH = 32u * C;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt = lanemask_lt();
  uint32_t cid[C], cx[C], hops[C];
  uint64_t acc[C];
  uint32_t act = 0;
  uint32_t q_base = 0, q_left = 0;  // warp-uniform local batch of ruler ids
  bool drained = false;             // warp-uniform
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
          if (mine) {
            const uint32_t id = q_base + my_rank;
            const uint32_t x0 = __ldg(ruler_elem + id);
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
      if (!(act & (1u << c))) continue;
      const uint32_t tg = rr[c].c;
      if (tag_unreached(tg)) {
        Rec wv;
        wv.a = acc[c];
        wv.b = rr[c].b;
        wv.c = cid[c];
        st_rec_cg(rec + cx[c], wv);
        acc[c] += rr[c].a;
        cx[c] = rr[c].b;
        if (++hops[c] > n) {
          set_error(st, KASCADE_ERR_CYCLE, cid[c]);
          end_chain_on_error(rec_next, cid[c]);
          act &= ~(1u << c);
        }
      } else if (tag_ruler(tg)) {
        // back at its own ruler: a cycle without a root that holds one ruler
        // (a valid chain only ends at another ruler)
        if (tag_id(tg) == cid[c])
          set_error(st, KASCADE_ERR_CYCLE, cid[c]);
        else if (has_pred && tag_id(tg) < pred_cap)
          atomicOr(has_pred + (tag_id(tg) >> 5), 1u << (tag_id(tg) & 31));  // that ruler has a predecessor
        Rec o;
        o.a = acc[c];
        o.b = tag_id(tg);
        o.c = TAG_UNREACHED;
        st_rec_cg(rec_next + cid[c], o);
        act &= ~(1u << c);
      } else {
        // already stamped by another chase: two predecessors
        set_error(st, KASCADE_ERR_NOT_A_LIST, cx[c]);
        end_chain_on_error(rec_next, cid[c]);
        act &= ~(1u << c);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// propagate: rank(x) = rank(ruler) - distance(ruler, x); elements no chase
// reached (ahead of their list's first ruler) walk forward to the first
// stamped element and add the weights they pass.
// ---------------------------------------------------------------------------
template <class Sink>
__global__ void __launch_bounds__(256) k_propagate(const Rec* __restrict__ rec, uint32_t n_out, uint32_t n_all,
                                                   const uint32_t* __restrict__ n_dev, uint64_t start,
                                                   const Out* __restrict__ out_next, uint32_t out_cap, Sink sink,
                                                   DevStatus* st) {
  // out_cap: entries of out_next.  Only the device-driven recursion can meet
  // a larger id (a level that outgrew its capacity, already reported as
  // KASCADE_ERR_TIMEOUT); such elements are skipped.
  if (n_dev) n_all = n_out = min(*n_dev, n_out);
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint64_t pol = l2_keep_policy();
  for (uint64_t base = start + (uint64_t)blockIdx.x * blockDim.x * PROP_ITEMS + threadIdx.x; base < n_out;
       base += (uint64_t)stride * PROP_ITEMS) {
    Rec rv[PROP_ITEMS];
#pragma unroll
    for (int i = 0; i < PROP_ITEMS; ++i) {
      uint64_t x = base + (uint64_t)i * blockDim.x;
      if (x < n_out) rv[i] = ld_rec_cs(rec + x);
    }
    // every stamped element's ruler result, all loads in flight together
    // (they would otherwise wait behind the previous element's stores)
    Out ov[PROP_ITEMS];
#pragma unroll
    for (int i = 0; i < PROP_ITEMS; ++i) {
      uint64_t x = base + (uint64_t)i * blockDim.x;
      ov[i] = Out{0, 0, 0};
      if (x < n_out && !tag_unreached(rv[i].c)) {
        const uint32_t id = tag_ruler(rv[i].c) ? tag_id(rv[i].c) : rv[i].c;
        if (id < out_cap) ov[i] = ld_out_keep(out_next + id, pol);
      }
    }
#pragma unroll
    for (int i = 0; i < PROP_ITEMS; ++i) {
      uint64_t x = base + (uint64_t)i * blockDim.x;
      if (x >= n_out) continue;
      Rec r = rv[i];
      Out o = ov[i];
      bool is_root = false;
      uint64_t acc = 0;
      if (tag_unreached(r.c)) {
        // Brent's cycle detection keeps an invalid (rootless, ruler-free)
        // cycle to O(cycle length) steps instead of n per element.
        uint32_t hops = 0, lam = 0, power = 1, mark = (uint32_t)x;
        bool cyc = false;
        while (tag_unreached(r.c)) {
          acc += r.a;
          const uint32_t y = r.b;
          if (y == mark || ++hops > n_all) {
            cyc = true;
            break;
          }
          if (++lam == power) {
            mark = y;
            power <<= 1;
            lam = 0;
          }
          r = ld_rec_cg(rec + y);
        }
        if (cyc) {
          set_error(st, KASCADE_ERR_CYCLE, x);
          continue;
        }
        const uint32_t id = tag_ruler(r.c) ? tag_id(r.c) : r.c;
        if (id >= out_cap) {
          set_error(st, KASCADE_ERR_TIMEOUT, id);
          continue;
        }
        o = ld_out(out_next + id);
      } else {
        if ((tag_ruler(r.c) ? tag_id(r.c) : r.c) >= out_cap) {
          set_error(st, KASCADE_ERR_TIMEOUT, x);
          continue;
        }
        if (tag_ruler(r.c)) is_root = (r.b == (uint32_t)x);
      }
      uint64_t rank;
      uint32_t root;
      if (tag_ruler(r.c)) {
        rank = o.rank + acc;
        root = o.root;
      } else {
        rank = o.rank - r.a + acc;
        root = o.root;
      }
      sink.put((uint32_t)x, rank, root, is_root);
    }
  }
}

// ---------------------------------------------------------------------------
// base case: one CTA, Wyllie pointer jumping in shared memory.
// ---------------------------------------------------------------------------
template <class Sink>
__global__ void __launch_bounds__(BASE_THREADS) k_base(const Rec* __restrict__ rec, uint32_t n,
                                                       const uint32_t* __restrict__ elem0, Sink sink,
                                                       DevStatus* st) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* rk = reinterpret_cast<uint64_t*>(smem);
  uint32_t* sc = reinterpret_cast<uint32_t*>(smem + 8ull * n);
  uint8_t* isroot = smem + 12ull * n;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    Rec r = rec[i];
    if (r.b >= n) {  // guard: treat as a root and report
      set_error(st, KASCADE_ERR_OUT_OF_RANGE, i);
      r.b = i;
    }
    bool root = (r.b == i);
    sc[i] = r.b;
    rk[i] = root ? 0ull : r.a;
    isroot[i] = root ? 1 : 0;
  }
  __syncthreads();
  int round = 0;
  while (true) {
    uint32_t ns[BASE_PER_THREAD];
    uint64_t nr[BASE_PER_THREAD];
    int changed = 0;
#pragma unroll
    for (int j = 0; j < BASE_PER_THREAD; ++j) {
      uint32_t i = threadIdx.x + j * blockDim.x;
      if (i < n) {
        uint32_t s = sc[i];
        if (!isroot[s]) {
          ns[j] = sc[s];
          nr[j] = rk[i] + rk[s];
          changed = 1;
        } else {
          ns[j] = s;
          nr[j] = rk[i];
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < BASE_PER_THREAD; ++j) {
      uint32_t i = threadIdx.x + j * blockDim.x;
      if (i < n) {
        sc[i] = ns[j];
        rk[i] = nr[j];
      }
    }
    if (!__syncthreads_or(changed)) break;
    if (++round > 40) {
      if (threadIdx.x == 0) set_error(st, KASCADE_ERR_CYCLE, 0);
      break;
    }
  }
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    uint32_t rt = sc[i];
    if (elem0) rt = elem0[rt];
    sink.put(i, rk[i], rt, isroot[i] != 0);
  }
}

// ---------------------------------------------------------------------------
// pointer doubling: double-buffered jump rounds over 16 B records.
// done bit 0: successor is a root; bit 1: the element is a root.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_pd_init(const Rec* __restrict__ rec, uint32_t n,
                                                 const uint32_t* __restrict__ n_dev, PdRec* __restrict__ a,
                                                 DevStatus* st) {
  if (n_dev) n = min(*n_dev, n);
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
    Rec r = rec[x];
    if (r.b >= n) {  // guard: treat as a root and report
      set_error(st, KASCADE_ERR_OUT_OF_RANGE, x);
      r.b = (uint32_t)x;
    }
    bool root = (r.b == (uint32_t)x);
    PdRec p;
    p.rank = root ? 0ull : r.a;
    p.succ = r.b;
    p.done = root ? 3u : 0u;
    a[x] = p;
  }
}

// One round of pointer jumping over the previous round's records `a`: an
// element not yet at its root follows its pointer JUMPS times there (a chain
// of dependent reads of `a` only, never of `b`), so a round multiplies every
// pointer's reach by JUMPS + 1.  JUMPS = 1 is classic doubling; the last level
// of the device-driven recursion (at most 2^17 elements, L2-resident, a fixed
// number of launches) takes JUMPS = 3: half the launches for three reads each.
template <int JUMPS>
__global__ void __launch_bounds__(256) k_pd_round(const PdRec* __restrict__ a, PdRec* __restrict__ b, uint32_t n,
                                                  const uint32_t* __restrict__ n_dev, uint32_t* __restrict__ active) {
  if (n_dev) n = min(*n_dev, n);
  uint32_t cnt = 0;
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
    PdRec e = a[x];
#pragma unroll
    for (int j = 0; j < JUMPS; ++j) {
      if (e.done & 1u) break;
      const PdRec t = a[e.succ];
      e.rank += t.rank;
      e.succ = t.succ;
      e.done = t.done & 1u;
    }
    cnt += (e.done & 1u) ? 0u : 1u;
    b[x] = e;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(FULL, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(active, cnt);
}

template <class Sink>
__global__ void __launch_bounds__(256) k_pd_final(const PdRec* __restrict__ a, uint32_t n,
                                                  const uint32_t* __restrict__ n_dev,
                                                  const uint32_t* __restrict__ elem0, Sink sink) {
  if (n_dev) n = min(*n_dev, n);
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
    PdRec e = a[x];
    uint32_t rt = e.succ;
    if (elem0) rt = elem0[rt];
    sink.put((uint32_t)x, e.rank, rt, (e.done & 2u) != 0u);
  }
}

// After a fixed number of rounds every element must point at a root; one that
// does not sits on a rootless cycle.
__global__ void __launch_bounds__(256) k_pd_check(const PdRec* __restrict__ a, uint32_t n,
                                                  const uint32_t* __restrict__ n_dev, DevStatus* st) {
  if (n_dev) n = min(*n_dev, n);
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x)
    if (!(a[x].done & 1u)) set_error(st, KASCADE_ERR_CYCLE, x);
}

// A level's size (device) against its capacity: more means the device-driven
// recursion cannot hold it; the caller reruns on the host-driven path.
__global__ void k_check_count(const uint32_t* __restrict__ cnt, uint32_t cap, uint32_t* __restrict__ copy,
                              DevStatus* st) {
  const uint32_t c = *cnt;
  if (copy) *copy = c;
  if (c > cap) set_error(st, KASCADE_ERR_TIMEOUT, c);
}

// ---------------------------------------------------------------------------
// is_list: count predecessors.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_count_preds(const uint64_t* __restrict__ succ, uint64_t n,
                                                     uint32_t* __restrict__ cnt, uint32_t* __restrict__ bad) {
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t s = succ[x];
    if (s >= n) {
      atomicOr(bad, 2u);
      continue;
    }
    if (s == x) continue;
    if (atomicAdd(cnt + s, 1u) >= 1u) atomicOr(bad, 1u);
  }
}

// ---------------------------------------------------------------------------
// Host-side launch helpers
// ---------------------------------------------------------------------------
template <class K>
int occupancy(K kernel, int block, size_t smem) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, smem) != cudaSuccess) {
    cudaGetLastError();
    nb = 1;
  }
  return nb < 1 ? 1 : nb;
}

template <int C>
kascade_status launch_chase_c(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* ruler_elem, uint32_t r,
                              Rec* rec_next, uint32_t* work, uint32_t block, cudaStream_t s) {
  static int occ[3] = {-1, -1, -1};  // blocks of 128, 256, 512 threads
  const int bi = block == 128 ? 0 : block == 512 ? 2 : 1;
  if (occ[bi] < 0) occ[bi] = occupancy(k_chase<C>, (int)block, 0);
  unsigned grid = (unsigned)(ctx.usable_sms() * occ[bi]);
  const uint64_t warps_per_block = block / 32;
  uint64_t need = ((uint64_t)r + 32ull * C - 1) / (32ull * C);  // warps worth of work
  uint64_t need_blocks = (need + warps_per_block - 1) / warps_per_block;
  if (need_blocks < grid) grid = (unsigned)(need_blocks ? need_blocks : 1);
  ProfScope ps(ctx, "chase", s);
  k_chase<C><<<grid, block, 0, s>>>(rec, n, nullptr, ruler_elem, r, nullptr, rec_next, work, nullptr, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status launch_chase(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* ruler_elem, uint32_t r,
                            Rec* rec_next, const Params& p, cudaStream_t s) {
  uint32_t* work = alloc<uint32_t>(ctx, 1);
  if (!work) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(work, 0, sizeof(uint32_t), s));
  switch (p.chains) {
    case 1:
      return launch_chase_c<1>(ctx, rec, n, ruler_elem, r, rec_next, work, p.block, s);
    case 4:
      return launch_chase_c<4>(ctx, rec, n, ruler_elem, r, rec_next, work, p.block, s);
    default:
      return launch_chase_c<2>(ctx, rec, n, ruler_elem, r, rec_next, work, p.block, s);
  }
}

// Chase with sizes in device memory: n and r are the capacities.
template <int C>
kascade_status launch_chase_dev_c(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* n_dev,
                                  const uint32_t* ruler_elem, uint32_t r, const uint32_t* r_dev, Rec* rec_next,
                                  uint32_t* work, uint32_t* has_pred, uint32_t block, cudaStream_t s) {
  static int occ[3] = {-1, -1, -1};
  const int bi = block == 128 ? 0 : block == 512 ? 2 : 1;
  if (occ[bi] < 0) occ[bi] = occupancy(k_chase<C>, (int)block, 0);
  unsigned grid = (unsigned)(ctx.usable_sms() * occ[bi]);
  const uint64_t warps_per_block = block / 32;
  const uint64_t need = ((uint64_t)r + 32ull * C - 1) / (32ull * C);
  const uint64_t need_blocks = (need + warps_per_block - 1) / warps_per_block;
  if (need_blocks < grid) grid = (unsigned)(need_blocks ? need_blocks : 1);
  ProfScope ps(ctx, "chase", s);
  k_chase<C><<<grid, block, 0, s>>>(rec, n, n_dev, ruler_elem, r, r_dev, rec_next, work, has_pred, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status launch_chase_dev(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* n_dev,
                                const uint32_t* ruler_elem, uint32_t r, const uint32_t* r_dev, Rec* rec_next,
                                uint32_t* work, uint32_t* has_pred, const Params& p, cudaStream_t s) {
  switch (p.chains) {
    case 1:
      return launch_chase_dev_c<1>(ctx, rec, n, n_dev, ruler_elem, r, r_dev, rec_next, work, has_pred, p.block, s);
    case 4:
      return launch_chase_dev_c<4>(ctx, rec, n, n_dev, ruler_elem, r, r_dev, rec_next, work, has_pred, p.block, s);
    default:
      return launch_chase_dev_c<2>(ctx, rec, n, n_dev, ruler_elem, r, r_dev, rec_next, work, has_pred, p.block, s);
  }
}

template <class Sink>
kascade_status launch_propagate(kascade_ctx& ctx, const Rec* rec, uint32_t n_out, uint32_t n_all, const Out* out_next,
                                uint32_t out_cap, const Sink& sink, cudaStream_t s) {
  ProfScope ps(ctx, "propagate", s);
  const unsigned grid = grid_for(ctx, ((uint64_t)n_out + PROP_ITEMS - 1) / PROP_ITEMS, 256, 8);
  k_propagate<Sink><<<grid, 256, 0, s>>>(rec, n_out, n_all, nullptr, 0, out_next, out_cap, sink, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

template <class Sink>
kascade_status launch_base(kascade_ctx& ctx, const Rec* rec, uint32_t n, const uint32_t* elem0, const Sink& sink,
                           cudaStream_t s) {
  if (n == 0) return KASCADE_OK;
  size_t smem = 13ull * n + 16;
  static bool configured = false;
  if (!configured) {
    KS_CUDA(cudaFuncSetAttribute(k_base<Sink>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(13 * BASE_THREADS * BASE_PER_THREAD + 16)));
    configured = true;
  }
  ProfScope ps(ctx, "base_case", s);
  k_base<Sink><<<1, BASE_THREADS, smem, s>>>(rec, n, elem0, sink, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status rank_deep(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* elem0, const SinkOut& sink,
                         int level, const Params& p, cudaStream_t s);

}  // namespace

// ---------------------------------------------------------------------------
// Public (library-internal) entry points
// ---------------------------------------------------------------------------
Params make_params(const kascade_ctx& ctx, const kascade_opts* o, uint64_t n) {
  Params p;
  // Spacing trades chase critical path (~ spacing * ln(n/spacing) hops)
  // against ruler-table size; these defaults are the tuned values for
  // random lists on B200 (see the autotune table in the batch path).
  {
    const int k = ctx.class_of(n);
    p.spacing0 = ctx.class_spacing_single[k];
    p.chains = ctx.class_chains[k];
    p.block = ctx.class_block[k];
  }
  if (o) {
    if (o->ruler_spacing) p.spacing0 = o->ruler_spacing;
    if (o->ruler_spacing_deep) p.spacing_deep = o->ruler_spacing_deep;
    if (o->max_levels) p.max_levels = o->max_levels;
    if (o->base_case_size) p.base_max = o->base_case_size;
    if (o->chains_per_thread) p.chains = o->chains_per_thread;
    if (o->block_size) p.block = o->block_size;
    if (o->seed) p.seed = o->seed;
    p.algorithm = o->algorithm;
    if (o->struct_size >= offsetof(kascade_opts, max_chain) + sizeof(uint32_t)) {
      if (o->level0_mode == 1) p.level0_log_min = 0xFFFFFFFFu;
      if (o->level0_mode == 2) p.level0_log_min = 0;
      p.max_chain = o->max_chain;
    }
  }
  if (p.base_max > (uint32_t)(BASE_THREADS * BASE_PER_THREAD)) p.base_max = BASE_THREADS * BASE_PER_THREAD;
  if (p.block != 128 && p.block != 512) p.block = 256;
  if (p.spacing0 < 2) p.spacing0 = 2;
  if (p.spacing_deep < 2) p.spacing_deep = 2;
  return p;
}

kascade_status prepare_arrays(kascade_ctx& ctx, const uint64_t* succ, WKind wk, const void* w, uint32_t n, Rec* rec,
                              uint32_t* ruler_elem, uint32_t* r_out, const Params& p, cudaStream_t s,
                              uint32_t** r_dev) {
  uint32_t* ctr = alloc<uint32_t>(ctx, 1);
  if (!ctr) return KASCADE_ERR_OOM;
  if (r_dev) *r_dev = ctr;
  KS_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t), s));
  uint32_t salt = salt_for(p.seed, 0), th = thresh_for(p.spacing0);
  {
    ProfScope ps(ctx, "prepare", s);
    // full tiles of 16 B-aligned inputs go through the bulk-copy kernel
    uint64_t start = 0;
    const bool aligned = (reinterpret_cast<uintptr_t>(succ) % 16 == 0) &&
                         (wk == WKind::Unit || (wk == WKind::U32 && reinterpret_cast<uintptr_t>(w) % 16 == 0));
    const uint32_t ntiles = n / PT_TILE;
    if (aligned && ntiles >= (uint32_t)ctx.usable_sms()) {
      const unsigned g = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)ctx.usable_sms() * 2);
      if (wk == WKind::U32) {
        constexpr int smem = PT_STAGES * PT_TILE * 12;
        static bool raised = false;
        if (!raised) {
          KS_CUDA(cudaFuncSetAttribute(k_prepare_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
          raised = true;
        }
        k_prepare_tma<true><<<g, 256, smem, s>>>(succ, (const uint32_t*)w, n, ntiles, rec, ruler_elem, ctr, salt, th,
                                                 ctx.d_status);
      } else {
        constexpr int smem = PT_STAGES * PT_TILE * 8;
        static bool raised = false;
        if (!raised) {
          KS_CUDA(cudaFuncSetAttribute(k_prepare_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
          raised = true;
        }
        k_prepare_tma<false><<<g, 256, smem, s>>>(succ, nullptr, n, ntiles, rec, ruler_elem, ctr, salt, th,
                                                  ctx.d_status);
      }
      KS_CHECK_LAUNCH();
      start = (uint64_t)ntiles * PT_TILE;
    }
    if (start < n) {
      const uint64_t rest = n - start;
      const unsigned grid = grid_for(ctx, (rest + 256 * PREP_ITEMS - 1) / (256 * PREP_ITEMS) * 256, 256, 8);
      switch (wk) {
        case WKind::Unit:
          k_prepare_arrays<WUnit><<<grid, 256, 0, s>>>(succ, WUnit{}, n, start, rec, ruler_elem, ctr, salt, th,
                                                       ctx.d_status);
          break;
        case WKind::U32:
          k_prepare_arrays<WU32><<<grid, 256, 0, s>>>(succ, WU32{(const uint32_t*)w}, n, start, rec, ruler_elem, ctr,
                                                      salt, th, ctx.d_status);
          break;
        case WKind::I64:
          k_prepare_arrays<WI64><<<grid, 256, 0, s>>>(succ, WI64{(const int64_t*)w}, n, start, rec, ruler_elem, ctr,
                                                      salt, th, ctx.d_status);
          break;
      }
      KS_CHECK_LAUNCH();
    }
  }
  // r_out == nullptr: the count stays on the device (*r_dev)
  return r_out ? read_u32(ctx, ctr, r_out, s) : KASCADE_OK;
}

template <class Sink>
kascade_status pointer_double_records(kascade_ctx& ctx, const Rec* rec, uint32_t n, const uint32_t* elem0,
                                      const Sink& sink, cudaStream_t s) {
  if (n == 0) return KASCADE_OK;
  PdRec* a = alloc<PdRec>(ctx, n);
  PdRec* b = alloc<PdRec>(ctx, n);
  uint32_t* active = alloc<uint32_t>(ctx, 1);
  if (!a || !b || !active) return KASCADE_ERR_OOM;
  unsigned grid = grid_for(ctx, n, 256, 8);
  {
    ProfScope ps(ctx, "pd_init", s);
    k_pd_init<<<grid, 256, 0, s>>>(rec, n, nullptr, a, ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  int rounds = 0;
  while (true) {
    KS_CUDA(cudaMemsetAsync(active, 0, sizeof(uint32_t), s));
    {
      ProfScope ps(ctx, "pd_round", s);
      k_pd_round<1><<<grid, 256, 0, s>>>(a, b, n, nullptr, active);
      KS_CHECK_LAUNCH();
    }
    PdRec* t = a;
    a = b;
    b = t;
    uint32_t left = 0;
    KS_TRY(read_u32(ctx, active, &left, s));
    if (left == 0) break;
    if (++rounds > 64) {
      ctx.error_info = left;
      return KASCADE_ERR_CYCLE;
    }
  }
  {
    ProfScope ps(ctx, "pd_final", s);
    k_pd_final<Sink><<<grid, 256, 0, s>>>(a, n, nullptr, elem0, sink);
    KS_CHECK_LAUNCH();
  }
  return KASCADE_OK;
}

namespace {

kascade_status rank_deep(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* elem0, const SinkOut& sink,
                         int level, const Params& p, cudaStream_t s) {
  ctx.last_levels.push_back(n);
  if (n <= p.base_max) return launch_base(ctx, rec, n, elem0, sink, s);
  uint32_t* ruler_elem = alloc<uint32_t>(ctx, n);
  uint32_t* elem0_next = alloc<uint32_t>(ctx, n);
  uint32_t* ctr = alloc<uint32_t>(ctx, 1);
  if (!ruler_elem || !elem0_next || !ctr) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(ctr, 0, sizeof(uint32_t), s));
  unsigned grid = grid_for(ctx, ((uint64_t)n + 256 * PREP_ITEMS - 1) / (256 * PREP_ITEMS) * 256, 256, 8);
  {
    ProfScope ps(ctx, "prepare_level", s);
    k_prepare_level<<<grid, 256, 0, s>>>(rec, n, nullptr, n, elem0, ruler_elem, elem0_next, ctr,
                                         salt_for(p.seed, level), thresh_for(p.spacing_deep), nullptr,
                                         ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  uint32_t r = 0;
  KS_TRY(read_u32(ctx, ctr, &r, s));
  if ((uint32_t)level >= p.max_levels || (uint64_t)r * 10 > (uint64_t)n * 7)
    return pointer_double_records(ctx, rec, n, elem0, sink, s);
  Rec* rec_next = alloc<Rec>(ctx, r);
  Out* out_next = alloc<Out>(ctx, r);
  if (!rec_next || !out_next) return KASCADE_ERR_OOM;
  KS_TRY(launch_chase(ctx, rec, n, ruler_elem, r, rec_next, p, s));
  KS_TRY(rank_deep(ctx, rec_next, r, elem0_next, SinkOut{out_next}, level + 1, p, s));
  return launch_propagate(ctx, rec, n, n, out_next, r, sink, s);
}

}  // namespace

template <class Sink>
kascade_status rank_records(kascade_ctx& ctx, Rec* rec, uint32_t n, uint32_t r0, uint32_t* ruler_elem0,
                            const Sink& sink, const Params& p, cudaStream_t s) {
  ctx.last_levels.clear();
  ctx.last_levels.push_back(n);
  if (n == 0) return KASCADE_OK;
  if (n <= p.base_max) return launch_base(ctx, rec, n, nullptr, sink, s);
  if (p.algorithm != KASCADE_ALGO_SPARSE_RULING_SET || p.max_levels == 0 || (uint64_t)r0 * 10 > (uint64_t)n * 7)
    return pointer_double_records(ctx, rec, n, nullptr, sink, s);
  if (Sink::kWriteFree && n >= p.level0_log_min && !sink.log_target(n).keep_roots) {
    const kascade_status st = rank_level0_log(ctx, rec, n, r0, ruler_elem0, sink.log_target(n), p, s);
    if (st != KASCADE_ERR_TIMEOUT) return st;
    // a chain exceeded the write-free path's hop cap (invalid input, or an
    // astronomically unlikely ruler gap): redo level 0 on the stamping path
    KS_CUDA(cudaMemsetAsync(&ctx.d_status->counter[0], 0, sizeof(unsigned long long), s));
  }
  Rec* rec1 = alloc<Rec>(ctx, r0);
  Out* out1 = alloc<Out>(ctx, r0);
  if (!rec1 || !out1) return KASCADE_ERR_OOM;
  KS_TRY(launch_chase(ctx, rec, n, ruler_elem0, r0, rec1, p, s));
  // level-1 elements are level-0 rulers: their level-0 index is ruler_elem0
  KS_TRY(rank_deep(ctx, rec1, r0, ruler_elem0, SinkOut{out1}, 1, p, s));
  return launch_propagate(ctx, rec, sink.limit(n), n, out1, r0, sink, s);
}

// ---------------------------------------------------------------------------
// Recursion without host waits.  Level sizes stay in device memory; every
// kernel is sized for its level's capacity and reads the size at run time.
// Capacities shrink by the deep-level ruler density (1.5x margin plus room for
// roots); the last level (at most DEV_FINAL elements, or the first that stops
// shrinking) runs pointer doubling for a fixed number of rounds.  A level that
// outgrows its capacity reports KASCADE_ERR_TIMEOUT and the caller reruns on
// the host-driven path.  The sequence of launches depends only on n and the
// capacities, so it can be captured in a CUDA graph.
// ---------------------------------------------------------------------------
constexpr uint32_t DEV_FINAL = 1u << 17;
constexpr uint32_t DEV_ROOT_MARGIN = 1u << 16;

uint32_t dev_cap_next(uint32_t cap, uint32_t spacing) {
  const uint64_t nx = (uint64_t)cap * 3 / (2ull * (spacing < 2 ? 2 : spacing)) + DEV_ROOT_MARGIN;
  return nx < cap ? (uint32_t)nx : cap;
}

// Levels 1.. of the device-driven recursion.  rec1 / out1 hold caps1
// elements; cnt[1] (device) holds level 1's size once the level-0 chase that
// writes rec1 has run, already checked against caps1; elem0_1 gives each
// level-1 element's level-0 index.  Fills out1 and cnt[2..L]; *levels = L.
kascade_status rank_deep_dev(kascade_ctx& ctx, Rec* rec1, Out* out1, uint32_t cap1, uint32_t* cnt,
                             const uint32_t* elem0_1, const uint32_t* pred1, const Params& p, cudaStream_t s,
                             int* levels) {
  uint32_t caps[MAX_DEV_LEVELS + 1];
  caps[1] = cap1;
  int L = 1;
  while (caps[L] > DEV_FINAL && L < MAX_DEV_LEVELS) {
    const uint32_t nx = dev_cap_next(caps[L], p.spacing_deep);
    if ((uint64_t)nx * 10 >= (uint64_t)caps[L] * 9) break;  // no longer shrinking: final level here
    caps[L + 1] = nx;
    ++L;
  }
  Rec* recs[MAX_DEV_LEVELS + 1];
  Out* outs[MAX_DEV_LEVELS + 1];
  uint32_t* rulers[MAX_DEV_LEVELS + 1];
  const uint32_t* elem0s[MAX_DEV_LEVELS + 1];
  const uint32_t* sizes[MAX_DEV_LEVELS + 1];
  uint32_t* preds[MAX_DEV_LEVELS + 1] = {};  // level k: which elements a chain of level k-1 ended at
  recs[1] = rec1;
  outs[1] = out1;
  elem0s[1] = elem0_1;
  sizes[1] = cnt + 1;
  preds[1] = const_cast<uint32_t*>(pred1);
  for (int k = 1; k <= L; ++k) {
    if (k > 1) {
      recs[k] = alloc<Rec>(ctx, caps[k]);
      outs[k] = alloc<Out>(ctx, caps[k]);
      if (!recs[k] || !outs[k]) return KASCADE_ERR_OOM;
    }
    if (k < L) {
      rulers[k] = alloc<uint32_t>(ctx, caps[k + 1]);
      uint32_t* e0 = alloc<uint32_t>(ctx, caps[k + 1]);
      if (!rulers[k] || !e0) return KASCADE_ERR_OOM;
      elem0s[k + 1] = e0;
      sizes[k + 1] = cnt + k + 1;
    }
    if (k > 1 && k < L) {  // the last level is ranked by doubling and samples no rulers
      const uint64_t words = ((uint64_t)caps[k] + 31) / 32;
      preds[k] = alloc<uint32_t>(ctx, words);
      if (!preds[k]) return KASCADE_ERR_OOM;
      KS_CUDA(cudaMemsetAsync(preds[k], 0, sizeof(uint32_t) * words, s));
    }
  }
  for (int k = 1; k < L; ++k) {
    {
      ProfScope ps(ctx, "prepare_level", s);
      const unsigned grid =
          grid_for(ctx, ((uint64_t)caps[k] + 256 * PREP_ITEMS - 1) / (256 * PREP_ITEMS) * 256, 256, 8);
      k_prepare_level<<<grid, 256, 0, s>>>(recs[k], caps[k], sizes[k], caps[k + 1], elem0s[k], rulers[k],
                                           const_cast<uint32_t*>(elem0s[k + 1]), cnt + k + 1,
                                           salt_for(p.seed, k), thresh_for(p.spacing_deep), preds[k],
                                           ctx.d_status);
      KS_CHECK_LAUNCH();
    }
    uint32_t* work = alloc<uint32_t>(ctx, 1);
    if (!work) return KASCADE_ERR_OOM;
    KS_CUDA(cudaMemsetAsync(work, 0, sizeof(uint32_t), s));
    KS_TRY(launch_chase_dev(ctx, recs[k], caps[k], sizes[k], rulers[k], caps[k + 1], sizes[k + 1], recs[k + 1], work,
                            k + 1 < L ? preds[k + 1] : nullptr, p, s));
  }
  // final level: pointer doubling, enough rounds for any list it can hold
  {
    const uint32_t m = caps[L];
    PdRec* a = alloc<PdRec>(ctx, m);
    PdRec* b = alloc<PdRec>(ctx, m);
    uint32_t* active = alloc<uint32_t>(ctx, 1);
    if (!a || !b || !active) return KASCADE_ERR_OOM;
    const unsigned grid = grid_for(ctx, m, 256, 8);
    ProfScope ps(ctx, "pd_final_level", s);
    k_pd_init<<<grid, 256, 0, s>>>(recs[L], m, sizes[L], a, ctx.d_status);
    KS_CHECK_LAUNCH();
    // rounds of reach x4 until 4^rounds >= 4m: any list of at most m elements
    int lg = 0;
    while ((1ull << lg) < m) ++lg;
    const int rounds = (lg + 1) / 2 + 1;
    for (int i = 0; i < rounds; ++i) {
      k_pd_round<3><<<grid, 256, 0, s>>>(a, b, m, sizes[L], active);
      KS_CHECK_LAUNCH();
      PdRec* t = a;
      a = b;
      b = t;
    }
    k_pd_check<<<grid, 256, 0, s>>>(a, m, sizes[L], ctx.d_status);
    KS_CHECK_LAUNCH();
    k_pd_final<SinkOut><<<grid, 256, 0, s>>>(a, m, sizes[L], elem0s[L], SinkOut{outs[L]});
    KS_CHECK_LAUNCH();
  }
  // propagate back up to level 1
  for (int k = L - 1; k >= 1; --k) {
    ProfScope ps(ctx, "propagate", s);
    const unsigned grid = grid_for(ctx, ((uint64_t)caps[k] + PROP_ITEMS - 1) / PROP_ITEMS, 256, 8);
    k_propagate<SinkOut><<<grid, 256, 0, s>>>(recs[k], caps[k], caps[k], sizes[k], 0, outs[k + 1], caps[k + 1],
                                              SinkOut{outs[k]}, ctx.d_status);
    KS_CHECK_LAUNCH();
  }
  *levels = L;
  return KASCADE_OK;
}

__global__ void k_set_level0(uint32_t* lv, uint32_t base, const uint32_t* add) { lv[0] = base + *add; }

kascade_status launch_set_level0(kascade_ctx& ctx, uint32_t* lv, uint32_t base, const uint32_t* add,
                                 cudaStream_t s) {
  (void)ctx;
  k_set_level0<<<1, 1, 0, s>>>(lv, base, add);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status launch_check_count(kascade_ctx& ctx, const uint32_t* cnt, uint32_t cap, uint32_t* copy,
                                  cudaStream_t s) {
  k_check_count<<<1, 1, 0, s>>>(cnt, cap, copy, ctx.d_status);
  KS_CHECK_LAUNCH();
  return KASCADE_OK;
}

kascade_status report_dev_levels(kascade_ctx& ctx, const uint32_t* cnt, int L, uint32_t n, cudaStream_t s) {
  KS_CUDA(cudaMemcpyAsync(reinterpret_cast<uint32_t*>(ctx.h_pinned + KS_PINNED_LEVELS), cnt,
                          sizeof(uint32_t) * (L + 1), cudaMemcpyDeviceToHost, s));
  ctx.pending_levels = L;
  ctx.pending_n = n;
  return KASCADE_OK;
}

// the device count to add to a sink's element count for level 0's size
// (tours sized for a bound), or null
template <class Sink>
const uint32_t* level0_add(const Sink&) {
  return nullptr;
}
template <>
const uint32_t* level0_add<SinkTour>(const SinkTour& t) {
  return t.downs_dev;
}

template <class Sink>
kascade_status rank_records_dev(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* r0_dev, uint32_t cap1,
                                uint32_t* ruler_elem0, const Sink& sink, const Params& p, cudaStream_t s) {
  ctx.last_levels.clear();
  ctx.last_levels.push_back(n);
  if (n == 0) return KASCADE_OK;
  if (cap1 > n) cap1 = n;
  uint32_t* cnt = alloc<uint32_t>(ctx, MAX_DEV_LEVELS + 2);
  Rec* rec1 = alloc<Rec>(ctx, cap1);
  Out* out1 = alloc<Out>(ctx, cap1);
  const uint64_t pwords = ((uint64_t)cap1 + 31) / 32;
  uint32_t* pred1 = alloc<uint32_t>(ctx, pwords);
  if (!cnt || !rec1 || !out1 || !pred1) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * (MAX_DEV_LEVELS + 2), s));
  KS_CUDA(cudaMemsetAsync(pred1, 0, sizeof(uint32_t) * pwords, s));
  if (const uint32_t* d = level0_add(sink)) KS_TRY(launch_set_level0(ctx, cnt, sink.limit(n), d, s));
  KS_TRY(launch_check_count(ctx, r0_dev, cap1, cnt + 1, s));
  // level 0 chase: capacities as bounds, the ruler count from device memory
  {
    uint32_t* work = alloc<uint32_t>(ctx, 1);
    if (!work) return KASCADE_ERR_OOM;
    KS_CUDA(cudaMemsetAsync(work, 0, sizeof(uint32_t), s));
    KS_TRY(launch_chase_dev(ctx, rec, n, nullptr, ruler_elem0, cap1, r0_dev, rec1, work, pred1, p, s));
  }
  // level-1 elements are level-0 rulers: their level-0 index is ruler_elem0
  int L = 1;
  KS_TRY(rank_deep_dev(ctx, rec1, out1, cap1, cnt, ruler_elem0, pred1, p, s, &L));
  KS_TRY(launch_propagate(ctx, rec, sink.limit(n), n, out1, cap1, sink, s));
  // the level sizes travel back with the call's status
  return report_dev_levels(ctx, cnt, L, n, s);
}

template kascade_status rank_records_dev<SinkBatch>(kascade_ctx&, Rec*, uint32_t, const uint32_t*, uint32_t,
                                                    uint32_t*, const SinkBatch&, const Params&, cudaStream_t);
template kascade_status rank_records_dev<SinkTour>(kascade_ctx&, Rec*, uint32_t, const uint32_t*, uint32_t,
                                                   uint32_t*, const SinkTour&, const Params&, cudaStream_t);
template kascade_status rank_records_dev<SinkPlain>(kascade_ctx&, Rec*, uint32_t, const uint32_t*, uint32_t,
                                                    uint32_t*, const SinkPlain&, const Params&, cudaStream_t);

kascade_status rank_sublist(kascade_ctx& ctx, Rec* rec, uint32_t n, const uint32_t* elem0, Out* out, int level,
                            const Params& p, cudaStream_t s) {
  return rank_deep(ctx, rec, n, elem0, SinkOut{out}, level, p, s);
}

kascade_status check_is_list(kascade_ctx& ctx, const uint64_t* succ, uint64_t n, int* ok, cudaStream_t s) {
  uint32_t* cnt = alloc<uint32_t>(ctx, n);
  uint32_t* bad = alloc<uint32_t>(ctx, 1);
  if (!cnt || !bad) return KASCADE_ERR_OOM;
  KS_CUDA(cudaMemsetAsync(cnt, 0, n * sizeof(uint32_t), s));
  KS_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), s));
  unsigned grid = grid_for(ctx, n, 256, 8);
  {
    ProfScope ps(ctx, "is_list", s);
    k_count_preds<<<grid, 256, 0, s>>>(succ, n, cnt, bad);
    KS_CHECK_LAUNCH();
  }
  uint32_t b = 0;
  KS_TRY(read_u32(ctx, bad, &b, s));
  if (b & 2u) return KASCADE_ERR_OUT_OF_RANGE;
  *ok = (b & 1u) ? 0 : 1;
  return KASCADE_OK;
}

// explicit instantiations for the level-0 sinks
template kascade_status rank_records<SinkPlain>(kascade_ctx&, Rec*, uint32_t, uint32_t, uint32_t*, const SinkPlain&,
                                                const Params&, cudaStream_t);
template kascade_status rank_records<SinkTour>(kascade_ctx&, Rec*, uint32_t, uint32_t, uint32_t*, const SinkTour&,
                                               const Params&, cudaStream_t);
template kascade_status rank_records<SinkBatch>(kascade_ctx&, Rec*, uint32_t, uint32_t, uint32_t*, const SinkBatch&,
                                                const Params&, cudaStream_t);
template kascade_status pointer_double_records<SinkBatch>(kascade_ctx&, const Rec*, uint32_t, const uint32_t*,
                                                          const SinkBatch&, cudaStream_t);
template kascade_status pointer_double_records<SinkPlain>(kascade_ctx&, const Rec*, uint32_t, const uint32_t*,
                                                          const SinkPlain&, cudaStream_t);
template kascade_status pointer_double_records<SinkTour>(kascade_ctx&, const Rec*, uint32_t, const uint32_t*,
                                                         const SinkTour&, cudaStream_t);

}  // namespace ks
